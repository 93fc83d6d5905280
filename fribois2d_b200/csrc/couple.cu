// Strong fluid-structure coupling iterated on the device, for one case or a
// batch: no host synchronisation per iteration.
//
// One coupled step (the loose step of src/main.F90:85-88 made implicit):
//   begin   initial guess F of the body load (Fy, Fz, M): the last two
//           converged loads extrapolated linearly, plus the learned
//           correction of the free coordinate's load when a perceptron is
//           set; the step's start state is saved (SNAP_SAVE);
//   loop    (a CUDA graph WHILE node, or a host loop)
//           restore the start state (from the second solve on), place the
//           body where F moves it (k_rigid PLACE), the fluid step, the loads
//           integrated at the trial position (k_rigid FORCES), then update:
//           F' = the fluid's load; converged when |F' - F|_q <=
//           tol max(1, |F'_q|); else F <- F + omega (F' - F) with Aitken's
//           factor from the free coordinate's residuals, starting from the
//           last factor Aitken computed in an earlier step (clamped to
//           [0.05, 2]; omega0 before the first);
//   accept  body back to the start of the step, the update with F'
//           (k_rigid COMMIT), then the converged step enters the history and
//           its (features, targets) the training-sample ring.
// oracle/fbo.c (fbo_coupled_step) restates the same iteration on the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "../../include/fribois2d.h"
#include "couple.h"
#include "pdl.h"

namespace fb {

namespace {

// Learned predictor's features of the free coordinate q: for each of the
// displacement, velocity and load, the second differences of its last
// kCplDepth converged values (newest first; formed in FP64), divided by
// their root mean square -- the shape of the history's recent curvature,
// bounded by sqrt(kCplDepth) whatever the case's amplitude -- then Re, mass
// ratio, reduced velocity.  scale[g] receives the root mean squares.  Needs
// kCplDepth + 2 converged steps.
__device__ bool features(const Couple &c, float *x, double *scale) {
    const int n = c.nh, q = c.q;
    if (n < kCplDepth + 2) return false;
    const double(*h[3])[3] = {c.hp, c.hv, c.hf};
    for (int g = 0; g < 3; ++g) {
        double d2[kCplDepth], ss = 0.0;
        for (int i = 0; i < kCplDepth; ++i) {
            const int a = n - 1 - i;
            d2[i] = h[g][a][q] - 2.0 * h[g][a - 1][q] + h[g][a - 2][q];
            ss = ss + d2[i] * d2[i];
        }
        const double rms = sqrt(ss / kCplDepth), sc = rms > 0.0 ? rms : 1.0;
        scale[g] = sc;
        for (int i = 0; i < kCplDepth; ++i) x[g * kCplDepth + i] = static_cast<float>(d2[i] / sc);
    }
    x[3 * kCplDepth] = static_cast<float>(c.feat_re);
    x[3 * kCplDepth + 1] = static_cast<float>(c.feat_mr);
    x[3 * kCplDepth + 2] = static_cast<float>(c.feat_ur);
    return true;
}

// The structured part of the learned guess, in units of the history's scale:
// the next second difference extrapolated linearly (2 x0 - x1: the cubic
// extrapolation of the history), unless one value dominates the window (a
// jump of the loads: max |x| > 2, where a smooth window stays near 1), then
// nothing (the linear extrapolation alone).
__device__ double prior(const float *x) {
    float m = 0.0f;
    for (int i = 0; i < kCplDepth; ++i) m = fmaxf(m, fabsf(x[i]));
    return (m > 2.0f) ? 0.0 : 2.0 * static_cast<double>(x[0]) - static_cast<double>(x[1]);
}

constexpr double kResidualBound = 0.02;

__device__ double extrap(const double (*h)[3], int n, int i) {
    if (n >= 2) return 2.0 * h[n - 1][i] - h[n - 2][i];
    if (n == 1) return h[0][i];
    return 0.0;
}

// the perceptron of mlp.cu on one sample: kCplH threads, one per hidden unit,
// the same accumulation order as k_mlp_fwd
__device__ void mlp_one(const float *__restrict__ P, const float *xs, float *h1, float *h2, float *y) {
    const int t = threadIdx.x;
    constexpr int oW1 = 0, ob1 = kCplH * kCplIn, oW2 = ob1 + kCplH, ob2 = oW2 + kCplH * kCplH, oW3 = ob2 + kCplH,
                  ob3 = oW3 + kCplOut * kCplH;
    float a = P[ob1 + t];
    for (int k = 0; k < kCplIn; ++k) a = fmaf(P[oW1 + t * kCplIn + k], xs[k], a);
    h1[t] = tanhf(a);
    __syncthreads();
    a = P[ob2 + t];
    for (int k = 0; k < kCplH; ++k) a = fmaf(P[oW2 + t * kCplH + k], h1[k], a);
    h2[t] = tanhf(a);
    __syncthreads();
    if (t < kCplOut) {
        a = P[ob3 + t];
        for (int k = 0; k < kCplH; ++k) a = fmaf(P[oW3 + t * kCplH + k], h2[k], a);
        y[t] = a;
    }
    __syncthreads();
}

}  // namespace

// one block (kCplH threads) per case.  Initial guess: the last two
// converged loads extrapolated linearly (the plain predictor); with the
// learned predictor the free coordinate's load adds scale x (prior + the
// network's residual, clamped to +-kResidualBound -- the range it was
// trained on: on smooth steps the prior's residual is ~1e-3 of the scale,
// and larger residuals are jumps of the loads that no history predicts).
__global__ void __launch_bounds__(kCplH) k_couple_begin(Couple *const *cs) {
    FB_GRID_WAIT();
    Couple &c = *cs[blockIdx.x];
    __shared__ float xs[kCplIn], h1[kCplH], h2[kCplH], y[kCplOut];
    __shared__ int have, net;
    __shared__ double corr, sF;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 3; ++i) c.F[i] = extrap(c.hf, c.nh, i);
        float x[kCplIn];
        double scale[3];
        have = (c.learned && features(c, x, scale)) ? 1 : 0;
        net = (have && c.mlp) ? 1 : 0;
        if (have) {
            sF = scale[2];
            corr = sF * prior(x + 2 * kCplDepth);
        }
        if (net)
            for (int k = 0; k < kCplIn; ++k) xs[k] = (x[k] - c.norm[k]) / c.norm[kCplIn + k];
    }
    __syncthreads();
    if (net) mlp_one(c.mlp, xs, h1, h2, y);
    if (threadIdx.x == 0) {
        if (net) {
            const double r = static_cast<double>(y[1] * c.norm[2 * kCplIn + kCplOut + 1] + c.norm[2 * kCplIn + 1]);
            corr = corr + sF * fmin(kResidualBound, fmax(-kResidualBound, r));
        }
        if (have) c.F[c.q] += corr;
        for (int i = 0; i < 3; ++i) c.fin[i] = c.F[i];
        c.fin[3] = 0.0;
        c.it = 0;
        c.active = 1;
        c.conv = 0;
        c.omega = c.have_omega ? fmin(2.0, fmax(0.05, c.omega_last)) : c.omega0;
    }
}

// blockIdx.z = case; the blocks of a case stride over its arrays
__global__ void __launch_bounds__(256) k_snap(const SnapList *__restrict__ ls, int mode) {
    FB_GRID_WAIT();
    const SnapList &l = ls[blockIdx.z];
    if (mode == SNAP_RESTORE_LOOP && !(l.c->active && l.c->it > 0)) return;
    const bool save = (mode == SNAP_SAVE);
    const int e0 = (mode == SNAP_RESTORE_BODY) ? l.nfield : 0;
    const long tid = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const long nt = static_cast<long>(gridDim.x) * blockDim.x;
    for (int e = e0; e < l.n; ++e) {
        const double *src = save ? l.arr[e] : l.copy[e];
        double *dst = save ? l.copy[e] : l.arr[e];
        const long len = l.len[e];
        for (long i = tid; i < len; i += nt) dst[i] = src[i];
    }
}

// one block; thread i updates case i (stride); then the WHILE condition
__global__ void __launch_bounds__(256) k_couple_update(Couple *const *cs, int n, cudaGraphConditionalHandle h,
                                                       int set_cond, int *any_out) {
    FB_GRID_WAIT();
    int any = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        Couple &c = *cs[i];
        if (!c.active) continue;
        const int q = c.q, it = c.it;
        double res[3];
        for (int k = 0; k < 3; ++k) {
            c.Ff[k] = c.forces[1 + k];
            res[k] = c.Ff[k] - c.F[k];
        }
        if (it == 0) c.res0 = c.res0 + fabs(res[q]) / fmax(1.0, fabs(c.Ff[q]));
        const bool conv = fabs(res[q]) <= c.tol * fmax(1.0, fabs(c.Ff[q]));
        c.it = it + 1;
        if (conv) {
            c.conv = 1;
            c.active = 0;
            continue;
        }
        if (it + 1 >= c.maxit) {   // not converged: the last fluid load is accepted
            c.active = 0;
            continue;
        }
        if (it > 0) {   // Aitken's factor from the free coordinate's residuals
            const double dr = res[q] - c.rprev[q];
            if (dr != 0.0) {
                c.omega = -c.omega * c.rprev[q] / dr;
                c.omega_last = c.omega;
                c.have_omega = 1;
            }
        }
        for (int k = 0; k < 3; ++k) {
            c.F[k] = c.F[k] + c.omega * res[k];
            c.rprev[k] = res[k];
            c.fin[k] = c.F[k];
        }
        any = 1;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) {
        if (set_cond) cudaGraphSetConditional(h, any ? 1u : 0u);
        if (any_out) *any_out = any ? 1 : 0;
    }
}

// after the loop: the accepted load F' for k_rigid COMMIT and the forcecomp row
__global__ void __launch_bounds__(256) k_couple_accept(Couple *const *cs, int n) {
    FB_GRID_WAIT();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        Couple &c = *cs[i];
        for (int k = 0; k < 3; ++k) {
            c.fin[k] = c.Ff[k];
            c.forces[1 + k] = c.Ff[k];
        }
        c.fin[3] = static_cast<double>(c.it);
        c.steps = c.steps + 1.0;
        c.solves = c.solves + static_cast<double>(c.it);
        if (!c.conv) c.maxit_hits = c.maxit_hits + 1.0;
    }
}

// after COMMIT: the converged step's sample (features of the history before
// it; targets = the corrections its displacement and load needed on top of
// their linear extrapolations, in units of the history's scale, less the
// prior), then the step joins the history
__global__ void __launch_bounds__(256) k_couple_record(Couple *const *cs, int n) {
    FB_GRID_WAIT();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        Couple &c = *cs[i];
        const int q = c.q;
        float x[kCplIn];
        double scale[3];
        if (c.cap > 0 && features(c, x, scale)) {
            const unsigned long long slot = c.nsamples % static_cast<unsigned long long>(c.cap);
            for (int k = 0; k < kCplIn; ++k) c.sx[slot * kCplIn + k] = x[k];
            c.st[slot * kCplOut] = static_cast<float>((c.rigid[q] - extrap(c.hp, c.nh, q)) / scale[0] - prior(x));
            c.st[slot * kCplOut + 1] =
                static_cast<float>((c.Ff[q] - extrap(c.hf, c.nh, q)) / scale[2] - prior(x + 2 * kCplDepth));
            c.nsamples = c.nsamples + 1ull;
        }
        if (c.nh == kCplHist) {
            for (int a = 1; a < kCplHist; ++a)
                for (int k = 0; k < 3; ++k) {
                    c.hp[a - 1][k] = c.hp[a][k];
                    c.hv[a - 1][k] = c.hv[a][k];
                    c.hf[a - 1][k] = c.hf[a][k];
                }
            c.nh = kCplHist - 1;
        }
        for (int k = 0; k < 3; ++k) {
            c.hp[c.nh][k] = c.rigid[k];
            c.hv[c.nh][k] = c.rigid[3 + k];
            c.hf[c.nh][k] = c.Ff[k];
        }
        c.nh = c.nh + 1;
    }
}

void launch_couple_begin(Couple *const *c, int n, cudaStream_t s) {
    pdl(k_couple_begin, dim3(n), dim3(kCplH), 0, s, c);
}

void launch_snap(const SnapList *l, int n, int mode, long longest, cudaStream_t s) {
    // about one wave of blocks over all cases, at least one per case
    const long want = (longest + 1023) / 1024;
    const int per_case = static_cast<int>(std::max(1L, std::min(want, static_cast<long>((2 * 148 * 8 + n - 1) / n))));
    pdl(k_snap, dim3(per_case, 1, n), dim3(256), 0, s, l, mode);
}

void launch_couple_update(Couple *const *c, int n, cudaGraphConditionalHandle h, int set_cond, int *any_out,
                          cudaStream_t s) {
    pdl(k_couple_update, dim3(1), dim3(256), 0, s, c, n, h, set_cond, any_out);
}

void launch_couple_accept(Couple *const *c, int n, cudaStream_t s) {
    pdl(k_couple_accept, dim3(1), dim3(256), 0, s, c, n);
}

void launch_couple_record(Couple *const *c, int n, cudaStream_t s) {
    pdl(k_couple_record, dim3(1), dim3(256), 0, s, c, n);
}

}  // namespace fb
