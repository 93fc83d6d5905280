// Batched tridiagonal line solves (solve_fluid.F90 solq2j/solq2k/solq3j/
// solq3k and the per-mode y solves of phcalc_outflow.F90:34-56).
//
// Every system is factorised once on the host (DGTTRF without row
// interchanges, which these diagonally dominant systems never need); a
// line solve is then the two first-order recurrences of the LU
// substitution,
//     forward   y(i) = a(i) y(i-1) + b(i),        a(0)   = 0
//     backward  x(i) = e(i) x(i+1) + g(i) y(i),   e(n-1) = 0
// A line is cut into contiguous chunks held in registers by consecutive
// threads.  Each thread composes the affine map of its chunk, a scan over
// the chunks (warp shuffles, plus shared memory across warps for long
// lines) gives every chunk its incoming value, and the chunk is applied.
// Depth is O(n/chunks + log chunks); every element is loaded and stored
// once, with all of a thread's loads independent and in flight together.
//
// Lines along y are contiguous in memory: one warp per line, staged through
// shared memory so that global accesses are coalesced.  Lines along z are
// strided: four neighbouring lines share each 32-byte sector, so a block
// interleaves four lines over its lanes and splits k among its warps.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.cuh"
#include "pdl.h"
#include "tri.h"

namespace fb {

#define Fv(a, j, k) (a)[fidx(d, (j), (k))]

namespace {

constexpr unsigned kFull = 0xffffffffu;

struct CoefShared {      // y or z systems: 1-D factors shared by all lines
    const double *a, *e, *g;
    template <int M>
    __device__ __forceinline__ void loadA(double (&c)[M], int i0, int cnt) const {
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) c[t] = __ldg(a + i0 + t);
    }
    template <int M>
    __device__ __forceinline__ void loadE(double (&c)[M], int i0, int cnt) const {
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) c[t] = __ldg(e + i0 + t);
    }
    template <int M>
    __device__ __forceinline__ void loadG(double (&c)[M], int i0, int cnt) const {
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) c[t] = __ldg(g + i0 + t);
    }
};

struct CoefModeS {       // Poisson mode: reciprocal pivots of the mode and the 1-based y
                         // off-diagonals, staged in shared memory
    const double *g, *amphj, *apphj;
    int n;
    template <int M>
    __device__ __forceinline__ void loadA(double (&c)[M], int i0, int cnt) const {
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) {
                const int i = i0 + t;
                c[t] = (i == 0) ? 0.0 : -(amphj[i + 1] * g[i - 1]);
            }
    }
    template <int M>
    __device__ __forceinline__ void loadE(double (&c)[M], int i0, int cnt) const {
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) {
                const int i = i0 + t;
                c[t] = (i == n - 1) ? 0.0 : -(apphj[i + 1] * g[i]);
            }
    }
    template <int M>
    __device__ __forceinline__ void loadG(double (&c)[M], int i0, int cnt) const {
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) c[t] = g[i0 + t];
    }
};

// The chains below only read registers: the coefficients of a chunk are
// loaded into c[] before each recurrence starts.
template <int M>
__device__ __forceinline__ void fwd_compose(const double (&v)[M], const double (&c)[M], int cnt, double &A,
                                            double &C) {
    A = 1.0;
    C = 0.0;
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) {
            C = fma(c[t], C, v[t]);
            A *= c[t];
        }
}

template <int M>
__device__ __forceinline__ void fwd_apply(double (&v)[M], const double (&c)[M], int cnt, double y) {
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) {
            y = fma(c[t], y, v[t]);
            v[t] = y;
        }
}

template <int M>
__device__ __forceinline__ void bwd_compose(const double (&v)[M], const double (&c)[M], int cnt, double &A,
                                            double &C) {
    A = 1.0;
    C = 0.0;
#pragma unroll
    for (int t = M - 1; t >= 0; --t)
        if (t < cnt) {
            C = fma(c[t], C, v[t]);
            A *= c[t];
        }
}

template <int M>
__device__ __forceinline__ void bwd_apply(double (&v)[M], const double (&c)[M], int cnt, double x) {
#pragma unroll
    for (int t = M - 1; t >= 0; --t)
        if (t < cnt) {
            x = fma(c[t], x, v[t]);
            v[t] = x;
        }
}

template <int M>
__device__ __forceinline__ void scale(double (&v)[M], const double (&c)[M], int cnt) {
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) v[t] = c[t] * v[t];
}

// one warp = one line of n unknowns, one contiguous chunk per lane
template <int M, class Co>
__device__ __forceinline__ void warp_line(double (&v)[M], int i0, int cnt, const Co &co) {
    const int lane = threadIdx.x & 31;
    double c[M], A, C;
    co.loadA(c, i0, cnt);
    fwd_compose(v, c, cnt, A, C);
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const double Ao = __shfl_up_sync(kFull, A, dd), Co_ = __shfl_up_sync(kFull, C, dd);
        if (lane >= dd) {
            C = fma(A, Co_, C);
            A *= Ao;
        }
    }
    double y = __shfl_up_sync(kFull, C, 1);
    if (lane == 0) y = 0.0;
    fwd_apply(v, c, cnt, y);
    co.loadG(c, i0, cnt);
    scale(v, c, cnt);  // g(i) y(i)
    co.loadE(c, i0, cnt);
    bwd_compose(v, c, cnt, A, C);
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const double Ao = __shfl_down_sync(kFull, A, dd), Co_ = __shfl_down_sync(kFull, C, dd);
        if (lane + dd < 32) {
            C = fma(A, Co_, C);
            A *= Ao;
        }
    }
    double x = __shfl_down_sync(kFull, C, 1);
    if (lane == 31) x = 0.0;
    bwd_apply(v, c, cnt, x);
}

// G consecutive warps share one line (lane chunks in warp-major order);
// warps exchange their chunk composites through sh (2 * G doubles per line).
template <int M, int G, class Co>
__device__ __forceinline__ void group_line(double (&v)[M], int i0, int cnt, const Co &co, double *sh) {
    const int lane = threadIdx.x & 31, gw = (threadIdx.x >> 5) % G;
    double c[M], A, C;
    co.loadA(c, i0, cnt);
    fwd_compose(v, c, cnt, A, C);
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const double Ao = __shfl_up_sync(kFull, A, dd), Co_ = __shfl_up_sync(kFull, C, dd);
        if (lane >= dd) {
            C = fma(A, Co_, C);
            A *= Ao;
        }
    }
    if (lane == 31) {
        sh[2 * gw] = A;
        sh[2 * gw + 1] = C;
    }
    double Cex = __shfl_up_sync(kFull, C, 1), Aex = __shfl_up_sync(kFull, A, 1);
    if (lane == 0) {
        Aex = 1.0;
        Cex = 0.0;
    }
    __syncthreads();
    double PC = 0.0;
    for (int q = 0; q < gw; ++q) PC = fma(sh[2 * q], PC, sh[2 * q + 1]);
    fwd_apply(v, c, cnt, fma(Aex, PC, Cex));
    co.loadG(c, i0, cnt);
    scale(v, c, cnt);
    co.loadE(c, i0, cnt);
    __syncthreads();
    bwd_compose(v, c, cnt, A, C);
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const double Ao = __shfl_down_sync(kFull, A, dd), Co_ = __shfl_down_sync(kFull, C, dd);
        if (lane + dd < 32) {
            C = fma(A, Co_, C);
            A *= Ao;
        }
    }
    if (lane == 0) {
        sh[2 * gw] = A;
        sh[2 * gw + 1] = C;
    }
    Cex = __shfl_down_sync(kFull, C, 1);
    Aex = __shfl_down_sync(kFull, A, 1);
    if (lane == 31) {
        Aex = 1.0;
        Cex = 0.0;
    }
    __syncthreads();
    double SC = 0.0;
    for (int q = G - 1; q > gw; --q) SC = fma(sh[2 * q], SC, sh[2 * q + 1]);
    bwd_apply(v, c, cnt, fma(Aex, SC, Cex));
}

// kZLines lines interleaved over the lanes (line = lane % 4), chunks over
// lane/4 and the block's warps; shA/shC hold one composite per (warp, line)
template <int M, class Co>
__device__ __forceinline__ void block_lines(double (&v)[M], int i0, int cnt, const Co &co, double *shA,
                                            double *shC) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, W = blockDim.x >> 5;
    const int l = lane & (kZLines - 1), sub = lane / kZLines;
    constexpr int kSub = 32 / kZLines;
    double c[M], A, C, Ao, Co_;
    // ---- forward
    co.loadA(c, i0, cnt);
    fwd_compose(v, c, cnt, A, C);
#pragma unroll
    for (int dd = kZLines; dd < 32; dd <<= 1) {
        Ao = __shfl_up_sync(kFull, A, dd);
        Co_ = __shfl_up_sync(kFull, C, dd);
        if (lane >= dd) {
            C = fma(A, Co_, C);
            A *= Ao;
        }
    }
    if (sub == kSub - 1) {
        shA[w * kZLines + l] = A;
        shC[w * kZLines + l] = C;
    }
    double Aex = __shfl_up_sync(kFull, A, kZLines), Cex = __shfl_up_sync(kFull, C, kZLines);
    if (sub == 0) {
        Aex = 1.0;
        Cex = 0.0;
    }
    __syncthreads();
    double PC = 0.0;
    for (int q = 0; q < w; ++q) PC = fma(shA[q * kZLines + l], PC, shC[q * kZLines + l]);
    fwd_apply(v, c, cnt, fma(Aex, PC, Cex));
    co.loadG(c, i0, cnt);
    scale(v, c, cnt);
    co.loadE(c, i0, cnt);
    __syncthreads();
    // ---- backward
    bwd_compose(v, c, cnt, A, C);
#pragma unroll
    for (int dd = kZLines; dd < 32; dd <<= 1) {
        Ao = __shfl_down_sync(kFull, A, dd);
        Co_ = __shfl_down_sync(kFull, C, dd);
        if (lane + dd < 32) {
            C = fma(A, Co_, C);
            A *= Ao;
        }
    }
    if (sub == 0) {
        shA[w * kZLines + l] = A;
        shC[w * kZLines + l] = C;
    }
    Aex = __shfl_down_sync(kFull, A, kZLines);
    Cex = __shfl_down_sync(kFull, C, kZLines);
    if (sub == kSub - 1) {
        Aex = 1.0;
        Cex = 0.0;
    }
    __syncthreads();
    double SC = 0.0;
    for (int q = W - 1; q > w; --q) SC = fma(shA[q * kZLines + l], SC, shC[q * kZLines + l]);
    bwd_apply(v, c, cnt, fma(Aex, SC, Cex));
}

}  // namespace

// ---------------------------------------------------------------- y lines

// Rows of a k-major field staged through shared memory: load row (scaled),
// solve with a warp per line, write back.  kind: 0 = solq2j, 1 = solq3j,
// 2 = Poisson mode (rows of hmn).
// kKind 0: the v and w systems of helsolve in one launch (solq2j on rows
// k = 1..n3m of rhs2, then solq3j on rows k = 2..n3m of rhs3; they are
// independent).  kKind 2: Poisson modes (rows of hmn).
// W: warps per line (the Poisson modes use 4: fewer values and registers per
// thread, more lines resident per SM)
template <int M, int kKind, int W = kYWarps>
__device__ __forceinline__ void ylines_body(const Dev &d, const ScanSys &s2, const double *by2, const ScanSys &s3, const double *by3) {
    extern __shared__ double sm[];
    __shared__ double shx[kYLines][2 * W];
    const int wl = (threadIdx.x >> 5) / W;       // line slot in the block
    const int tl = threadIdx.x % (32 * W);       // thread within the line group
    int line = blockIdx.x * kYLines + wl;
    int sys = 0, n, r;
    if (kKind == 2) {
        n = d.n2m;
        r = line;
        if (r >= d.n3m) r = -1;
    } else if (line < d.n3m) {
        sys = 0;
        n = d.n2;
        r = line + 1;
    } else {
        sys = 1;
        n = d.n2m;
        r = line - d.n3m + 2;
        if (r > d.n3m) r = -1;
    }
    const bool live = (r >= 0);
    if (!live) n = d.n2m;  // idle line slot: still takes part in the block barriers
    double *row = nullptr;
    if (live) row = (kKind == 2) ? d.hmn + static_cast<size_t>(r) * d.ldh : (sys == 0 ? d.rhs2 : d.rhs3) + fidx(d, 1, r);
    const double *by = (sys == 0) ? by2 : by3;
    double *buf = sm + wl * (d.n2 + 1);
    constexpr int kT = 32 * W;
    // Poisson modes: the mode's reciprocal pivots and the y off-diagonals
    // are staged with the line, so the recurrences read shared memory only
    double *pgs = sm + kYLines * (d.n2 + 1) + wl * (d.n2m + 1);
    double *ams = sm + kYLines * (d.n2 + 1) + kYLines * (d.n2m + 1), *aps = ams + (d.n2m + 2);
    if (kKind == 2) {
        for (int i = threadIdx.x; i <= d.n2m; i += blockDim.x) {
            ams[i] = __ldg(d.amphj + i);
            aps[i] = __ldg(d.apphj + i);
        }
    }
    // coalesced staging: thread-strided loads, all independent
    if (live) {
        const double *pgr = d.pg + static_cast<size_t>(r) * d.ldh;
#pragma unroll
        for (int it = 0; it < M; ++it) {
            const int i = tl + kT * it;
            if (i < n) {
                double v = __ldcg(row + i);
                if (kKind != 2) {
                    if (sys == 0) v = (i >= 1 && i <= n - 2) ? v * __ldg(by + i + 1) : 0.0;
                    else v = v * __ldg(by + i + 1);
                } else {
                    pgs[i] = __ldg(pgr + i);
                }
                buf[i] = v;
            }
        }
    }
    __syncthreads();
    const int m = ((n + kT - 1) / kT) | 1;  // odd chunk: conflict-free 64-bit shared loads
    const int i0 = min(tl * m, n), cnt = live ? min(m, n - i0) : 0;
    double v[M];
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) v[t] = buf[i0 + t];
    if (kKind == 2) {
        group_line<M, W>(v, i0, cnt, CoefModeS{pgs, ams, aps, n}, shx[wl]);
    } else {
        const ScanSys &s = (sys == 0) ? s2 : s3;
        group_line<M, W>(v, i0, cnt, CoefShared{s.a, s.e, s.g}, shx[wl]);
    }
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) buf[i0 + t] = v[t];
    __syncthreads();
    if (live) {
#pragma unroll
        for (int it = 0; it < M; ++it) {
            const int i = tl + kT * it;
            if (i < n) row[i] = buf[i];
        }
    }
}

template <int M, int kKind, int W = kYWarps>
__global__ void __launch_bounds__(kYLines * W * 32) k_ylines(Dev d, ScanSys s2, const double *by2, ScanSys s3, const double *by3) {
    FB_GRID_WAIT();
    ylines_body<M, kKind, W>(d, s2, by2, s3, by3);
}

// ---------------------------------------------------------------- Poisson modes

// The per-mode y solves of phcalc (phcalc_outflow.F90:34-56): one warp per
// mode.  The block copies the y off-diagonals once and each warp its mode's
// right-hand side (a row of hmn) and reciprocal pivots to its own
// shared-memory rows, all with cp.async in flight together (one wait instead
// of a round trip per element group), then solves with lane chunks of
// an odd length m (conflict-free 8-byte shared accesses): each lane composes
// its chunk of the forward recurrence y(i) = a(i) y(i-1) + b(i),
// a(i) = -amphj(i+1) g(i-1), the warp scans the composites, the lanes apply
// them, scale by g(i), and do the same backward with
// e(i) = -apphj(i+1) g(i); only warp-level synchronisation inside the
// solve.  nw warps (modes) per block, as many as the shared memory holds.
// one warp's mode: the forward and backward recurrences of the staged line
// (in place), then the line stored to its row of hmn
__device__ __forceinline__ void ymodes_solve(int n, int lane, const double *am, const double *ap, double *line,
                                             const double *piv, double *row) {
    const int m = ((n + 31) / 32) | 1;
    const int i0 = min(lane * m, n), cnt = min(m, n - i0);
    // forward: composite of the chunk, y_out = A y_in + C
    double A = 1.0, C = 0.0;
    for (int t = 0; t < cnt; ++t) {
        const int i = i0 + t;
        const double a = (i == 0) ? 0.0 : -(am[i + 1] * piv[i - 1]);
        C = fma(a, C, line[i]);
        A *= a;
    }
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const double Ao = __shfl_up_sync(kFull, A, dd), Co = __shfl_up_sync(kFull, C, dd);
        if (lane >= dd) {
            C = fma(A, Co, C);
            A *= Ao;
        }
    }
    double y = __shfl_up_sync(kFull, C, 1);
    if (lane == 0) y = 0.0;
    for (int t = 0; t < cnt; ++t) {
        const int i = i0 + t;
        const double a = (i == 0) ? 0.0 : -(am[i + 1] * piv[i - 1]);
        y = fma(a, y, line[i]);
        line[i] = piv[i] * y;   // g(i) y(i)
    }
    // backward: x(i) = e(i) x(i+1) + g(i) y(i)
    A = 1.0;
    C = 0.0;
    for (int t = cnt - 1; t >= 0; --t) {
        const int i = i0 + t;
        const double e = (i == n - 1) ? 0.0 : -(ap[i + 1] * piv[i]);
        C = fma(e, C, line[i]);
        A *= e;
    }
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
        const double Ao = __shfl_down_sync(kFull, A, dd), Co = __shfl_down_sync(kFull, C, dd);
        if (lane + dd < 32) {
            C = fma(A, Co, C);
            A *= Ao;
        }
    }
    double x = __shfl_down_sync(kFull, C, 1);
    if (lane == 31) x = 0.0;
    for (int t = cnt - 1; t >= 0; --t) {
        const int i = i0 + t;
        const double e = (i == n - 1) ? 0.0 : -(ap[i + 1] * piv[i]);
        x = fma(e, x, line[i]);
        line[i] = x;
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) row[i] = line[i];
}

// rmax (may be null): the maxima of |hmn| over each row j (over the modes:
// the rows of the INT8 transform's data operand) are accumulated into rmax[j]
// from the block's modes, for the digit cut that follows
__device__ __forceinline__ void ymodes_body(const Dev &d, int nw, double *rmax = nullptr) {
    extern __shared__ double sm[];
    const int n = d.n2m, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double *am = sm, *ap = sm + (n + 2);                       // 1-based off-diagonals
    double *line = sm + 2 * (n + 2) + static_cast<size_t>(w) * 2 * (n + 1);
    double *piv = line + (n + 1);
    // every copy of the block in flight at once (cp.async), one wait
    for (int i = threadIdx.x; i <= n + 1; i += blockDim.x) {
        cp8(am + i, d.amphj + i);
        cp8(ap + i, d.apphj + i);
    }
    const int r = blockIdx.x * nw + w;
    const bool live = (w < nw) && (r < d.n3m);
    double *row = live ? d.hmn + static_cast<size_t>(r) * d.ldh : nullptr;
    if (live) {
        const double *pgr = d.pg + static_cast<size_t>(r) * d.ldh;
        for (int i = lane; i < n; i += 32) {
            cp8(line + i, row + i);
            cp8(piv + i, pgr + i);
        }
    }
    cp_wait();
    __syncthreads();   // the off-diagonals (and every line) are staged
    if (live) ymodes_solve(n, lane, am, ap, line, piv, row);
    if (!rmax) return;
    __syncthreads();   // every live warp's solved line is in shared memory
    const int nlive = max(0, min(nw, d.n3m - blockIdx.x * nw));
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double mx = 0.0;
        for (int q = 0; q < nlive; ++q)
            mx = fmax(mx, fabs(sm[2 * (n + 2) + static_cast<size_t>(q) * 2 * (n + 1) + j]));
        if (mx > 0.0) atomic_max_nonneg(rmax + j, mx);
    }
}

__global__ void __launch_bounds__(256) k_ymodes(Dev d, int nw, double *rmax) {
    FB_GRID_WAIT();
    ymodes_body(d, nw, rmax);
}

__global__ void __launch_bounds__(256) kg_ymodes(const GroupCase *__restrict__ g, int nw) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    ymodes_body(d, nw);
}

// ---------------------------------------------------------------- z lines

// solq2k (+ helsolve wall columns) on blocks [0, nb2) and solq3k on the
// rest, one launch (the two are independent).  Lines j0..j0+3.
template <int M, int kMaxThreads>
__global__ void __launch_bounds__(kMaxThreads) k_zlines(Dev d, SubDev sd, int nb2) {
    FB_GRID_WAIT();
    __shared__ double shA[16 * kZLines], shC[16 * kZLines];
    const int kKind = (static_cast<int>(blockIdx.x) < nb2) ? 0 : 1;
    const int blk = (kKind == 0) ? blockIdx.x : blockIdx.x - nb2;
    const ScanSys &s = (kKind == 0) ? sd.sz2 : sd.sz3;
    const double *bz = (kKind == 0) ? sd.bz2 : sd.bz3;
    const double ugkks = sd.ugkks, ugkkn = sd.ugkkn;
    const int n = (kKind == 0) ? d.n3m : d.n3;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, W = blockDim.x >> 5;
    const int l = lane & (kZLines - 1);
    const int c = w * (32 / kZLines) + lane / kZLines;  // chunk index within the line
    const int nc = W * (32 / kZLines);
    const int m = (n + nc - 1) / nc;
    const int i0 = min(c * m, n), cnt = min(m, n - i0);
    const int j0 = blk * kZLines + 1, j = j0 + l;
    const bool live = (j <= d.n2m) && (kKind == 1 || j >= 2);
    const int jj = live ? j : 2;  // a valid column for the (discarded) loads of idle lanes
    const double *src = (kKind == 0) ? d.rhs2 : d.rhs3;
    double v[M];
    // gather this thread's chunk (row k = i + 1 of column j): loads first
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) v[t] = __ldcg(src + fidx(d, jj, i0 + t + 1));
    double *qf = (kKind == 0) ? d.q2 : d.q3;
    double bs = 0.0, bn = 0.0;
    if (kKind == 0) {
        bs = d.dqb2s[jj] * ugkks;
        bn = d.dqb2n[jj] * ugkkn;
    } else {
        bs = d.dqb3s[jj];
        bn = d.dqb3n[jj];
    }
#pragma unroll
    for (int t = 0; t < M; ++t)
        if (t < cnt) {
            const int k = i0 + t + 1;
            double x = 0.0;
            if (live) {
                if (kKind == 0) {
                    x = v[t] * __ldg(bz + k);
                    if (k == 1) x = x + bs;
                    if (k == n) x = x + bn;
                } else {
                    if (k == 1) x = bs;
                    else if (k == n) x = bn;
                    else x = v[t] * __ldg(bz + k);
                }
            }
            v[t] = x;
        }
    block_lines(v, i0, cnt, CoefShared{s.a, s.e, s.g}, shA, shC);
    if (live) {
        double q[M];
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) q[t] = __ldcg(qf + fidx(d, j, i0 + t + 1));
#pragma unroll
        for (int t = 0; t < M; ++t)
            if (t < cnt) {
                const int k = i0 + t + 1;
                const double add = (kKind == 1 && k == n) ? bn : v[t];
                qf[fidx(d, j, k)] = q[t] + add;
            }
    }
    if (kKind == 0 && j0 == 1) {
        for (int k = threadIdx.x; k <= d.n3; k += blockDim.x) {
            Fv(d.q2, 1, k) = 0.0;
            Fv(d.q2, d.n2, k) = 0.0;
        }
    }
}

// ---------------------------------------------------------------- windowed ADI

// helsolve (helsolve.F90:4-56 with solq2j/solq2k/solq3j/solq3k) as one
// launch over 2-D tiles, both velocity components.  The four Helmholtz
// operators are strongly diagonally dominant (off-diagonals ~ beta*al/h^2
// against a unit diagonal), so the influence of a value on the LU
// recurrences dies out geometrically: the products of K+1 consecutive
// multipliers a(i) (forward) and e(i) (backward) fall below 2^-56 for a
// window K that the host measures from the factors of each substep
// (overlapped, truncated partitions: the truncated-SPIKE idea of Polizzi and
// Sameh for diagonally dominant banded systems).  A thread computes a
// segment of kWSeg values of one recurrence exactly as the sequential
// recurrence would, except that it starts K positions early from zero;
// segments need no communication.  A tile runs four phases through shared
// memory: forward and backward y recurrences over the tile's rows plus a
// halo of K rows on either side in k, then forward and backward z
// recurrences over its columns, adding the result to q2/q3.  rhs2/rhs3 are
// read once and q2/q3 read and written once; the recurrence coefficients of
// the tile are staged in shared memory with it.
constexpr int kWTj = 32;        // tile columns (j): one lane each in the z phases
constexpr int kWSeg = 16;       // values per thread segment
constexpr int kWSegY = 24;      // values per forward-y segment (2 cover a tile row and its halo)
constexpr int kWThreads = 256;
constexpr int kWXp = kWTj + 1;  // row stride of the z right-hand side tile (odd: conflict-free column stores)

namespace {

// y(i) = a(i) y(i-1) + F(i) for the TS positions from s, started from zero K
// positions earlier; a and F are indexed relative to the segment start
// (a[u], F(u) for u = -K .. TS-1).  Positions at or past nmax are not set.
template <int TS, int KM, class FA, class FF>
__device__ __forceinline__ void seg_fwd(const FA &A, const FF &F, int K, int lo, int nmax, double (&y)[TS]) {
    double v = 0.0;
#pragma unroll
    for (int u = -KM; u < 0; ++u)
        if (u >= -K && u >= lo) v = fma(A(u), v, F(u));
#pragma unroll
    for (int t = 0; t < TS; ++t) {
        y[t] = 0.0;
        if (t < nmax) {
            v = fma(A(t), v, F(t));
            y[t] = v;
        }
    }
}

// x(i) = e(i) x(i+1) + g(i) Y(i) for the TS positions from s, started from
// zero K positions after the segment; positions at or past nmax are not used
template <int TS, int KM, class FE, class FG, class FY>
__device__ __forceinline__ void seg_bwd(const FE &E, const FG &G, const FY &Y, int K, int nmax, double (&x)[TS]) {
    double v = 0.0;
#pragma unroll
    for (int u = TS + KM - 1; u >= TS; --u)
        if (u < TS + K && u < nmax) v = fma(E(u), v, G(u) * Y(u));
#pragma unroll
    for (int t = TS - 1; t >= 0; --t) {
        x[t] = 0.0;
        if (t < nmax) {
            v = fma(E(t), v, G(t) * Y(t));
            x[t] = v;
        }
    }
}

template <int kWTk>
struct WinShape {            // shared-memory layout of one tile of kWTk rows (in doubles)
    int nyf, cols, pitch, rows;  // forward y segments per row; rhs tile rows x cols (stride pitch, odd)
    int ypitch, nzf;             // row stride of the forward y values; forward z segments per column
    int ncy, ncz;                // staged coefficient counts (y: a e g; z: a e g)
    int a_size, b_size, c_size;  // regions A (rhs, then z rhs), B (y, then z partials), C (coefficients)
    __host__ __device__ WinShape(int Ky, int Kz) {
        nyf = (kWTj + Ky + kWSegY - 1) / kWSegY;
        cols = nyf * kWSegY + Ky;  // every forward y segment reads inside its row
        pitch = cols | 1;
        rows = kWTk + 2 * Kz;
        ypitch = (nyf * kWSegY) | 1;
        nzf = (kWTk + Kz + kWSeg - 1) / kWSeg;
        ncy = cols;
        ncz = nzf * kWSeg + Kz;
        const int a1 = rows * pitch, a2 = rows * kWXp;
        a_size = a1 > a2 ? a1 : a2;
        const int b1 = rows * ypitch, b2 = nzf * kWSeg * kWTj;
        b_size = b1 > b2 ? b1 : b2;
        c_size = 4 * ncy + 3 * ncz;   // y: a e g and the row normalisers; z: a e g
    }
};

}  // namespace

// blockIdx.y = 0: v (solq2j + solq2k + walls), 1: w (solq3j + solq3k);
// blockIdx.x = tile (tj fastest).
template <int KM, int kWTk>
__device__ __forceinline__ void helsolve_win_body(const Dev &d, const SubDev &sd, int ntj, int Ky, int Kz) {
    extern __shared__ double sm[];
    const WinShape<kWTk> sh(Ky, Kz);
    double *A = sm, *B = sm + sh.a_size, *C = B + sh.b_size;
    const int fld = blockIdx.y;
    const int tj = blockIdx.x % ntj, tk = blockIdx.x / ntj;
    const int j0 = 1 + tj * kWTj, k0 = 1 + tk * kWTk;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int kWarps = kWThreads / 32;
    const ScanSys sy = fld ? sd.sy3 : sd.sy2, sz = fld ? sd.sz3 : sd.sz2;
    const double *by = fld ? sd.by3 : sd.by2, *bz = fld ? sd.bz3 : sd.bz2;
    const double *rhs = fld ? d.rhs3 : d.rhs2;
    double *q = fld ? d.q3 : d.q2;
    const int ny = fld ? d.n2m : d.n2;   // y unknowns (j = 1..ny, line index j-1)
    const int nz = fld ? d.n3 : d.n3m;   // z unknowns (k = 1..nz, line index k-1)
    const int jlo = fld ? 1 : 2;          // columns with a right-hand side
    const int klo = fld ? 2 : 1;          // rows whose y lines are solved
    const int rows = sh.rows, cols = sh.cols;
    const int iy0 = j0 - 1 - Ky;          // y line index of tile column 0
    const int iz0 = k0 - 1 - Kz;          // z line index of tile row 0
    double *cya = C, *cye = C + sh.ncy, *cyg = C + 2 * sh.ncy, *cys = C + 3 * sh.ncy;
    double *cza = C + 4 * sh.ncy, *cze = cza + sh.ncz, *czg = cza + 2 * sh.ncz;

    // 1. coefficients, the y row normalisers of the tile's columns (cys) and
    //    the right-hand side tile; A[r * pitch + c] holds (j0 - Ky + c, k0 - Kz + r).
    //    All of the tile's copies are issued at once (cp.async); the forward
    //    y recurrences scale the right-hand side as they read it
    for (int c = threadIdx.x; c < sh.ncy; c += kWThreads) {
        const int i = iy0 + c;
        if (i >= 0 && i < ny) {
            cp8(cya + c, sy.a + i);
            cp8(cye + c, sy.e + i);
            cp8(cyg + c, sy.g + i);
        } else {
            cya[c] = cye[c] = cyg[c] = 0.0;
        }
        const int jc = j0 - Ky + c;
        if (c < cols && jc >= jlo && jc <= d.n2m) cp8(cys + c, by + jc);
        else cys[c] = 0.0;
    }
    for (int c = threadIdx.x; c < sh.ncz; c += kWThreads) {
        const int i = iz0 + c;
        if (i >= 0 && i < nz) {
            cp8(cza + c, sz.a + i);
            cp8(cze + c, sz.e + i);
            cp8(czg + c, sz.g + i);
        } else {
            cza[c] = cze[c] = czg[c] = 0.0;
        }
    }
    {
        constexpr int kCC = 3;   // column chunks of 32 (cols <= 96)
        int jc[kCC];
        bool okc[kCC];
#pragma unroll
        for (int cc = 0; cc < kCC; ++cc) {
            const int c = lane + 32 * cc;
            jc[cc] = j0 - Ky + c;
            okc[cc] = (c < cols) && (jc[cc] >= jlo && jc[cc] <= d.n2m);
        }
        for (int r = w; r < rows; r += kWarps) {
            const int k = k0 - Kz + r;
            const bool kok = (k >= klo && k <= d.n3m);
#pragma unroll
            for (int cc = 0; cc < kCC; ++cc) {
                if (lane + 32 * cc >= cols) continue;
                double *dst = A + r * sh.pitch + lane + 32 * cc;
                if (kok && okc[cc]) cp8(dst, rhs + fidx(d, jc[cc], k));
                else *dst = 0.0;
            }
        }
        cp_wait();
    }
    __syncthreads();

    // 2. forward y recurrences: lanes = rows, warps = (row group, segment);
    //    B[r * ypitch + c] = y at tile column c (j = j0 + c), c < nyf * kWSegY
    const int nrg = (rows + 31) / 32;
    for (int task = w; task < nrg * sh.nyf; task += kWarps) {
        const int rg = task / sh.nyf, sg = task - rg * sh.nyf;
        const int r = rg * 32 + lane, rr = min(r, rows - 1);
        const int c0 = Ky + sg * kWSegY;  // coefficient/rhs column of the segment start
        const double *arow = A + rr * sh.pitch + c0;
        const int lo = -(j0 - 1 + sg * kWSegY);  // line index 0 relative to the segment start
        double y[kWSegY];
        seg_fwd<kWSegY, KM>([&](int u) { return cya[c0 + u]; }, [&](int u) { return arow[u] * cys[c0 + u]; }, Ky,
                           lo, ny - (j0 - 1 + sg * kWSegY), y);
        if (r < rows) {
#pragma unroll
            for (int t = 0; t < kWSegY; ++t) B[r * sh.ypitch + sg * kWSegY + t] = y[t];
        }
    }
    __syncthreads();

    // 3. backward y recurrences over the tile's columns, then the z right-hand
    //    side: A[r * kWXp + c] = f at (j0 + c, k0 - Kz + r), scaled by the z
    //    row normalisers, with the inflow/outflow terms (solve_fluid.F90:208-209,
    //    266-275)
    for (int task = w; task < nrg * (kWTj / kWSeg); task += kWarps) {
        const int rg = task / (kWTj / kWSeg), sg = task - rg * (kWTj / kWSeg);
        const int r = rg * 32 + lane, rr = min(r, rows - 1);
        const int k = k0 - Kz + r;
        const bool live = (r < rows) && k >= klo && k <= d.n3m;
        const int c0 = Ky + sg * kWSeg;
        const double *brow = B + rr * sh.ypitch + sg * kWSeg;
        double x[kWSeg];
        seg_bwd<kWSeg, KM>([&](int u) { return cye[c0 + u]; }, [&](int u) { return cyg[c0 + u]; },
                           [&](int u) { return brow[u]; }, Ky, ny - (j0 - 1 + sg * kWSeg), x);
        if (r < rows) {
            const double bzk = (k >= 1 && k <= nz) ? __ldg(bz + k) : 0.0;
            double *arow = A + r * kWXp + sg * kWSeg;
            if (k != 1 && k != nz) {   // interior rows: no inflow/outflow term
#pragma unroll
                for (int t = 0; t < kWSeg; ++t) arow[t] = live ? x[t] * bzk : 0.0;
            } else {
#pragma unroll
                for (int t = 0; t < kWSeg; ++t) {
                    const int j = j0 + sg * kWSeg + t;
                    const int jj = min(max(j, 1), d.n2m);
                    double f = live ? x[t] * bzk : 0.0;
                    if (fld == 0) {
                        if (k == 1) f = f + d.dqb2s[jj] * sd.ugkks;
                        if (k == nz) f = f + d.dqb2n[jj] * sd.ugkkn;
                    } else {
                        if (k == 1) f = d.dqb3s[jj];
                        if (k == nz) f = d.dqb3n[jj];
                    }
                    arow[t] = f;
                }
            }
        }
    }
    __syncthreads();

    // 4. forward z recurrences: lanes = columns, warps = segments of rows;
    //    B[c * kWTj + lane] = z partial at tile row c from k0, c < nzf * kWSeg
    const int j = j0 + lane;
    const bool jlive = (j >= jlo && j <= d.n2m);
    const double *acol = A + lane;
    for (int sg = w; sg < sh.nzf; sg += kWarps) {
        const int c0 = Kz + sg * kWSeg;  // tile row and coefficient index of the segment start
        double y[kWSeg];
        // rows past the tile's halo (c0 + u >= rows, last segment only) read
        // whatever region A holds there, inside its allocation ((rows + 15) x
        // kWXp < rows x pitch): they feed only positions past the halo, which
        // the backward z phase never reads
        seg_fwd<kWSeg, KM>([&](int u) { return cza[c0 + u]; }, [&](int u) { return acol[(c0 + u) * kWXp]; }, Kz,
                           -(k0 - 1 + sg * kWSeg), nz - (k0 - 1 + sg * kWSeg), y);
#pragma unroll
        for (int t = 0; t < kWSeg; ++t) B[(sg * kWSeg + t) * kWTj + lane] = y[t];
    }
    __syncthreads();

    // 5. backward z recurrences over the tile's rows; q += result
    for (int sg = w; sg < kWTk / kWSeg; sg += kWarps) {
        const int s = k0 - 1 + sg * kWSeg;
        if (s >= d.n3m) continue;
        const int c0 = Kz + sg * kWSeg;
        const double *bcol = B + sg * kWSeg * kWTj + lane;
        double x[kWSeg];
        seg_bwd<kWSeg, KM>([&](int u) { return cze[c0 + u]; }, [&](int u) { return czg[c0 + u]; },
                           [&](int u) { return bcol[u * kWTj]; }, Kz, nz - s, x);
        if (jlive) {
            double qv[kWSeg];
#pragma unroll
            for (int t = 0; t < kWSeg; ++t)
                if (s + 1 + t <= d.n3m) qv[t] = __ldcg(q + fidx(d, j, s + 1 + t));
#pragma unroll
            for (int t = 0; t < kWSeg; ++t)
                if (s + 1 + t <= d.n3m) q[fidx(d, j, s + 1 + t)] = qv[t] + x[t];
        }
    }
    if (fld == 1 && jlive && w == 0 && k0 <= d.n3m && k0 + kWTk > d.n3m)
        Fv(q, j, d.n3) = Fv(q, j, d.n3) + d.dqb3n[j];
    if (fld == 0 && blockIdx.x == 0) {  // helsolve.F90:35-36: wall values of v
        for (int k = threadIdx.x; k <= d.n3; k += kWThreads) {
            Fv(d.q2, 1, k) = 0.0;
            Fv(d.q2, d.n2, k) = 0.0;
        }
    }
}

template <int KM, int kWTk>
__global__ void __launch_bounds__(kWThreads, 3) k_helsolve_win(Dev d, SubDev sd, int ntj, int Ky, int Kz) {
    FB_GRID_WAIT();
    helsolve_win_body<KM, kWTk>(d, sd, ntj, Ky, Kz);
}

// grouped forms (blockIdx.z = case; substep n 0-based): each case keeps its
// own windows, the group's shared memory fits the largest
template <int KM, int kWTk>
__global__ void __launch_bounds__(kWThreads, 3) kg_helsolve_win(const GroupCase *__restrict__ g, int n, int ntj) {
    __shared__ Dev d;
    __shared__ SubDev s;
    if (!stage_case(g, &d, &s, n)) return;
    helsolve_win_body<KM, kWTk>(d, s, ntj, s.win_y, s.win_z);
}


// ---------------------------------------------------------------- dispatch

namespace {

// line buffers; for the Poisson modes also the pivot rows and the two y
// off-diagonal arrays
size_t ylines_smem(const Dev &d, int kind) {
    size_t n = static_cast<size_t>(kYLines) * (d.n2 + 1);
    if (kind == 2) n += static_cast<size_t>(kYLines) * (d.n2m + 1) + 2 * static_cast<size_t>(d.n2m + 2);
    return n * sizeof(double);
}

template <int kKind>
void ylaunch(const Dev &d, const SubDev *sd, cudaStream_t st) {
    constexpr int W = (kKind == 2) ? kYPoissonWarps : kYWarps;
    const int lines = (kKind == 2) ? d.n3m : d.n3m + (d.n3m - 1);
    const int blocks = (lines + kYLines - 1) / kYLines;
    const int m = ((d.n2 + 32 * W - 1) / (32 * W)) | 1;
    const size_t smem = ylines_smem(d, kKind);
    const ScanSys z{nullptr, nullptr, nullptr};
    const ScanSys s2 = sd ? sd->sy2 : z, s3 = sd ? sd->sy3 : z;
    const double *b2 = sd ? sd->by2 : nullptr, *b3 = sd ? sd->by3 : nullptr;
    const int threads = kYLines * W * 32;
    if (m <= 9) pdl(k_ylines<9, kKind, W>, dim3(blocks), dim3(threads), smem, st, d, s2, b2, s3, b3);
    else if (m <= 17) pdl(k_ylines<17, kKind, W>, dim3(blocks), dim3(threads), smem, st, d, s2, b2, s3, b3);
    else pdl(k_ylines<33, kKind, W>, dim3(blocks), dim3(threads), smem, st, d, s2, b2, s3, b3);
}

void zlaunch(const Dev &d, const SubDev &sd, cudaStream_t st) {
    const int nb2 = (d.n2m + kZLines - 1) / kZLines;
    const int blocks = 2 * nb2;
    const int n = d.n3;  // the longer of the two systems sets the chunking
    constexpr int kChunksPerWarp = 32 / kZLines;
    int warps = (n + kChunksPerWarp * 16 - 1) / (kChunksPerWarp * 16);
    if (warps <= 16) {
        pdl(k_zlines<16, 512>, dim3(blocks), dim3(warps * 32), 0, st, d, sd, nb2);
        return;
    }
    warps = (n + kChunksPerWarp * 32 - 1) / (kChunksPerWarp * 32);
    if (warps <= 10) {
        pdl(k_zlines<32, 320>, dim3(blocks), dim3(warps * 32), 0, st, d, sd, nb2);
        return;
    }
    warps = (n + kChunksPerWarp * 64 - 1) / (kChunksPerWarp * 64);
    pdl(k_zlines<64, 256>, dim3(blocks), dim3(warps * 32), 0, st, d, sd, nb2);
}

template <class K>
cudaError_t allow_smem(K kern) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

}  // namespace

cudaError_t scan_configure() {
    cudaError_t e;
#define AL(K)                                  \
    if ((e = allow_smem(K)) != cudaSuccess) return e;
    AL((k_ylines<9, 0>)) AL((k_ylines<17, 0>)) AL((k_ylines<33, 0>))
    AL((k_helsolve_win<9, 32>)) AL((k_helsolve_win<9, 64>))
    AL((k_helsolve_win<12, 32>)) AL((k_helsolve_win<12, 64>))
    AL((k_helsolve_win<16, 32>)) AL((k_helsolve_win<16, 64>))
    AL((k_helsolve_win<kWinMax, 32>)) AL((k_helsolve_win<kWinMax, 64>))
    AL((kg_helsolve_win<9, 32>)) AL((kg_helsolve_win<9, 64>))
    AL((kg_helsolve_win<12, 32>)) AL((kg_helsolve_win<12, 64>))
    AL((kg_helsolve_win<16, 32>)) AL((kg_helsolve_win<16, 64>))
    AL((kg_helsolve_win<kWinMax, 32>)) AL((kg_helsolve_win<kWinMax, 64>))
    if ((e = cudaFuncSetAttribute(k_ymodes, cudaFuncAttributeMaxDynamicSharedMemorySize, 225 * 1024)) != cudaSuccess ||
        (e = cudaFuncSetAttribute(kg_ymodes, cudaFuncAttributeMaxDynamicSharedMemorySize, 225 * 1024)) != cudaSuccess)
        return e;
#undef AL
    return cudaSuccess;
}

template <int TK>
void win_launch(const Dev &d, const SubDev &s, cudaStream_t st) {
    const int ntj = (d.n2m + kWTj - 1) / kWTj, ntk = (d.n3m + TK - 1) / TK;
    const dim3 grid(ntj * ntk, 2);
    const WinShape<TK> sh(s.win_y, s.win_z);
    const size_t smem = static_cast<size_t>(sh.a_size + sh.b_size + sh.c_size) * sizeof(double);
    // the warm-up of every segment runs KM predicated steps: the smallest
    // instantiated KM that covers both windows
    const int km = std::max(s.win_y, s.win_z);
    if (km <= 9)
        pdl(k_helsolve_win<9, TK>, dim3(grid), dim3(kWThreads), smem, st, d, s, ntj, s.win_y, s.win_z);
    else if (km <= 12)
        pdl(k_helsolve_win<12, TK>, dim3(grid), dim3(kWThreads), smem, st, d, s, ntj, s.win_y, s.win_z);
    else if (km <= 16)
        pdl(k_helsolve_win<16, TK>, dim3(grid), dim3(kWThreads), smem, st, d, s, ntj, s.win_y, s.win_z);
    else
        pdl(k_helsolve_win<kWinMax, TK>, dim3(grid), dim3(kWThreads), smem, st, d, s, ntj, s.win_y, s.win_z);
}

void launch_win_helsolve(const Dev &d, const SubDev &s, cudaStream_t st) {
    if (s.win_tk == 32) win_launch<32>(d, s, st);
    else win_launch<64>(d, s, st);
}

void launch_scan_helsolve(const Dev &d, const SubDev &s, cudaStream_t st) {
    ylaunch<0>(d, &s, st);
    zlaunch(d, s, st);
}

namespace {
// modes per block and shared bytes of k_ymodes: as many warps as fit (<= 8)
int ymodes_shape(const Dev &d, size_t *smem) {
    const size_t shared = 2 * static_cast<size_t>(d.n2m + 2) * sizeof(double);
    const size_t per = 2 * static_cast<size_t>(d.n2m + 1) * sizeof(double);
    const size_t cap = 225u * 1024u;   // the 227 KB opt-in less the grouped kernel's static Dev
    int nw = static_cast<int>(std::min<size_t>(8, (cap - shared) / per));
    if (nw < 1) nw = 1;
    *smem = shared + per * static_cast<size_t>(nw);
    return nw;
}
}  // namespace

void launch_scan_poisson(const Dev &d, cudaStream_t st, double *rmax) {
    size_t smem = 0;
    const int nw = ymodes_shape(d, &smem);
    pdl(k_ymodes, dim3((d.n3m + nw - 1) / nw), dim3(32 * nw), smem, st, d, nw, rmax);
}

template <int TK>
void gwin_launch(const Group &g, int n, cudaStream_t st) {
    const Dev &d = g.rep;
    const int ntj = (d.n2m + kWTj - 1) / kWTj, ntk = (d.n3m + TK - 1) / TK;
    const dim3 grid(ntj * ntk, 2, g.n);
    const int ky = g.win_ky[n], kz = g.win_kz[n];
    const WinShape<TK> sh(ky, kz);   // sizes grow with the windows: fits every case
    const size_t smem = static_cast<size_t>(sh.a_size + sh.b_size + sh.c_size) * sizeof(double);
    const int km = std::max(ky, kz);
    if (km <= 9)
        pdl(kg_helsolve_win<9, TK>, grid, dim3(kWThreads), smem, st, g.cases, n, ntj);
    else if (km <= 12)
        pdl(kg_helsolve_win<12, TK>, grid, dim3(kWThreads), smem, st, g.cases, n, ntj);
    else if (km <= 16)
        pdl(kg_helsolve_win<16, TK>, grid, dim3(kWThreads), smem, st, g.cases, n, ntj);
    else
        pdl(kg_helsolve_win<kWinMax, TK>, grid, dim3(kWThreads), smem, st, g.cases, n, ntj);
}

void glaunch_win_helsolve(const Group &g, int n, cudaStream_t st) {
    if (g.win_tk == 32) gwin_launch<32>(g, n, st);
    else gwin_launch<64>(g, n, st);
}

void glaunch_scan_poisson(const Group &g, cudaStream_t st) {
    const Dev &d = g.rep;
    size_t smem = 0;
    const int nw = ymodes_shape(d, &smem);
    pdl(kg_ymodes, dim3((d.n3m + nw - 1) / nw, 1, g.n), dim3(32 * nw), smem, st, g.cases, nw);
}

}  // namespace fb
