// C ABI of the B200-native FRiBoIS2D fluid time step (include/fribois2d.h):
// context set-up, device memory, substep orchestration, CUDA-graph replay.
#include <cublasLt.h>
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/fribois2d.h"
#include "couple.h"
#include "device.cuh"
#include "host.h"
#include "kernels.h"
#include "tc_gemm.h"
#include "tri.h"

using fb::Dev;
using fb::SubDev;
using fb::TriDev;

struct fb_host {
    fb::HostCase hc;
};

struct fb_ctx {
    fb::HostCase hc;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;              // marker set-up branch
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // fb_set_markers: pinned staging of the four marker arrays, free again once
    // stage_ev (recorded after their copies) has completed
    double *stage_h = nullptr;
    cudaEvent_t stage_ev = nullptr;
    // fb_fluid_tsch / fb_rigid: status and forcecomp row written by the GPU
    // into mapped host memory (k_publish), read after the stream sync
    double *mbox_h = nullptr, *mbox_d = nullptr;
    double *rigid_mbox = nullptr;   // set by fb_rigid around its rigid stage: k_rigid publishes itself
    cublasHandle_t blas = nullptr;
    void *blas_ws = nullptr;                  // 32 MB workspace of cuBLAS / cuBLASLt
    // FP64 transforms through cuBLASLt with an algorithm timed per grid size
    // (fb_autotune); [0] forward hmn = dph zmmt^T, [1] backward dph = hmn zmm^T
    cublasLtHandle_t lt = nullptr;
    cublasLtMatmulDesc_t lt_op = nullptr;
    cublasLtMatrixLayout_t lt_l[6] = {};      // A, B, C of the forward, then of the backward product
    cublasLtMatmulAlgo_t lt_algo[2] = {};
    bool lt_on[2] = {false, false};
    Dev d{};
    fb::NlMaps nlmaps{};                      // TMA descriptors of the stencil tiles' fields
    SubDev sub[3]{};
    double usdtal[3] = {0, 0, 0};
    std::vector<void *> allocs;
    int hist_cap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    cudaGraph_t fgraph = nullptr;             // fluid step alone (fb_fluid_tsch), fixed dt
    cudaGraphExec_t fgraph_exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    double *zmm = nullptr, *zmmt = nullptr;  // Poisson eigenvectors and inverse
    int null_mode = -1;
    bool allow_win = true;    // windowed helsolve allowed (FRIBOIS2D_HELSOLVE=scan turns it off)
    bool report = false;      // end-of-step diagnostics (ttime.F90) into the history rows
    // substep coefficients (Helmholtz factors, row normalisers) of all
    // substeps in one device block, rebuilt for every step when dt varies:
    // host image, pinned staging copy, device copy, pointer fix-ups
    std::vector<double> coef_h;
    std::vector<int> coef_hi;
    double *coef_d = nullptr, *coef_pin = nullptr;
    int *coef_di = nullptr, *coef_pini = nullptr;
    std::vector<std::pair<const double **, size_t>> coef_fix;
    std::vector<std::pair<const int **, size_t>> coef_fixi;
    size_t coef_cap = 0, coef_capi = 0;
    bool vardt = false;       // idtv = .false.: dt from the CFL number every step
    // strong fluid-structure coupling (fb_set_coupling), iterated on the device
    int coupling = FB_COUPLING_LOOSE;
    int cmaxit = 50;
    fb::Couple *cpl = nullptr;                 // device: the iteration's set-up, state, history
    fb::Couple **cpl_list = nullptr;           // device: {cpl}, the form the coupling kernels take
    fb::SnapList snapl{};                      // the saved start-of-step state's arrays
    fb::SnapList *snapl_d = nullptr;           // ... in device memory
    long snap_longest = 0;
    double *snap = nullptr;                    // device copy of the step's starting state
    float *smp_x = nullptr, *smp_t = nullptr;  // device ring of training samples
    int smp_cap = 8192;
    unsigned long long smp_drained = 0;
    fb_mlp *mlp = nullptr;
    float *mlp_norm_d = nullptr;               // x mean, x std, t mean, t std
    bool cond_graph = true;                    // coupled step as a graph WHILE node (else a host loop)
    int tune_tk = 64;         // windowed helsolve tile height (autotuned per grid size)
    int tune_bn = 128;        // 3xTF32 GEMM tile width (autotuned per grid size)
    int tune_i8bn = fb::kI8BN;  // INT8 digit-product tile width, 32, 48 or 64 (autotuned per grid size)
    bool i8_fixed = false;      // the width set by FRIBOIS2D_I8_TILE: not tuned
    // precision form of the Poisson solve (3xTF32 tensor-core transforms + one
    // FP64 refinement sweep); planes of TF32 splits, tensor maps, FP64 scratch
    int poisson_mode = FB_POISSON_FP64;
    int tf32_sweeps = 2;      // FP64 refinement sweeps of the precision form
    fb::SplitPlane pl_a{}, pl_a2{}, pl_zt{}, pl_z{};
    double *zs_d = nullptr, *zsinv_d = nullptr;  // S and S^-1 of zmm = S U (the transforms use U)
    fb::Tf32x3Plan plan_fwd{}, plan_bwd{};
    double *pw = nullptr;
    // FP64 transforms on the INT8 tensor cores: digit planes of the data
    // operand (dph, then hmn) and of the two eigenvector matrices
    fb::I8Plan i8a{}, i8f{}, i8b{};
    // row maxima of the data operand for the digit cut, accumulated by its
    // producer: [0, ldh) dph's (divg), [ldh, 2 ldh) hmn's (the mode solves);
    // each cut clears the other half for the next producer
    double *i8max = nullptr;
    bool i8_ready = false;
    int own_launches = 0;     // own kernels enqueued (counted while capturing)
    int step_kernels = 0;     // own kernels per captured step (coupled: with one fluid solve)
    int iter_kernels = 0;     // own kernels per fluid solve of a coupled step
    // host copies of the scalar state the reference keeps in modules
    double dt = 0, dt_o = 0, beta = 0, al = 0, ga = 0, ro = 0;
    int cur_ns = 0, cur_n = 1;
    std::string err;
};

namespace {

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            std::fprintf(stderr, "fribois2d: %s failed: %s (%s:%d)\n", #call,            \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                    \
            return FB_ERR_CUDA;                                                          \
        }                                                                                \
    } while (0)
#define CB(call)                                                                         \
    do {                                                                                 \
        cublasStatus_t s_ = (call);                                                      \
        if (s_ != CUBLAS_STATUS_SUCCESS) {                                               \
            std::fprintf(stderr, "fribois2d: %s failed: %d (%s:%d)\n", #call,            \
                         static_cast<int>(s_), __FILE__, __LINE__);                      \
            return FB_ERR_CUDA;                                                          \
        }                                                                                \
    } while (0)

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

// Device allocations are zeroed and filled on the context stream and waited
// for: the stream is non-blocking, so work issued on the legacy default
// stream (cudaMemset, pageable cudaMemcpy, which may return before its DMA
// lands) would not be ordered before the context's kernels.
template <class T>
int dnew(fb_ctx *c, T **p, size_t n) {
    void *q = nullptr;
    CK(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    c->allocs.push_back(q);
    CK(cudaMemsetAsync(q, 0, std::max<size_t>(n, 1) * sizeof(T), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    *p = static_cast<T *>(q);
    return FB_OK;
}

// host -> device copy ordered on the context stream and complete on return
int h2d(fb_ctx *c, void *dst, const void *src, size_t bytes) {
    if (!bytes) return FB_OK;
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FB_OK;
}

template <class T>
int dup(fb_ctx *c, T **p, const std::vector<T> &v) {
    int st = dnew(c, p, v.size());
    if (st) return st;
    return h2d(c, *p, v.data(), v.size() * sizeof(T));
}

// Smallest K such that every product of K+1 consecutive |c(i)| is at most
// 2^-56: a recurrence x(i) = c(i) x(i-1) + ... started K positions early from
// zero then agrees with the full recurrence to below the rounding of FP64.
int window_len(const std::vector<double> &c, int kmax) {
    const int n = static_cast<int>(c.size());
    std::vector<double> L(c.size());
    for (int i = 0; i < n; ++i)
        L[static_cast<size_t>(i)] = (c[static_cast<size_t>(i)] == 0.0) ? -HUGE_VAL : std::log2(std::fabs(c[static_cast<size_t>(i)]));
    for (int K = 0; K <= kmax; ++K) {
        bool ok = true;
        for (int m = 0; m + K < n && ok; ++m) {
            double sum = 0.0;
            for (int i = m; i <= m + K; ++i) sum += L[static_cast<size_t>(i)];
            if (sum > -56.0) ok = false;
        }
        if (ok) return K;
    }
    return kmax + 1;
}

// appends v to the coefficient image; *slot points at it once uploaded
void put(fb_ctx *c, const double **slot, const std::vector<double> &v) {
    c->coef_fix.emplace_back(slot, c->coef_h.size());
    c->coef_h.insert(c->coef_h.end(), v.begin(), v.end());
    c->coef_h.resize((c->coef_h.size() + 31) / 32 * 32, 0.0);  // 256-byte aligned arrays
}

void put(fb_ctx *c, const int **slot, const std::vector<int> &v) {
    c->coef_fixi.emplace_back(slot, c->coef_hi.size());
    c->coef_hi.insert(c->coef_hi.end(), v.begin(), v.end());
    c->coef_hi.resize((c->coef_hi.size() + 63) / 64 * 64, 0);
}

// tridiagonal system (lower(2:n), diag, upper(1:n-1)) -> factors in the image
int upload_tri(fb_ctx *c, TriDev &t, fb::ScanSys &sc, const std::vector<double> &lo,
               const std::vector<double> &di, const std::vector<double> &up, int *win = nullptr) {
    fb::TriLU f = fb::factor(lo, di, up);
    if (f.info != 0) return FB_ERR_NUMERIC;
    std::vector<double> dinv(f.d.size());
    for (size_t i = 0; i < f.d.size(); ++i) dinv[i] = 1.0 / f.d[i];
    {   // recurrence form of DGTTS2 without interchanges (tri.cu)
        const int n = f.n;
        std::vector<double> a(static_cast<size_t>(n), 0.0), e(static_cast<size_t>(n), 0.0);
        for (int i = 1; i < n; ++i) a[static_cast<size_t>(i)] = -f.dl[static_cast<size_t>(i - 1)];
        for (int i = 0; i + 1 < n; ++i)
            e[static_cast<size_t>(i)] = -f.du[static_cast<size_t>(i)] * dinv[static_cast<size_t>(i)];
        if (win) *win = std::max(window_len(a, fb::kWinMax), window_len(e, fb::kWinMax));
        put(c, &sc.a, a);
        put(c, &sc.e, e);
        put(c, &sc.g, dinv);
    }
    t.n = f.n;
    t.pivoted = f.pivoted ? 1 : 0;
    put(c, &t.dl, f.dl);
    put(c, &t.dinv, dinv);
    put(c, &t.du, f.du);
    put(c, &t.du2, f.du2);
    put(c, &t.ipiv, f.ipiv);
    return FB_OK;
}

// solve_fluid.F90: the four Helmholtz systems of one substep, normalised to
// a unit diagonal exactly as the reference builds them before DGTTRF.
int build_substep(fb_ctx *c, int n, double al) {
    const fb::Grid &g = c->hc.grid;
    SubDev &s = c->sub[n];
    const int n2 = g.n2, n3 = g.n3, n2m = g.n2m, n3m = g.n3m;
    s.al = al;
    s.beta = c->dt / g.ren * 0.5;
    s.betadx = s.beta * al;
    const double betadx = s.betadx;
    std::vector<double> b(static_cast<size_t>(std::max(n2, n3)) + 2, 0.0);
    int st;
    int wy2 = 0, wz2 = 0, wy3 = 0, wz3 = 0;
    {   // solq2j (solve_fluid.F90:126-153)
        std::vector<double> am(n2 + 1, 0.0), ap(n2 + 1, 0.0), lo, di(n2, 1.0), up;
        std::fill(b.begin(), b.end(), 0.0);
        for (int jc = 2; jc <= n2m; ++jc) {
            double acjl_b = 1.0 / (1.0 - betadx * g.ac2j[jc]);
            ap[jc] = -betadx * g.ap2j[jc] * acjl_b;
            am[jc] = -betadx * g.am2j[jc] * acjl_b;
            b[jc] = acjl_b;
        }
        for (int j = 2; j <= n2; ++j) lo.push_back(am[j]);
        for (int j = 1; j <= n2 - 1; ++j) up.push_back(ap[j]);
        if ((st = upload_tri(c, s.y2, s.sy2, lo, di, up, &wy2))) return st;
        put(c, &s.by2, std::vector<double>(b.begin(), b.begin() + n2 + 2));
    }
    {   // solq2k (solve_fluid.F90:185-212)
        std::vector<double> am(n3m + 1, 0.0), ap(n3m + 1, 0.0), lo, di(n3m, 1.0), up;
        std::fill(b.begin(), b.end(), 0.0);
        for (int kc = 1; kc <= n3m; ++kc) {
            double ackl_b = 1.0 / (1.0 - g.ac3sk[kc] * betadx);
            am[kc] = -g.am3sk[kc] * betadx * ackl_b;
            ap[kc] = -g.ap3sk[kc] * betadx * ackl_b;
            b[kc] = ackl_b;
        }
        for (int k = 2; k <= n3m; ++k) lo.push_back(am[k]);
        for (int k = 1; k <= n3m - 1; ++k) up.push_back(ap[k]);
        if ((st = upload_tri(c, s.z2, s.sz2, lo, di, up, &wz2))) return st;
        put(c, &s.bz2, std::vector<double>(b.begin(), b.begin() + n3 + 2));
        s.ugkks = 1.0 / (g.g3rm[1] * g.g3rc[1]) * g.dx3q * 2.0 * betadx;
        s.ugkkn = 1.0 / (g.g3rm[n3m] * g.g3rc[n3]) * g.dx3q * 2.0 * betadx;
    }
    {   // solq3j (solve_fluid.F90:77-97)
        std::vector<double> am(n2m + 1, 0.0), ap(n2m + 1, 0.0), lo, di(n2m, 1.0), up;
        std::fill(b.begin(), b.end(), 0.0);
        for (int jc = 1; jc <= n2m; ++jc) {
            double acjl_b = 1.0 / (1.0 - betadx * g.ac3j[jc]);
            ap[jc] = -betadx * g.ap3j[jc] * acjl_b;
            am[jc] = -betadx * g.am3j[jc] * acjl_b;
            b[jc] = acjl_b;
        }
        for (int j = 2; j <= n2m; ++j) lo.push_back(am[j]);
        for (int j = 1; j <= n2m - 1; ++j) up.push_back(ap[j]);
        if ((st = upload_tri(c, s.y3, s.sy3, lo, di, up, &wy3))) return st;
        put(c, &s.by3, std::vector<double>(b.begin(), b.begin() + n2 + 2));
    }
    {   // solq3k (solve_fluid.F90:260-288)
        std::vector<double> am(n3 + 1, 0.0), ap(n3 + 1, 0.0), lo, di(n3, 1.0), up;
        std::fill(b.begin(), b.end(), 0.0);
        for (int kc = 2; kc <= n3m; ++kc) {
            double ackl_b = 1.0 / (1.0 - g.ac3sk[kc] * betadx);
            am[kc] = -g.am3sk[kc] * betadx * ackl_b;
            ap[kc] = -g.ap3sk[kc] * betadx * ackl_b;
            b[kc] = ackl_b;
        }
        for (int k = 2; k <= n3; ++k) lo.push_back(am[k]);
        for (int k = 1; k <= n3 - 1; ++k) up.push_back(ap[k]);
        if ((st = upload_tri(c, s.z3, s.sz3, lo, di, up, &wz3))) return st;
        put(c, &s.bz3, std::vector<double>(b.begin(), b.begin() + n3 + 2));
    }
    c->usdtal[n] = 1.0 / (c->dt * al);
    // the constants grouped launches read from the substep (the single-case
    // launches take them as arguments): RK3 coefficients, 1/(dt al)
    s.usdtal = c->usdtal[n];
    if (c->hc.deck.nsst == 3) {
        s.ga = c->hc.gam[n];
        s.ro = c->hc.rom[n];
    }
    s.scan_ok = !(s.y2.pivoted || s.z2.pivoted || s.y3.pivoted || s.z3.pivoted);
    s.win_y = std::max(wy2, wy3);
    s.win_z = std::max(wz2, wz3);
    if (!s.scan_ok || !c->allow_win || s.win_y > fb::kWinMax || s.win_z > fb::kWinMax) s.win_y = s.win_z = 0;
    s.win_tk = c->tune_tk;
    return FB_OK;
}

// (Re)builds the coefficients of every substep for the current dt and
// uploads them: allocated on the first call, then refreshed in place with one
// asynchronous copy on the context stream (ordered before the next kernels).
int build_substeps(fb_ctx *c) {
    c->coef_h.clear();
    c->coef_hi.clear();
    c->coef_fix.clear();
    c->coef_fixi.clear();
    const int nsst = c->hc.deck.nsst;
    int st;
    for (int n = 0; n < nsst; ++n) {
        const double al = (nsst == 3) ? c->hc.alm[n] : 1.0;
        if ((st = build_substep(c, n, al))) return st;
    }
    const size_t nd = c->coef_h.size(), ni = std::max<size_t>(c->coef_hi.size(), 1);
    if (!c->coef_d) {
        if ((st = dnew(c, &c->coef_d, nd))) return st;
        if ((st = dnew(c, &c->coef_di, ni))) return st;
        CK(cudaMallocHost(&c->coef_pin, nd * sizeof(double)));
        CK(cudaMallocHost(&c->coef_pini, ni * sizeof(int)));
        c->coef_cap = nd;
        c->coef_capi = ni;
    }
    if (nd != c->coef_cap || ni != c->coef_capi) return FB_ERR_STATE;  // sizes never change with dt
    for (auto &f : c->coef_fix) *f.first = c->coef_d + f.second;
    for (auto &f : c->coef_fixi) *f.first = c->coef_di + f.second;
    std::memcpy(c->coef_pin, c->coef_h.data(), nd * sizeof(double));
    if (!c->coef_hi.empty()) std::memcpy(c->coef_pini, c->coef_hi.data(), c->coef_hi.size() * sizeof(int));
    CK(cudaMemcpyAsync(c->coef_d, c->coef_pin, nd * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->coef_di, c->coef_pini, ni * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    return FB_OK;
}

// phcalc_outflow.F90:34-56: one y system per z mode, (A_y + wr(k) I) x = h.
// The reference divides each row by its diagonal before DGTTRF; the same
// solution is obtained here from the LU of the unscaled system, of which only
// the reciprocal pivots depend on the mode (multipliers are rebuilt on the
// device from amphj/apphj).  The Neumann null mode (wr = 0 up to round-off)
// is singular: the reference's answer there is fixed only up to an arbitrary
// constant, which updvp differentiates away and pr_submean removes, so its
// last unknown is pinned to zero instead of dividing by a round-off pivot.
int build_poisson(fb_ctx *c) {
    const fb::Grid &g = c->hc.grid;
    const int n2m = g.n2m, n3m = g.n3m, ldh = c->d.ldh;
    std::vector<double> pg(static_cast<size_t>(n3m) * ldh, 0.0);
    double wmax = 0.0;
    int k0 = 0;
    for (int m = 0; m < n3m; ++m) {
        wmax = std::max(wmax, std::fabs(c->hc.wr[static_cast<size_t>(m)]));
        if (std::fabs(c->hc.wr[static_cast<size_t>(m)]) < std::fabs(c->hc.wr[static_cast<size_t>(k0)])) k0 = m;
    }
    int nnull = 0;
    for (int m = 0; m < n3m; ++m)
        if (std::fabs(c->hc.wr[static_cast<size_t>(m)]) < 1e-9 * wmax) ++nnull;
    if (nnull != 1) return FB_ERR_NUMERIC;
    c->null_mode = k0;
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (int m = 0; m < n3m; ++m) {
        const double wrk = c->hc.wr[static_cast<size_t>(m)];
        double *gm = pg.data() + static_cast<size_t>(m) * ldh;
        double dprev = g.acphj[1] + wrk;
        gm[0] = 1.0 / dprev;
        for (int i = 1; i < n2m; ++i) {
            const double l = g.amphj[i + 1] / dprev;
            const double di = (g.acphj[i + 1] + wrk) - l * g.apphj[i];
            if (m == k0 && i == n2m - 1) {
                gm[i] = 0.0;  // gauge of the null mode
                break;
            }
            if (!(std::fabs(di) > 0.0) || !std::isfinite(di)) ++bad;
            gm[i] = 1.0 / di;
            dprev = di;
        }
    }
    if (bad) return FB_ERR_NUMERIC;
    double *p;
    int st;
    if ((st = dup(c, &p, pg))) return st;
    c->d.pg = p;
    return FB_OK;
}

int setup_i8(fb_ctx *c);

int create_impl(const char *dir, int device, fb_ctx *c) {
    std::string err = fb::setup_case(dir, c->hc);
    if (!err.empty()) {
        c->err = err;
        std::fprintf(stderr, "fribois2d: %s\n", err.c_str());
        return FB_ERR_INPUT;
    }
    const fb::Deck &dk = c->hc.deck;
    const fb::Grid &g = c->hc.grid;
    c->vardt = !dk.idtv;
    if (g.n3 > 4096 || g.n2 > 2080) {
        std::fprintf(stderr, "fribois2d: grid larger than the line solvers support (n3 <= 4096, n2 <= 2080)\n");
        return FB_ERR_UNSUPPORTED;
    }
    c->device = device;
    if (const char *hv = std::getenv("FRIBOIS2D_HELSOLVE")) c->allow_win = std::strcmp(hv, "scan") != 0;
    if (const char *tw = std::getenv("FRIBOIS2D_I8_TILE")) {   // fixed INT8 product tile width (32, 48 or 64)
        const int w = std::atoi(tw);
        if (w == 32 || w == 48 || w == 64) {
            c->tune_i8bn = w;
            c->i8_fixed = true;
        }
    }
    CK(cudaSetDevice(device));
    CK(fb::scan_configure());
    CK(fb::kernels_configure());
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    CB(cublasCreate(&c->blas));
    CB(cublasSetStream(c->blas, c->stream));
    CB(cublasSetPointerMode(c->blas, CUBLAS_POINTER_MODE_HOST));
    {   // a fixed workspace keeps cuBLAS from allocating inside graph capture
        void *ws = nullptr;
        CK(cudaMalloc(&ws, 32u << 20));
        c->allocs.push_back(ws);
        c->blas_ws = ws;
        CB(cublasSetWorkspace(c->blas, ws, 32u << 20));
    }

    Dev &d = c->d;
    d.n2 = g.n2;
    d.n3 = g.n3;
    d.n2m = g.n2m;
    d.n3m = g.n3m;
    d.P = round_up(g.n2, 32);
    d.NK = g.n3 + 1;
    d.ldh = round_up(g.n2m, 32);
    d.vardt = c->vardt ? 1 : 0;
    {   // getintvort (utils_proc.F90:605-609): the zz node nearest z = 18.5; the
        // line needs row indz + 1, so a domain without it has no vorticity line
        int best = 1;
        for (int k = 2; k <= g.n3; ++k)
            if (std::fabs(g.zz[k] - 18.5) < std::fabs(g.zz[best] - 18.5)) best = k;
        d.indz = (best < g.n3) ? best : 0;
    }
    d.nlm = dk.ibact ? dk.nlm : 0;
    d.nsst = dk.nsst;
    d.wfun = dk.wfun;
    d.dx2 = g.dx2;
    d.dx3 = g.dx3;
    d.dx2q = g.dx2q;
    d.dx3q = g.dx3q;
    d.ren = g.ren;
    d.visc = dk.visc;
    d.dt = dk.dt;
    d.cou = dk.cou;
    d.q3uw = dk.q3uw;
    d.q3lw = dk.q3lw;
    d.rext2 = dk.rext2;
    d.alx3 = dk.alx3;
    d.radiusSD = dk.radiusSD;
    d.kprobe = dk.kprobe;
    d.ddmin = g.ddmin;
    d.cfllim = dk.cfllim;
    {   // iobcs.F90:54-59: the outflow section area (constant)
        double area = 0.0;
        for (int j = 1; j <= g.n2m; ++j) area = area + g.g2rm[j] / g.dx2;
        d.area_out = area;
    }
    c->dt = dk.dt;
    c->dt_o = dk.dt;
    int st;
    double *p;
    int *ip;
#define UP1(name)                                           \
    if ((st = dup(c, &p, g.name))) return st;               \
    d.name = p;
#define UPI(name)                                           \
    if ((st = dup(c, &ip, g.name))) return st;              \
    d.name = ip;
    UP1(rc) UP1(rm) UP1(zz) UP1(zm) UP1(g2rc) UP1(g2rm) UP1(g3rc) UP1(g3rm)
    UP1(udx2c) UP1(udx2m) UP1(udx3c) UP1(udx3m)
    UPI(jmv) UPI(jpv) UPI(kmv) UPI(kpv)
    UP1(am2j) UP1(ac2j) UP1(ap2j) UP1(am3j) UP1(ac3j) UP1(ap3j)
    UP1(am3ck) UP1(ac3ck) UP1(ap3ck) UP1(am3sk) UP1(ac3sk) UP1(ap3sk)
    UP1(amphj) UP1(acphj) UP1(apphj) UP1(amphk) UP1(acphk) UP1(apphk)
#undef UP1
#undef UPI

    const size_t nf = static_cast<size_t>(d.NK) * d.P;
    double **fields[] = {&d.q2, &d.q3, &d.pr, &d.dph, &d.rhs2, &d.rhs3, &d.ru2, &d.ru3};
    for (double **f : fields)
        if ((st = dnew(c, f, nf))) return st;
    if ((st = dnew(c, &d.hmn, static_cast<size_t>(d.n3m) * d.ldh))) return st;
    if ((st = fb::encode_nl_maps(&c->nlmaps, d))) return st;
    {   // inqpr (initial_sol.F90:268-296): q2 = 0, q3 = velin = 1, pr = 0
        std::vector<double> one(nf, 0.0);
        for (int k = 0; k <= g.n3; ++k)
            for (int j = 1; j <= g.n2; ++j) one[fb::fidx(d, j, k)] = 1.0;
        if ((st = h2d(c, d.q3, one.data(), nf * sizeof(double)))) return st;
    }
    double **bnd[] = {&d.qb2s, &d.qb2n, &d.dqb2s, &d.dqb2n, &d.qb3s, &d.qb3n, &d.dqb3s, &d.dqb3n, &d.dq2x2o, &d.dq3x2o};
    for (double **b : bnd)
        if ((st = dnew(c, b, static_cast<size_t>(g.n2) + 2))) return st;
    {
        std::vector<double> v(static_cast<size_t>(g.n2) + 2, 0.0);
        for (int j = 1; j <= g.n2m; ++j) v[j] = 1.0;
        if ((st = h2d(c, d.qb3s, v.data(), v.size() * sizeof(double)))) return st;
        if ((st = h2d(c, d.qb3n, v.data(), v.size() * sizeof(double)))) return st;
    }
    const size_t nlm = static_cast<size_t>(std::max(d.nlm, 1));
    {   // the four marker arrays in one allocation, in this order, so that a
        // host's per-step marker exchange is one copy each way
        const size_t m = c->hc.lmcc.size();
        if (c->hc.lmvel.size() != m || c->hc.lmacc.size() != m || c->hc.lmnor.size() != m) return FB_ERR_STATE;
        double *mk = nullptr;
        if ((st = dnew(c, &mk, 4 * std::max<size_t>(m, 1)))) return st;
        d.lmcc = mk;
        d.lmvel = mk + m;
        d.lmacc = mk + 2 * m;
        d.lmnor = mk + 3 * m;
        if ((st = h2d(c, d.lmcc, c->hc.lmcc.data(), m * sizeof(double))) ||
            (st = h2d(c, d.lmvel, c->hc.lmvel.data(), m * sizeof(double))) ||
            (st = h2d(c, d.lmacc, c->hc.lmacc.data(), m * sizeof(double))) ||
            (st = h2d(c, d.lmnor, c->hc.lmnor.data(), m * sizeof(double))))
            return st;
    }
    if ((st = dup(c, &d.lmA, c->hc.lmA))) return st;
    if ((st = dup(c, &d.vert, c->hc.vert))) return st;
    if ((st = dnew(c, &d.lmind, nlm * 4))) return st;
    if ((st = dnew(c, &d.eulins, nlm * 2 * 2 * fb::kSD))) return st;
    if ((st = dnew(c, &d.phi, nlm * 2 * fb::kSD))) return st;
    if ((st = dnew(c, &d.cl, nlm * 2))) return st;
    if ((st = dnew(c, &d.contrib, nlm * 2 * fb::kSD))) return st;
    // spreading table: at least 8 entries per (marker, direction), a load of 1/8 at most
    d.hlog = 10;
    while ((static_cast<size_t>(1) << d.hlog) < 16 * nlm) ++d.hlog;
    if (d.nlm) {
        const size_t hcap = static_cast<size_t>(1) << d.hlog;
        if ((st = dnew(c, &d.hkey, hcap))) return st;
        if ((st = dnew(c, &d.hcnt, hcap))) return st;
        if ((st = dnew(c, &d.hval, hcap * fb::kBucket))) return st;
        if ((st = dnew(c, &d.hslot, nlm * 2))) return st;
        if ((st = dnew(c, &d.chain, nlm * 2 * fb::kSD))) return st;
        if ((st = dnew(c, &d.chead, nlm * 2 * fb::kSD))) return st;
        if ((st = dnew(c, &d.hlist, nlm * 2 * fb::kSD * fb::kHeadList))) return st;
        if ((st = dnew(c, &d.hlen, nlm * 2 * fb::kSD))) return st;
    }
    if ((st = dnew(c, &d.probe, nlm * 24))) return st;
    if ((st = dnew(c, &d.press, nlm))) return st;
    if ((st = dnew(c, &d.tau, nlm * 2))) return st;
    if ((st = dnew(c, &d.bcerrv, nlm))) return st;
    if ((st = dnew(c, &d.bcerrw, nlm))) return st;
    if ((st = dnew(c, &d.rigid, 18))) return st;
    if ((st = h2d(c, d.rigid, c->hc.rigid, 18 * sizeof(double)))) return st;
    if ((st = dnew(c, &d.forces, 8))) return st;
    if ((st = dnew(c, &d.scal, fb::S_SLOTS))) return st;
    c->hist_cap = 4096;
    if ((st = dnew(c, &d.hist, static_cast<size_t>(c->hist_cap) * FB_HIST_COLS))) return st;
    if ((st = dnew(c, &d.red, static_cast<size_t>(3) * fb::kRedSlot))) return st;
    if ((st = dnew(c, &d.count, 4))) return st;
    if ((st = dnew(c, &d.status, 1))) return st;
    const size_t gridblocks = static_cast<size_t>((d.n2m + 31) / 32) * ((d.n3m + 7) / 8);
    if (gridblocks > static_cast<size_t>(fb::kRedSlot)) return FB_ERR_UNSUPPORTED;
    d.rbden = dk.rbden;
    d.rba0 = dk.rba[0];
    d.rba1 = dk.rba[1];
    d.cmposi0 = dk.cmposi[0];
    d.cmposi1 = dk.cmposi[1];
    d.cmroti = dk.cmroti;
    d.rbgravF0 = dk.rbgravF[0];
    d.rbgravF1 = dk.rbgravF[1];
    d.rrr = dk.rrr;
    for (int i = 0; i < 3; ++i) {
        d.kk[i] = dk.kk[i];
        d.kk3[i] = dk.kk3[i];
        d.cc[i] = dk.cc[i];
        d.rbmcon[i] = dk.rbmcon[i];
    }
    for (int i = 0; i < 9; ++i) d.kinori[i] = c->hc.kinori[i];
    d.rtcoup = dk.rtcoup ? 1 : 0;

    if ((st = build_substeps(c))) return st;
    CK(cudaStreamSynchronize(c->stream));
    c->beta = c->dt / g.ren * 0.5;
    if ((st = build_poisson(c))) return st;
    if ((st = dup(c, &c->zmm, c->hc.zmm))) return st;
    if ((st = dup(c, &c->zmmt, c->hc.zmmt))) return st;
    // the default Poisson transforms: FP64-accurate products of this
    // library's INT8 tensor-core kernel (cuBLAS DGEMM stays selectable with
    // fb_set_poisson(FB_POISSON_FP64) as the comparison arm)
    if ((st = setup_i8(c))) return st;
    c->poisson_mode = FB_POISSON_INT8X8;
    CK(cudaDeviceSynchronize());
    return FB_OK;
}

}  // namespace

namespace {

// substep coefficients (fluid_tsch.F90:64-77)
void coefs(const fb_ctx *c, int ns, int n, double &al, double &ga, double &ro) {
    if (c->hc.deck.nsst == 3) {
        al = c->hc.alm[n - 1];
        ga = c->hc.gam[n - 1];
        ro = c->hc.rom[n - 1];
    } else {
        if (ns == 0) {
            ga = 1.0;
            ro = 0.0;
        } else {
            ga = 1.0 + 0.5 * c->dt / c->dt_o;
            ro = -0.5 * c->dt / c->dt_o;
        }
        al = ga + ro;
    }
}

// cuBLASLt form of product w (0 forward, 1 backward) with algorithm a
int gemm_lt(fb_ctx *c, int w, const cublasLtMatmulAlgo_t *a) {
    const Dev &d = c->d;
    const double one = 1.0, zero = 0.0;
    const double *A = w ? d.hmn : d.dph + d.P, *B = w ? c->zmm : c->zmmt;
    double *C = w ? d.dph + d.P : d.hmn;
    cublasLtMatrixLayout_t *l = c->lt_l + 3 * w;
    CB(cublasLtMatmul(c->lt, c->lt_op, &one, A, l[0], B, l[1], &zero, C, l[2], C, l[2], a, c->blas_ws, 32u << 20,
                      c->stream));
    return FB_OK;
}

int gemm_fwd(fb_ctx *c) {   // phcalc_outflow.F90:31, hmn = dph * zmmt^T
    if (c->lt_on[0]) return gemm_lt(c, 0, &c->lt_algo[0]);
    const Dev &d = c->d;
    const double one = 1.0, zero = 0.0;
    CB(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, d.n2m, d.n3m, d.n3m, &one, d.dph + d.P, d.P,
                   c->zmmt, d.n3m, &zero, d.hmn, d.ldh));
    return FB_OK;
}

int gemm_bwd(fb_ctx *c) {   // phcalc_outflow.F90:61,65-69, dph = vmn * zmm^T
    if (c->lt_on[1]) return gemm_lt(c, 1, &c->lt_algo[1]);
    const Dev &d = c->d;
    const double one = 1.0, zero = 0.0;
    CB(cublasDgemm(c->blas, CUBLAS_OP_N, CUBLAS_OP_T, d.n2m, d.n3m, d.n3m, &one, d.hmn, d.ldh, c->zmm,
                   d.n3m, &zero, d.dph + d.P, d.P));
    return FB_OK;
}

// mean device ms of `reps` calls of fn after one warm-up call (-1 on error)
template <class F>
double time_calls(fb_ctx *c, int reps, F fn) {
    if (fn()) return -1.0;
    if (cudaEventRecord(c->ev0, c->stream) != cudaSuccess) return -1.0;
    for (int i = 0; i < reps; ++i)
        if (fn()) return -1.0;
    float ms = 0.f;
    if (cudaEventRecord(c->ev1, c->stream) != cudaSuccess || cudaEventSynchronize(c->ev1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, c->ev0, c->ev1) != cudaSuccess)
        return -1.0;
    return static_cast<double>(ms) / reps;
}

// The FP64 transforms' algorithms: cuBLASLt's heuristic candidates for each
// product timed against cublasDgemm on the live buffers (hmn and dph are
// work arrays between steps; both are saved and restored all the same).
// The fastest is kept, so the products follow the reference's DGEMMs with
// a summation order that cuBLAS picks per shape.  The choice is cached per
// (n2, n3) for the process.
int tune_dgemm(fb_ctx *c) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, std::array<std::pair<bool, cublasLtMatmulAlgo_t>, 2>> cache;
    const Dev &d = c->d;
    const std::pair<int, int> key(d.n2, d.n3);
    if (!c->lt) {
        CB(cublasLtCreate(&c->lt));
        CB(cublasLtMatmulDescCreate(&c->lt_op, CUBLAS_COMPUTE_64F, CUDA_R_64F));
        const cublasOperation_t tn = CUBLAS_OP_N, tt = CUBLAS_OP_T;
        CB(cublasLtMatmulDescSetAttribute(c->lt_op, CUBLASLT_MATMUL_DESC_TRANSA, &tn, sizeof(tn)));
        CB(cublasLtMatmulDescSetAttribute(c->lt_op, CUBLASLT_MATMUL_DESC_TRANSB, &tt, sizeof(tt)));
        const uint64_t m = d.n2m, n = d.n3m;
        CB(cublasLtMatrixLayoutCreate(&c->lt_l[0], CUDA_R_64F, m, n, d.P));
        CB(cublasLtMatrixLayoutCreate(&c->lt_l[1], CUDA_R_64F, n, n, n));
        CB(cublasLtMatrixLayoutCreate(&c->lt_l[2], CUDA_R_64F, m, n, d.ldh));
        CB(cublasLtMatrixLayoutCreate(&c->lt_l[3], CUDA_R_64F, m, n, d.ldh));
        CB(cublasLtMatrixLayoutCreate(&c->lt_l[4], CUDA_R_64F, n, n, n));
        CB(cublasLtMatrixLayoutCreate(&c->lt_l[5], CUDA_R_64F, m, n, d.P));
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            for (int w = 0; w < 2; ++w) {
                c->lt_on[w] = it->second[static_cast<size_t>(w)].first;
                c->lt_algo[w] = it->second[static_cast<size_t>(w)].second;
            }
            return FB_OK;
        }
    }
    const size_t fbytes = static_cast<size_t>(d.NK) * d.P * sizeof(double);
    const size_t hbytes = static_cast<size_t>(d.n3m) * d.ldh * sizeof(double);
    char *save = nullptr;
    CK(cudaMalloc(&save, fbytes + hbytes));
    CK(cudaMemcpyAsync(save, d.dph, fbytes, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(save + fbytes, d.hmn, hbytes, cudaMemcpyDeviceToDevice, c->stream));
    cublasLtMatmulPreference_t pref = nullptr;
    int r = FB_OK;
    const uint64_t wsb = 32u << 20;
    if (cublasLtMatmulPreferenceCreate(&pref) != CUBLAS_STATUS_SUCCESS ||
        cublasLtMatmulPreferenceSetAttribute(pref, CUBLASLT_MATMUL_PREF_MAX_WORKSPACE_BYTES, &wsb, sizeof(wsb)) !=
            CUBLAS_STATUS_SUCCESS)
        r = FB_ERR_CUDA;
    for (int w = 0; w < 2 && !r; ++w) {
        c->lt_on[w] = false;
        const double base = time_calls(c, 5, [&] { return w ? gemm_bwd(c) : gemm_fwd(c); });
        if (base < 0.0) {
            r = FB_ERR_CUDA;
            break;
        }
        cublasLtMatmulHeuristicResult_t res[16];
        int cnt = 0;
        cublasLtMatrixLayout_t *l = c->lt_l + 3 * w;
        if (cublasLtMatmulAlgoGetHeuristic(c->lt, c->lt_op, l[0], l[1], l[2], l[2], pref, 16, res, &cnt) !=
            CUBLAS_STATUS_SUCCESS)
            cnt = 0;
        double best = 0.98 * base;   // a candidate must beat cublasDgemm clearly
        for (int i = 0; i < cnt; ++i) {
            if (res[i].state != CUBLAS_STATUS_SUCCESS || res[i].workspaceSize > wsb) continue;
            const double t = time_calls(c, 5, [&] { return gemm_lt(c, w, &res[i].algo); });
            if (t > 0.0 && t < best) {
                best = t;
                c->lt_algo[w] = res[i].algo;
                c->lt_on[w] = true;
            }
        }
        cudaGetLastError();
    }
    if (pref) cublasLtMatmulPreferenceDestroy(pref);
    cudaMemcpyAsync(d.dph, save, fbytes, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(d.hmn, save + fbytes, hbytes, cudaMemcpyDeviceToDevice, c->stream);
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    cudaFree(save);
    if (r) return r;
    if (e != cudaSuccess) return FB_ERR_CUDA;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = {std::make_pair(c->lt_on[0], c->lt_algo[0]), std::make_pair(c->lt_on[1], c->lt_algo[1])};
    return FB_OK;
}

// phcalc in the precision form: phi = Z T^-1 Z^-1 dph with 3xTF32 tensor-core
// transforms (TF32 high/low splits, FP32 accumulation) and FP64 tridiagonal
// solves, then one FP64 refinement sweep on the Poisson residual:
// r = dph - L phi, dph <- phi + Z T^-1 Z^-1 r.
int phcalc_tf32(fb_ctx *c) {
    const Dev &d = c->d;
    cudaStream_t st = c->stream;
    // phi_0 = Z T^-1 Z^-1 dph into pw
    fb::launch_split_t(d.dph + d.P, d.P, d.n2m, d.n3m, c->pl_a, st, c->zsinv_d);
    fb::launch_tf32x3(c->plan_fwd, d.hmn, d.ldh, nullptr, 0, d.status, st);
    fb::launch_scan_poisson(d, st);
    fb::launch_split_t(d.hmn, d.ldh, d.n2m, d.n3m, c->pl_a2, st);
    fb::launch_tf32x3(c->plan_bwd, c->pw + d.P, d.P, nullptr, 0, d.status, st, c->zs_d);
    // refinement sweeps: phi += Z T^-1 Z^-1 (dph - L phi); the last lands in dph
    for (int sw = 1; sw <= c->tf32_sweeps; ++sw) {
        const bool last = (sw == c->tf32_sweeps);
        fb::launch_poisson_residual(d, c->pw, c->pl_a, st, c->zsinv_d);
        fb::launch_tf32x3(c->plan_fwd, d.hmn, d.ldh, nullptr, 0, d.status, st);
        fb::launch_scan_poisson(d, st);
        fb::launch_split_t(d.hmn, d.ldh, d.n2m, d.n3m, c->pl_a2, st);
        fb::launch_tf32x3(c->plan_bwd, (last ? d.dph : c->pw) + d.P, d.P, c->pw + d.P, d.P, d.status, st, c->zs_d);
    }
    c->own_launches += 5 + 5 * c->tf32_sweeps;
    return FB_OK;
}

// allocates the precision-form buffers and splits the eigenvector matrices
int setup_tf32(fb_ctx *c) {
    if (c->pw) return FB_OK;
    const Dev &d = c->d;
    const long ld = round_up(d.n3m, 32);
    auto plane = [&](fb::SplitPlane &pl, int rows) -> int {
        int st;
        if ((st = dnew(c, &pl.hi, static_cast<size_t>(rows) * ld))) return st;
        if ((st = dnew(c, &pl.lo, static_cast<size_t>(rows) * ld))) return st;
        pl.ld = ld;
        return FB_OK;
    };
    int st;
    if ((st = fb::tf32x3_configure())) return st;
    if ((st = plane(c->pl_a, d.n2m)) || (st = plane(c->pl_a2, d.n2m)) || (st = plane(c->pl_zt, d.n3m)) ||
        (st = plane(c->pl_z, d.n3m)))
        return st;
    double *pw = nullptr;
    if ((st = dnew(c, &pw, static_cast<size_t>(d.NK) * d.P))) return st;
    // zmm = S U with U orthogonal: the tensor cores transform with U, which is
    // perfectly conditioned, and the diagonal S is applied in FP64 (to the
    // forward operand and to the backward output)
    const int n = d.n3m;
    const std::vector<double> &zs = c->hc.zs;
    std::vector<double> zinv(static_cast<size_t>(n)), urm(static_cast<size_t>(n) * n), ucm(urm.size());
    for (int r = 0; r < n; ++r) zinv[static_cast<size_t>(r)] = 1.0 / zs[static_cast<size_t>(r)];
    for (int col = 0; col < n; ++col)
        for (int r = 0; r < n; ++r) {
            const double u = c->hc.zmm[static_cast<size_t>(col) * n + r] / zs[static_cast<size_t>(r)];
            urm[static_cast<size_t>(r) * n + col] = u;
            ucm[static_cast<size_t>(col) * n + r] = u;
        }
    if ((st = dup(c, &c->zs_d, zs)) || (st = dup(c, &c->zsinv_d, zinv))) return st;
    double *tmp = nullptr;
    CK(cudaMalloc(&tmp, 2 * urm.size() * sizeof(double)));
    if ((st = h2d(c, tmp, urm.data(), urm.size() * sizeof(double))) ||
        (st = h2d(c, tmp + urm.size(), ucm.data(), ucm.size() * sizeof(double)))) {
        cudaFree(tmp);
        return st;
    }
    // B of the forward transform: U(k, m) as [m][k]; of the backward one: U(k, m) as [k][m]
    fb::launch_split_t(tmp, n, n, n, c->pl_zt, c->stream);
    fb::launch_split_t(tmp + urm.size(), n, n, n, c->pl_z, c->stream);
    const cudaError_t e1 = cudaGetLastError(), e2 = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return FB_ERR_CUDA;
    if ((st = fb::tf32x3_plan(c->plan_fwd, c->pl_a, c->pl_zt, d.n2m, d.n3m, d.n3m, c->tune_bn))) return st;
    if ((st = fb::tf32x3_plan(c->plan_bwd, c->pl_a2, c->pl_z, d.n2m, d.n3m, d.n3m, c->tune_bn))) return st;
    c->pw = pw;
    return FB_OK;
}

// allocates the INT8 digit planes and cuts the eigenvector matrices once
int setup_i8(fb_ctx *c) {
    if (c->i8_ready) return FB_OK;
    const Dev &d = c->d;
    int st;
    if ((st = fb::i8_configure())) return st;
    const long ldk = (d.n3m + fb::kI8BK - 1) / fb::kI8BK * fb::kI8BK;
    auto make = [&](fb::I8Plan &p, int rows, int box) -> int {
        p.ldk = ldk;
        p.rows_pad = (rows + 127) / 128 * 128;
        int r;
        if ((r = dnew(c, &p.dig, static_cast<size_t>(fb::kI8S) * p.rows_pad * ldk))) return r;
        if ((r = dnew(c, &p.scale, static_cast<size_t>(p.rows_pad)))) return r;
        return fb::i8_plan(p, rows, d.n3m, box);
    };
    if ((st = make(c->i8a, d.n2m, 128)) || (st = make(c->i8f, d.n3m, c->tune_i8bn)) ||
        (st = make(c->i8b, d.n3m, c->tune_i8bn)))
        return st;
    if ((st = dnew(c, &c->i8max, 2 * static_cast<size_t>(d.ldh)))) return st;   // zeroed
    // forward B(m, k) = zmmt(m, k); backward B(k, m) = zmm(k, m): both column-major
    fb::launch_i8_split(c->zmmt, d.n3m, d.n3m, d.n3m, c->i8f, c->stream);
    fb::launch_i8_split(c->zmm, d.n3m, d.n3m, d.n3m, c->i8b, c->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    c->i8_ready = true;
    return FB_OK;
}

// phcalc with the transforms on the INT8 tensor cores (phcalc_outflow.F90:31,
// 61-69): hmn = dph zmmt^T, per-mode y solves, dph = hmn zmm^T
int phcalc_i8(fb_ctx *c) {
    const Dev &d = c->d;
    cudaStream_t st = c->stream;
    // dph's row maxima come from divg, hmn's from the mode solves
    double *mx_dph = c->i8max, *mx_hmn = c->i8max + d.ldh;
    fb::launch_i8_cut_rows(d.dph + d.P, d.P, d.n2m, d.n3m, c->i8a, mx_dph, mx_hmn, st);
    fb::launch_i8x8(c->i8a, c->i8f, d.hmn, d.ldh, d.status, st, true);   // i8f, i8b: cut once at set-up
    fb::launch_scan_poisson(d, st, mx_hmn);
    fb::launch_i8_cut_rows(d.hmn, d.ldh, d.n2m, d.n3m, c->i8a, mx_hmn, mx_dph, st);
    fb::launch_i8x8(c->i8a, c->i8b, d.dph + d.P, d.P, d.status, st, true);
    c->own_launches += 5;   // two digit cuts, two products, the mode solves
    return FB_OK;
}

int stage_impl(fb_ctx *c, int stage, int ns, int n) {
    double al, ga, ro;
    coefs(c, ns, n, al, ga, ro);
    c->al = al;
    c->ga = ga;
    c->ro = ro;
    const Dev &d = c->d;
    const SubDev &s = c->sub[n - 1];
    cudaStream_t st = c->stream;
    int r = FB_OK;
    static const int kOwn[18] = {1, 1, 1, 0, 0, 0, 1, 2, 4, 1, 1, 1, 0, 1, 0, 2, 2, 1};
    if (stage >= 0 && stage < 18) c->own_launches += kOwn[stage] + ((stage == FB_ST_FORCING && n == 1) ? 2 : 0);
    switch (stage) {
    case FB_ST_CFL: fb::launch_cfl(d, st); break;
    case FB_ST_BOUCDQ: fb::launch_boucdq(d, ga, ro, st); break;
    case FB_ST_NL_RHS: fb::launch_nl_rhs(d, al, ga, ro, st, false, &c->nlmaps); break;
    case FB_ST_LGRDIST: fb::launch_lgrdist(d, st); break;
    case FB_ST_FORCING:
        if (!d.nlm) break;
        if (n == 1) {
            fb::launch_mls_setup(d, st);
            fb::launch_spread_chains(d, st);
        }
        fb::launch_mls_interp(d, st);
        fb::launch_mls_spread(d, st);
        break;
    case FB_ST_HELSOLVE:
        if (s.win_y > 0) {
            fb::launch_win_helsolve(d, s, st);
            c->own_launches -= 3;
        } else if (s.scan_ok) {
            fb::launch_scan_helsolve(d, s, st);
            c->own_launches -= 2;
        } else {
            fb::launch_helsolve(d, s, st);
        }
        break;
    case FB_ST_DIVG:   // with the INT8 transforms: dph's row maxima for their digit cut
        fb::launch_divg(d, c->usdtal[n - 1], st, c->poisson_mode == FB_POISSON_INT8X8 ? c->i8max : nullptr);
        break;
    case FB_ST_PHCALC:
        // kOwn counts the mode solves of the DGEMM form; the tensor-core forms
        // count all of their own launches themselves
        if (c->poisson_mode == FB_POISSON_TF32X3) {
            c->own_launches -= 1;
            if ((r = phcalc_tf32(c))) return r;
            break;
        }
        if (c->poisson_mode == FB_POISSON_INT8X8) {
            c->own_launches -= 1;
            if ((r = phcalc_i8(c))) return r;
            break;
        }
        if ((r = gemm_fwd(c))) return r;
        fb::launch_scan_poisson(d, st);
        if ((r = gemm_bwd(c))) return r;
        break;
    case FB_ST_UPDVP: fb::launch_updvp_prcalc(d, al, al * c->beta, st, false, &c->nlmaps); break;
    case FB_ST_PRSUBMEAN: fb::launch_submean_boucqt(d, st); break;
    case FB_ST_CHECKBCS:
    case FB_ST_LOADS: fb::launch_loads(d, st); break;
    case FB_ST_RIGID: fb::launch_rigid(d, c->hist_cap, st, fb::RIGID_STEP, nullptr, c->rigid_mbox); break;
    case FB_TK_GEMM_FWD: return gemm_fwd(c);
    case FB_TK_POISSON_TRI: fb::launch_scan_poisson(d, st); break;
    case FB_TK_GEMM_BWD: return gemm_bwd(c);
    case FB_TK_TF32X3_GEMM:
        if (!c->pw) return FB_ERR_STATE;
        fb::launch_tf32x3(c->plan_fwd, d.hmn, d.ldh, nullptr, 0, d.status, st);
        break;
    case FB_TK_I8_SPLIT:   // the step's form: dph's row maxima from the last divg (kept)
        if (!c->i8_ready) return FB_ERR_STATE;
        fb::launch_i8_cut_rows(d.dph + d.P, d.P, d.n2m, d.n3m, c->i8a, c->i8max, nullptr, st);
        break;
    case FB_TK_I8X8_GEMM:
        if (!c->i8_ready) return FB_ERR_STATE;
        fb::launch_i8x8(c->i8a, c->i8f, d.hmn, d.ldh, d.status, st, true);
        break;
    default: return FB_ERR_STATE;
    }
    if (cudaGetLastError() != cudaSuccess) return FB_ERR_CUDA;
    return FB_OK;
}

// fluid_tsch.F90:30-182 enqueued on the context stream (no host sync)
// variable dt (fluid_tsch.F90:34-48): the CFL number of the current field
// sets dt = cflmax / cflm (at most dtmax) from the second step on; the
// substep coefficients are rebuilt for it.  Runs cfl and waits for it.
int vardt_update(fb_ctx *c, int ns) {
    int r;
    if ((r = stage_impl(c, FB_ST_CFL, ns, 1))) return r;
    double am = 0.0;
    CK(cudaMemcpyAsync(&am, c->d.scal + fb::S_CFLRAW, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double dt = c->dt;
    if (ns > 0) {
        dt = c->hc.deck.cflmax / am;
        if (dt > c->hc.deck.dtmax) dt = c->hc.deck.dtmax;
    }
    if (!(dt >= 1.0e-8)) return FB_ERR_CFL;
    if (dt != c->dt) {
        c->dt = dt;
        c->d.dt = dt;
        if ((r = build_substeps(c))) return r;
    }
    return FB_OK;
}

int enqueue_fluid(fb_ctx *c, int ns) {
    const Dev &d = c->d;
    int r;
    if (c->vardt && (r = vardt_update(c, ns))) return r;
    // The marker set-up of substep 1 (lgrdistribution, MLS weights) reads
    // only marker data: it runs on a side branch while cfl, boucdq and the
    // explicit terms run on the main stream.
    if (d.nlm) {
        CK(cudaEventRecord(c->ev_fork, c->stream));
        CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
        c->own_launches += 3;
        fb::launch_lgrdist(d, c->side);
        fb::launch_mls_setup(d, c->side);
        fb::launch_spread_chains(d, c->side);
        CK(cudaGetLastError());
        CK(cudaEventRecord(c->ev_join, c->side));
    }
    if (!c->vardt && (r = stage_impl(c, FB_ST_CFL, ns, 1))) return r;
    c->beta = c->dt / c->hc.grid.ren * 0.5;
    // RK3: pr_submean of substeps 1 and 2 is deferred; nl_rhs and updvp of
    // the next substep subtract the mean as they read pr, and the mean is
    // kept for the entries updvp does not rewrite, which the last pr_submean
    // brings up to date.  boucqt and the next boucdq share one launch.
    const bool defer = (d.nsst == 3);
    for (int n = 1; n <= d.nsst; ++n) {
        const bool pend = defer && n > 1;
        double al, ga, ro;
        coefs(c, ns, n, al, ga, ro);
        if (!pend && (r = stage_impl(c, FB_ST_BOUCDQ, ns, n))) return r;
        if (pend) {
            fb::launch_nl_rhs(d, al, ga, ro, c->stream, true, &c->nlmaps);
            c->own_launches += 1;
        } else if ((r = stage_impl(c, FB_ST_NL_RHS, ns, n))) {
            return r;
        }
        if (d.nlm) {
            if (n == 1) CK(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
            // the weights are ready: interpolation and spreading only
            if ((r = stage_impl(c, FB_ST_FORCING, ns, n == 1 ? 2 : n))) return r;
        }
        if ((r = stage_impl(c, FB_ST_HELSOLVE, ns, n))) return r;
        if ((r = stage_impl(c, FB_ST_DIVG, ns, n))) return r;
        if ((r = stage_impl(c, FB_ST_PHCALC, ns, n))) return r;
        if (pend) {
            fb::launch_updvp_prcalc(d, al, al * c->beta, c->stream, true, &c->nlmaps);
            c->own_launches += 1;
        } else if ((r = stage_impl(c, FB_ST_UPDVP, ns, n))) {
            return r;
        }
        if (defer && n < d.nsst) {
            double al1, ga1, ro1;
            coefs(c, ns, n + 1, al1, ga1, ro1);
            fb::launch_substep_mid(d, n == 1 ? fb::S_PRAVG1 : fb::S_PRAVG2, ga1, ro1, c->stream);
            c->own_launches += 1;
        } else if (defer) {
            fb::launch_submean_boucqt(d, c->stream, true);
            c->own_launches += 1;
        } else if ((r = stage_impl(c, FB_ST_PRSUBMEAN, ns, n))) {
            return r;
        }
        CK(cudaGetLastError());
    }
    if (d.nlm && c->hc.deck.cbody && (r = stage_impl(c, FB_ST_LOADS, ns, 1))) return r;
    return FB_OK;
}

int enqueue_report(fb_ctx *c) {
    if (!c->report || !c->d.nlm) return FB_OK;
    fb::launch_diag(c->d, c->hist_cap, c->stream);
    c->own_launches += 1;
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

int enqueue_step(fb_ctx *c, int ns) {
    int r = enqueue_fluid(c, ns);
    if (r) return r;
    if (c->d.nlm) {
        if ((r = stage_impl(c, FB_ST_RIGID, ns, 1))) return r;
        return enqueue_report(c);
    }
    return FB_OK;
}

void drop_graph(fb_ctx *c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->fgraph_exec) cudaGraphExecDestroy(c->fgraph_exec);
    if (c->fgraph) cudaGraphDestroy(c->fgraph);
    c->graph_exec = nullptr;
    c->graph = nullptr;
    c->fgraph_exec = nullptr;
    c->fgraph = nullptr;
}

int read_status(fb_ctx *c, int *status) {
    CK(cudaMemcpyAsync(status, c->d.status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FB_OK;
}

// advances the host clock the way main.F90:92,96 does
void host_clock(fb_ctx *c, int nsteps) {
    for (int i = 0; i < nsteps; ++i) c->dt_o = c->dt;
}

int capture_coupled(fb_ctx *c);

int capture_step(fb_ctx *c) {
    if (c->graph_exec) return FB_OK;
    if (c->coupling != FB_COUPLING_LOOSE) return capture_coupled(c);
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    c->own_launches = 0;
    int r = enqueue_step(c, 1);
    c->step_kernels = c->own_launches;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (e != cudaSuccess) return FB_ERR_CUDA;
    c->graph = g;
    CK(cudaGraphInstantiate(&c->graph_exec, g, 0));
    return FB_OK;
}

// field (j, k) <-> host (k, j) dense copies
int field_ptr(fb_ctx *c, int id, double **p) {
    Dev &d = c->d;
    switch (id) {
    case FB_Q2: *p = d.q2; return FB_OK;
    case FB_Q3: *p = d.q3; return FB_OK;
    case FB_PR: *p = d.pr; return FB_OK;
    case FB_DPH: *p = d.dph; return FB_OK;
    case FB_RHS2: *p = d.rhs2; return FB_OK;
    case FB_RHS3: *p = d.rhs3; return FB_OK;
    case FB_RU2: *p = d.ru2; return FB_OK;
    case FB_RU3: *p = d.ru3; return FB_OK;
    }
    return FB_ERR_STATE;
}

// 1-based device vectors and plain marker arrays
int vec_ptr(fb_ctx *c, int id, double **p, int64_t *n, bool *one_based) {
    Dev &d = c->d;
    const int64_t n2 = d.n2, n3 = d.n3, nlm = d.nlm, n3m = d.n3m;
    *one_based = true;
    switch (id) {
    case FB_QB2S: *p = d.qb2s; *n = n2; return FB_OK;
    case FB_QB2N: *p = d.qb2n; *n = n2; return FB_OK;
    case FB_DQB2S: *p = d.dqb2s; *n = n2; return FB_OK;
    case FB_DQB2N: *p = d.dqb2n; *n = n2; return FB_OK;
    case FB_QB3S: *p = d.qb3s; *n = n2; return FB_OK;
    case FB_QB3N: *p = d.qb3n; *n = n2; return FB_OK;
    case FB_DQB3S: *p = d.dqb3s; *n = n2; return FB_OK;
    case FB_DQB3N: *p = d.dqb3n; *n = n2; return FB_OK;
    case FB_DQ2X2O: *p = d.dq2x2o; *n = n2; return FB_OK;
    case FB_DQ3X2O: *p = d.dq3x2o; *n = n2; return FB_OK;
    case FB_RC: *p = const_cast<double *>(d.rc); *n = n2; return FB_OK;
    case FB_RM: *p = const_cast<double *>(d.rm); *n = n2; return FB_OK;
    case FB_ZZ: *p = const_cast<double *>(d.zz); *n = n3; return FB_OK;
    case FB_ZM: *p = const_cast<double *>(d.zm); *n = n3; return FB_OK;
    case FB_UDX2C: *p = const_cast<double *>(d.udx2c); *n = n2; return FB_OK;
    case FB_UDX2M: *p = const_cast<double *>(d.udx2m); *n = n2; return FB_OK;
    case FB_UDX3C: *p = const_cast<double *>(d.udx3c); *n = n3; return FB_OK;
    case FB_UDX3M: *p = const_cast<double *>(d.udx3m); *n = n3; return FB_OK;
    case FB_AMPHJ: *p = const_cast<double *>(d.amphj); *n = n2; return FB_OK;
    case FB_ACPHJ: *p = const_cast<double *>(d.acphj); *n = n2; return FB_OK;
    case FB_APPHJ: *p = const_cast<double *>(d.apphj); *n = n2; return FB_OK;
    case FB_AMPHK: *p = const_cast<double *>(d.amphk); *n = n3; return FB_OK;
    case FB_ACPHK: *p = const_cast<double *>(d.acphk); *n = n3; return FB_OK;
    case FB_APPHK: *p = const_cast<double *>(d.apphk); *n = n3; return FB_OK;
    }
    *one_based = false;
    switch (id) {
    case FB_ZMM: *p = c->zmm; *n = n3m * n3m; return FB_OK;
    case FB_ZMMT: *p = c->zmmt; *n = n3m * n3m; return FB_OK;
    case FB_LMCC: *p = d.lmcc; *n = 2 * nlm; return FB_OK;
    case FB_LMVEL: *p = d.lmvel; *n = 2 * nlm; return FB_OK;
    case FB_LMACC: *p = d.lmacc; *n = 2 * nlm; return FB_OK;
    case FB_LMNOR: *p = d.lmnor; *n = 2 * nlm; return FB_OK;
    case FB_LMA: *p = d.lmA; *n = nlm; return FB_OK;
    case FB_VERT: *p = d.vert; *n = 2 * (nlm + 1); return FB_OK;
    case FB_PHI: *p = d.phi; *n = 18 * nlm; return FB_OK;
    case FB_CL: *p = d.cl; *n = 2 * nlm; return FB_OK;
    case FB_PRESS: *p = d.press; *n = nlm; return FB_OK;
    case FB_TAU: *p = d.tau; *n = 2 * nlm; return FB_OK;
    case FB_BCERRV: *p = d.bcerrv; *n = nlm; return FB_OK;
    case FB_BCERRW: *p = d.bcerrw; *n = nlm; return FB_OK;
    case FB_RIGID: *p = d.rigid; *n = 18; return FB_OK;
    case FB_FORCES: *p = d.forces; *n = 8; return FB_OK;
    case FB_HMN: *p = d.hmn; *n = n3m * d.ldh; return FB_OK;
    }
    return FB_ERR_STATE;
}

}  // namespace

// =================================================================== C ABI

extern "C" {

const char *fb_version(void) { return "fribois2d_b200 0.1 (sm_100a)"; }

const char *fb_status_string(int status) {
    switch (status) {
    case FB_OK: return "ok";
    case FB_ERR_CFL: return "CFL number above cfllim (fluid_tsch.F90:51-54)";
    case FB_ERR_MLS: return "MLS partition of unity violated (MLSint.F90:157-163)";
    case FB_ERR_MARKER_OUT: return "Lagrangian marker outside the grid (lgrdistribution.F90:217-221)";
    case FB_ERR_INPUT: return "malformed or missing input deck";
    case FB_ERR_CUDA: return "CUDA runtime or cuBLAS failure";
    case FB_ERR_STATE: return "invalid argument for this context";
    case FB_ERR_UNSUPPORTED: return "deck option not supported on the device path";
    case FB_ERR_NUMERIC: return "singular set-up system or non-finite value";
    case FB_ERR_TIMEOUT: return "a device-side wait gave up";
    }
    return "unknown status";
}

int fb_create(const char *input_dir, int device, fb_ctx **out) {
    if (!input_dir || !out) return FB_ERR_STATE;
    *out = nullptr;
    fb_ctx *c = new (std::nothrow) fb_ctx();
    if (!c) return FB_ERR_STATE;
    int r = create_impl(input_dir, device, c);
    if (r) {
        fb_destroy(c);
        return r;
    }
    *out = c;
    return FB_OK;
}

int fb_destroy(fb_ctx *c) {
    if (!c) return FB_OK;
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    for (void *p : c->allocs)
        if (p) cudaFree(p);
    if (c->coef_pin) cudaFreeHost(c->coef_pin);
    if (c->coef_pini) cudaFreeHost(c->coef_pini);
    if (c->stage_h) cudaFreeHost(c->stage_h);
    if (c->mbox_h) cudaFreeHost(c->mbox_h);
    if (c->stage_ev) cudaEventDestroy(c->stage_ev);
    if (c->blas) cublasDestroy(c->blas);
    for (cublasLtMatrixLayout_t l : c->lt_l)
        if (l) cublasLtMatrixLayoutDestroy(l);
    if (c->lt_op) cublasLtMatmulDescDestroy(c->lt_op);
    if (c->lt) cublasLtDestroy(c->lt);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return FB_OK;
}

// the mapped host words of k_publish (allocated once, outside any capture)
static int mbox_ready(fb_ctx *c) {
    if (c->mbox_h) return FB_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaHostAlloc(&c->mbox_h, 16 * sizeof(double), cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer(reinterpret_cast<void **>(&c->mbox_d), c->mbox_h, 0));
    return FB_OK;
}

static int mbox_status(const fb_ctx *c) {
    return static_cast<int>(static_cast<const volatile double *>(c->mbox_h)[0]);
}

int fb_fluid_tsch(fb_ctx *c, int ns) {
    if (!c) return FB_ERR_STATE;
    int r;
    if ((r = mbox_ready(c))) return r;
    if (!c->vardt && ns >= 1) {
        // fixed dt after the first step: the same launches every step,
        // replayed from a graph captured at the first such call (with the
        // status published at its end)
        if (!c->fgraph_exec) {
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            r = enqueue_fluid(c, ns);
            if (!r) {
                fb::launch_publish(c->d, false, c->mbox_d, c->stream);
                c->own_launches += 1;
            }
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (r || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                return r ? r : FB_ERR_CUDA;
            }
            c->fgraph = g;
            CK(cudaGraphInstantiate(&c->fgraph_exec, g, 0));
        }
        CK(cudaGraphLaunch(c->fgraph_exec, c->stream));
    } else {
        if ((r = enqueue_fluid(c, ns))) return r;
        fb::launch_publish(c->d, false, c->mbox_d, c->stream);
        c->own_launches += 1;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    return mbox_status(c);
}

int fb_rigid(fb_ctx *c, int ns, double *forcecomp) {
    if (!c) return FB_ERR_STATE;
    int r;
    if ((r = mbox_ready(c))) return r;
    if (!c->report || !c->d.nlm) {   // k_rigid publishes the status and the forcecomp row itself
        c->rigid_mbox = c->d.nlm ? c->mbox_d : nullptr;
        r = stage_impl(c, FB_ST_RIGID, ns, 1);
        c->rigid_mbox = nullptr;
        if (r) return r;
        if (!c->d.nlm) {   // no rigid launch without markers
            fb::launch_publish(c->d, true, c->mbox_d, c->stream);
            c->own_launches += 1;
        }
    } else {
        if ((r = stage_impl(c, FB_ST_RIGID, ns, 1))) return r;
        if ((r = enqueue_report(c))) return r;
        fb::launch_publish(c->d, true, c->mbox_d, c->stream);   // status and the forcecomp row
        c->own_launches += 1;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
    if (forcecomp) std::memcpy(forcecomp, c->mbox_h + 1, 8 * sizeof(double));
    host_clock(c, 1);
    return mbox_status(c);
}

int fb_last_history(fb_ctx *c, double *row);

}  // extern "C"

namespace {

// ---- strong fluid-structure coupling ----------------------------------------
// The reference couples explicitly: the fluid step sees the body where the
// previous rigid update left it.  Optionally each step iterates on the body
// load instead (couple.cu: device-side initial guess, restore, trial
// placement, fluid step, loads, Aitken update, accept), either as a CUDA
// graph WHILE node whose condition the update kernel sets -- no host
// synchronisation inside the step -- or, where such a graph cannot be
// built, as a host loop over the same kernels.

constexpr int kNoConditionalGraph = -1;

// the saved state (the fluid step's inputs that a trial step overwrites) and
// the device structures of the iteration
int couple_alloc(fb_ctx *c) {
    if (c->cpl) return FB_OK;
    Dev &d = c->d;
    const long nf = static_cast<long>(d.NK) * d.P, nb = static_cast<long>(d.n2) + 2;
    fb::SnapList &l = c->snapl;
    std::memset(static_cast<void *>(&l), 0, sizeof(l));
    auto add = [&](double *a, long n) {
        l.arr[l.n] = a;
        l.len[l.n] = n;
        ++l.n;
    };
    for (double *f : {d.q2, d.q3, d.pr, d.ru2, d.ru3}) add(f, nf);
    for (double *b : {d.qb2s, d.qb2n, d.dqb2s, d.dqb2n, d.qb3s, d.qb3n, d.dqb3s, d.dqb3n, d.dq2x2o, d.dq3x2o})
        add(b, nb);
    add(d.scal, fb::S_COUNT);
    l.nfield = l.n;
    const long nm = static_cast<long>(c->hc.lmcc.size());
    for (double *m : {d.lmcc, d.lmvel, d.lmacc, d.lmnor}) add(m, nm);
    add(d.vert, static_cast<long>(c->hc.vert.size()));
    add(d.rigid, 18);
    long total = 0;
    for (int i = 0; i < l.n; ++i) {
        total += l.len[i];
        c->snap_longest = std::max(c->snap_longest, l.len[i]);
    }
    int st;
    if ((st = dnew(c, &c->snap, static_cast<size_t>(total)))) return st;
    long off = 0;
    for (int i = 0; i < l.n; ++i) {
        l.copy[i] = c->snap + off;
        off += l.len[i];
    }
    if ((st = dnew(c, &c->smp_x, static_cast<size_t>(c->smp_cap) * fb::kCplIn)) ||
        (st = dnew(c, &c->smp_t, static_cast<size_t>(c->smp_cap) * fb::kCplOut)))
        return st;
    fb::Couple *cpl = nullptr;
    if ((st = dnew(c, &cpl, 1)) || (st = dnew(c, &c->cpl_list, 1)) || (st = dnew(c, &c->snapl_d, 1))) return st;
    l.c = cpl;
    if ((st = h2d(c, c->cpl_list, &cpl, sizeof(cpl))) || (st = h2d(c, c->snapl_d, &l, sizeof(l)))) return st;
    c->cpl = cpl;
    return FB_OK;
}

// reads the device iteration state, lets fn change it, writes it back
template <class F>
int couple_edit(fb_ctx *c, F fn) {
    fb::Couple h;
    CK(cudaMemcpyAsync(&h, c->cpl, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    fn(h);
    return h2d(c, c->cpl, &h, sizeof(h));
}

double *couple_fin(fb_ctx *c) {
    return reinterpret_cast<double *>(reinterpret_cast<char *>(c->cpl) + offsetof(fb::Couple, fin));
}

// the flag that gates a coupled case's grouped launches (null: loose case)
const int *couple_gate(const fb_ctx *c) {
    if (c->coupling == FB_COUPLING_LOOSE || !c->cpl) return nullptr;
    return reinterpret_cast<const int *>(reinterpret_cast<const char *>(c->cpl) + offsetof(fb::Couple, active));
}

// initial guess and the saved start state
int enqueue_couple_begin(fb_ctx *c) {
    fb::launch_couple_begin(c->cpl_list, 1, c->stream);
    fb::launch_snap(c->snapl_d, 1, fb::SNAP_SAVE, c->snap_longest, c->stream);
    c->own_launches += 2;
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// one fluid solve of the iteration (restore, trial placement, fluid step,
// loads at the trial position, update); set_cond: write the WHILE condition
int enqueue_couple_iter(fb_ctx *c, int ns, cudaGraphConditionalHandle h, int set_cond) {
    fb::launch_snap(c->snapl_d, 1, fb::SNAP_RESTORE_LOOP, c->snap_longest, c->stream);
    fb::launch_rigid(c->d, c->hist_cap, c->stream, fb::RIGID_PLACE, couple_fin(c));
    c->own_launches += 2;
    int r = enqueue_fluid(c, ns);
    if (r) return r;
    fb::launch_rigid(c->d, c->hist_cap, c->stream, fb::RIGID_FORCES, nullptr);
    fb::launch_couple_update(c->cpl_list, 1, h, set_cond, nullptr, c->stream);
    c->own_launches += 2;
    return cudaGetLastError() == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}

// accept: body back to the start of the step, commit with the fluid's load,
// record the step for the predictors
int enqueue_couple_end(fb_ctx *c) {
    fb::launch_snap(c->snapl_d, 1, fb::SNAP_RESTORE_BODY, c->snap_longest, c->stream);
    fb::launch_couple_accept(c->cpl_list, 1, c->stream);
    fb::launch_rigid(c->d, c->hist_cap, c->stream, fb::RIGID_COMMIT, couple_fin(c));
    fb::launch_couple_record(c->cpl_list, 1, c->stream);
    c->own_launches += 4;
    if (cudaGetLastError() != cudaSuccess) return FB_ERR_CUDA;
    return enqueue_report(c);
}

// the coupled step as one graph: begin -> WHILE(any iterating){iteration} -> end
int capture_coupled(fb_ctx *c) {
    cudaGraph_t G = nullptr, ga = nullptr, gb = nullptr, gd = nullptr;
    int r = FB_OK;
    auto cap = [&](cudaGraph_t *out, auto fn) -> int {
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FB_ERR_CUDA;
        const int rr = fn();
        const cudaError_t e = cudaStreamEndCapture(c->stream, out);
        return rr ? rr : (e == cudaSuccess ? FB_OK : FB_ERR_CUDA);
    };
    auto cleanup = [&] {
        for (cudaGraph_t g : {ga, gb, gd, G})
            if (g) cudaGraphDestroy(g);
    };
    cudaGraphConditionalHandle h{};
    if (cudaGraphCreate(&G, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&h, G, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return kNoConditionalGraph;
    }
    c->own_launches = 0;
    if ((r = cap(&ga, [&] { return enqueue_couple_begin(c); }))) {
        cleanup();
        return r;
    }
    const int k_begin = c->own_launches;
    if ((r = cap(&gb, [&] { return enqueue_couple_iter(c, 1, h, 1); }))) {
        cleanup();
        return r;
    }
    const int k_iter = c->own_launches - k_begin;
    if ((r = cap(&gd, [&] { return enqueue_couple_end(c); }))) {
        cleanup();
        return r;
    }
    c->step_kernels = c->own_launches;   // begin, one fluid solve, end
    c->iter_kernels = k_iter;
    cudaGraphNode_t na = nullptr, nc = nullptr, nb = nullptr, nd = nullptr;
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    bool ok = cudaGraphAddChildGraphNode(&na, G, nullptr, 0, ga) == cudaSuccess &&
              cudaGraphAddNode(&nc, G, &na, 1, &p) == cudaSuccess &&
              cudaGraphAddChildGraphNode(&nb, p.conditional.phGraph_out[0], nullptr, 0, gb) == cudaSuccess &&
              cudaGraphAddChildGraphNode(&nd, G, &nc, 1, gd) == cudaSuccess;
    if (ok) ok = cudaGraphInstantiate(&c->graph_exec, G, 0) == cudaSuccess;
    for (cudaGraph_t g : {ga, gb, gd}) cudaGraphDestroy(g);
    ga = gb = gd = nullptr;
    if (!ok) {
        cudaGetLastError();
        c->graph_exec = nullptr;
        cleanup();
        return kNoConditionalGraph;
    }
    c->graph = G;
    return FB_OK;
}

// the same step with the iteration driven from the host (one read of the
// device flag per fluid solve): the first Adams-Bashforth step, and devices
// where the conditional graph is not available
int coupled_step_host(fb_ctx *c, int ns) {
    int r;
    if ((r = enqueue_couple_begin(c))) return r;
    for (int it = 0; it < c->cmaxit; ++it) {
        if ((r = enqueue_couple_iter(c, ns, cudaGraphConditionalHandle{}, 0))) return r;
        int active = 0;
        CK(cudaMemcpyAsync(&active, reinterpret_cast<char *>(c->cpl) + offsetof(fb::Couple, active), sizeof(int),
                           cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (!active) break;
    }
    return enqueue_couple_end(c);
}

}  // namespace

extern "C" {

int fb_advance(fb_ctx *c, int ns0, int nsteps, double *hist) {
    if (!c || nsteps < 0) return FB_ERR_STATE;
    if (!c->d.nlm) return FB_ERR_UNSUPPORTED;
    int r, status = 0, done = 0;
    if (c->coupling != FB_COUPLING_LOOSE && c->cond_graph && !c->graph_exec) {
        r = capture_step(c);
        if (r == kNoConditionalGraph) c->cond_graph = false;
        else if (r) return r;
    }
    const bool host_loop = c->coupling != FB_COUPLING_LOOSE && !c->cond_graph;
    if (host_loop || (c->coupling != FB_COUPLING_LOOSE && c->hc.deck.nsst == 1 && ns0 == 0)) {
        // coupled steps driven from the host: all of them, or the first
        // Adams-Bashforth step (its own coefficients) before the graph
        c->last_ms = 0.0;
        for (; done < nsteps && (host_loop || done < 1); ++done) {
            CK(cudaEventRecord(c->ev0, c->stream));
            if ((r = coupled_step_host(c, ns0 + done))) return r;
            CK(cudaEventRecord(c->ev1, c->stream));
            if ((r = read_status(c, &status))) return r;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
            c->last_ms += ms;
            if (hist && (r = fb_last_history(c, hist + static_cast<size_t>(done) * FB_HIST_COLS))) return r;
            host_clock(c, 1);
            if (status) return status;
        }
        if (done == nsteps) return FB_OK;
    }
    if (c->vardt) {   // dt changes every step: eager launches, no captured graph
        c->last_ms = 0.0;
        for (; done < nsteps; ++done) {
            CK(cudaEventRecord(c->ev0, c->stream));
            if ((r = enqueue_step(c, ns0 + done))) return r;
            CK(cudaEventRecord(c->ev1, c->stream));
            if ((r = read_status(c, &status))) return r;
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
            c->last_ms += ms;
            if (hist && (r = fb_last_history(c, hist + static_cast<size_t>(done) * FB_HIST_COLS))) return r;
            host_clock(c, 1);
            if (status) return status;
        }
        return FB_OK;
    }
    // the first Adams-Bashforth step has its own coefficients: run it eagerly
    if (c->coupling == FB_COUPLING_LOOSE && c->hc.deck.nsst == 1 && ns0 == 0 && nsteps > 0) {
        CK(cudaEventRecord(c->ev0, c->stream));
        if ((r = enqueue_step(c, 0))) return r;
        CK(cudaEventRecord(c->ev1, c->stream));
        if ((r = read_status(c, &status))) return r;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        c->last_ms = ms;
        if (hist) {
            double row0;
            CK(cudaMemcpy(&row0, c->d.scal + fb::S_STEP, sizeof(double), cudaMemcpyDeviceToHost));
            int row = (static_cast<int>(row0) - 1 + c->hist_cap) % c->hist_cap;
            CK(cudaMemcpy(hist, c->d.hist + static_cast<size_t>(row) * FB_HIST_COLS, FB_HIST_COLS * sizeof(double),
                          cudaMemcpyDeviceToHost));
        }
        host_clock(c, 1);
        if (status) return status;
        done = 1;
    } else if (done == 0) {
        c->last_ms = 0.0;
    }
    if ((r = capture_step(c))) return r;
    while (done < nsteps) {
        const int chunk = std::min(nsteps - done, c->hist_cap);
        double row0;
        CK(cudaMemcpyAsync(&row0, c->d.scal + fb::S_STEP, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaEventRecord(c->ev0, c->stream));
        for (int i = 0; i < chunk; ++i) CK(cudaGraphLaunch(c->graph_exec, c->stream));
        CK(cudaEventRecord(c->ev1, c->stream));
        if ((r = read_status(c, &status))) return r;
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
        c->last_ms += ms;
        if (hist) {
            for (int i = 0; i < chunk; ++i) {
                int row = (static_cast<int>(row0) + i) % c->hist_cap;
                CK(cudaMemcpy(hist + static_cast<size_t>(done + i) * FB_HIST_COLS,
                              c->d.hist + static_cast<size_t>(row) * FB_HIST_COLS, FB_HIST_COLS * sizeof(double),
                              cudaMemcpyDeviceToHost));
            }
        }
        host_clock(c, chunk);
        done += chunk;
        if (status) return status;
    }
    return FB_OK;
}

int fb_last_history(fb_ctx *c, double *row) {
    if (!c || !row || !c->d.nlm) return FB_ERR_STATE;
    double step = 0.0;
    CK(cudaMemcpyAsync(&step, c->d.scal + fb::S_STEP, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (step < 1.0) return FB_ERR_STATE;
    const int r = (static_cast<int>(step) - 1) % c->hist_cap;
    CK(cudaMemcpy(row, c->d.hist + static_cast<size_t>(r) * FB_HIST_COLS, FB_HIST_COLS * sizeof(double),
                  cudaMemcpyDeviceToHost));
    return FB_OK;
}

// ---- checkpoint / restart: raw little-endian FP64 files in place of the
// reference's HDF5 restart set (mpi_routines.F90:532-806 rest_*.h5,
// iobcs.F90:114-205 outflow.h5 / inflow.h5) and its text master_rigid.dat
// (ttime.F90:117-124).  Each .bin file holds a 32-byte header (magic, format
// version, n2, n3, nlm, count) followed by `count` doubles.
namespace {

struct RestartHeader {
    char magic[8];
    int32_t version, n2, n3, nlm;
    int64_t count;
};

int write_blob(fb_ctx *c, const std::string &path, const std::vector<double> &v) {
    RestartHeader h{};
    std::memcpy(h.magic, "FBRST01", 8);
    h.version = 1;
    h.n2 = c->d.n2;
    h.n3 = c->d.n3;
    h.nlm = c->d.nlm;
    h.count = static_cast<int64_t>(v.size());
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return FB_ERR_INPUT;
    const bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
                    std::fwrite(v.data(), sizeof(double), v.size(), f) == v.size();
    return (std::fclose(f) == 0 && ok) ? FB_OK : FB_ERR_INPUT;
}

int read_blob(fb_ctx *c, const std::string &path, std::vector<double> &v) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return FB_ERR_INPUT;
    RestartHeader h{};
    bool ok = std::fread(&h, sizeof(h), 1, f) == 1 && std::memcmp(h.magic, "FBRST01", 8) == 0 && h.version == 1 &&
              h.n2 == c->d.n2 && h.n3 == c->d.n3 && h.nlm == c->d.nlm && h.count >= 0 && h.count < (1LL << 34);
    if (ok) {
        v.resize(static_cast<size_t>(h.count));
        ok = std::fread(v.data(), sizeof(double), v.size(), f) == v.size();
    }
    std::fclose(f);
    return ok ? FB_OK : FB_ERR_INPUT;
}

// arrays of one restart file, in order
struct RestartFile {
    const char *name;
    std::vector<int> ids;
};

const std::vector<RestartFile> &restart_files() {
    static const std::vector<RestartFile> files = {
        {"rest_q2.bin", {FB_Q2}},
        {"rest_q3.bin", {FB_Q3}},
        {"rest_pr.bin", {FB_PR}},
        {"rest_ru2.bin", {FB_RU2}},
        {"rest_ru3.bin", {FB_RU3}},
        {"outflow.bin", {FB_QB2N, FB_QB3N, FB_DQ2X2O, FB_DQ3X2O}},
        {"inflow.bin", {FB_QB2S, FB_QB3S}},
        // state the reference rebuilds on restart, kept so that a restarted run
        // continues bit for bit: boundary increments and the marker set
        {"device_state.bin", {FB_DQB2S, FB_DQB2N, FB_DQB3S, FB_DQB3N, FB_LMCC, FB_LMVEL, FB_LMACC, FB_LMNOR,
                              FB_VERT, FB_RIGID, FB_FORCES}},
    };
    return files;
}

int64_t array_len(fb_ctx *c, int id) {
    double *p = nullptr;
    if (field_ptr(c, id, &p) == FB_OK) return static_cast<int64_t>(c->d.NK) * c->d.n2;
    int64_t n = 0;
    bool ob = false;
    return vec_ptr(c, id, &p, &n, &ob) == FB_OK ? n : -1;
}

}  // namespace

int fb_write_restart(fb_ctx *c, const char *dir) {
    if (!c || !dir) return FB_ERR_STATE;
    const std::string root(dir);
    int r;
    for (const RestartFile &rf : restart_files()) {
        std::vector<double> blob;
        for (int id : rf.ids) {
            const int64_t n = array_len(c, id);
            if (n < 0) return FB_ERR_STATE;
            std::vector<double> v(static_cast<size_t>(n));
            if ((r = fb_get_array(c, id, v.data(), n))) return r;
            blob.insert(blob.end(), v.begin(), v.end());
        }
        if ((r = write_blob(c, root + "/" + rf.name, blob))) return r;
    }
    {   // device scalars (clock, step counter, running sums) and host scalars
        std::vector<double> sc(fb::S_COUNT + 2);
        CK(cudaMemcpyAsync(sc.data(), c->d.scal, fb::S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        sc[fb::S_COUNT] = c->dt;
        sc[fb::S_COUNT + 1] = c->dt_o;
        if ((r = write_blob(c, root + "/scalars.bin", sc))) return r;
        std::vector<double> rg(18);
        if ((r = fb_get_array(c, FB_RIGID, rg.data(), 18))) return r;
        std::FILE *f = std::fopen((root + "/master_rigid.dat").c_str(), "w");
        if (!f) return FB_ERR_INPUT;
        // list-directed layout: time / dt, dt_o / cmp_np1 / cmv_np1 / cma_np1
        std::fprintf(f, " %25.17E\n %25.17E %25.17E\n", sc[fb::S_TIME], c->dt, c->dt_o);
        for (int q = 0; q < 3; ++q)
            std::fprintf(f, " %25.17E %25.17E %25.17E\n", rg[9 + 3 * q], rg[10 + 3 * q], rg[11 + 3 * q]);
        if (std::fclose(f) != 0) return FB_ERR_INPUT;
    }
    return FB_OK;
}

int fb_read_restart(fb_ctx *c, const char *dir) {
    if (!c || !dir) return FB_ERR_STATE;
    const std::string root(dir);
    int r;
    for (const RestartFile &rf : restart_files()) {
        std::vector<double> blob;
        if ((r = read_blob(c, root + "/" + rf.name, blob))) return r;
        size_t off = 0;
        for (int id : rf.ids) {
            const int64_t n = array_len(c, id);
            if (n < 0 || off + static_cast<size_t>(n) > blob.size()) return FB_ERR_INPUT;
            if ((r = fb_set_array(c, id, blob.data() + off, n))) return r;
            off += static_cast<size_t>(n);
        }
        if (off != blob.size()) return FB_ERR_INPUT;
    }
    std::vector<double> sc;
    if ((r = read_blob(c, root + "/scalars.bin", sc))) return r;
    if (sc.size() != static_cast<size_t>(fb::S_COUNT + 2)) return FB_ERR_INPUT;
    CK(cudaMemcpyAsync(c->d.scal, sc.data(), fb::S_COUNT * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (sc[fb::S_COUNT] != c->dt) return FB_ERR_INPUT;  // the deck's dt must match the checkpoint's
    c->dt_o = sc[fb::S_COUNT + 1];
    return FB_OK;
}

int fb_get_loads(fb_ctx *c, double *press, double *tau) {
    if (!c) return FB_ERR_STATE;
    const size_t nlm = static_cast<size_t>(c->d.nlm);
    if (press) CK(cudaMemcpyAsync(press, c->d.press, nlm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (tau) CK(cudaMemcpyAsync(tau, c->d.tau, 2 * nlm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FB_OK;
}

// The arrays are copied into pinned staging memory before the call returns
// (the caller may reuse its buffers at once); the host-to-device copies are
// ordered on the context stream ahead of the next step, without a wait here.
int fb_set_markers(fb_ctx *c, const double *lmcc, const double *lmvel, const double *lmacc, const double *lmnor) {
    if (!c) return FB_ERR_STATE;
    const size_t n = 2 * static_cast<size_t>(c->d.nlm), b = n * sizeof(double);
    if (!n) return FB_OK;
    CK(cudaSetDevice(c->device));
    if (!c->stage_h) {
        CK(cudaMallocHost(&c->stage_h, 4 * b));
        CK(cudaEventCreateWithFlags(&c->stage_ev, cudaEventDisableTiming));
    } else {
        CK(cudaEventSynchronize(c->stage_ev));   // the previous call's copies have left the staging
    }
    const double *src[4] = {lmcc, lmvel, lmacc, lmnor};
    double *dst[4] = {c->d.lmcc, c->d.lmvel, c->d.lmacc, c->d.lmnor};
    const bool all = lmcc && lmvel && lmacc && lmnor;   // the device arrays are contiguous: one copy
    for (int i = 0; i < 4; ++i) {
        if (!src[i]) continue;
        std::memcpy(c->stage_h + i * n, src[i], b);
        if (!all) CK(cudaMemcpyAsync(dst[i], c->stage_h + i * n, b, cudaMemcpyHostToDevice, c->stream));
    }
    if (all) CK(cudaMemcpyAsync(c->d.lmcc, c->stage_h, 4 * b, cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->stage_ev, c->stream));
    return FB_OK;
}

int fb_get_markers(fb_ctx *c, double *lmcc, double *lmvel, double *lmacc, double *lmnor) {
    if (!c) return FB_ERR_STATE;
    const size_t n = 2 * static_cast<size_t>(c->d.nlm), b = n * sizeof(double);
    if (!b) return FB_OK;
    CK(cudaSetDevice(c->device));
    double *dst[4] = {lmcc, lmvel, lmacc, lmnor};
    if (!c->stage_h) {
        CK(cudaMallocHost(&c->stage_h, 4 * b));
        CK(cudaEventCreateWithFlags(&c->stage_ev, cudaEventDisableTiming));
        CK(cudaEventRecord(c->stage_ev, c->stream));
    }
    // the contiguous device arrays in one copy through the pinned staging,
    // once fb_set_markers' copies out of it are done (stream order)
    CK(cudaMemcpyAsync(c->stage_h, c->d.lmcc, 4 * b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < 4; ++i)
        if (dst[i]) std::memcpy(dst[i], c->stage_h + i * n, b);
    return FB_OK;
}

int fb_step_markers(fb_ctx *c, int ns, double *lmcc, double *lmvel, double *lmacc, double *lmnor,
                    double *forcecomp) {
    if (!c) return FB_ERR_STATE;
    int r;
    if ((r = mbox_ready(c))) return r;
    if ((r = fb_set_markers(c, lmcc, lmvel, lmacc, lmnor))) return r;
    if (!c->vardt && ns >= 1 && c->fgraph_exec) {
        CK(cudaGraphLaunch(c->fgraph_exec, c->stream));   // the fluid step (status into the mapped words)
    } else {
        // the first fixed-dt step captures the graph, a variable dt needs the host: as fb_fluid_tsch
        const int st = fb_fluid_tsch(c, ns);
        if (st) return st;
    }
    // the rigid update publishes the (sticky) status and the forcecomp row itself
    c->rigid_mbox = c->d.nlm ? c->mbox_d : nullptr;
    r = stage_impl(c, FB_ST_RIGID, ns, 1);
    c->rigid_mbox = nullptr;
    if (r) return r;
    if (!c->d.nlm || c->report) {
        if ((r = enqueue_report(c))) return r;
        fb::launch_publish(c->d, true, c->mbox_d, c->stream);
        c->own_launches += 1;
    }
    const size_t n = 2 * static_cast<size_t>(c->d.nlm), b = n * sizeof(double);
    if (b) CK(cudaMemcpyAsync(c->stage_h, c->d.lmcc, 4 * b, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));   // the one wait
    double *dst[4] = {lmcc, lmvel, lmacc, lmnor};
    for (int i = 0; b && i < 4; ++i)
        if (dst[i]) std::memcpy(dst[i], c->stage_h + i * n, b);
    if (forcecomp) std::memcpy(forcecomp, c->mbox_h + 1, 8 * sizeof(double));
    host_clock(c, 1);
    return mbox_status(c);
}

int fb_get_dims(fb_ctx *c, int32_t dims[8]) {
    if (!c || !dims) return FB_ERR_STATE;
    dims[0] = c->d.n2;
    dims[1] = c->d.n3;
    dims[2] = c->d.nlm;
    dims[3] = c->d.nsst;
    dims[4] = c->d.P;
    dims[5] = c->d.ldh;
    dims[6] = c->sub[0].y2.pivoted | (c->sub[0].z3.pivoted << 1);
    dims[7] = c->sub[0].win_y | (c->sub[0].win_z << 8);  // windowed helsolve (0: line scans)
    return FB_OK;
}

int fb_get_array(fb_ctx *c, int id, double *host, int64_t n) {
    if (!c || !host) return FB_ERR_STATE;
    Dev &d = c->d;
    double *p = nullptr;
    // every copy below is ordered on the context stream after the work that
    // writes the array, and waited for before returning
    if (field_ptr(c, id, &p) == FB_OK) {
        if (n != static_cast<int64_t>(d.NK) * d.n2) return FB_ERR_STATE;
        CK(cudaMemcpy2DAsync(host, d.n2 * sizeof(double), p, d.P * sizeof(double), d.n2 * sizeof(double), d.NK,
                             cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return FB_OK;
    }
    if (id == FB_SCALARS) {
        if (n != 13) return FB_ERR_STATE;
        double s[fb::S_COUNT];
        CK(cudaMemcpyAsync(s, d.scal, sizeof(s), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        const double v[13] = {s[fb::S_TIME], c->dt, c->dt_o, c->beta, c->al, c->ga, c->ro, s[fb::S_CFLM],
                              s[fb::S_Q3AVG], s[fb::S_NBCV], s[fb::S_NBCW], d.ddmin, s[fb::S_PRAVG]};
        std::memcpy(host, v, sizeof(v));
        return FB_OK;
    }
    if (id == FB_WR) {
        if (n != d.n3m) return FB_ERR_STATE;
        std::memcpy(host, c->hc.wr.data(), static_cast<size_t>(n) * sizeof(double));
        return FB_OK;
    }
    int64_t cnt = 0;
    bool one_based = false;
    if (vec_ptr(c, id, &p, &cnt, &one_based) != FB_OK || n != cnt) return FB_ERR_STATE;
    CK(cudaMemcpyAsync(host, p + (one_based ? 1 : 0), static_cast<size_t>(n) * sizeof(double),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FB_OK;
}

int fb_set_array(fb_ctx *c, int id, const double *host, int64_t n) {
    if (!c || !host) return FB_ERR_STATE;
    Dev &d = c->d;
    double *p = nullptr;
    CK(cudaStreamSynchronize(c->stream));
    if (field_ptr(c, id, &p) == FB_OK) {
        if (n != static_cast<int64_t>(d.NK) * d.n2) return FB_ERR_STATE;
        CK(cudaMemcpy2DAsync(p, d.P * sizeof(double), host, d.n2 * sizeof(double), d.n2 * sizeof(double), d.NK,
                             cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return FB_OK;
    }
    if (id == FB_WR || id == FB_ZMM || id == FB_ZMMT) return FB_ERR_STATE;  // set-up data is immutable
    int64_t cnt = 0;
    bool one_based = false;
    if (vec_ptr(c, id, &p, &cnt, &one_based) != FB_OK || n != cnt) return FB_ERR_STATE;
    if (one_based && id >= FB_RC) return FB_ERR_STATE;  // grid data is immutable
    CK(cudaMemcpyAsync(p + (one_based ? 1 : 0), host, static_cast<size_t>(n) * sizeof(double),
                       cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FB_OK;
}

int fb_get_iarray(fb_ctx *c, int id, int32_t *host, int64_t n) {
    if (!c || !host) return FB_ERR_STATE;
    CK(cudaStreamSynchronize(c->stream));
    const int64_t nlm = c->d.nlm;
    if (id == FB_LMIND && n == 4 * nlm) {
        CK(cudaMemcpyAsync(host, c->d.lmind, static_cast<size_t>(n) * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return FB_OK;
    }
    if (id == FB_EULINS && n == 36 * nlm) {
        CK(cudaMemcpyAsync(host, c->d.eulins, static_cast<size_t>(n) * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return FB_OK;
    }
    return FB_ERR_STATE;
}

int fb_synchronize(fb_ctx *c) {
    if (!c) return FB_ERR_STATE;
    int status = 0;
    int r = read_status(c, &status);
    return r ? r : status;
}

int fb_set_substep(fb_ctx *c, int ns, int n) {
    if (!c || n < 1 || n > c->d.nsst) return FB_ERR_STATE;
    c->cur_ns = ns;
    c->cur_n = n;
    double al, ga, ro;
    coefs(c, ns, n, al, ga, ro);
    c->al = al;
    c->ga = ga;
    c->ro = ro;
    c->beta = c->dt / c->hc.grid.ren * 0.5;
    return FB_OK;
}

int fb_stage(fb_ctx *c, int stage, int n) {
    if (!c || n < 1 || n > c->d.nsst) return FB_ERR_STATE;
    int r = stage_impl(c, stage, c->cur_ns, n);
    if (r) return r;
    int status = 0;
    if ((r = read_status(c, &status))) return r;
    return status;
}

int fb_time_stage(fb_ctx *c, int stage, int n, int reps, double *ms) {
    if (!c || !ms || reps < 1 || n < 1 || n > c->d.nsst) return FB_ERR_STATE;
    // reps launches captured into one graph, so that host launch cost does
    // not enter the device time of short kernels
    int r = stage_impl(c, stage, c->cur_ns, n);
    if (r) return r;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < reps && !r; ++i) r = stage_impl(c, stage, c->cur_ns, n);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    if (r || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return r ? r : FB_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&ge, g, 0);
    if (e == cudaSuccess) e = cudaGraphLaunch(ge, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev0, c->stream);
    if (e == cudaSuccess) e = cudaGraphLaunch(ge, c->stream);
    if (e == cudaSuccess) e = cudaEventRecord(c->ev1, c->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(c->ev1);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, c->ev0, c->ev1);
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return FB_ERR_CUDA;
    *ms = static_cast<double>(t) / reps;
    CK(cudaMemsetAsync(c->d.status, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return FB_OK;
}

int fb_kernel_count(fb_ctx *c, int32_t *per_step) {
    if (!c || !per_step) return FB_ERR_STATE;
    int r = capture_step(c);
    if (r) return r;
    *per_step = c->step_kernels;
    return FB_OK;
}

int fb_last_advance_ms(fb_ctx *c, double *ms) {
    if (!c || !ms) return FB_ERR_STATE;
    *ms = c->last_ms;
    return FB_OK;
}

// ---- host-only set-up -------------------------------------------------------

int fb_host_create(const char *input_dir, fb_host **out) {
    if (!input_dir || !out) return FB_ERR_STATE;
    fb_host *h = new (std::nothrow) fb_host();
    if (!h) return FB_ERR_STATE;
    std::string err = fb::setup_case(input_dir, h->hc);
    if (!err.empty()) {
        std::fprintf(stderr, "fribois2d: %s\n", err.c_str());
        delete h;
        *out = nullptr;
        return FB_ERR_INPUT;
    }
    *out = h;
    return FB_OK;
}

int fb_host_destroy(fb_host *h) {
    delete h;
    return FB_OK;
}

int fb_host_dims(fb_host *h, int32_t dims[8]) {
    if (!h || !dims) return FB_ERR_STATE;
    const fb::HostCase &hc = h->hc;
    dims[0] = hc.grid.n2;
    dims[1] = hc.grid.n3;
    dims[2] = hc.deck.nlm;
    dims[3] = hc.deck.nsst;
    dims[4] = hc.deck.idtv ? 1 : 0;
    dims[5] = hc.deck.ibact ? 1 : 0;
    dims[6] = hc.deck.wfun;
    dims[7] = hc.deck.forst;
    return FB_OK;
}

int fb_host_array(fb_host *h, int id, double *out, int64_t n) {
    if (!h || !out) return FB_ERR_STATE;
    const fb::HostCase &hc = h->hc;
    const fb::Grid &g = hc.grid;
    const std::vector<double> *v = nullptr;
    bool one_based = true;
    switch (id) {
    case FB_RC: v = &g.rc; break;
    case FB_RM: v = &g.rm; break;
    case FB_ZZ: v = &g.zz; break;
    case FB_ZM: v = &g.zm; break;
    case FB_UDX2C: v = &g.udx2c; break;
    case FB_UDX2M: v = &g.udx2m; break;
    case FB_UDX3C: v = &g.udx3c; break;
    case FB_UDX3M: v = &g.udx3m; break;
    case FB_AMPHJ: v = &g.amphj; break;
    case FB_ACPHJ: v = &g.acphj; break;
    case FB_APPHJ: v = &g.apphj; break;
    case FB_AMPHK: v = &g.amphk; break;
    case FB_ACPHK: v = &g.acphk; break;
    case FB_APPHK: v = &g.apphk; break;
    default: one_based = false;
    }
    if (one_based) {
        const int64_t cnt = static_cast<int64_t>(v->size()) - 2;
        if (n != cnt) return FB_ERR_STATE;
        std::memcpy(out, v->data() + 1, static_cast<size_t>(n) * sizeof(double));
        return FB_OK;
    }
    switch (id) {
    case FB_WR: v = &hc.wr; break;
    case FB_ZMM: v = &hc.zmm; break;
    case FB_ZMMT: v = &hc.zmmt; break;
    case FB_LMCC: v = &hc.lmcc; break;
    case FB_LMVEL: v = &hc.lmvel; break;
    case FB_LMACC: v = &hc.lmacc; break;
    case FB_LMNOR: v = &hc.lmnor; break;
    case FB_LMA: v = &hc.lmA; break;
    case FB_VERT: v = &hc.vert; break;
    case FB_RIGID:
        if (n != 18) return FB_ERR_STATE;
        std::memcpy(out, hc.rigid, sizeof(hc.rigid));
        return FB_OK;
    default: return FB_ERR_STATE;
    }
    if (n != static_cast<int64_t>(v->size())) return FB_ERR_STATE;
    std::memcpy(out, v->data(), static_cast<size_t>(n) * sizeof(double));
    return FB_OK;
}

int fb_set_poisson(fb_ctx *c, int mode) {
    if (!c || (mode != FB_POISSON_FP64 && mode != FB_POISSON_TF32X3 && mode != FB_POISSON_INT8X8)) return FB_ERR_STATE;
    CK(cudaSetDevice(c->device));
    if (mode == FB_POISSON_TF32X3) {
        const int st = setup_tf32(c);
        if (st) return st;
    }
    if (mode == FB_POISSON_INT8X8) {
        const int st = setup_i8(c);
        if (st) return st;
    }
    if (mode != c->poisson_mode) {   // the captured step no longer matches
        CK(cudaStreamSynchronize(c->stream));
        drop_graph(c);
        c->poisson_mode = mode;
    }
    return FB_OK;
}

int fb_set_refinement(fb_ctx *c, int sweeps) {
    if (!c || sweeps < 1 || sweeps > 4) return FB_ERR_STATE;
    if (sweeps != c->tf32_sweeps) {   // the captured step no longer matches
        CK(cudaSetDevice(c->device));
        CK(cudaStreamSynchronize(c->stream));
        drop_graph(c);
        c->tf32_sweeps = sweeps;
    }
    return FB_OK;
}

int fb_autotune(fb_ctx *c, int32_t choice[2]);

// ---- batches: independent cases advanced by one graph launch per step
//
// FB_BATCH_GROUPED: cases of one launch geometry (grid, marker count,
// helsolve tile height, options) form a group, and every stage of the step
// is one launch over the whole group (gridDim.z = cases, the case's view
// staged from a device array) plus, per transform, one batched cuBLAS DGEMM
// (FP64) or one grouped 3xTF32 tensor-core launch (precision form, tensor
// maps of every case in device memory); the groups run on parallel branches
// of one graph.  Cases that cannot be grouped (line-scan helsolve) run their
// own captured step on a branch of the same graph.  FB_BATCH_GRAPH: every case runs its own
// captured step on its own branch (bitwise equal to stepping it alone).
struct BatchGroup {
    fb::Group g{};
    fb::GroupCase *dcases = nullptr;
    std::vector<fb_ctx *> members;
    double **ptr = nullptr;     // device: 6 arrays of n pointers (forward A, B, C; backward A, B, C)
    cublasHandle_t blas = nullptr;
    void *ws = nullptr;
    cudaStream_t st = nullptr, side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, done = nullptr;
    bool cbody = false, report = false;
    int launches = 0;           // own kernels per step
    // precision form: the products, splits and residuals of every case
    bool tf32 = false;
    int sweeps = 1;                  // refinement sweeps (one value per group)
    fb::Tf32x3Plan plan_fwd{}, plan_bwd{};   // launch geometry (the first case's plans)
    fb::GemmTask *gt = nullptr;      // 4 x n: forward -> hmn; backward -> pw; -> dph (+ pw); -> pw (+ pw)
    fb::SplitTask *sp = nullptr;     // 2 x n: dph S^-1 -> a; hmn -> a2
    fb::ResidualTask *rt = nullptr;  // n: pw -> a (S^-1)
    // FP64 transforms on the INT8 tensor cores: digit cuts and products of every case
    bool i8 = false;
    fb::I8Plan i8rep{};              // split geometry (the first case's data operand)
    int i8bn = fb::kI8BN;            // product tile width of the group
    fb::I8SplitTask *i8s = nullptr;  // 2 x n: dph, then hmn, into the case's digit planes
    fb::I8Task *i8t = nullptr;       // 2 x n: forward -> hmn, backward -> dph
};

struct fb_batch {
    std::vector<fb_ctx *> ctx;
    int device = 0;
    int mode = FB_BATCH_GROUPED;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> done;   // per ungrouped case
    std::vector<fb_ctx *> singles;   // cases stepped by their own captured step
    std::vector<BatchGroup *> groups;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int *status_h = nullptr;   // pinned: one status per case
    double last_ms = 0.0;
    int launches = 0;          // own kernels per step (coupled: with one fluid solve)
    // strongly coupled cases: one iteration over the whole batch, converged
    // cases gated out of every launch until all have converged
    bool coupled = false;
    fb::Couple **cpls = nullptr;    // device: the cases' iteration states
    fb::SnapList *snaps = nullptr;  // device: the cases' saved states
    long snap_longest = 0;
    int maxit = 1;                  // the largest iteration limit of the cases
    int *any_d = nullptr;           // device flag of the host-driven loop
    bool cond_graph = true;
    cudaGraphExec_t exec_a = nullptr, exec_b = nullptr, exec_d = nullptr;   // host-driven loop's parts
};

namespace {

void group_free(BatchGroup *bg) {
    if (!bg) return;
    if (bg->st) cudaStreamSynchronize(bg->st);
    if (bg->blas) cublasDestroy(bg->blas);
    if (bg->ws) cudaFree(bg->ws);
    if (bg->dcases) cudaFree(bg->dcases);
    if (bg->ptr) cudaFree(bg->ptr);
    if (bg->gt) cudaFree(bg->gt);
    if (bg->sp) cudaFree(bg->sp);
    if (bg->rt) cudaFree(bg->rt);
    if (bg->i8s) cudaFree(bg->i8s);
    if (bg->i8t) cudaFree(bg->i8t);
    for (cudaEvent_t e : {bg->fork, bg->join, bg->done})
        if (e) cudaEventDestroy(e);
    if (bg->st) cudaStreamDestroy(bg->st);
    if (bg->side) cudaStreamDestroy(bg->side);
    delete bg;
}

// grouped launches need the windowed helsolve in every substep
bool groupable(const fb_ctx *c) {
    if (c->hc.deck.nsst != 3) return false;
    if (c->poisson_mode == FB_POISSON_TF32X3 && !c->pw) return false;
    if (c->poisson_mode == FB_POISSON_INT8X8 && !c->i8_ready) return false;
    for (int n = 0; n < 3; ++n)
        if (c->sub[n].win_y <= 0 || c->sub[n].win_tk != c->sub[0].win_tk) return false;
    return true;
}

// cases that may share launches: same launch geometry and options
using GroupKey = std::array<int, 13>;
GroupKey group_key(const fb_ctx *c) {
    const Dev &d = c->d;
    const bool tf = c->poisson_mode == FB_POISSON_TF32X3, i8 = c->poisson_mode == FB_POISSON_INT8X8;
    return {d.n2, d.n3, d.nlm, d.P, d.ldh, d.NK, c->sub[0].win_tk, c->hc.deck.cbody ? 1 : 0,
            (c->report && d.nlm) ? 1 : 0, c->poisson_mode, tf ? c->plan_fwd.bn : 0, tf ? c->tf32_sweeps : 0,
            i8 ? c->i8b.box : 0};
}

// The product tile of a group's grouped launches, timed over the whole group
// (the per-grid choice of fb_autotune is made on one case, whose few tiles
// fill the GPU differently): forward products of every case into one
// scratch output (their inputs untouched), a few launches per candidate.
int group_gemm_tile(BatchGroup *bg, int *best) {
    const int n = static_cast<int>(bg->members.size());
    const Dev &d0 = bg->members[0]->d;
    *best = bg->members[0]->plan_fwd.bn;
    double *scratch = nullptr;
    fb::GemmTask *tasks = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int r = FB_OK;
    if (cudaMalloc(&scratch, sizeof(double) * static_cast<size_t>(d0.n3m) * d0.ldh) != cudaSuccess ||
        cudaMalloc(&tasks, sizeof(fb::GemmTask) * n) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        r = FB_ERR_CUDA;
    double best_ms = 1e30;
    std::vector<fb::GemmTask> h(static_cast<size_t>(n));
    for (int cand : {64, 128, fb::kPairTile + 128, fb::kPairTile + 192, fb::kPairTile + 256}) {
        if (r) break;
        for (int i = 0; i < n && !r; ++i) {
            const fb_ctx *c = bg->members[static_cast<size_t>(i)];
            const Dev &d = c->d;
            fb::GemmTask &t = h[static_cast<size_t>(i)];
            r = fb::tf32x3_plan(t.p, c->pl_a, c->pl_zt, d.n2m, d.n3m, d.n3m, cand);
            t.o = fb::GemmOut{scratch, d.ldh, nullptr, 0, nullptr, d.n2m, d.n3m};
            t.status = d.status;
        }
        if (r) break;
        if (cudaMemcpyAsync(tasks, h.data(), sizeof(fb::GemmTask) * n, cudaMemcpyHostToDevice, bg->st) != cudaSuccess) {
            r = FB_ERR_CUDA;
            break;
        }
        fb::launch_tf32x3_group(tasks, h[0].p, n, bg->st);
        cudaEventRecord(e0, bg->st);
        for (int k = 0; k < 3; ++k) fb::launch_tf32x3_group(tasks, h[0].p, n, bg->st);
        cudaEventRecord(e1, bg->st);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            r = FB_ERR_CUDA;
            break;
        }
        if (ms < best_ms) {
            best_ms = ms;
            *best = cand;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (tasks) cudaFree(tasks);
    if (scratch) cudaFree(scratch);
    return r;
}

// The windowed helsolve's tile height for the group's launches, timed over
// the whole group like the GEMM tile (q2 and q3 of every case saved and
// restored around the trial launches; rhs2/rhs3 are only read).
int group_helsolve_tile(BatchGroup *bg) {
    const int n = static_cast<int>(bg->members.size());
    const Dev &d0 = bg->members[0]->d;
    const size_t fb = static_cast<size_t>(d0.NK) * d0.P;
    double *save = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int r = FB_OK;
    if (cudaMalloc(&save, sizeof(double) * 2 * fb * n) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess)
        r = FB_ERR_CUDA;
    for (int i = 0; i < n && !r; ++i) {
        const Dev &d = bg->members[static_cast<size_t>(i)]->d;
        if (cudaMemcpyAsync(save + 2 * fb * i, d.q2, fb * sizeof(double), cudaMemcpyDeviceToDevice, bg->st) !=
                cudaSuccess ||
            cudaMemcpyAsync(save + 2 * fb * i + fb, d.q3, fb * sizeof(double), cudaMemcpyDeviceToDevice, bg->st) !=
                cudaSuccess)
            r = FB_ERR_CUDA;
    }
    double best_ms = 1e30;
    int best = bg->g.win_tk;
    for (int cand : {32, 64}) {
        if (r) break;
        bg->g.win_tk = cand;
        fb::glaunch_win_helsolve(bg->g, 0, bg->st);
        cudaEventRecord(e0, bg->st);
        for (int k = 0; k < 3; ++k) fb::glaunch_win_helsolve(bg->g, 0, bg->st);
        cudaEventRecord(e1, bg->st);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            r = FB_ERR_CUDA;
            break;
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = cand;
        }
    }
    bg->g.win_tk = best;
    for (int i = 0; i < n && save && !r; ++i) {
        const Dev &d = bg->members[static_cast<size_t>(i)]->d;
        if (cudaMemcpyAsync(d.q2, save + 2 * fb * i, fb * sizeof(double), cudaMemcpyDeviceToDevice, bg->st) !=
                cudaSuccess ||
            cudaMemcpyAsync(d.q3, save + 2 * fb * i + fb, fb * sizeof(double), cudaMemcpyDeviceToDevice, bg->st) !=
                cudaSuccess)
            r = FB_ERR_CUDA;
    }
    if (cudaStreamSynchronize(bg->st) != cudaSuccess && !r) r = FB_ERR_CUDA;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (save) cudaFree(save);
    return r;
}

// the INT8 form's task arrays (phcalc_i8's launches, per case)
int group_setup_i8(BatchGroup *bg) {
    const int n = static_cast<int>(bg->members.size());
    std::vector<fb::I8SplitTask> sp(static_cast<size_t>(2 * n));
    std::vector<fb::I8Task> gt(static_cast<size_t>(2 * n));
    for (int i = 0; i < n; ++i) {
        const fb_ctx *c = bg->members[static_cast<size_t>(i)];
        const Dev &d = c->d;
        const size_t k = static_cast<size_t>(i), m = static_cast<size_t>(n);
        const fb::I8Plan &a = c->i8a;
        const int *gate = couple_gate(c);
        sp[k] = {d.dph + d.P, d.P, a.dig, a.ldk, a.scale, a.rows_pad, gate};
        sp[m + k] = {d.hmn, d.ldh, a.dig, a.ldk, a.scale, a.rows_pad, gate};
        gt[k] = {a.map, c->i8f.map, fb::I8Out{d.hmn, d.ldh, a.scale, c->i8f.scale, d.n2m, d.n3m}, d.n3m, d.status,
                 gate};
        gt[m + k] = {a.map, c->i8b.map, fb::I8Out{d.dph + d.P, d.P, a.scale, c->i8b.scale, d.n2m, d.n3m}, d.n3m,
                     d.status, gate};
    }
    CK(cudaMalloc(&bg->i8s, sizeof(fb::I8SplitTask) * sp.size()));
    CK(cudaMalloc(&bg->i8t, sizeof(fb::I8Task) * gt.size()));
    CK(cudaMemcpyAsync(bg->i8s, sp.data(), sizeof(fb::I8SplitTask) * sp.size(), cudaMemcpyHostToDevice, bg->st));
    CK(cudaMemcpyAsync(bg->i8t, gt.data(), sizeof(fb::I8Task) * gt.size(), cudaMemcpyHostToDevice, bg->st));
    CK(cudaStreamSynchronize(bg->st));
    bg->i8rep = bg->members[0]->i8a;
    bg->i8bn = bg->members[0]->i8b.box;
    bg->i8 = true;
    return FB_OK;
}

// the precision form's task arrays (phcalc_tf32's launches, per case)
int group_setup_tf32(BatchGroup *bg) {
    const int n = static_cast<int>(bg->members.size());
    int bn = 0, r;
    if ((r = group_gemm_tile(bg, &bn))) return r;
    std::vector<fb::GemmTask> gt(static_cast<size_t>(4 * n));
    std::vector<fb::SplitTask> sp(static_cast<size_t>(2 * n));
    std::vector<fb::ResidualTask> rt(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        const fb_ctx *c = bg->members[static_cast<size_t>(i)];
        const Dev &d = c->d;
        const size_t k = static_cast<size_t>(i), m = static_cast<size_t>(n);
        const int M = c->plan_fwd.M, N = c->plan_fwd.N;
        fb::Tf32x3Plan pf{}, pb{};
        if ((r = fb::tf32x3_plan(pf, c->pl_a, c->pl_zt, d.n2m, d.n3m, d.n3m, bn)) ||
            (r = fb::tf32x3_plan(pb, c->pl_a2, c->pl_z, d.n2m, d.n3m, d.n3m, bn)))
            return r;
        if (i == 0) {
            bg->plan_fwd = pf;
            bg->plan_bwd = pb;
        }
        const int *gate = couple_gate(c);
        gt[k] = {pf, fb::GemmOut{d.hmn, d.ldh, nullptr, 0, nullptr, M, N}, d.status, gate};
        gt[m + k] = {pb, fb::GemmOut{c->pw + d.P, d.P, nullptr, 0, c->zs_d, M, N}, d.status, gate};
        gt[2 * m + k] = {pb, fb::GemmOut{d.dph + d.P, d.P, c->pw + d.P, d.P, c->zs_d, M, N}, d.status, gate};
        gt[3 * m + k] = {pb, fb::GemmOut{c->pw + d.P, d.P, c->pw + d.P, d.P, c->zs_d, M, N}, d.status, gate};
        sp[k] = {d.dph + d.P, d.P, c->pl_a.hi, c->pl_a.lo, c->pl_a.ld, c->zsinv_d, gate};
        sp[m + k] = {d.hmn, d.ldh, c->pl_a2.hi, c->pl_a2.lo, c->pl_a2.ld, nullptr, gate};
        rt[k] = {c->pw, c->pl_a.hi, c->pl_a.lo, c->pl_a.ld, c->zsinv_d};
    }
    CK(cudaMalloc(&bg->gt, sizeof(fb::GemmTask) * gt.size()));
    CK(cudaMalloc(&bg->sp, sizeof(fb::SplitTask) * sp.size()));
    CK(cudaMalloc(&bg->rt, sizeof(fb::ResidualTask) * rt.size()));
    CK(cudaMemcpyAsync(bg->gt, gt.data(), sizeof(fb::GemmTask) * gt.size(), cudaMemcpyHostToDevice, bg->st));
    CK(cudaMemcpyAsync(bg->sp, sp.data(), sizeof(fb::SplitTask) * sp.size(), cudaMemcpyHostToDevice, bg->st));
    CK(cudaMemcpyAsync(bg->rt, rt.data(), sizeof(fb::ResidualTask) * rt.size(), cudaMemcpyHostToDevice, bg->st));
    CK(cudaStreamSynchronize(bg->st));
    bg->tf32 = true;
    bg->sweeps = bg->members[0]->tf32_sweeps;
    return FB_OK;
}

int group_setup(BatchGroup *bg) {
    const int n = static_cast<int>(bg->members.size());
    const fb_ctx *c0 = bg->members[0];
    CK(cudaStreamCreateWithFlags(&bg->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&bg->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&bg->fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&bg->join, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&bg->done, cudaEventDisableTiming));
    std::vector<fb::GroupCase> hc(static_cast<size_t>(n));
    std::vector<double *> ptr(static_cast<size_t>(6 * n));
    fb::Group &g = bg->g;
    g.n = n;
    g.rep = c0->d;
    g.win_tk = c0->sub[0].win_tk;
    for (int k = 0; k < 3; ++k) g.win_ky[k] = g.win_kz[k] = 0;
    for (int i = 0; i < n; ++i) {
        const fb_ctx *c = bg->members[static_cast<size_t>(i)];
        fb::GroupCase &gc = hc[static_cast<size_t>(i)];
        std::memset(static_cast<void *>(&gc), 0, sizeof(gc));
        gc.d = c->d;
        for (int k = 0; k < 3; ++k) {
            gc.s[k] = c->sub[k];
            g.win_ky[k] = std::max(g.win_ky[k], c->sub[k].win_y);
            g.win_kz[k] = std::max(g.win_kz[k], c->sub[k].win_z);
        }
        gc.hist_rows = c->hist_cap;
        gc.gate = couple_gate(c);
        gc.fin = c->coupling != FB_COUPLING_LOOSE ? couple_fin(const_cast<fb_ctx *>(c)) : nullptr;
        const Dev &d = c->d;
        ptr[static_cast<size_t>(0 * n + i)] = d.dph + d.P;
        ptr[static_cast<size_t>(1 * n + i)] = c->zmmt;
        ptr[static_cast<size_t>(2 * n + i)] = d.hmn;
        ptr[static_cast<size_t>(3 * n + i)] = d.hmn;
        ptr[static_cast<size_t>(4 * n + i)] = c->zmm;
        ptr[static_cast<size_t>(5 * n + i)] = d.dph + d.P;
    }
    CK(cudaMalloc(&bg->dcases, sizeof(fb::GroupCase) * n));
    CK(cudaMalloc(&bg->ptr, sizeof(double *) * 6 * n));
    CK(cudaMemcpyAsync(bg->dcases, hc.data(), sizeof(fb::GroupCase) * n, cudaMemcpyHostToDevice, bg->st));
    CK(cudaMemcpyAsync(bg->ptr, ptr.data(), sizeof(double *) * 6 * n, cudaMemcpyHostToDevice, bg->st));
    CK(cudaStreamSynchronize(bg->st));
    g.cases = bg->dcases;
    CB(cublasCreate(&bg->blas));
    CB(cublasSetStream(bg->blas, bg->st));
    CB(cublasSetPointerMode(bg->blas, CUBLAS_POINTER_MODE_HOST));
    CK(cudaMalloc(&bg->ws, 32u << 20));
    CB(cublasSetWorkspace(bg->blas, bg->ws, 32u << 20));
    bg->cbody = c0->hc.deck.cbody;
    bg->report = c0->report && c0->d.nlm;
    int r;
    if ((r = group_helsolve_tile(bg))) return r;
    if (c0->poisson_mode == FB_POISSON_TF32X3) return group_setup_tf32(bg);
    if (c0->poisson_mode == FB_POISSON_INT8X8) return group_setup_i8(bg);
    return FB_OK;
}

// the fluid step of a group (fluid_tsch.F90:30-182 + loads, in the order
// enqueue_fluid uses), enqueued on the group's stream; k counts launches
int enqueue_group_fluid(BatchGroup *bg, int &k) {
    const fb::Group &g = bg->g;
    const Dev &d = g.rep;
    const int n = g.n;
    cudaStream_t st = bg->st;
    CK(cudaEventRecord(bg->fork, st));
    CK(cudaStreamWaitEvent(bg->side, bg->fork, 0));
    fb::glaunch_marker_setup(g, bg->side);
    k += 3;
    CK(cudaEventRecord(bg->join, bg->side));
    fb::glaunch_cfl(g, st);
    k += 1;
    const double one = 1.0, zero = 0.0;
    double **p = bg->ptr;
    for (int s = 0; s < 3; ++s) {   // pr_submean deferred as in enqueue_fluid
        if (s == 0) {
            fb::glaunch_boucdq(g, s, st);
            k += 1;
        }
        fb::glaunch_nl_rhs(g, s, st, s > 0);
        if (s == 0) CK(cudaStreamWaitEvent(st, bg->join, 0));
        fb::glaunch_forcing(g, st);
        fb::glaunch_win_helsolve(g, s, st);
        fb::glaunch_divg(g, s, st);
        if (bg->tf32) {   // phcalc_tf32's launches, each over the whole group
            fb::launch_split_t_group(bg->sp, d.n2m, d.n3m, n, st);
            fb::launch_tf32x3_group(bg->gt, bg->plan_fwd, n, st);
            fb::glaunch_scan_poisson(g, st);
            fb::launch_split_t_group(bg->sp + n, d.n2m, d.n3m, n, st);
            fb::launch_tf32x3_group(bg->gt + n, bg->plan_bwd, n, st);
            for (int sw = 1; sw <= bg->sweeps; ++sw) {   // the last sweep lands in dph
                fb::launch_poisson_residual_group(g, bg->rt, st);
                fb::launch_tf32x3_group(bg->gt, bg->plan_fwd, n, st);
                fb::glaunch_scan_poisson(g, st);
                fb::launch_split_t_group(bg->sp + n, d.n2m, d.n3m, n, st);
                fb::launch_tf32x3_group(bg->gt + (sw == bg->sweeps ? 2 : 3) * n, bg->plan_bwd, n, st);
            }
            k += 5 + 5 * bg->sweeps;
        } else if (bg->i8) {   // phcalc_i8's launches, each over the whole group
            fb::launch_i8_split_group(bg->i8s, bg->i8rep, d.n2m, d.n3m, n, st);
            fb::launch_i8x8_group(bg->i8t, d.n2m, d.n3m, n, bg->i8bn, st);
            fb::glaunch_scan_poisson(g, st);
            fb::launch_i8_split_group(bg->i8s + n, bg->i8rep, d.n2m, d.n3m, n, st);
            fb::launch_i8x8_group(bg->i8t + n, d.n2m, d.n3m, n, bg->i8bn, st);
            k += 5;
        } else {
            // phcalc_outflow.F90:31,61-69: hmn = dph zmmt^T, dph = vmn zmm^T
            CB(cublasDgemmBatched(bg->blas, CUBLAS_OP_N, CUBLAS_OP_T, d.n2m, d.n3m, d.n3m, &one, p, d.P, p + n,
                                  d.n3m, &zero, p + 2 * n, d.ldh, n));
            fb::glaunch_scan_poisson(g, st);
            CB(cublasDgemmBatched(bg->blas, CUBLAS_OP_N, CUBLAS_OP_T, d.n2m, d.n3m, d.n3m, &one, p + 3 * n, d.ldh,
                                  p + 4 * n, d.n3m, &zero, p + 5 * n, d.P, n));
            k += 1;
        }
        fb::glaunch_updvp_prcalc(g, s, st, s > 0);
        if (s < 2) fb::glaunch_substep_mid(g, s + 1, s == 0 ? fb::S_PRAVG1 : fb::S_PRAVG2, st);
        else fb::glaunch_submean_boucqt(g, st, true);
        k += 7;
    }
    if (bg->cbody) {
        fb::glaunch_loads(g, st);
        k += 2;
    }
    CK(cudaGetLastError());
    return FB_OK;
}

// one loose step of a group: the fluid step, then rigid (rigid.F90:4-138)
int enqueue_group(BatchGroup *bg) {
    int k = 0;
    int r = enqueue_group_fluid(bg, k);
    if (r) return r;
    fb::glaunch_rigid(bg->g, bg->st);
    k += 1;
    if (bg->report) {
        fb::glaunch_diag(bg->g, bg->st);
        k += 1;
    }
    CK(cudaGetLastError());
    bg->launches = k;
    return FB_OK;
}

}  // namespace

int fb_batch_destroy(fb_batch *b) {
    if (!b) return FB_OK;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (BatchGroup *bg : b->groups) group_free(bg);
    for (cudaEvent_t e : b->done)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->status_h) cudaFreeHost(b->status_h);
    for (cudaGraphExec_t e : {b->exec_a, b->exec_b, b->exec_d})
        if (e) cudaGraphExecDestroy(e);
    if (b->cpls) cudaFree(b->cpls);
    if (b->snaps) cudaFree(b->snaps);
    if (b->any_d) cudaFree(b->any_d);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return FB_OK;
}

}  // extern "C"

namespace {

// The parts of one strongly coupled step of a batch: begin (initial guesses,
// saved states), one fluid solve of every case still iterating (converged
// cases sit out every launch), end (accept, commit, record).
int enqueue_batch_begin(fb_batch *b) {
    const int n = static_cast<int>(b->ctx.size());
    fb::launch_couple_begin(b->cpls, n, b->stream);
    fb::launch_snap(b->snaps, n, fb::SNAP_SAVE, b->snap_longest, b->stream);
    CK(cudaGetLastError());
    return FB_OK;
}

// forks every group off the batch stream, runs fn(group) on it, joins back
template <class F>
int over_groups(fb_batch *b, F fn) {
    CK(cudaEventRecord(b->fork, b->stream));
    for (BatchGroup *bg : b->groups) {
        CK(cudaStreamWaitEvent(bg->st, b->fork, 0));
        int r = fn(bg);
        if (r) return r;
        CK(cudaEventRecord(bg->done, bg->st));
        CK(cudaStreamWaitEvent(b->stream, bg->done, 0));
    }
    return FB_OK;
}

int enqueue_batch_iter(fb_batch *b, cudaGraphConditionalHandle h, int set_cond, int *launches) {
    const int n = static_cast<int>(b->ctx.size());
    fb::launch_snap(b->snaps, n, fb::SNAP_RESTORE_LOOP, b->snap_longest, b->stream);
    int k = 2;
    int r = over_groups(b, [&](BatchGroup *bg) -> int {
        fb::glaunch_rigid(bg->g, bg->st, fb::RIGID_PLACE);
        int kk = 2;
        const int rr = enqueue_group_fluid(bg, kk);
        fb::glaunch_rigid(bg->g, bg->st, fb::RIGID_FORCES);
        k += kk;
        return rr;
    });
    if (r) return r;
    fb::launch_couple_update(b->cpls, n, h, set_cond, set_cond ? nullptr : b->any_d, b->stream);
    CK(cudaGetLastError());
    if (launches) *launches = k;
    return FB_OK;
}

int enqueue_batch_end(fb_batch *b, int *launches) {
    const int n = static_cast<int>(b->ctx.size());
    fb::launch_snap(b->snaps, n, fb::SNAP_RESTORE_BODY, b->snap_longest, b->stream);
    fb::launch_couple_accept(b->cpls, n, b->stream);
    int k = 3;
    int r = over_groups(b, [&](BatchGroup *bg) -> int {
        fb::glaunch_rigid(bg->g, bg->st, fb::RIGID_COMMIT);
        k += 1;
        return FB_OK;
    });
    if (r) return r;
    fb::launch_couple_record(b->cpls, n, b->stream);
    r = over_groups(b, [&](BatchGroup *bg) -> int {
        if (bg->report) {
            fb::glaunch_diag(bg->g, bg->st);
            k += 1;
        }
        return FB_OK;
    });
    if (r) return r;
    CK(cudaGetLastError());
    if (launches) *launches = k;
    return FB_OK;
}

// the coupled batch step: one graph with a WHILE node around the fluid solves
// (or, without conditional graphs, three graphs that the host loop replays)
int capture_batch_coupled(fb_batch *b) {
    auto cap = [&](cudaGraph_t *out, auto fn) -> int {
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return FB_ERR_CUDA;
        const int rr = fn();
        const cudaError_t e = cudaStreamEndCapture(b->stream, out);
        return rr ? rr : (e == cudaSuccess ? FB_OK : FB_ERR_CUDA);
    };
    cudaGraph_t G = nullptr, ga = nullptr, gb = nullptr, gd = nullptr;
    auto cleanup = [&] {
        for (cudaGraph_t g : {ga, gb, gd, G})
            if (g) cudaGraphDestroy(g);
    };
    int r, ki = 0, ke = 0;
    cudaGraphConditionalHandle h{};
    b->cond_graph = cudaGraphCreate(&G, 0) == cudaSuccess &&
                    cudaGraphConditionalHandleCreate(&h, G, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGetLastError();
    if ((r = cap(&ga, [&] { return enqueue_batch_begin(b); })) ||
        (r = cap(&gb, [&] { return enqueue_batch_iter(b, h, b->cond_graph ? 1 : 0, &ki); })) ||
        (r = cap(&gd, [&] { return enqueue_batch_end(b, &ke); }))) {
        cleanup();
        return r;
    }
    b->launches = 2 + ki + ke;
    if (b->cond_graph) {
        cudaGraphNode_t na = nullptr, nc = nullptr, nb = nullptr, nd = nullptr;
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        b->cond_graph = cudaGraphAddChildGraphNode(&na, G, nullptr, 0, ga) == cudaSuccess &&
                        cudaGraphAddNode(&nc, G, &na, 1, &p) == cudaSuccess &&
                        cudaGraphAddChildGraphNode(&nb, p.conditional.phGraph_out[0], nullptr, 0, gb) == cudaSuccess &&
                        cudaGraphAddChildGraphNode(&nd, G, &nc, 1, gd) == cudaSuccess &&
                        cudaGraphInstantiate(&b->exec, G, 0) == cudaSuccess;
        cudaGetLastError();
        if (b->cond_graph) {
            b->graph = G;
            G = nullptr;
            cleanup();
            return FB_OK;
        }
        b->exec = nullptr;
        // the iteration graph was captured to set the condition: capture it again
        cudaGraphDestroy(gb);
        gb = nullptr;
        if ((r = cap(&gb, [&] { return enqueue_batch_iter(b, h, 0, nullptr); }))) {
            cleanup();
            return r;
        }
    }
    const bool ok = cudaGraphInstantiate(&b->exec_a, ga, 0) == cudaSuccess &&
                    cudaGraphInstantiate(&b->exec_b, gb, 0) == cudaSuccess &&
                    cudaGraphInstantiate(&b->exec_d, gd, 0) == cudaSuccess;
    cleanup();
    return ok ? FB_OK : FB_ERR_CUDA;
}

}  // namespace

extern "C" {

int fb_batch_create_mode(fb_ctx *const *ctxs, int n, int mode, fb_batch **out) {
    if (!ctxs || n < 1 || !out || (mode != FB_BATCH_GROUPED && mode != FB_BATCH_GRAPH)) return FB_ERR_STATE;
    *out = nullptr;
    fb_batch *b = new (std::nothrow) fb_batch;
    if (!b) return FB_ERR_CUDA;
    b->device = ctxs[0]->device;
    b->mode = mode;
    for (int i = 0; i < n; ++i) {
        fb_ctx *c = ctxs[i];
        if (!c || c->device != b->device || !c->d.nlm) {
            delete b;
            return FB_ERR_STATE;
        }
        if (c->vardt || c->hc.deck.nsst != 3) {  // per-step host control or first-step coefficients
            delete b;
            return FB_ERR_UNSUPPORTED;
        }
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == c) {   // a case may appear once
                delete b;
                return FB_ERR_STATE;
            }
        b->ctx.push_back(c);
    }
    // strongly coupled cases iterate together: all of a batch or none, every
    // case in a grouped launch with a transform form whose launches can sit
    // a converged case out (the library's own tensor-core kernels)
    int ncoupled = 0;
    for (fb_ctx *c : b->ctx) ncoupled += (c->coupling != FB_COUPLING_LOOSE) ? 1 : 0;
    if (ncoupled) {
        bool ok = ncoupled == n && mode == FB_BATCH_GROUPED;
        for (fb_ctx *c : b->ctx) ok = ok && c->poisson_mode != FB_POISSON_FP64;
        if (!ok) {
            delete b;
            return FB_ERR_UNSUPPORTED;
        }
        b->coupled = true;
    }
    int r = FB_OK;
    auto fail = [&](int code) {
        fb_batch_destroy(b);
        return code;
    };
    if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaMallocHost(&b->status_h, sizeof(int) * n) != cudaSuccess)
        return fail(FB_ERR_CUDA);
    for (fb_ctx *c : b->ctx) {   // tile shapes per grid size, then the contexts go quiet
        if ((r = fb_autotune(c, nullptr))) return fail(r);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(FB_ERR_CUDA);
    }
    // groups in order of first appearance
    std::map<GroupKey, BatchGroup *> by_key;
    for (fb_ctx *c : b->ctx) {
        if (mode != FB_BATCH_GROUPED || !groupable(c)) {
            b->singles.push_back(c);
            continue;
        }
        const auto key = group_key(c);
        auto it = by_key.find(key);
        if (it == by_key.end()) {
            BatchGroup *bg = new (std::nothrow) BatchGroup;
            if (!bg) return fail(FB_ERR_CUDA);
            b->groups.push_back(bg);
            it = by_key.emplace(key, bg).first;
        }
        it->second->members.push_back(c);
    }
    if (b->coupled && !b->singles.empty()) return fail(FB_ERR_UNSUPPORTED);   // every case grouped
    for (BatchGroup *bg : b->groups)
        if ((r = group_setup(bg))) return fail(r);
    if (b->coupled) {
        std::vector<fb::Couple *> cp;
        std::vector<fb::SnapList> sl;
        for (fb_ctx *c : b->ctx) {
            if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(FB_ERR_CUDA);
            cp.push_back(c->cpl);
            sl.push_back(c->snapl);
            b->snap_longest = std::max(b->snap_longest, c->snap_longest);
            b->maxit = std::max(b->maxit, c->cmaxit);
        }
        if (cudaMalloc(&b->cpls, sizeof(fb::Couple *) * n) != cudaSuccess ||
            cudaMalloc(&b->snaps, sizeof(fb::SnapList) * n) != cudaSuccess ||
            cudaMalloc(&b->any_d, sizeof(int)) != cudaSuccess ||
            cudaMemcpy(b->cpls, cp.data(), sizeof(fb::Couple *) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(b->snaps, sl.data(), sizeof(fb::SnapList) * n, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(FB_ERR_CUDA);
        if ((r = capture_batch_coupled(b))) return fail(r);
        *out = b;
        return FB_OK;
    }
    b->done.assign(b->singles.size(), nullptr);
    for (auto &e : b->done)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(FB_ERR_CUDA);
    // one step of every group and every ungrouped case captured from the
    // master stream: each branch forks from it and joins back
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return fail(FB_ERR_CUDA);
    cudaError_t e = cudaEventRecord(b->fork, b->stream);
    b->launches = 0;
    for (BatchGroup *bg : b->groups) {
        if (e != cudaSuccess || r) break;
        e = cudaStreamWaitEvent(bg->st, b->fork, 0);
        if (e != cudaSuccess) break;
        r = enqueue_group(bg);
        b->launches += bg->launches;
        if (!r) e = cudaEventRecord(bg->done, bg->st);
        if (!r && e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, bg->done, 0);
    }
    for (size_t i = 0; i < b->singles.size() && e == cudaSuccess && !r; ++i) {
        fb_ctx *c = b->singles[i];
        e = cudaStreamWaitEvent(c->stream, b->fork, 0);
        if (e != cudaSuccess) break;
        c->own_launches = 0;
        r = enqueue_step(c, 1);
        c->step_kernels = c->own_launches;
        b->launches += c->own_launches;
        if (!r) e = cudaEventRecord(b->done[i], c->stream);
        if (!r && e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->done[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
    if (r || e != cudaSuccess || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(r ? r : FB_ERR_CUDA);
    }
    b->graph = g;
    if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) return fail(FB_ERR_CUDA);
    *out = b;
    return FB_OK;
}

int fb_batch_create(fb_ctx *const *ctxs, int n, fb_batch **out) {
    return fb_batch_create_mode(ctxs, n, FB_BATCH_GROUPED, out);
}

int fb_batch_info(fb_batch *b, int32_t info[3]) {
    if (!b || !info) return FB_ERR_STATE;
    info[0] = static_cast<int32_t>(b->groups.size());
    info[1] = static_cast<int32_t>(b->singles.size());
    info[2] = b->launches;
    return FB_OK;
}

int fb_batch_advance(fb_batch *b, int nsteps) {
    if (!b || nsteps < 0) return FB_ERR_STATE;
    CK(cudaSetDevice(b->device));
    // work the contexts queued on their own streams (marker uploads) comes first
    for (fb_ctx *x : b->ctx) CK(cudaStreamSynchronize(x->stream));
    CK(cudaEventRecord(b->ev0, b->stream));
    if (b->coupled && !b->cond_graph) {   // the fluid solves driven from the host
        for (int i = 0; i < nsteps; ++i) {
            CK(cudaGraphLaunch(b->exec_a, b->stream));
            for (int it = 0; it < b->maxit; ++it) {
                CK(cudaGraphLaunch(b->exec_b, b->stream));
                int any = 0;
                CK(cudaMemcpyAsync(&any, b->any_d, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
                CK(cudaStreamSynchronize(b->stream));
                if (!any) break;
            }
            CK(cudaGraphLaunch(b->exec_d, b->stream));
        }
    } else {
        for (int i = 0; i < nsteps; ++i) CK(cudaGraphLaunch(b->exec, b->stream));
    }
    CK(cudaEventRecord(b->ev1, b->stream));
    for (size_t i = 0; i < b->ctx.size(); ++i)
        CK(cudaMemcpyAsync(b->status_h + i, b->ctx[i]->d.status, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    int status = FB_OK;
    for (size_t i = 0; i < b->ctx.size(); ++i) {
        host_clock(b->ctx[i], nsteps);
        if (!status && b->status_h[i]) status = b->status_h[i];
    }
    return status;
}

int fb_batch_last_ms(fb_batch *b, double *ms) {
    if (!b || !ms) return FB_ERR_STATE;
    *ms = b->last_ms;
    return FB_OK;
}

// Tile shapes per grid size: the windowed helsolve's tile height (32 or 64
// rows) and, once the precision form is on, the 3xTF32 GEMM's tile width
// (64 or 128 columns), each chosen by timing both on this context.  The
// choice is remembered per (n2, n3) for the process, so a batch of cases of
// a few grid sizes tunes each size once.  The timed stages' outputs (q2, q3,
// hmn) are saved and restored around the measurement.
int fb_autotune(fb_ctx *c, int32_t choice[2]) {
    if (!c) return FB_ERR_STATE;
    static std::mutex mu;
    // (n2, n3) -> (tk, bn, i8 bn); bn 0: untuned
    static std::map<std::pair<int, int>, std::array<int, 3>> cache;
    const std::pair<int, int> key(c->d.n2, c->d.n3);
    int tk = 0, bn = 0, ibn = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            tk = it->second[0];
            bn = it->second[1];
            ibn = it->second[2];
        }
    }
    const bool want_bn = (c->pw != nullptr), want_ibn = c->i8_ready && !c->i8_fixed;
    auto i8_tile = [&](int w) -> int {   // the B operands' boxes set the product tile width
        int r = fb::i8_plan(c->i8f, c->d.n3m, c->d.n3m, w);
        if (!r) r = fb::i8_plan(c->i8b, c->d.n3m, c->d.n3m, w);
        if (!r) c->tune_i8bn = w;
        return r;
    };
    if (!tk || (want_bn && !bn) || (want_ibn && !ibn)) {
        CK(cudaSetDevice(c->device));
        const Dev &d = c->d;
        const size_t fbytes = static_cast<size_t>(d.NK) * d.P * sizeof(double);
        const size_t hbytes = static_cast<size_t>(d.n3m) * d.ldh * sizeof(double);
        void *save = nullptr;
        CK(cudaMalloc(&save, 2 * fbytes + hbytes));
        char *sv = static_cast<char *>(save);
        CK(cudaMemcpyAsync(sv, d.q2, fbytes, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(sv + fbytes, d.q3, fbytes, cudaMemcpyDeviceToDevice, c->stream));
        CK(cudaMemcpyAsync(sv + 2 * fbytes, d.hmn, hbytes, cudaMemcpyDeviceToDevice, c->stream));
        int r = FB_OK;
        // each candidate is timed in three interleaved rounds and judged by
        // its best round: single timings of a few launches flip the choice
        constexpr int kRounds = 3;
        if (!tk) {
            const int cands[2] = {32, 64};
            double bm[2] = {1e30, 1e30};
            if (c->sub[0].win_y == 0) tk = 64;   // line scans: no tile to tune
            for (int rd = 0; rd < kRounds && !tk && !r; ++rd)
                for (int k = 0; k < 2 && !r; ++k) {
                    for (int n = 0; n < d.nsst; ++n) c->sub[n].win_tk = cands[k];
                    double ms = 0.0;
                    if (!(r = fb_time_stage(c, FB_ST_HELSOLVE, 1, 10, &ms))) bm[k] = std::min(bm[k], ms);
                }
            if (!tk && !r) tk = (bm[0] < bm[1]) ? 32 : 64;
        }
        if (!r && want_ibn && !ibn) {
            // The INT8 product's tile width from its waves, not from timing: a
            // CTA's time grows with its width, so the step pays waves x width
            // (148 SMs, one CTA each); ties go to the wider tile (fewer MMA
            // instructions per column).  Timed alone, back-to-back launches
            // overlap one launch's last wave with the next one's first, which
            // favours narrow two-wave tiles; inside the time step the next
            // kernel is another stage (galloping rectangle, the same process:
            // 480 us per step with 48 columns, 513 with 64).
            ibn = fb::i8_tile_width(d.n2m, d.n3m);   // C = dph (n2m rows) x eigenvectors (n3m)
            r = i8_tile(ibn);
        }
        if (!r && want_bn && !bn) {
            double best = 1e30;
            for (int cand : {64, 128, fb::kPairTile + 128, fb::kPairTile + 192, fb::kPairTile + 256}) {
                if ((r = fb::tf32x3_plan(c->plan_fwd, c->pl_a, c->pl_zt, d.n2m, d.n3m, d.n3m, cand))) break;
                double ms = 0.0;
                if ((r = fb_time_stage(c, FB_TK_TF32X3_GEMM, 1, 10, &ms))) break;
                if (ms < best) {
                    best = ms;
                    bn = cand;
                }
            }
        }
        cudaMemcpyAsync(d.q2, sv, fbytes, cudaMemcpyDeviceToDevice, c->stream);
        cudaMemcpyAsync(d.q3, sv + fbytes, fbytes, cudaMemcpyDeviceToDevice, c->stream);
        cudaMemcpyAsync(d.hmn, sv + 2 * fbytes, hbytes, cudaMemcpyDeviceToDevice, c->stream);
        cudaStreamSynchronize(c->stream);
        cudaFree(save);
        if (r) return r;
        std::lock_guard<std::mutex> lk(mu);
        cache[key] = {tk, bn, ibn};
    }
    if (want_ibn && ibn) {
        int r;
        if ((r = i8_tile(ibn))) return r;
    }
    {
        int rt;
        if ((rt = tune_dgemm(c))) return rt;
    }
    c->tune_tk = tk;
    for (int n = 0; n < c->d.nsst; ++n) c->sub[n].win_tk = tk;
    if (want_bn && bn) {
        c->tune_bn = bn;
        int r;
        if ((r = fb::tf32x3_plan(c->plan_fwd, c->pl_a, c->pl_zt, c->d.n2m, c->d.n3m, c->d.n3m, bn))) return r;
        if ((r = fb::tf32x3_plan(c->plan_bwd, c->pl_a2, c->pl_z, c->d.n2m, c->d.n3m, c->d.n3m, bn))) return r;
    }
    CK(cudaStreamSynchronize(c->stream));
    drop_graph(c);
    if (choice) {
        choice[0] = c->tune_tk;
        choice[1] = c->tune_bn;
    }
    return FB_OK;
}

int fb_set_coupling(fb_ctx *c, int mode, double tol, int max_iter) {
    if (!c || mode < FB_COUPLING_LOOSE || mode > FB_COUPLING_LEARNED || !(tol > 0.0) || max_iter < 1)
        return FB_ERR_STATE;
    if (mode != FB_COUPLING_LOOSE && (c->vardt || !c->d.nlm)) return FB_ERR_UNSUPPORTED;
    CK(cudaSetDevice(c->device));
    if (mode == FB_COUPLING_LOOSE) {
        if (c->coupling != FB_COUPLING_LOOSE) {   // the captured step changes
            CK(cudaStreamSynchronize(c->stream));
            drop_graph(c);
        }
        c->coupling = mode;
        return FB_OK;
    }
    int st = couple_alloc(c);
    if (st) return st;
    const bool fresh = (c->coupling == FB_COUPLING_LOOSE);
    // the predictor's history: the steps already taken (history ring)
    std::vector<std::array<double, 9>> seed;
    if (fresh) {
        double step = 0.0;
        CK(cudaMemcpyAsync(&step, c->d.scal + fb::S_STEP, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        const int done = static_cast<int>(step), take = std::min(done, std::min(fb::kCplHist, c->hist_cap));
        std::vector<double> row(FB_HIST_COLS);
        for (int i = done - take; i < done; ++i) {
            CK(cudaMemcpy(row.data(), c->d.hist + static_cast<size_t>(i % c->hist_cap) * FB_HIST_COLS,
                          FB_HIST_COLS * sizeof(double), cudaMemcpyDeviceToHost));
            seed.push_back({row[9], row[10], row[11], row[12], row[13], row[14], row[1], row[2], row[3]});
        }
    }
    const fb::Deck &dk = c->hc.deck;
    int q = 0;
    for (int i = 0; i < 3; ++i)
        if (dk.rbmcon[i] == 0) {
            q = i;
            break;
        }
    const double mass = dk.rbden * (q == 2 ? dk.rba[1] : dk.rba[0]);
    const double kq = dk.kk[q];
    int nin = 0, nout = 0;
    const float *params = c->mlp ? fb::mlp_params_device(c->mlp, &nin, &nout) : nullptr;
    st = couple_edit(c, [&](fb::Couple &h) {
        h.tol = tol;
        h.omega0 = 0.5;
        h.maxit = max_iter;
        h.q = q;
        h.learned = (mode == FB_COUPLING_LEARNED) ? 1 : 0;
        h.cap = c->smp_cap;
        h.feat_re = 1.0 / dk.visc;
        h.feat_mr = dk.rbden;
        h.feat_ur = kq > 0.0 ? 2.0 * M_PI * std::sqrt(mass / kq) : 0.0;
        h.mlp = params;
        h.norm = c->mlp_norm_d;
        h.forces = c->d.forces;
        h.rigid = c->d.rigid;
        h.sx = c->smp_x;
        h.st = c->smp_t;
        if (fresh) {
            h.nh = static_cast<int>(seed.size());
            for (int i = 0; i < h.nh; ++i)
                for (int k = 0; k < 3; ++k) {
                    h.hp[i][k] = seed[static_cast<size_t>(i)][k];
                    h.hv[i][k] = seed[static_cast<size_t>(i)][3 + k];
                    h.hf[i][k] = seed[static_cast<size_t>(i)][6 + k];
                }
        }
    });
    if (st) return st;
    if (fresh) {   // the captured step changes
        CK(cudaStreamSynchronize(c->stream));
        drop_graph(c);
    }
    c->coupling = mode;
    c->cmaxit = max_iter;
    return FB_OK;
}

int fb_set_predictor(fb_ctx *c, fb_mlp *m, const float *norm) {
    if (!c || (m && !norm)) return FB_ERR_STATE;
    int nin = 0, nout = 0;
    const float *params = m ? fb::mlp_params_device(m, &nin, &nout) : nullptr;
    if (m && (nin != fb::kCplIn || nout != fb::kCplOut)) return FB_ERR_STATE;
    CK(cudaSetDevice(c->device));
    int st;
    const size_t nn = 2 * fb::kCplIn + 2 * fb::kCplOut;
    if (m) {
        if (!c->mlp_norm_d && (st = dnew(c, &c->mlp_norm_d, nn))) return st;
        if ((st = h2d(c, c->mlp_norm_d, norm, nn * sizeof(float)))) return st;
    }
    c->mlp = m;
    if (c->cpl)
        return couple_edit(c, [&](fb::Couple &h) {
            h.mlp = params;
            h.norm = m ? c->mlp_norm_d : nullptr;
        });
    return FB_OK;
}

int fb_coupling_stats(fb_ctx *c, double out[4]) {
    if (!c || !out) return FB_ERR_STATE;
    for (int i = 0; i < 4; ++i) out[i] = 0.0;
    if (!c->cpl) return FB_OK;
    fb::Couple h;
    CK(cudaMemcpyAsync(&h, c->cpl, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out[0] = h.steps;
    out[1] = h.solves;
    out[2] = h.maxit_hits;
    out[3] = h.steps > 0 ? h.res0 / h.steps : 0.0;
    return FB_OK;
}

// the samples written since the last call, oldest first (a ring of smp_cap:
// samples older than that are lost)
int fb_coupling_samples(fb_ctx *c, float *x, float *t, int cap, int *n) {
    if (!c || !n) return FB_ERR_STATE;
    *n = 0;
    if (!c->cpl) return FB_OK;
    unsigned long long written = 0;
    CK(cudaMemcpyAsync(&written, reinterpret_cast<char *>(c->cpl) + offsetof(fb::Couple, nsamples), sizeof(written),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const unsigned long long ring = static_cast<unsigned long long>(c->smp_cap);
    if (written - c->smp_drained > ring) c->smp_drained = written - ring;
    const int have = static_cast<int>(written - c->smp_drained);
    *n = have;
    if (!x || !t) return FB_OK;
    const int m = std::max(0, std::min(cap, have));
    for (int done = 0; done < m;) {   // up to the ring's end, then from its start
        const size_t slot = static_cast<size_t>((c->smp_drained + static_cast<unsigned long long>(done)) % ring);
        const int run = std::min(m - done, static_cast<int>(ring - slot));
        CK(cudaMemcpy(x + static_cast<size_t>(done) * fb::kCplIn, c->smp_x + slot * fb::kCplIn,
                      sizeof(float) * static_cast<size_t>(run) * fb::kCplIn, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(t + static_cast<size_t>(done) * fb::kCplOut, c->smp_t + slot * fb::kCplOut,
                      sizeof(float) * static_cast<size_t>(run) * fb::kCplOut, cudaMemcpyDeviceToHost));
        done += run;
    }
    c->smp_drained += static_cast<unsigned long long>(m);
    *n = m;
    return FB_OK;
}

int fb_set_report(fb_ctx *c, int on) {
    if (!c) return FB_ERR_STATE;
    if ((on != 0) != c->report) {
        CK(cudaStreamSynchronize(c->stream));
        drop_graph(c);
        c->report = (on != 0);
    }
    return FB_OK;
}

int fb_gemm_tf32x3(int device, int M, int N, int K, int bn, const double *A, const double *B, double *C) {
    if (M < 1 || N < 1 || K < 1 || !A || !B || !C || !fb::tf32x3_shape_ok(bn)) return FB_ERR_STATE;
    CK(cudaSetDevice(device));
    int st = fb::tf32x3_configure();
    if (st) return st;
    const long ld = (K + 31) / 32 * 32;
    std::vector<void *> mem;
    auto alloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        mem.push_back(p);
        return p;
    };
    double *dA = static_cast<double *>(alloc(sizeof(double) * M * K));
    double *dB = static_cast<double *>(alloc(sizeof(double) * N * K));
    double *dC = static_cast<double *>(alloc(sizeof(double) * M * N));
    float *ah = static_cast<float *>(alloc(sizeof(float) * M * ld)), *al = static_cast<float *>(alloc(sizeof(float) * M * ld));
    float *bh = static_cast<float *>(alloc(sizeof(float) * N * ld)), *bl = static_cast<float *>(alloc(sizeof(float) * N * ld));
    int *status = static_cast<int *>(alloc(sizeof(int)));
    st = FB_OK;
    if (!dA || !dB || !dC || !ah || !al || !bh || !bl || !status) st = FB_ERR_CUDA;
    fb::Tf32x3Plan plan{};
    fb::SplitPlane pa{ah, al, ld}, pb{bh, bl, ld};
    if (!st && (cudaMemcpy(dA, A, sizeof(double) * M * K, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(dB, B, sizeof(double) * N * K, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemset(status, 0, sizeof(int)) != cudaSuccess))
        st = FB_ERR_CUDA;
    if (!st) {
        fb::launch_split_t(dA, M, M, K, pa, nullptr);  // A(m, k) at A[k * M + m] -> [m][k]
        fb::launch_split_t(dB, N, N, K, pb, nullptr);
        st = fb::tf32x3_plan(plan, pa, pb, M, N, K, bn);
    }
    if (!st) {
        fb::launch_tf32x3(plan, dC, M, nullptr, 0, status, nullptr);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = FB_ERR_CUDA;
    }
    int dev_status = 0;
    if (!st && cudaMemcpy(&dev_status, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) st = FB_ERR_CUDA;
    if (!st && dev_status) st = dev_status;
    if (!st && cudaMemcpy(C, dC, sizeof(double) * M * N, cudaMemcpyDeviceToHost) != cudaSuccess) st = FB_ERR_CUDA;
    for (void *p : mem) cudaFree(p);
    return st;
}

int fb_gemm_i8x8(int device, int M, int N, int K, const double *A, const double *B, double *C) {
    if (M < 1 || N < 1 || K < 1 || !A || !B || !C) return FB_ERR_STATE;
    if (K > fb::kI8MaxK) return FB_ERR_UNSUPPORTED;   // int32 class sums would overflow
    CK(cudaSetDevice(device));
    int st = fb::i8_configure();
    if (st) return st;
    const long ldk = (K + fb::kI8BK - 1) / fb::kI8BK * fb::kI8BK;
    std::vector<void *> mem;
    auto alloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        mem.push_back(p);
        return p;
    };
    fb::I8Plan pa{}, pb{};
    pa.ldk = pb.ldk = ldk;
    pa.rows_pad = (M + 127) / 128 * 128;
    pb.rows_pad = (N + 127) / 128 * 128;
    double *dA = static_cast<double *>(alloc(sizeof(double) * M * K));
    double *dB = static_cast<double *>(alloc(sizeof(double) * N * K));
    double *dC = static_cast<double *>(alloc(sizeof(double) * M * N));
    pa.dig = static_cast<int8_t *>(alloc(static_cast<size_t>(fb::kI8S) * pa.rows_pad * ldk));
    pb.dig = static_cast<int8_t *>(alloc(static_cast<size_t>(fb::kI8S) * pb.rows_pad * ldk));
    pa.scale = static_cast<double *>(alloc(sizeof(double) * pa.rows_pad));
    pb.scale = static_cast<double *>(alloc(sizeof(double) * pb.rows_pad));
    int *status = static_cast<int *>(alloc(sizeof(int)));
    double *mxA = static_cast<double *>(alloc(sizeof(double) * M));
    double *mxB = static_cast<double *>(alloc(sizeof(double) * N));
    st = FB_OK;
    if (!dA || !dB || !dC || !pa.dig || !pb.dig || !pa.scale || !pb.scale || !status || !mxA || !mxB)
        st = FB_ERR_CUDA;
    if (!st && (cudaMemcpy(dA, A, sizeof(double) * M * K, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(dB, B, sizeof(double) * N * K, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemset(status, 0, sizeof(int)) != cudaSuccess ||
                cudaMemset(mxA, 0, sizeof(double) * M) != cudaSuccess ||
                cudaMemset(mxB, 0, sizeof(double) * N) != cudaSuccess))
        st = FB_ERR_CUDA;
    if (!st) st = fb::i8_plan(pa, M, K, 128);
    if (!st) st = fb::i8_plan(pb, N, K, fb::kI8BN);
    if (!st) {
        // row maxima, then the cut of each operand (the step's kernels)
        fb::launch_i8_rowmax(dA, M, M, K, mxA, nullptr);
        fb::launch_i8_rowmax(dB, N, N, K, mxB, nullptr);
        fb::launch_i8_cut_rows(dA, M, M, K, pa, mxA, nullptr, nullptr);
        fb::launch_i8_cut_rows(dB, N, N, K, pb, mxB, nullptr, nullptr);
        fb::launch_i8x8(pa, pb, dC, M, status, nullptr);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) st = FB_ERR_CUDA;
    }
    int dev_status = 0;
    if (!st && cudaMemcpy(&dev_status, status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) st = FB_ERR_CUDA;
    if (!st && dev_status) st = dev_status;
    if (!st && cudaMemcpy(C, dC, sizeof(double) * M * N, cudaMemcpyDeviceToHost) != cudaSuccess) st = FB_ERR_CUDA;
    for (void *p : mem) cudaFree(p);
    return st;
}

int fb_eigen_tridiag(int n, const double *am, const double *ac, const double *ap, double *wr, double *zmm,
                     double *zmmt) {
    if (n < 1 || !am || !ac || !ap || !wr || !zmm || !zmmt) return FB_ERR_STATE;
    return fb::eigen_tridiag(n, am, ac, ap, wr, zmm, zmmt) ? FB_ERR_NUMERIC : FB_OK;
}

}  // extern "C"
