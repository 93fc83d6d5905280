// CUDA kernels of the FRiBoIS2D fluid time step (sm_100a, FP64).
//
// This translation unit is compiled with -fmad=false: every expression keeps
// the reference's left-to-right evaluation without fused multiply-adds, so
// the stencil stages reproduce the CPU restatement bit for bit.  Each kernel
// cites the reference routine it implements.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include <cudaTypedefs.h>

#include "device.cuh"
#include "kernels.h"
#include "pdl.h"
#include "tma.cuh"
#include "../../include/fribois2d.h"

namespace fb {

#define Fv(a, j, k) (a)[fidx(d, (j), (k))]

// ------------------------------------------------------------ helpers

__device__ __forceinline__ void raise_status(const Dev &d, int code) {
    atomicCAS(d.status, 0, code);
}

// indic.F90:276-303 as arithmetic (no dependent index loads)
__device__ __forceinline__ int jmv_(int jc) { return jc == 1 ? 1 : jc - 1; }
__device__ __forceinline__ int jpv_(const Dev &d, int jc) { return jc >= d.n2m ? jc : jc + 1; }
__device__ __forceinline__ int kmv_(int kc) { return kc == 1 ? 1 : kc - 1; }
__device__ __forceinline__ int kpv_(const Dev &d, int kc) { return kc == d.n3m ? kc : kc + 1; }

template <bool kMax>
__device__ __forceinline__ double warp_reduce(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, v, o);
        v = kMax ? fmax(v, x) : v + x;
    }
    return v;
}

// block reduction with shuffles; sh holds 32 doubles; result in every thread
template <bool kMax>
__device__ double block_reduce_fast(double v, double *sh) {
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    v = warp_reduce<kMax>(v);
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double r = (t < nw) ? sh[t] : (kMax ? -INFINITY : 0.0);
    if (t < 32) r = warp_reduce<kMax>(r);
    if (t == 0) sh[0] = r;
    __syncthreads();
    r = sh[0];
    __syncthreads();
    return r;
}

// block_reduce_fast<false> of N values at once (the same shuffle tree for
// each, so the same sums), three barriers in all; sh holds 32 N doubles
template <int N>
__device__ void block_sum_n(double (&v)[N], double *sh) {
    const int t = threadIdx.x + threadIdx.y * blockDim.x;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = warp_reduce<false>(v[i]);
    if ((t & 31) == 0)
#pragma unroll
        for (int i = 0; i < N; ++i) sh[32 * i + (t >> 5)] = v[i];
    __syncthreads();
    if (t < 32) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double r = (t < nw) ? sh[32 * i + t] : 0.0;
            r = warp_reduce<false>(r);
            v[i] = r;
        }
    }
    if (t == 0)   // (lane 0 read slot 32 i itself before; the other lanes read other slots)
#pragma unroll
        for (int i = 0; i < N; ++i) sh[32 * i] = v[i];
    __syncthreads();
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = sh[32 * i];
    __syncthreads();
}

// ------------------------------------------------------------ cfl

// cfl.F90 (fluid_tsch.F90:211-258) and the fixed-dt check fluid_tsch.F90:49-55.
// Both reductions (max for the CFL number, sum for the mean w) share one
// last-block pass so that a single block finalises them.
__device__ __forceinline__ void cfl_body(const Dev &d) {
    __shared__ double sh[32];
    __shared__ bool last;
    const int t = threadIdx.x, nt = blockDim.x;
    const int b = blockIdx.x, nb = gridDim.x;
    double qcf = 1.0e-8, q3a = 0.0;
    // rows k over the blocks, columns j over the threads (no index division);
    // kR rows (k, k + nb, ...) by kU columns of a thread per pass, their loads
    // all issued before the first use; a row's terms are summed before the
    // next row's (for rows of up to kU x blockDim columns, the per-thread
    // order of the sum is that of one value at a time)
    constexpr int kU = 4, kR = 2;
    for (int k0 = b + 1; k0 <= d.n3m; k0 += kR * nb) {
        double udx3[kR], dz[kR];
#pragma unroll
        for (int r = 0; r < kR; ++r) {
            const int k = min(k0 + r * nb, d.n3m);
            udx3[r] = d.udx3m[k];
            dz[r] = d.zz[k + 1] - d.zz[k];
        }
        for (int j0 = t + 1; j0 <= d.n2m; j0 += kU * nt) {
            double a2[kR][kU], b2[kR][kU], a3[kR][kU], b3[kR][kU], u2[kU], rj[kU], rjp[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int j = min(j0 + u * nt, d.n2m), jp = j + 1;
                u2[u] = d.udx2m[j];
                rj[u] = d.rc[j];
                rjp[u] = d.rc[jp];
#pragma unroll
                for (int r = 0; r < kR; ++r) {
                    const int k = min(k0 + r * nb, d.n3m);
                    a2[r][u] = Fv(d.q2, j, k);
                    b2[r][u] = Fv(d.q2, jp, k);
                    a3[r][u] = Fv(d.q3, j, k);
                    b3[r][u] = Fv(d.q3, j, k + 1);
                }
            }
#pragma unroll
            for (int r = 0; r < kR; ++r) {
                if (k0 + r * nb > d.n3m) break;
#pragma unroll
                for (int u = 0; u < kU; ++u) {
                    if (j0 + u * nt > d.n2m) break;
                    const double q = (fabs((a2[r][u] + b2[r][u]) * 0.5 * u2[u]) +
                                      fabs((a3[r][u] + b3[r][u]) * 0.5 * udx3[r]));
                    // fmax drops a NaN: a non-finite velocity turns into +inf, which
                    // every later fmax keeps, so the CFL test below catches it
                    qcf = fmax(qcf, (q == q) ? q : INFINITY);
                    q3a = q3a + a3[r][u] * dz[r] * (rjp[u] - rj[u]);
                }
            }
        }
    }
    const double pm = block_reduce_fast<true>(qcf, sh);
    const double ps = block_reduce_fast<false>(q3a, sh);
    double *rm = d.red, *rs = d.red + kRedSlot;
    if (t == 0) {
        rm[b] = pm;
        rs[b] = ps;
        __threadfence();
        last = (atomicAdd(d.count, 1u) == static_cast<unsigned>(nb - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double am = 1.0e-8, as = 0.0;
    for (int i = t; i < nb; i += nt) {
        am = fmax(am, __ldcg(rm + i));
        as = as + __ldcg(rs + i);
    }
    am = block_reduce_fast<true>(am, sh);
    as = block_reduce_fast<false>(as, sh);
    if (t == 0) {
        d.count[0] = 0u;
        const double cflm = am * d.dt;
        d.scal[S_CFLM] = cflm;
        d.scal[S_CFLRAW] = am;
        d.scal[S_Q3AVG] = as / (d.rext2 * d.alx3);
        // fixed dt: the stability check of fluid_tsch.F90:49-55; variable dt
        // is set from am on the host (fluid_tsch.F90:34-48)
        if (!d.vardt && !(cflm <= d.cfllim)) raise_status(d, FB_ERR_CFL);
    }
}

__global__ void __launch_bounds__(256) k_cfl(Dev d) {
    FB_GRID_WAIT();
    cfl_body(d);
}

// ------------------------------------------------------------ boundaries

// iobcs.F90:5-77 (boucdq): radiative outflow increments + mass-flux correction
__device__ __forceinline__ void boucdq_body(const Dev &d, double ga, double ro) {
    __shared__ double sh[32];
    const int n3 = d.n3, n3m = d.n3m;
    double qout = 0.0;
    for (int j = threadIdx.x + 1; j <= d.n2; j += blockDim.x) {
        d.dqb2s[j] = 0.0;
        d.dqb3s[j] = 0.0;
    }
    for (int j = threadIdx.x + 1; j <= d.n2m; j += blockDim.x) {
        double dq2x2 = (d.qb2n[j] - Fv(d.q2, j, n3m)) * 2.0 * d.udx3c[n3];
        double dqb2n = -d.dt * (ga * dq2x2 + ro * d.dq2x2o[j]) * d.cou;
        double dq3x2 = (d.qb3n[j] - Fv(d.q3, j, n3m)) * d.udx3c[n3];
        double dqb3n = -d.dt * (ga * dq3x2 + ro * d.dq3x2o[j]) * d.cou;
        d.dqb2n[j] = dqb2n;
        d.dqb3n[j] = dqb3n;
        d.dq2x2o[j] = dq2x2;
        d.dq3x2o[j] = dq3x2;
        qout = qout + dqb3n * (d.g2rm[j] / d.dx2);
    }
    double q = block_reduce_fast<false>(qout, sh);
    const double cor = (0.0 - q) / d.area_out;
    __syncthreads();
    for (int j = threadIdx.x + 1; j <= d.n2m; j += blockDim.x) d.dqb3n[j] = d.dqb3n[j] + cor;
}

__global__ void __launch_bounds__(1024) k_boucdq(Dev d, double ga, double ro) {
    FB_GRID_WAIT();
    boucdq_body(d, ga, ro);
}

// ------------------------------------------------------------ explicit terms

// HDNL.F90:5-171 (hdnl2, hdnl3) fused with INVTR.F90:4-280 (invtr2, invtr3).
// The convective terms stay in registers; ru2/ru3 receive them as the
// reference's invtr does (ru2 = dph, ru3 = qcap).  q2f/q3f are not stored:
// the forcing stage forms q + rhs at the few support nodes it reads.
// Tiles of kNlJ x kNlK cells: a block holds q2, q3 and pr of a tile plus a
// one-cell halo, and the tile's j and k coefficients, in shared memory, so
// each cell's stencil reads shared memory instead of issuing ~24 global
// loads.  Blocks are persistent over tiles with two buffers: the copies of
// the next tile (cp.async) and its ru2/ru3 (registers) are in flight while
// the current tile is computed.  Thread (tx, ty) of the 32 x 8 block computes
// the cells j = j0 + tx, k = k0 + 4 ty + i, i = 0..3 of a tile (consecutive
// rows share their stencil loads).
constexpr int kNlJ = 32, kNlK = 32, kNlS = kNlJ + 3;  // odd row stride
constexpr int kNlBlocksPerSM = 2;
struct NlTile {
    double q2[kNlK + 2][kNlS], q3[kNlK + 2][kNlS], pr[kNlK + 2][kNlS];  // rows k0-1.., cols j0-1..
    double udx3m[kNlK], ap3sk[kNlK], ac3sk[kNlK], am3sk[kNlK];           // k coefficients, rows k0..
    double udx3c[kNlK], ap3ck[kNlK], ac3ck[kNlK], am3ck[kNlK];
    double udx2c[kNlJ], am2j[kNlJ], ac2j[kNlJ], ap2j[kNlJ];              // j coefficients, columns j0..
    double udx2m[kNlJ], am3j[kNlJ], ac3j[kNlJ], ap3j[kNlJ];
};
constexpr size_t kNlSmem = 2 * sizeof(NlTile);

// The TMA-staged tile: one box per field of kNlTH rows (k0 - 1 .. k0 + 32) by
// kNlTW columns.  A box must start on a 16-byte boundary, so it starts one
// column left of the halo: column c holds j = j0 - 2 + c, and the stencil
// reads columns 1 .. 34.  Each field array starts on a 128-byte boundary.
constexpr int kNlTW = kNlJ + 4, kNlTH = kNlK + 2;
struct alignas(128) NlTileT {
    alignas(128) double q2[kNlTH][kNlTW];
    alignas(128) double q3[kNlTH][kNlTW];
    alignas(128) double pr[kNlTH][kNlTW];
    double udx3m[kNlK], ap3sk[kNlK], ac3sk[kNlK], am3sk[kNlK];
    double udx3c[kNlK], ap3ck[kNlK], ac3ck[kNlK], am3ck[kNlK];
    double udx2c[kNlJ], am2j[kNlJ], ac2j[kNlJ], ap2j[kNlJ];
    double udx2m[kNlJ], am3j[kNlJ], ac3j[kNlJ], ap3j[kNlJ];
};
constexpr uint32_t kNlBoxBytes = kNlTH * kNlTW * 8;
static_assert(kNlBoxBytes % 16 == 0 && (kNlTW * 8) % 16 == 0, "TMA box rows in 16-byte units");
// two tiles, their two mbarriers, and the slack to align the tiles to 128 bytes
constexpr size_t kNlSmemT = 2 * sizeof(NlTileT) + 128 + 128;

// ru2v, ru3v: ru2/ru3 at the cell, read before any cell of the thread is
// stored (0 when ro = 0)
// kC0: the tile column of j = j0 (1 for the cp.async tile, 2 for the TMA tile)
template <int kC0, class Tile>
__device__ __forceinline__ void nl_cell(const Dev &d, const Tile &t, int j0, int k0, int jc, int kc, double al,
                                        double ga, double ro, double ru2v, double ru3v) {
#define S2(j, k) t.q2[(k) - k0 + 1][(j) - j0 + kC0]
#define S3(j, k) t.q3[(k) - k0 + 1][(j) - j0 + kC0]
#define SP(j, k) t.pr[(k) - k0 + 1][(j) - j0 + kC0]
    const int n2m = d.n2m, n3m = d.n3m;
    const double dt = d.dt, alre = al / d.ren;

    // ---- v momentum at (jc, kc), jc = 2..n2m
    if (jc >= 2) {
        const int jm = jc - 1, jp = jc + 1;
        double h22 = ((S2(jp, kc) + S2(jc, kc)) * (S2(jp, kc) + S2(jc, kc)) -
                      (S2(jm, kc) + S2(jc, kc)) * (S2(jm, kc) + S2(jc, kc))) *
                     t.udx2c[jc - j0] * 0.25;
        double dph = -h22;
        const int jmv = jc - 1;  // jmv(jc) for jc >= 2
        if (kc >= 2 && kc <= n3m - 1) {
            const int kmm = kc - 1, kpp = kc + 1, kp = kc + 1;  // kmv, kpv in the interior
            double h23 = ((S3(jc, kp) + S3(jmv, kp)) * (S2(jc, kpp) + S2(jc, kc)) -
                          (S3(jc, kc) + S3(jmv, kc)) * (S2(jc, kc) + S2(jc, kmm))) *
                         t.udx3m[kc - k0] * 0.25;
            dph = dph - h23;
        } else if (kc == n3m) {
            const int kmm = kc - 1;
            double h23 = (d.qb2n[jc] * (d.qb3n[jc] + d.qb3n[jmv]) -
                          (S3(jc, kc) + S3(jmv, kc)) * (S2(jc, kc) + S2(jc, kmm)) * 0.5) *
                         t.udx3m[kc - k0] * 0.5;
            dph = dph - h23;
        }
        if (kc == 1) {
            const int kp = kc + 1;
            double h23 = ((S3(jc, kp) + S3(jmv, kp)) * (S2(jc, kc) + S2(jc, kp)) * 0.5 -
                          d.qb2s[jc] * (d.qb3s[jc] + d.qb3s[jmv])) *
                         t.udx3m[kc - k0] * 0.5;
            dph = dph - h23;
        }
        const double ammj = t.am2j[jc - j0], accj = t.ac2j[jc - j0], appj = t.ap2j[jc - j0];
        const double d22q2 = S2(jp, kc) * appj + S2(jc, kc) * accj + S2(jm, kc) * ammj;
        double d33q2, dpx22;
        if (kc >= 2 && kc <= n3m - 1) {
            const int km = kc - 1, kp = kc + 1;
            d33q2 = S2(jc, kp) * t.ap3sk[kc - k0] + S2(jc, kc) * t.ac3sk[kc - k0] + S2(jc, km) * t.am3sk[kc - k0];
            const double udx2 = al * t.udx2c[jc - j0];
            dpx22 = (SP(jc, kc) - SP(jm, kc)) * udx2;
        } else if (kc == 1) {
            const int kp = kc + 1;
            const double codea = d.dx3q / (d.g3rc[kp] * d.g3rm[kc]);
            const double codeb = d.dx3q / (d.g3rc[kc] * d.g3rm[kc]);
            d33q2 = ((S2(jc, kp) - S2(jc, kc)) * codea - (S2(jc, kc) - d.qb2s[jc]) * codeb * 2.0);
            dpx22 = (SP(jc, kc) - SP(jm, kc)) * t.udx2c[jc - j0] * al;
        } else {
            const int km = kc - 1, kp = kc + 1;
            const double codea = d.dx3q / (d.g3rc[kp] * d.g3rm[kc]);
            const double codeb = d.dx3q / (d.g3rc[kc] * d.g3rm[kc]);
            d33q2 = ((d.qb2n[jc] - S2(jc, kc)) * codea * 2.0 - (S2(jc, kc) - S2(jc, km)) * codeb);
            dpx22 = (SP(jc, kc) - SP(jm, kc)) * t.udx2c[jc - j0] * al;
        }
        const double dcq2 = d22q2 + d33q2;
        const size_t i = fidx(d, jc, kc);
        // the first RK3 substep has ro = 0: ru2 is not read (one field pass less)
        const double ru = ru2v;
        // global stores (st.global): the compiler then knows they do not
        // alias the shared-memory tile and reuses the tile loads across the
        // thread's consecutive cells
        __stcg(d.rhs2 + i, (ga * dph + ro * ru + alre * dcq2 - dpx22) * dt);
        __stcg(d.ru2 + i, dph);
    }

    // ---- w momentum at (jc, kc), kc = 2..n3m
    if (kc >= 2) {
        double qcap = 0.0;  // hdnl3 never writes kc = n3m (HDNL.F90:143)
        if (kc <= n3m - 1) {
            const int kmm = kc - 1, km = kc - 1, kp = kc + 1;
            const int jmm = jmv_(jc), jpp = jpv_(d, jc), jp = jc + 1;
            double h32 = (((S2(jp, kc) + S2(jp, km)) * (S3(jpp, kc) + S3(jc, kc))) -
                          ((S2(jc, kc) + S2(jc, km)) * (S3(jc, kc) + S3(jmm, kc)))) *
                         t.udx2m[jc - j0] * 0.25;
            double h33 = ((S3(jc, kp) + S3(jc, kc)) * (S3(jc, kp) + S3(jc, kc)) -
                          (S3(jc, kc) + S3(jc, kmm)) * (S3(jc, kc) + S3(jc, kmm))) *
                         t.udx3c[kc - k0] * 0.25;
            qcap = -(h32 + h33);
        }
        const int km = kc - 1, kp = kc + 1;
        const double udx3 = al * t.udx3c[kc - k0];
        const double ammj = t.am3j[jc - j0], accj = t.ac3j[jc - j0], appj = t.ap3j[jc - j0];
        double dq32;
        if (jc == 1) {
            dq32 = S3(jc + 1, kc) * appj + S3(jc, kc) * accj + d.q3lw * ammj;
        } else if (jc == n2m) {
            dq32 = d.q3uw * appj + S3(jc, kc) * accj + S3(jc - 1, kc) * ammj;
        } else {
            dq32 = S3(jpv_(d, jc), kc) * appj + S3(jc, kc) * accj + S3(jmv_(jc), kc) * ammj;
        }
        const double dq33 = S3(jc, kp) * t.ap3ck[kc - k0] + S3(jc, kc) * t.ac3ck[kc - k0] + S3(jc, km) * t.am3ck[kc - k0];
        const double dcq3 = dq32 + dq33;
        const double dpx33 = (SP(jc, kc) - SP(jc, km)) * udx3;
        const size_t i = fidx(d, jc, kc);
        const double ru = ru3v;
        __stcg(d.rhs3 + i, (ga * qcap + ro * ru + alre * dcq3 - dpx33) * dt);
        __stcg(d.ru3 + i, qcap);
    }
}
#undef S2
#undef S3
#undef SP

// the tile's coefficient vectors (cp.async), and the commit of the thread's
// cp.async group
template <class Tile>
__device__ __forceinline__ void nl_prefetch_coef(const Dev &d, Tile &t, int j0, int k0, int tid) {
    if (tid < kNlK) {
        const int k = min(k0 + tid, d.n3m);
        cp8(&t.udx3m[tid], d.udx3m + k);
        cp8(&t.ap3sk[tid], d.ap3sk + k);
        cp8(&t.ac3sk[tid], d.ac3sk + k);
        cp8(&t.am3sk[tid], d.am3sk + k);
        cp8(&t.udx3c[tid], d.udx3c + k);
        cp8(&t.ap3ck[tid], d.ap3ck + k);
        cp8(&t.ac3ck[tid], d.ac3ck + k);
        cp8(&t.am3ck[tid], d.am3ck + k);
    } else if (tid < kNlK + kNlJ) {
        const int c = tid - kNlK, j = min(j0 + c, d.n2m);
        cp8(&t.udx2c[c], d.udx2c + j);
        cp8(&t.am2j[c], d.am2j + j);
        cp8(&t.ac2j[c], d.ac2j + j);
        cp8(&t.ap2j[c], d.ap2j + j);
        cp8(&t.udx2m[c], d.udx2m + j);
        cp8(&t.am3j[c], d.am3j + j);
        cp8(&t.ac3j[c], d.ac3j + j);
        cp8(&t.ap3j[c], d.ap3j + j);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// issues the copies of one tile into t (one cp.async group per thread)
__device__ __forceinline__ void nl_prefetch(const Dev &d, NlTile &t, int tile, int ntj, int tid) {
    const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
    // tile + halo: j = j0-1 .. j0+kNlJ, k = k0-1 .. k0+kNlK (entries outside
    // the stored arrays, j < 1, j > n2, k > n3, are never read by a cell)
    constexpr int kW = kNlJ + 2, kH = kNlK + 2;
    for (int e = tid; e < kW * kH; e += 256) {
        const int r = e / kW, c = e % kW;
        const int j = j0 - 1 + c, k = k0 - 1 + r;
        if (j >= 1 && j <= d.n2 && k >= 0 && k <= d.n3) {
            const size_t i = fidx(d, j, k);
            cp8(&t.q2[r][c], d.q2 + i);
            cp8(&t.q3[r][c], d.q3 + i);
            cp8(&t.pr[r][c], d.pr + i);
        } else {
            t.q2[r][c] = 0.0;
            t.q3[r][c] = 0.0;
            t.pr[r][c] = 0.0;
        }
    }
    nl_prefetch_coef(d, t, j0, k0, tid);
}

// ru2/ru3 at this thread's cells of a tile (0 when ro = 0)
__device__ __forceinline__ void nl_ru(const Dev &d, int tile, int ntj, double ro, double (&r2)[kNlK / 8],
                                      double (&r3)[kNlK / 8]) {
    const int jc = 1 + (tile % ntj) * kNlJ + threadIdx.x, k0 = 1 + (tile / ntj) * kNlK;
#pragma unroll
    for (int i = 0; i < kNlK / 8; ++i) {
        const int kc = k0 + (kNlK / 8) * threadIdx.y + i;
        const bool ok = jc <= d.n2m && kc <= d.n3m && ro != 0.0;
        const size_t x = fidx(d, min(jc, d.n2m), min(kc, d.n3m));
        r2[i] = ok ? d.ru2[x] : 0.0;
        r3[i] = ok ? d.ru3[x] : 0.0;
    }
}

// tiles blockIdx.x, blockIdx.x + gridDim.x, ...; buf: two NlTile in shared memory
// pend: the previous substep's pressure mean (scal[S_PRAVG]) is still to be
// subtracted from pr (the fused step defers pr_submean of RK3 substeps 1 and
// 2): the staged tile gets pr - pravg, the value pr_submean would have stored.
__device__ __forceinline__ void nl_rhs_body(const Dev &d, double al, double ga, double ro, NlTile *buf,
                                            bool pend = false) {
    const double pravg = pend ? d.scal[S_PRAVG] : 0.0;
    const int ntj = (d.n2m + kNlJ - 1) / kNlJ, ntk = (d.n3m + kNlK - 1) / kNlK, ntiles = ntj * ntk;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    int tile = blockIdx.x;
    if (tile >= ntiles) return;
    nl_prefetch(d, buf[0], tile, ntj, tid);
    double r2n[kNlK / 8], r3n[kNlK / 8];
    nl_ru(d, tile, ntj, ro, r2n, r3n);
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        const NlTile &t = buf[it & 1];
        double r2[kNlK / 8], r3[kNlK / 8];
#pragma unroll
        for (int i = 0; i < kNlK / 8; ++i) {
            r2[i] = r2n[i];
            r3[i] = r3n[i];
        }
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) {
            nl_prefetch(d, buf[(it + 1) & 1], nxt, ntj, tid);
            nl_ru(d, nxt, ntj, ro, r2n, r3n);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        if (pend) {
            NlTile &tw = buf[it & 1];
            for (int e = tid; e < (kNlK + 2) * (kNlJ + 2); e += 256) {
                double &x = tw.pr[e / (kNlJ + 2)][e % (kNlJ + 2)];
                x = x - pravg;
            }
            __syncthreads();
        }
        const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
        const int jc = j0 + threadIdx.x;
        if (jc <= d.n2m) {
#pragma unroll
            for (int i = 0; i < kNlK / 8; ++i) {
                const int kc = k0 + (kNlK / 8) * threadIdx.y + i;
                if (kc > d.n3m) break;
                nl_cell<1>(d, t, j0, k0, jc, kc, al, ga, ro, r2[i], r3[i]);
            }
        }
        __syncthreads();   // this buffer is refilled two tiles on
    }
}

__global__ void __launch_bounds__(256, kNlBlocksPerSM) k_nl_rhs(Dev d, double al, double ga, double ro, int pend) {
    extern __shared__ __align__(16) unsigned char nl_smem[];
    FB_GRID_WAIT();
    nl_rhs_body(d, al, ga, ro, reinterpret_cast<NlTile *>(nl_smem), pend != 0);
}

// the three field boxes of a tile, issued by one thread on the buffer's
// mbarrier.  The proxy fence orders the threads' earlier reads (and the pend
// pass's writes) of this buffer before the copies overwrite it.  Boxes that
// reach past the fields (j < 1, j > n2, k > n3) are zero-filled there; no cell
// reads those entries.
__device__ __forceinline__ void nl_issue_tma(const NlMaps &m, NlTileT &t, uint32_t bar, int tile, int ntj) {
    const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
    const int x = j0 - 3, y = k0 - 1;   // x: element j - 1 of the column j = j0 - 2 (even: 16-byte aligned)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, 3u * kNlBoxBytes);
    tma_load_2d(smem_u32(&t.q2[0][0]), &m.q2, bar, x, y);
    tma_load_2d(smem_u32(&t.q3[0][0]), &m.q3, bar, x, y);
    tma_load_2d(smem_u32(&t.pr[0][0]), &m.pr, bar, x, y);
}

// nl_rhs_body with the field tiles staged by TMA: tile it waits on phase
// it / 2 of its buffer's mbarrier; the coefficient vectors stay cp.async.  A
// wait that gives up (one second) records FB_ERR_TIMEOUT and ends the block's
// tiles.
__device__ __forceinline__ void nl_rhs_tma_body(const Dev &d, const NlMaps &m, double al, double ga, double ro,
                                                NlTileT *buf, uint64_t *bars, bool pend) {
    const double pravg = pend ? d.scal[S_PRAVG] : 0.0;
    const int ntj = (d.n2m + kNlJ - 1) / kNlJ, ntk = (d.n3m + kNlK - 1) / kNlK, ntiles = ntj * ntk;
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    int tile = blockIdx.x;
    if (tile >= ntiles) return;
    const uint32_t bar0 = smem_u32(bars), bar1 = smem_u32(bars + 1);
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        nl_issue_tma(m, buf[0], bar0, tile, ntj);
    }
    {
        const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
        nl_prefetch_coef(d, buf[0], j0, k0, tid);
    }
    double r2n[kNlK / 8], r3n[kNlK / 8];
    nl_ru(d, tile, ntj, ro, r2n, r3n);
    __syncthreads();   // the barriers are initialised before any thread waits on them
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        NlTileT &t = buf[it & 1];
        double r2[kNlK / 8], r3[kNlK / 8];
#pragma unroll
        for (int i = 0; i < kNlK / 8; ++i) {
            r2[i] = r2n[i];
            r3[i] = r3n[i];
        }
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) {
            if (tid == 0) nl_issue_tma(m, buf[(it + 1) & 1], (it & 1) ? bar0 : bar1, nxt, ntj);
            nl_prefetch_coef(d, buf[(it + 1) & 1], 1 + (nxt % ntj) * kNlJ, 1 + (nxt / ntj) * kNlK, tid);
            nl_ru(d, nxt, ntj, ro, r2n, r3n);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        const bool landed = mbar_wait((it & 1) ? bar1 : bar0, static_cast<uint32_t>(it >> 1) & 1u);
        if (__syncthreads_or(!landed)) {
            if (tid == 0) atomicCAS(d.status, 0, FB_ERR_TIMEOUT);
            return;
        }
        if (pend) {
            for (int e = tid; e < kNlTH * kNlTW; e += 256) {
                double &x = t.pr[e / kNlTW][e % kNlTW];
                x = x - pravg;
            }
            __syncthreads();
        }
        const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
        const int jc = j0 + threadIdx.x;
        if (jc <= d.n2m) {
#pragma unroll
            for (int i = 0; i < kNlK / 8; ++i) {
                const int kc = k0 + (kNlK / 8) * threadIdx.y + i;
                if (kc > d.n3m) break;
                nl_cell<2>(d, t, j0, k0, jc, kc, al, ga, ro, r2[i], r3[i]);
            }
        }
        __syncthreads();   // this buffer is refilled two tiles on
    }
}

__global__ void __launch_bounds__(256, kNlBlocksPerSM)
    k_nl_rhs_tma(const __grid_constant__ Dev d, const __grid_constant__ NlMaps m, double al, double ga, double ro,
                 int pend) {
    extern __shared__ __align__(16) unsigned char nl_smem[];
    const uint32_t raw = smem_u32(nl_smem);
    unsigned char *base = nl_smem + ((128u - (raw & 127u)) & 127u);   // the tiles on 128-byte boundaries
    NlTileT *buf = reinterpret_cast<NlTileT *>(base);
    uint64_t *bars = reinterpret_cast<uint64_t *>(base + 2 * sizeof(NlTileT));
    FB_GRID_WAIT();
    nl_rhs_tma_body(d, m, al, ga, ro, buf, bars, pend != 0);
}

// ------------------------------------------------------------ MLS forcing

__device__ int nearest_sorted(const double *a, int lo, int hi, double x, int guess) {
    // first index of min |a(i) - x| over a(lo..hi), a strictly increasing.
    // The bracket a(l) <= x < a(l+1) is unique: it is searched from the
    // marker's index of the previous step (a few steps) and by bisection
    // when that guess is off; both give the same l.
    if (x <= a[lo]) return lo;
    if (x >= a[hi]) return hi;
    int l = -1;
    if (guess >= lo && guess < hi) {
        int g = guess;
        for (int s = 0; s < 16 && g > lo && a[g] > x; ++s) --g;
        for (int s = 0; s < 16 && g < hi - 1 && a[g + 1] <= x; ++s) ++g;
        if (a[g] <= x && x < a[g + 1]) l = g;
    }
    if (l < 0) {
        int h = hi;
        l = lo;
        while (h - l > 1) {
            int m = (l + h) >> 1;
            if (a[m] <= x) l = m;
            else h = m;
        }
    }
    const int h = l + 1;
    double dl = fabs(a[l] - x), dh = fabs(a[h] - x);
    return (dh < dl) ? h : l;
}

// entry of a spreading-table key (Fibonacci hashing: the top hlog bits of
// key x 2^64 / golden ratio)
__device__ __forceinline__ unsigned bucket_hash(unsigned long long key, int hlog) {
    return static_cast<unsigned>((key * 0x9E3779B97F4A7C15ull) >> (64 - hlog));
}

// lgrdistribution.F90:189-267: nearest nodes per marker and direction
__device__ __forceinline__ void lgrdist_body(const Dev &d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d.nlm) return;
    // empty the spreading-table entries this marker filled at the previous
    // step: every used entry is some marker's own entry, so the table is
    // empty again before the set-up fills it
    for (int dir = 0; dir < 2; ++dir) {
        const int e = d.hslot[2 * i + dir];
        if (e) {
            d.hkey[e - 1] = 0ull;
            d.hcnt[e - 1] = 0;
            d.hslot[2 * i + dir] = 0;
        }
    }
    const double y = d.lmcc[2 * i], z = d.lmcc[2 * i + 1];
    if (y > d.rext2 || y < 0.0 || z > d.alx3 || z < 0.0 || !(y == y) || !(z == z)) {
        raise_status(d, FB_ERR_MARKER_OUT);
        for (int c = 0; c < 4; ++c) d.lmind[4 * i + c] = -1;
        return;
    }
    int ind;
    const int g0 = d.lmind[4 * i + 0], g1 = d.lmind[4 * i + 1], g2 = d.lmind[4 * i + 2], g3 = d.lmind[4 * i + 3];
    d.lmind[4 * i + 0] = nearest_sorted(d.rc, 1, d.n2, y, g0);
    if (z < d.zm[1] && z > 0.0) ind = 1;
    else if (z > d.zm[d.n3m] && z < d.alx3) ind = d.n3m;
    else ind = nearest_sorted(d.zm, 1, d.n3, z, g1);
    d.lmind[4 * i + 1] = ind;
    if (y < d.rm[1] && y > 0.0) ind = 1;
    else if (y > d.rm[d.n2m] && y < d.rext2) ind = d.n2m;
    else ind = nearest_sorted(d.rm, 1, d.n2, y, g2);
    d.lmind[4 * i + 2] = ind;
    d.lmind[4 * i + 3] = nearest_sorted(d.zz, 1, d.n3, z, g3);
}

__global__ void k_lgrdist(Dev d) {
    FB_GRID_WAIT();
    lgrdist_body(d);
}

// utils_math.f90:637-725 (GEsolve), n = 3, scaled partial pivoting
__device__ __forceinline__ bool gesolve3(const double ai[3][3], const double bi[3], double x[3]) {
    // every loop unrolled and the row exchange written per candidate row, so
    // that the matrix stays in registers
    double a[3][3], b[3], s[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        b[i] = bi[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) a[i][j] = ai[i][j];
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
#pragma unroll
        for (int i = k; i < 3; ++i) {
            s[i] = 0.0;
#pragma unroll
            for (int j = k; j < 3; ++j) s[i] = fmax(s[i], fabs(a[i][j]));
        }
        double pivot = fabs(a[k][k] / s[k]);
        int l = k;
#pragma unroll
        for (int j = k + 1; j < 3; ++j) {
            double q = fabs(a[j][k] / s[j]);
            if (q > pivot) {
                pivot = q;
                l = j;
            }
        }
        if (pivot == 0.0) return false;
#pragma unroll
        for (int r = k + 1; r < 3; ++r) {
            if (l != r) continue;
#pragma unroll
            for (int j = k; j < 3; ++j) {
                double t = a[k][j];
                a[k][j] = a[r][j];
                a[r][j] = t;
            }
            double t = b[k];
            b[k] = b[r];
            b[r] = t;
        }
#pragma unroll
        for (int i = k + 1; i < 3; ++i) {
            double c = a[i][k] / a[k][k];
            a[i][k] = 0.0;
            b[i] = b[i] - c * b[k];
#pragma unroll
            for (int j = k + 1; j < 3; ++j) a[i][j] = a[i][j] - c * a[k][j];
        }
    }
    x[2] = b[2] / a[2][2];
#pragma unroll
    for (int i = 1; i >= 0; --i) {
        double c = 0.0;
#pragma unroll
        for (int j = i + 1; j < 3; ++j) c = c + a[i][j] * x[j];
        x[i] = (b[i] - c) / a[i][i];
    }
    return true;
}

// MLSint.F90:406-486 (one axis of the weight function) and its derivative
// MLSint.F90:492-593
__device__ void wkernel(int wfun, double difc, double sdds, double &wc, double &dw) {
    double drdc = (fabs(difc) <= 1.0e-20) ? 0.0 : (difc / fabs(difc)) / sdds;
    double rc = fabs(difc) / sdds;
    double rc2 = rc * rc, rc3 = rc * rc * rc, rc4 = rc * rc * rc * rc;
    wc = 0.0;
    dw = 0.0;
    if (wfun == 1) {
        if (rc > 1.0) {
        } else if (rc <= 0.5) {
            wc = (2.0 / 3.0) - 4.0 * rc2 + 4.0 * rc3;
            dw = (-8.0 * rc + 12.0 * rc2) * drdc;
        } else {
            wc = (4.0 / 3.0) - 4.0 * rc + 4.0 * rc2 - (4.0 / 3.0) * rc3;
            dw = (-4.0 + 8.0 * rc - 4.0 * rc2) * drdc;
        }
    } else if (wfun == 2) {
        if (rc <= 1.0) {
            double e = exp(-((rc / 0.3) * (rc / 0.3)));
            wc = e;
            dw = (-1.0 / (0.3 * 0.3) * 2.0 * rc * e) * drdc;
        }
    } else if (wfun == 3) {
        if (rc <= 1.0) {
            wc = 1.0 - 6.0 * rc2 + 8.0 * rc3 - 3.0 * rc4;
            dw = -12.0 * rc + 24.0 * rc2 - 12.0 * rc3;
        }
    } else if (wfun == 4) {
        if (rc > 1.0) {
        } else if (rc < 0.5) {
            wc = 1.0 / 3.0 * (1.0 + sqrt(-3.0 * rc2 + 1.0));
            dw = -rc * pow(-3.0 * rc2 - 1.0, -0.5);
        } else {
            wc = 1.0 / 6.0 * (5.0 - 3.0 * rc - sqrt(-3.0 * ((1.0 - rc) * (1.0 - rc)) + 1.0));
            dw = -(1.0 - rc) / (2.0 * sqrt(1.0 - 3.0 * ((1.0 - rc) * (1.0 - rc)))) - 0.5;
        }
    }
}

// Groups of kNodeLanes lanes work on one (marker, direction) each, support
// node m on lane m < kSD; a sum over the support is formed in node order from
// the group's shuffles (the sequential loop's sum).  Every lane of a warp
// reaches every shuffle: a group that stops (outside the channel, an error)
// carries on with its loads and stores switched off.
constexpr int kNodeLanes = 16;

// x summed over the group's first kSD lanes in lane order, on every lane
__device__ __forceinline__ double group_sum_nodes(double x, int base) {
    double s = 0.0;
#pragma unroll
    for (int mm = 0; mm < kSD; ++mm) s = s + __shfl_sync(0xffffffffu, x, base + mm);
    return s;
}

// the group's lane index of the least v, the first of equal values (as a
// sequential search with a strict comparison finds it); lanes past the
// searched range hold +inf
__device__ __forceinline__ int group_argmin(double v, int m) {
    int i = m;
#pragma unroll
    for (int o = kNodeLanes / 2; o; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (ov < v || (ov == v && oi < i)) {
            v = ov;
            i = oi;
        }
    }
    return i;
}

// true when no lane of the group (base .. base + kNodeLanes - 1) has flag set
__device__ __forceinline__ bool group_none(bool flag, int base) {
    return (__ballot_sync(0xffffffffu, flag) & (((1u << kNodeLanes) - 1u) << base)) == 0u;
}

// the support arrays of MLS_SD_ind (MLSint.F90:4-104) for direction idir
__device__ __forceinline__ void sd_axes(const Dev &d, int idir, const double *&y, int &dimy, const double *&z,
                                        int &dimz) {
    if (idir == 1) {
        y = d.rc; dimy = d.n2; z = d.zm; dimz = d.n3m;
    } else if (idir == 2) {
        y = d.rm; dimy = d.n2m; z = d.zz; dimz = d.n3;
    } else {
        y = d.rm; dimy = d.n2m; z = d.zm; dimz = d.n3m;
    }
}

// Marker set-up at substep 1: MLS_SD_ind + MLS_SF + momentum coefficient cl
// (forcing_MLS.F90:57-94, MLSint.F90:115-166, compute_AB :284-338), and the
// spreading keys.  One (marker, direction) per group of kNodeLanes lanes.
__device__ __forceinline__ void mls_setup_body(const Dev &d) {
    if (!d.nlm) return;
    const int T = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = T / kNodeLanes, m = T % kNodeLanes;
    const int base = (threadIdx.x & 31) & ~(kNodeLanes - 1);
    const bool have = t < 2 * d.nlm;
    const int tt = have ? t : 0;
    const int n = tt >> 1, idir = (tt & 1) + 1;
    const bool node = m < kSD;
    double *phi = d.phi + static_cast<size_t>(tt) * kSD;
    int *eu = d.eulins + static_cast<size_t>(tt) * 2 * kSD;
    if (have && node) phi[m] = 0.0;
    if (have && m == 0) d.cl[tt] = 0.0;
    const bool stopped = __shfl_sync(0xffffffffu, static_cast<int>(*d.status != 0), base) != 0;
    const double pos[2] = {d.lmcc[2 * n], d.lmcc[2 * n + 1]};
    const bool ok = have && !stopped && (d.zz[1] < pos[1] && pos[1] < d.zz[d.n3]);
    const int i0 = d.lmind[4 * n + 2 * (idir - 1)], k0 = d.lmind[4 * n + 2 * (idir - 1) + 1];
    // MLS_SD_ind: node m = 3 (j - 1) + (k - 1) of the 3 x 3 support, moved
    // inside the field
    const double *y, *z;
    int dimy, dimz;
    sd_axes(d, idir, y, dimy, z, dimz);
    const int sj = (i0 == 1) ? 1 : (i0 == d.n2m ? -1 : 0);
    const int sk = (k0 == 1) ? 1 : (k0 == d.n3m ? -1 : 0);
    const int mm = node ? m : 0;
    const int ej = i0 + (mm / 3 + 1 + sj) - 2, ek = k0 + (mm % 3 + 1 + sk) - 2;
    const bool bad = ok && node && (ej < 1 || ej + 1 > dimy || ek < 1 || ek + 1 > dimz);
    const bool good = group_none(bad, base) && ok && i0 >= 1 && k0 >= 1;
    if (ok && !good && m == 0) raise_status(d, FB_ERR_MARKER_OUT);
    double sc0 = 0.0, sc1 = 0.0, sd0 = 0.0, sd1 = 0.0, w = 0.0;
    if (good && node) {
        sc0 = y[ej];
        sd0 = y[ej + 1] - y[ej];
        sc1 = z[ek];
        sd1 = z[ek + 1] - z[ek];
        double wc0, wc1, dw;
        wkernel(d.wfun, pos[0] - sc0, d.radiusSD * sd0, wc0, dw);
        wkernel(d.wfun, pos[1] - sc1, d.radiusSD * sd1, wc1, dw);
        w = wc0 * wc1;
    }
    const double pk[3] = {1.0, sc0, sc1};
    double A[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b)   // pk[a] pk[b] = pk[b] pk[a]: the same terms, the same sums
            A[a][b] = (b < a) ? A[b][a] : group_sum_nodes(w * (pk[a] * pk[b]), base);
    const double gps[3] = {1.0, pos[0], pos[1]};
    double ptA[3];
    gesolve3(A, gps, ptA);
    const double B0 = 1.0 * w, B1 = sc0 * w, B2 = sc1 * w;
    double ph = 0.0;
    ph = ph + ptA[0] * B0;
    ph = ph + ptA[1] * B1;
    ph = ph + ptA[2] * B2;
    const double sumphi = group_sum_nodes(ph, base);
    if (good && m == 0 && !(fabs(1.0 - fabs(sumphi)) <= 1.0e-10)) raise_status(d, FB_ERR_MLS);
    const double vol = sd0 * sd1;
    const double dvel = group_sum_nodes(ph * vol, base);
    const double lgr_h = group_sum_nodes(1.0 / 2.0 * ph * (sd0 + sd1), base);
    if (!good) return;   // (after the group's last shuffle)
    if (node) {
        phi[m] = ph;
        eu[m] = ej;
        eu[kSD + m] = ek;
    }
    if (m != 0) return;
    d.cl[tt] = d.lmA[n] * lgr_h / dvel;
    // register the support box (start cell = node m = 0, this lane's) for the spreading
    const unsigned long long cell = static_cast<unsigned long long>(idir - 1) * d.NK * d.P + fidx(d, ej, ek);
    const unsigned mask = (1u << d.hlog) - 1u;
    for (int lev = 0; lev < kBucketLevels; ++lev) {
        const unsigned long long key = cell * kBucketLevels + lev + 1;
        unsigned h = bucket_hash(key, d.hlog);
        for (unsigned probes = 0;; ++probes) {   // find or claim the key's entry
            const unsigned long long prev = atomicCAS(d.hkey + h, 0ull, key);
            if (prev == 0ull || prev == key) break;
            if (probes == mask) {   // full: cannot happen at the table's sizing
                raise_status(d, FB_ERR_UNSUPPORTED);
                return;
            }
            h = (h + 1) & mask;
        }
        const int slot = atomicAdd(d.hcnt + h, 1);
        if (slot < kBucket) {
            d.hval[static_cast<size_t>(h) * kBucket + slot] = n;
            d.hslot[tt] = static_cast<int>(h) + 1;
            return;
        }
    }
    raise_status(d, FB_ERR_UNSUPPORTED);   // more than kBucket x kBucketLevels boxes start in one cell
}

__global__ void k_mls_setup(Dev d) {
    FB_GRID_WAIT();
    mls_setup_body(d);
}

// interp_spread (forcing_MLS.F90:135-182), interpolation half: the
// provisional velocity q* = q + rhs (INVTR.F90:147,275) at the support,
// direct forcing F = (V - u*)/dt and the per-node contributions cl*phi*F.
// One (marker, direction) per 16 lanes, node m on lane m < kSD: the nine
// support loads are independent, and each lane forms the sum of the nine
// products in node order from the group's shuffles (the sequential sum).
constexpr int kInterpLanes = 16;
__device__ __forceinline__ void mls_interp_body(const Dev &d) {
    const int T = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = T / kInterpLanes, m = T % kInterpLanes, lane = threadIdx.x & 31;
    const bool have = t < 2 * d.nlm;
    const bool stopped = (*d.status != 0);
    const int tt = have ? t : 0;
    const int n = tt >> 1, idir = (tt & 1) + 1;
    const double pos2 = d.lmcc[2 * n + 1];
    const bool inside = (d.zz[1] < pos2 && pos2 < d.zz[d.n3]);
    double phim = 0.0, prod = 0.0;
    if (have && inside && m < kSD) {
        const int *eu = d.eulins + static_cast<size_t>(tt) * 2 * kSD;
        const double *q = (idir == 1) ? d.q2 : d.q3;
        const double *r = (idir == 1) ? d.rhs2 : d.rhs3;
        phim = d.phi[static_cast<size_t>(tt) * kSD + m];
        const int j = eu[m], k = eu[kSD + m];
        // q2f/q3f are written only where invtr2/invtr3 write them; elsewhere
        // the reference reads storage that was never set (zero here)
        const bool written = (idir == 1) ? (j >= 2 && j <= d.n2m && k >= 1 && k <= d.n3m)
                                         : (j >= 1 && j <= d.n2m && k >= 2 && k <= d.n3m);
        double qf = 0.0;
        if (written) {
            const size_t i = fidx(d, j, k);
            qf = q[i] + r[i];
        }
        prod = phim * qf;
    }
    double u = 0.0;
#pragma unroll
    for (int mm = 0; mm < kSD; ++mm) u = u + __shfl_sync(0xffffffffu, prod, (lane & ~(kInterpLanes - 1)) + mm);
    if (!have || stopped || m >= kSD) return;
    double *c = d.contrib + static_cast<size_t>(tt) * kSD;
    if (!inside) {
        c[m] = 0.0;
        return;
    }
    const double f = (d.lmvel[2 * n + idir - 1] - u) / d.dt;
    c[m] = d.cl[tt] * phim * f;
}

__global__ void k_mls_interp(Dev d) {
    FB_GRID_WAIT();
    mls_interp_body(d);
}

// interp_spread, spreading half, without atomics on the field.  Once per
// step (the supports are fixed for the three substeps) every cell's touchers
// are found in the buckets of the 3 x 3 possible box start cells and chained
// in increasing marker index (the reference's loop order,
// forcing_MLS.F90:51-104); the head of each chain is the lowest-index
// toucher.  Every substep the heads then add their chain's sum fe*dt to rhs
// (helsolve.F90:22,47).
__device__ __forceinline__ void spread_chains_body(const Dev &d) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 2 * d.nlm * kSD) return;
    d.chead[g] = 0;
    if (*d.status) return;
    const int t = g / kSD, m = g % kSD, n = t >> 1, dir = t & 1;
    const double pos2 = d.lmcc[2 * n + 1];
    if (!(d.zz[1] < pos2 && pos2 < d.zz[d.n3])) return;
    const int *eu = d.eulins + static_cast<size_t>(t) * 2 * kSD;
    const int j = eu[m], k = eu[kSD + m];
    // cells helsolve reads: v at j = 2..n2m, k = 1..n3m; w at j = 1..n2m, k = 2..n3m
    const bool used = (dir == 0) ? (j >= 2 && j <= d.n2m && k >= 1 && k <= d.n3m)
                                 : (j >= 1 && j <= d.n2m && k >= 2 && k <= d.n3m);
    if (!used) return;
    const size_t plane = static_cast<size_t>(dir) * d.NK * d.P;
    // the cell's touchers are the markers registered at the 3 x 3 possible
    // box start cells (table lookups); a lower-index toucher means this slot
    // is not the head
    constexpr int kMaxTouch = 9 * kBucket;   // touchers of one cell kept at most
    int ln[kMaxTouch], ls[kMaxTouch];         // touchers after n, ascending marker index
    int L = 0;
    bool over = false;
    const unsigned mask = (1u << d.hlog) - 1u;
    for (int q = 0; q < 9; ++q) {
        const int sj = j - q / 3, sk = k - q % 3;
        if (sj < 1 || sk < 0) continue;
        const unsigned long long cell = plane + fidx(d, sj, sk);
        for (int lev = 0; lev < kBucketLevels; ++lev) {
            const unsigned long long key = cell * kBucketLevels + lev + 1;
            unsigned h = bucket_hash(key, d.hlog);
            unsigned long long kh = d.hkey[h];
            for (unsigned probes = 0; kh != key && kh != 0ull && probes < mask; ++probes) {
                h = (h + 1) & mask;
                kh = d.hkey[h];
            }
            if (kh != key) break;   // no (further) boxes start in this cell
            const int cnt = d.hcnt[h];
            for (int e = 0; e < min(cnt, kBucket); ++e) {
                const int nn = d.hval[static_cast<size_t>(h) * kBucket + e];
                if (nn < n) return;
                if (nn == n) continue;
                if (L >= kMaxTouch) {   // denser than the marker spacing the spreading is built for
                    over = true;
                    continue;
                }
                // insertion in increasing marker index (a marker has one box start cell)
                int p = L++;
                while (p > 0 && ln[p - 1] > nn) {
                    ln[p] = ln[p - 1];
                    ls[p] = ls[p - 1];
                    --p;
                }
                ln[p] = nn;
                ls[p] = (2 * nn + dir) * kSD + q;   // node (dj, dk) = (q / 3, q % 3) of marker nn
            }
            if (cnt <= kBucket) break;   // the cell's last entry
        }
    }
    if (over) {
        raise_status(d, FB_ERR_UNSUPPORTED);
        return;
    }
    // this slot heads the cell's chain: link the touchers in marker order;
    // the head also keeps the first kHeadList of them in line
    d.chead[g] = 1;
    int prev_slot = g;
    for (int p = 0; p < L; ++p) {
        d.chain[prev_slot] = ls[p];
        prev_slot = ls[p];
    }
    d.chain[prev_slot] = -1;
    d.hlen[g] = L;
    int *hl = d.hlist + static_cast<size_t>(g) * kHeadList;
    for (int p = 0; p < kHeadList; ++p) hl[p] = (p < L) ? ls[p] : g;
}

__global__ void k_spread_chains(Dev d) {
    FB_GRID_WAIT();
    spread_chains_body(d);
}

__device__ __forceinline__ void mls_spread_body(const Dev &d) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 2 * d.nlm * kSD) return;
    if (*d.status) return;
    if (!d.chead[g]) return;  // not the head of a cell's chain
    const int t = g / kSD, dir = t & 1;
    const int *eu = d.eulins + static_cast<size_t>(t) * 2 * kSD;
    const int m = g % kSD;
    // the head's in-line list gives the first kHeadList members at once
    // (independent loads); a longer chain continues along chain[]; the sum
    // runs in chain order
    const int L = d.hlen[g];
    const int4 *hl = reinterpret_cast<const int4 *>(d.hlist + static_cast<size_t>(g) * kHeadList);
    const int4 h0 = hl[0], h1 = hl[1];
    const int idx[kHeadList] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
    double cv[kHeadList];
#pragma unroll
    for (int p = 0; p < kHeadList; ++p) cv[p] = d.contrib[idx[p]];   // the head's own slot past the end
    double fe = 0.0;
    fe = fe + d.contrib[g];
#pragma unroll
    for (int p = 0; p < kHeadList; ++p)
        if (p < L) fe = fe + cv[p];
    if (L > kHeadList)
        for (int s = d.chain[idx[kHeadList - 1]]; s >= 0; s = d.chain[s]) fe = fe + d.contrib[s];
    double *r = (dir == 0) ? d.rhs2 : d.rhs3;
    const size_t i = fidx(d, eu[m], eu[kSD + m]);
    r[i] = r[i] + fe * d.dt;
}

__global__ void k_mls_spread(Dev d) {
    FB_GRID_WAIT();
    mls_spread_body(d);
}

// ------------------------------------------------------------ tridiagonal

// DGTTS2 (LAPACK) for one line with precomputed DGTTRF factors; b strided.
// The pivots are stored as reciprocals, so the back substitution multiplies.
__device__ __forceinline__ void gtts2(const TriDev &f, size_t off, double *b, size_t s) {
    const int n = f.n;
    const double *dl = f.dl + off, *dinv = f.dinv + off, *du = f.du + off, *du2 = f.du2 + off;
    if (!f.pivoted) {
        double prev = b[0];
        for (int i = 0; i < n - 1; ++i) {
            double cur = b[(i + 1) * s] - dl[i] * prev;
            b[(i + 1) * s] = cur;
            prev = cur;
        }
        double x1 = b[(n - 1) * s] * dinv[n - 1];
        b[(n - 1) * s] = x1;
        for (int i = n - 2; i >= 0; --i) {
            double x0 = (b[i * s] - du[i] * x1) * dinv[i];
            b[i * s] = x0;
            x1 = x0;
        }
    } else {
        const int *ipiv = f.ipiv + off;
        for (int i = 0; i < n - 1; ++i) {
            if (ipiv[i] == i + 1) {
                b[(i + 1) * s] = b[(i + 1) * s] - dl[i] * b[i * s];
            } else {
                double temp = b[i * s] - dl[i] * b[(i + 1) * s];
                b[i * s] = b[(i + 1) * s];
                b[(i + 1) * s] = temp;
            }
        }
        b[(n - 1) * s] = b[(n - 1) * s] * dinv[n - 1];
        if (n > 1) b[(n - 2) * s] = (b[(n - 2) * s] - du[n - 2] * b[(n - 1) * s]) * dinv[n - 2];
        for (int i = n - 3; i >= 0; --i)
            b[i * s] = (b[i * s] - du[i] * b[(i + 1) * s] - du2[i] * b[(i + 2) * s]) * dinv[i];
    }
}

// solve_fluid.F90:110-160 (solq2j): v, y lines of n2 unknowns, k = 1..n3m
__global__ void k_tri_y2(Dev d, SubDev s) {
    FB_GRID_WAIT();
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (k > d.n3m) return;
    double *b = d.rhs2 + fidx(d, 1, k);
    b[0] = 0.0;
    for (int j = 2; j <= d.n2m; ++j) b[j - 1] = b[j - 1] * s.by2[j];
    b[d.n2 - 1] = 0.0;
    gtts2(s.y2, 0, b, 1);
}

// solve_fluid.F90:164-229 (solq2k) then helsolve.F90:32-33: v, z lines of
// n3m unknowns with the inflow/outflow terms, q2 += x, wall columns zeroed
__global__ void k_tri_z2(Dev d, SubDev s) {
    FB_GRID_WAIT();
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > d.n2m) return;
    if (j == 1) {
        for (int k = 0; k <= d.n3; ++k) {
            Fv(d.q2, 1, k) = 0.0;
            Fv(d.q2, d.n2, k) = 0.0;
        }
        return;
    }
    double *b = d.rhs2 + fidx(d, j, 1);
    const size_t P = static_cast<size_t>(d.P);
    for (int k = 1; k <= d.n3m; ++k) b[(k - 1) * P] = b[(k - 1) * P] * s.bz2[k];
    b[0] = b[0] + d.dqb2s[j] * s.ugkks;
    b[(d.n3m - 1) * P] = b[(d.n3m - 1) * P] + d.dqb2n[j] * s.ugkkn;
    gtts2(s.z2, 0, b, P);
    for (int k = 1; k <= d.n3m; ++k) Fv(d.q2, j, k) = Fv(d.q2, j, k) + b[(k - 1) * P];
}

// solve_fluid.F90:61-104 (solq3j): w, y lines of n2m unknowns, k = 2..n3m
// (the k = 1 line of the reference is overwritten by solq3k and skipped)
__global__ void k_tri_y3(Dev d, SubDev s) {
    FB_GRID_WAIT();
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 2;
    if (k > d.n3m) return;
    double *b = d.rhs3 + fidx(d, 1, k);
    for (int j = 1; j <= d.n2m; ++j) b[j - 1] = b[j - 1] * s.by3[j];
    gtts2(s.y3, 0, b, 1);
}

// solve_fluid.F90:233-312 (solq3k): w, z lines of n3 unknowns with
// Dirichlet end rows, q3 += x, outflow row advanced by dqb3n
__global__ void k_tri_z3(Dev d, SubDev s) {
    FB_GRID_WAIT();
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (j > d.n2m) return;
    double *b = d.rhs3 + fidx(d, j, 1);
    const size_t P = static_cast<size_t>(d.P);
    b[0] = d.dqb3s[j];
    for (int k = 2; k <= d.n3m; ++k) b[(k - 1) * P] = b[(k - 1) * P] * s.bz3[k];
    b[(d.n3 - 1) * P] = d.dqb3n[j];
    gtts2(s.z3, 0, b, P);
    for (int k = 1; k <= d.n3m; ++k) Fv(d.q3, j, k) = Fv(d.q3, j, k) + b[(k - 1) * P];
    Fv(d.q3, j, d.n3) = Fv(d.q3, j, d.n3) + d.dqb3n[j];
}

// ------------------------------------------------------------ Poisson

// divergence.F90:88-115 (divg)
// Blocks of 32 x 8 threads over 32 x (8 kDivK) cells: thread (x, y) takes j0 + x
// and the rows k0 + y + 8 i.  rmax (may be null): the maxima of |dph| over
// each row j (the rows of the INT8 transform's data operand) are accumulated
// into rmax[j - 1], one atomic per block and row, for the digit cut that follows
constexpr int kDivK = 4;
__device__ __forceinline__ void divg_body(const Dev &d, double usdtal, double *rmax = nullptr) {
    const int jc = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int kb = blockIdx.y * blockDim.y * kDivK + threadIdx.y + 1;
    double m = 0.0;
    if (jc <= d.n2m) {
#pragma unroll
        for (int i = 0; i < kDivK; ++i) {
            const int kc = kb + static_cast<int>(blockDim.y) * i;
            if (kc > d.n3m) break;
            const double dqcap = (Fv(d.q2, jc + 1, kc) - Fv(d.q2, jc, kc)) * d.udx2m[jc] +
                                 (Fv(d.q3, jc, kc + 1) - Fv(d.q3, jc, kc)) * d.udx3m[kc];
            const double v = dqcap * usdtal;
            Fv(d.dph, jc, kc) = v;
            m = fmax(m, fabs(v));   // fmax drops a NaN, as the cut's maximum does
        }
    }
    if (!rmax) return;
    __shared__ double part[8][32];
    part[threadIdx.y][threadIdx.x] = m;
    __syncthreads();
    if (threadIdx.y == 0 && jc <= d.n2m) {
        for (int q = 1; q < 8; ++q) m = fmax(m, part[q][threadIdx.x]);
        if (m > 0.0) atomic_max_nonneg(rmax + jc - 1, m);
    }
}

__global__ void k_divg(Dev d, double usdtal, double *rmax) {
    FB_GRID_WAIT();
    divg_body(d, usdtal, rmax);
}

// updvp.F90:5-59 (updvp) fused with updvp.F90:68-105 (prcalc) and the
// partial sums of pr_submean (updvp.F90:320-333).  Tiles of kNlJ x kNlK cells
// as in nl_rhs: dph with its halo in shared memory; the block partial sums
// of the pressure mean are finished by the case's last block.
struct UpTile {
    double dph[kNlK + 2][kNlS];   // dph tile + one-cell halo (rows k0-1.., cols j0-1..)
    double kc[6][kNlK];           // udx3c, apphk, acphk, amphk, zz(k), zz(k+1) at rows k0..
    double jc[6][kNlJ];           // udx2c, apphj, acphj, amphj, rc(j), rc(j+1) at columns j0..
};
constexpr size_t kUpSmem = 2 * sizeof(UpTile);
constexpr int kUpBlocksPerSM = 3;

// the TMA-staged form: the dph box of kNlTH x kNlTW (column c holds j = j0 - 2 + c)
struct alignas(128) UpTileT {
    alignas(128) double dph[kNlTH][kNlTW];
    double kc[6][kNlK];
    double jc[6][kNlJ];
};
constexpr size_t kUpSmemT = 2 * sizeof(UpTileT) + 128 + 128;   // tiles, two mbarriers, alignment slack

// the dph box of a tile, issued by one thread (see nl_issue_tma)
__device__ __forceinline__ void up_issue_tma(const NlMaps &m, UpTileT &t, uint32_t bar, int tile, int ntj) {
    const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, kNlBoxBytes);
    tma_load_2d(smem_u32(&t.dph[0][0]), &m.dph, bar, j0 - 3, k0 - 1);
}

// the tile's coefficient vectors (cp.async) and the commit of the thread's group
template <class Tile>
__device__ __forceinline__ void up_prefetch_coef(const Dev &d, Tile &t, int j0, int k0, int tid) {
    if (tid < kNlK) {
        const int k = min(k0 + tid, d.n3m);
        cp8(&t.kc[0][tid], d.udx3c + k);
        cp8(&t.kc[1][tid], d.apphk + k);
        cp8(&t.kc[2][tid], d.acphk + k);
        cp8(&t.kc[3][tid], d.amphk + k);
        cp8(&t.kc[4][tid], d.zz + k);
        cp8(&t.kc[5][tid], d.zz + k + 1);
    } else if (tid < kNlK + kNlJ) {
        const int c = tid - kNlK, j = min(j0 + c, d.n2m);
        cp8(&t.jc[0][c], d.udx2c + j);
        cp8(&t.jc[1][c], d.apphj + j);
        cp8(&t.jc[2][c], d.acphj + j);
        cp8(&t.jc[3][c], d.amphj + j);
        cp8(&t.jc[4][c], d.rc + j);
        cp8(&t.jc[5][c], d.rc + j + 1);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void up_prefetch(const Dev &d, UpTile &t, int tile, int ntj, int tid) {
    const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
    constexpr int kW = kNlJ + 2, kH = kNlK + 2;
    for (int e = tid; e < kW * kH; e += 256) {
        const int r = e / kW, c = e % kW;
        const int j = j0 - 1 + c, k = k0 - 1 + r;
        if (j >= 1 && j <= d.n2 && k >= 0 && k <= d.n3) cp8(&t.dph[r][c], d.dph + fidx(d, j, k));
        else t.dph[r][c] = 0.0;
    }
    up_prefetch_coef(d, t, j0, k0, tid);
}

// q2, q3, pr at this thread's cells of a tile, read before any is written
__device__ __forceinline__ void up_own(const Dev &d, int tile, int ntj, double (&q2)[kNlK / 8], double (&q3)[kNlK / 8],
                                       double (&pr)[kNlK / 8]) {
    const int jc = 1 + (tile % ntj) * kNlJ + threadIdx.x, k0 = 1 + (tile / ntj) * kNlK;
#pragma unroll
    for (int i = 0; i < kNlK / 8; ++i) {
        const int kc = k0 + threadIdx.y + 8 * i;
        const bool ok = jc <= d.n2m && kc <= d.n3m;
        const size_t x = fidx(d, min(jc, d.n2m), min(kc, d.n3m));
        q2[i] = ok ? d.q2[x] : 0.0;
        q3[i] = ok ? d.q3[x] : 0.0;
        pr[i] = ok ? d.pr[x] : 0.0;
    }
}

// pend: as for nl_rhs, pr - pravg of the previous substep is the pressure
// this update starts from (read before this grid's last block stores the new
// mean).  kTma: the dph tiles are TMA boxes on the mbarriers bars (maps m);
// a wait that gives up records FB_ERR_TIMEOUT and ends the block's tiles (the
// block still takes part in the mean)
template <bool kTma, class Tile>
__device__ __forceinline__ void updvp_prcalc_body(const Dev &d, double al, double be, Tile *buf, bool pend = false,
                                                  const NlMaps *m = nullptr, uint64_t *bars = nullptr) {
    __shared__ double sh[32];
    __shared__ bool last;
    constexpr int kC0 = kTma ? 2 : 1;   // the tile column of j = j0
    const double pravg = pend ? d.scal[S_PRAVG] : 0.0;
    const int ntj = (d.n2m + kNlJ - 1) / kNlJ, ntk = (d.n3m + kNlK - 1) / kNlK, ntiles = ntj * ntk;
    const int t = threadIdx.x + blockDim.x * threadIdx.y, nt = blockDim.x * blockDim.y;
    const int b = blockIdx.x, nb = gridDim.x;
    constexpr int kC = kNlK / 8;
    double part = 0.0;
    int tile = blockIdx.x;
    double q2n[kC], q3n[kC], prn[kC];
    uint32_t bar0 = 0, bar1 = 0;
    if constexpr (kTma) {
        bar0 = smem_u32(bars);
        bar1 = smem_u32(bars + 1);
    }
    if (tile < ntiles) {
        if constexpr (kTma) {
            if (t == 0) {
                mbar_init(bar0, 1);
                mbar_init(bar1, 1);
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
                up_issue_tma(*m, buf[0], bar0, tile, ntj);
            }
            up_prefetch_coef(d, buf[0], 1 + (tile % ntj) * kNlJ, 1 + (tile / ntj) * kNlK, t);
            __syncthreads();   // the barriers are initialised before any thread waits on them
        } else {
            up_prefetch(d, buf[0], tile, ntj, t);
        }
        up_own(d, tile, ntj, q2n, q3n, prn);
    }
    for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
        const Tile &u = buf[it & 1];
        double q2v[kC], q3v[kC], prv[kC];
#pragma unroll
        for (int i = 0; i < kC; ++i) {
            q2v[i] = q2n[i];
            q3v[i] = q3n[i];
            prv[i] = prn[i];
        }
        const int nxt = tile + gridDim.x;
        if (nxt < ntiles) {
            if constexpr (kTma) {
                if (t == 0) up_issue_tma(*m, buf[(it + 1) & 1], (it & 1) ? bar0 : bar1, nxt, ntj);
                up_prefetch_coef(d, buf[(it + 1) & 1], 1 + (nxt % ntj) * kNlJ, 1 + (nxt / ntj) * kNlK, t);
            } else {
                up_prefetch(d, buf[(it + 1) & 1], nxt, ntj, t);
            }
            up_own(d, nxt, ntj, q2n, q3n, prn);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        if constexpr (kTma) {
            const bool landed = mbar_wait((it & 1) ? bar1 : bar0, static_cast<uint32_t>(it >> 1) & 1u);
            if (__syncthreads_or(!landed)) {
                if (t == 0) atomicCAS(d.status, 0, FB_ERR_TIMEOUT);
                break;
            }
        } else {
            __syncthreads();
        }
        const int j0 = 1 + (tile % ntj) * kNlJ, k0 = 1 + (tile / ntj) * kNlK;
        const int jc = j0 + threadIdx.x;
#define TD(j, k) u.dph[(k) - k0 + 1][(j) - j0 + kC0]
        if (jc <= d.n2m) {
            const int cj = jc - j0;
            const int jm = jmv_(jc), jp = jpv_(d, jc);
            const double usujm = al * d.dt * u.jc[0][cj];
            const double apj = u.jc[1][cj], acj = u.jc[2][cj], amj = u.jc[3][cj];
            const double dyc = u.jc[5][cj] - u.jc[4][cj];
#pragma unroll
            for (int i = 0; i < kC; ++i) {
                const int kc = k0 + threadIdx.y + 8 * i;
                if (kc > d.n3m) break;
                const int r = kc - k0;
                const double locdph = TD(jc, kc);
                Fv(d.q2, jc, kc) = q2v[i] - (locdph - TD(jm, kc)) * usujm;
                if (kc >= 2) {
                    const double usukm = al * d.dt * u.kc[0][r];
                    Fv(d.q3, jc, kc) = q3v[i] - (TD(jc, kc) - TD(jc, kc - 1)) * usukm;
                }
                const int kp = kpv_(d, kc), km = kmv_(kc);
                const double pr0 = pend ? prv[i] - pravg : prv[i];
                const double p = pr0 + TD(jc, kc) -
                                 be * ((TD(jp, kc) * apj + TD(jc, kc) * acj + TD(jm, kc) * amj) +
                                       (TD(jc, kp) * u.kc[1][r] + TD(jc, kc) * u.kc[2][r] + TD(jc, km) * u.kc[3][r]));
                Fv(d.pr, jc, kc) = p;
                part = part + p * (u.kc[5][r] - u.kc[4][r]) * dyc;
            }
        }
#undef TD
        __syncthreads();   // this buffer is refilled two tiles on
    }
    const double bsum = block_reduce_fast<false>(part, sh);
    double *red = d.red + 2 * static_cast<size_t>(kRedSlot);
    if (t == 0) {
        red[b] = bsum;
        __threadfence();
        last = (atomicAdd(d.count + 2, 1u) == static_cast<unsigned>(nb - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double acc = 0.0;
    for (int i = t; i < nb; i += nt) acc = acc + __ldcg(red + i);
    acc = block_reduce_fast<false>(acc, sh);
    if (t == 0) {
        d.count[2] = 0u;
        d.scal[S_PRAVG] = acc / (d.rext2 * d.alx3);
    }
}

__global__ void __launch_bounds__(256, kUpBlocksPerSM) k_updvp_prcalc(Dev d, double al, double be, int pend) {
    extern __shared__ __align__(16) unsigned char up_smem[];
    FB_GRID_WAIT();
    updvp_prcalc_body<false>(d, al, be, reinterpret_cast<UpTile *>(up_smem), pend != 0);
}

__global__ void __launch_bounds__(256, kUpBlocksPerSM)
    k_updvp_prcalc_tma(const __grid_constant__ Dev d, const __grid_constant__ NlMaps m, double al, double be,
                       int pend) {
    extern __shared__ __align__(16) unsigned char up_smem[];
    const uint32_t raw = smem_u32(up_smem);
    unsigned char *base = up_smem + ((128u - (raw & 127u)) & 127u);   // the tiles on 128-byte boundaries
    FB_GRID_WAIT();
    updvp_prcalc_body<true>(d, al, be, reinterpret_cast<UpTileT *>(base), pend != 0, &m,
                            reinterpret_cast<uint64_t *>(base + 2 * sizeof(UpTileT)));
}

// pr_submean (updvp.F90:336: the whole array) and boucqt (iobcs.F90:97-105)
// deferred: the means of RK3 substeps 1 and 2 were applied to the cells that
// updvp rewrites (j <= n2m, 1 <= k <= n3m) as it read them; the other
// entries of the array get all three subtractions here, in order.
__device__ __forceinline__ void submean_boucqt_body(const Dev &d, bool deferred = false) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int k = blockIdx.y * blockDim.y + threadIdx.y;
    const double pravg = d.scal[S_PRAVG];
    if (j <= d.n2 && k <= d.n3) {
        double p = Fv(d.pr, j, k);
        if (deferred && (j > d.n2m || k < 1 || k > d.n3m)) p = (p - d.scal[S_PRAVG1]) - d.scal[S_PRAVG2];
        Fv(d.pr, j, k) = p - pravg;
    }
    if (blockIdx.y == 0 && threadIdx.y == 0 && j <= d.n2m) {
        d.qb2s[j] = d.qb2s[j] + d.dqb2s[j];
        d.qb3s[j] = d.qb3s[j] + d.dqb3s[j];
        d.qb2n[j] = d.qb2n[j] + d.dqb2n[j];
        d.qb3n[j] = d.qb3n[j] + d.dqb3n[j];
    }
}

__global__ void k_submean_boucqt(Dev d, int deferred) {
    FB_GRID_WAIT();
    submean_boucqt_body(d, deferred != 0);
}

// The end of RK3 substep 1 or 2 in the fused step: boucqt (iobcs.F90:97-105),
// the substep's pressure mean kept in slot for the final pr_submean, then
// boucdq of the next substep (iobcs.F90:5-77) in the same block.  The mean
// itself is subtracted by the next nl_rhs and updvp as they read pr.
__device__ __forceinline__ void substep_mid_body(const Dev &d, int slot, double ga, double ro) {
    for (int j = threadIdx.x + 1; j <= d.n2m; j += blockDim.x) {
        d.qb2s[j] = d.qb2s[j] + d.dqb2s[j];
        d.qb3s[j] = d.qb3s[j] + d.dqb3s[j];
        d.qb2n[j] = d.qb2n[j] + d.dqb2n[j];
        d.qb3n[j] = d.qb3n[j] + d.dqb3n[j];
    }
    if (threadIdx.x == 0) d.scal[slot] = d.scal[S_PRAVG];
    __syncthreads();
    boucdq_body(d, ga, ro);
}

__global__ void __launch_bounds__(1024) k_substep_mid(Dev d, int slot, double ga, double ro) {
    FB_GRID_WAIT();
    substep_mid_body(d, slot, ga, ro);
}

// ------------------------------------------------------------ loads

// loads_transfer_c (loads_transfer.F90:143-185), per-marker part: the probe
// interpolation of v, w or p with first and second derivatives; the v and w
// groups also form checkbcs (ckbcs.F90:29-60) with the substep-1 weights.
// One (marker, quantity) per group of kLoadLanes lanes, support node m on
// lane m < kSD: the nodes' weights, moment terms and field reads are
// independent, and every sum over the nodes is formed in node order from the
// group's shuffles, so each result is that of the sequential loops.  Every
// lane of a warp reaches every shuffle: a group that stops (outside the
// channel, an error) carries on with its loads and stores switched off.
constexpr int kLoadLanes = kNodeLanes;
constexpr int kLoadMk = 2;   // markers per block: the three groups of a marker in one block
constexpr int kLoadThreads = 3 * kLoadMk * kLoadLanes;

__device__ __forceinline__ void loads_probe_body(const Dev &d) {
    constexpr unsigned kAll = 0xffffffffu;
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    const int T = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = T / kLoadLanes, m = T % kLoadLanes;
    const int base = (threadIdx.x & 31) & ~(kLoadLanes - 1);
    const bool have = t < 3 * d.nlm;
    const int tt = have ? t : 0;
    const int n = tt / 3, idir = tt % 3 + 1;
    const bool node = m < kSD;
    double *pb = d.probe + static_cast<size_t>(n) * 24;
    const double pos[2] = {d.lmcc[2 * n], d.lmcc[2 * n + 1]};
    const bool inside = (d.zz[1] < pos[1] && pos[1] < d.zz[d.n3]);
    if (have && m == 0) {
        if (idir == 1) {
            pb[23] = inside ? 0.0 : -1.0;
            d.bcerrv[n] = 0.0;
        }
        if (idir == 2) d.bcerrw[n] = 0.0;
    }
    const bool stopped = __shfl_sync(kAll, static_cast<int>(*d.status != 0), base) != 0;
    const bool ok = have && !stopped && inside;

    // checkbcs: the velocity at the marker from the substep-1 weights
    double prod = 0.0;
    if (ok && idir <= 2 && node) {
        const int t2 = 2 * n + idir - 1;
        const int *eu = d.eulins + static_cast<size_t>(t2) * 2 * kSD;
        const double *q = (idir == 1) ? d.q2 : d.q3;
        prod = d.phi[static_cast<size_t>(t2) * kSD + m] * q[fidx(d, eu[m], eu[kSD + m])];
    }
    const double u = group_sum_nodes(prod, base);
    if (ok && idir <= 2 && m == 0) {
        if (idir == 1) d.bcerrv[n] = d.lmvel[2 * n] - u;
        else d.bcerrw[n] = d.lmvel[2 * n + 1] - u;
    }

    const double hpr = d.ddmin * d.kprobe;
    const double probe[2] = {pos[0] + d.lmnor[2 * n] * hpr, pos[1] + d.lmnor[2 * n + 1] * hpr};
    int mj, mk;
    if (idir == 3) {
        mj = d.lmind[4 * n + 2];
        mk = d.lmind[4 * n + 1];
    } else {
        mj = d.lmind[4 * n + 2 * (idir - 1)];
        mk = d.lmind[4 * n + 2 * (idir - 1) + 1];
    }

    // probeind (loads_transfer.F90:238-281): the nearest y and z lines to the
    // probe within 5 lines of the marker's own; lane i holds lines js + i, ks + i
    constexpr int off = 5;
    const int js = mj - off, ks = mk - off;
    const bool inrange = ok && js >= 1 && mj + off <= d.n2 && ks >= 1 && mk + off <= d.n3;
    const double *ya = (idir == 1) ? d.rc : d.rm;
    const double *za = (idir == 2) ? d.zz : d.zm;
    double vy = inf, vz = inf;
    if (inrange && m <= 2 * off) {
        vy = fabs(ya[js + m] - probe[0]);
        vz = fabs(za[ks + m] - probe[1]);
    }
    // a NaN distance never wins the strict comparison; one at the first line
    // keeps the first line
    const bool y0nan = isnan(__shfl_sync(kAll, vy, base)), z0nan = isnan(__shfl_sync(kAll, vz, base));
    const int iy = group_argmin(isnan(vy) ? inf : vy, m);
    const int iz = group_argmin(isnan(vz) ? inf : vz, m);
    const int ij = js + (y0nan ? 0 : iy), ik = ks + (z0nan ? 0 : iz);

    // MLS_SD_ind (MLSint.F90:4-104): node m = 3 (j - 1) + (k - 1) of the 3 x 3
    // support, moved inside the field
    const double *y, *z;
    int dimy, dimz;
    sd_axes(d, idir, y, dimy, z, dimz);
    const int sj = (ij == 1) ? 1 : (ij == d.n2m ? -1 : 0);
    const int sk = (ik == 1) ? 1 : (ik == d.n3m ? -1 : 0);
    const int mm = node ? m : 0;
    const int ej = ij + (mm / 3 + 1 + sj) - 2, ek = ik + (mm % 3 + 1 + sk) - 2;
    const bool bad = inrange && node && (ej < 1 || ej + 1 > dimy || ek < 1 || ek + 1 > dimz);
    const bool supported = group_none(bad, base) && inrange;
    const int ej0 = __shfl_sync(kAll, ej, base);
    const bool good = supported && ej0 >= 2;
    if (ok && !good && m == 0) raise_status(d, FB_ERR_MARKER_OUT);
    const bool act = good && node;

    // the field values that getpbup reads, requested before the MLS algebra
    // so that their latency overlaps it
    double f0 = 0.0, fym = 0.0, fzm = 0.0, g2r = 1.0, g3r = 1.0;
    if (act) {
        const double *f = (idir == 1) ? d.q2 : (idir == 2 ? d.q3 : d.pr);
        f0 = Fv(f, ej, ek);
        fym = Fv(f, ej - 1, ek);
        fzm = Fv(f, ej, ek - 1);
        g2r = d.g2rc[ej];
        g3r = d.g3rc[ek];
    }

    // MLS_SF_d (MLSint.F90:173-258) with compute_AB_d (:342-402)
    double sc0 = 0.0, sc1 = 0.0, w0 = 0.0, w1 = 0.0, w2 = 0.0;
    if (act) {
        sc0 = y[ej];
        sc1 = z[ek];
        const double sd0 = y[ej + 1] - y[ej], sd1 = z[ek + 1] - z[ek];
        double wc[2], dw[2];
        wkernel(d.wfun, probe[0] - sc0, d.radiusSD * sd0, wc[0], dw[0]);
        wkernel(d.wfun, probe[1] - sc1, d.radiusSD * sd1, wc[1], dw[1]);
        w0 = wc[0] * wc[1];
        w1 = wc[1] * dw[0];
        w2 = wc[0] * dw[1];
    }
    const double pk[3] = {1.0, sc0, sc1};
    double A[3][3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            if (b < a) {   // pk[a] pk[b] = pk[b] pk[a]: the same terms, the same sums
#pragma unroll
                for (int l = 0; l < 3; ++l) A[a][b][l] = A[b][a][l];
                continue;
            }
            const double pp = pk[a] * pk[b];
            A[a][b][0] = group_sum_nodes(w0 * pp, base);
            A[a][b][1] = group_sum_nodes(w1 * pp, base);
            A[a][b][2] = group_sum_nodes(w2 * pp, base);
        }
    double Aa[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) Aa[a][b] = A[a][b][0];
    double gam[3][3];
    const double gps[3] = {1.0, probe[0], probe[1]};
    double g0[3];
    gesolve3(Aa, gps, g0);
#pragma unroll
    for (int l = 1; l <= 2; ++l) {
        double C[3], gx[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double acc = 0.0;
#pragma unroll
            for (int b = 0; b < 3; ++b) acc = acc + A[a][b][l] * g0[b];
            const double gpl = (a == l) ? 1.0 : 0.0;
            C[a] = gpl - acc;
        }
        gesolve3(Aa, C, gx);
#pragma unroll
        for (int a = 0; a < 3; ++a) gam[a][l] = gx[a];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) gam[a][0] = g0[a];
    double p0 = 0.0, p1 = 0.0, p2 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double B0 = pk[a] * w0, B1 = pk[a] * w1, B2 = pk[a] * w2;
        p0 = p0 + gam[a][0] * B0;
        p1 = p1 + gam[a][1] * B0 + gam[a][0] * B1;
        p2 = p2 + gam[a][2] * B0 + gam[a][0] * B2;
    }
    const double sumphi = group_sum_nodes(p0, base);
    if (good && m == 0 && !(fabs(1.0 - fabs(sumphi)) <= 1.0e-10)) raise_status(d, FB_ERR_MLS);

    // getpbup (loads_transfer.F90:285-357) for this quantity
    double o[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (act) {
        const double uk1 = (f0 - fym) * d.dx2 / g2r;
        const double uk2 = (f0 - fzm) * d.dx3 / g3r;
        o[0] = p0 * f0;
        o[1] = p1 * f0;
        o[2] = p2 * f0;
        o[3] = p1 * uk1;
        o[4] = p1 * uk2;
        o[5] = p2 * uk1;
        o[6] = p2 * uk2;
    }
    double res = 0.0;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const double s = group_sum_nodes(o[i], base);
        if (m == i) res = s;
    }
    if (good && m < 7) pb[7 * (idir - 1) + m] = res;
}

// the probes of kLoadMk markers per block, then each probed marker's own
// tangent (loads_transfer.F90:177-185) from its first two probes
__device__ __forceinline__ void loads_probe_tan_body(const Dev &d) {
    if (!d.nlm) return;
    loads_probe_body(d);
    __syncthreads();
    const int T = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = T / kLoadLanes;
    if (t >= 3 * d.nlm || t % 3 != 0 || T % kLoadLanes != 0 || *d.status) return;
    const int n = t / 3;
    double *pb = d.probe + static_cast<size_t>(n) * 24;
    if (pb[23] < 0.0) return;
    const double nory = d.lmnor[2 * n], norz = d.lmnor[2 * n + 1];
    const double vel0 = pb[0], vel1 = pb[7];
    const double veln_md = vel0 * nory + vel1 * norz;
    const double velt0 = vel0 - veln_md * nory, velt1 = vel1 - veln_md * norz;
    const double velt_md = sqrt(velt0 * velt0 + velt1 * velt1);
    if (velt_md != 0.0) {
        pb[21] = velt0 / sqrt(velt0 * velt0 + velt1 * velt1);
        pb[22] = velt1 / sqrt(velt0 * velt0 + velt1 * velt1);
        pb[23] = 1.0;
    } else {
        pb[23] = 0.0;
    }
}

__global__ void __launch_bounds__(kLoadThreads, 5) k_loads_probe(Dev d) {
    FB_GRID_WAIT();
    loads_probe_tan_body(d);
}

// loads_transfer_c (loads_transfer.F90:187-214): the tangent carries over
// from the previous marker when the probe's tangential velocity vanishes;
// pressure extrapolation (Wang et al. 2019 eq. 20) and wall shear (eq. 26).
// Also the L2 norms of checkbcs (ckbcs.F90:76-81).  Single block.
__device__ __forceinline__ void loads_finish_body(const Dev &d) {
    __shared__ double sh[32];
    __shared__ bool last;
    const double hpr = d.ddmin * d.kprobe, visc = d.visc;
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    double sv = 0.0, sw = 0.0;
    if (n < d.nlm) {
        const double *pb = d.probe + static_cast<size_t>(n) * 24;
        if (*d.status == 0) {
            d.press[n] = 0.0;
            d.tau[2 * n] = 0.0;
            d.tau[2 * n + 1] = 0.0;
            if (pb[23] >= 0.0) {
                double tany = 0.0, tanz = 0.0;
                for (int m = n; m >= 0; --m) {   // the last marker up to n with a tangent of its own
                    const double *pm = d.probe + static_cast<size_t>(m) * 24;
                    if (pm[23] > 0.5) {
                        tany = pm[21];
                        tanz = pm[22];
                        break;
                    }
                }
                const double *ucy = pb, *ucz = pb + 7, *pc = pb + 14;
                const double nory = d.lmnor[2 * n], norz = d.lmnor[2 * n + 1];
                double dpdnw = d.lmacc[2 * n] * nory + d.lmacc[2 * n + 1] * norz;
                dpdnw = -1.0 * dpdnw;
                const double dpdne = pc[1] * nory + pc[2] * norz;
                d.press[n] = pc[0] - 0.5 * (dpdnw + dpdne) * hpr;
                const double ducdn = (ucy[1] * tany * nory + ucy[2] * tany * norz + ucz[1] * tanz * nory +
                                      ucz[2] * tanz * norz);
                const double d3ucdn3 = (pc[3] * nory * nory + pc[4] * nory * norz + pc[5] * norz * nory +
                                        pc[6] * norz * norz) * 1.0 / visc;
                const double d2ucdn2 = (ucy[3] * tany * nory * nory + ucy[4] * tany * nory * norz +
                                        ucy[5] * tany * norz * nory + ucy[6] * tany * norz * norz +
                                        ucz[3] * tanz * nory * nory + ucz[4] * tanz * nory * norz +
                                        ucz[5] * tanz * norz * nory + ucz[6] * tanz * norz * norz);
                const double ducdnm = ducdn - d2ucdn2 * hpr - 0.5 * d3ucdn3 * (hpr * hpr);
                d.tau[2 * n] = visc * ducdnm * tany;
                d.tau[2 * n + 1] = visc * ducdnm * tanz;
            }
        }
        sv = d.bcerrv[n] * d.bcerrv[n];
        sw = d.bcerrw[n] * d.bcerrw[n];
    }
    // the L2 norms of checkbcs (ckbcs.F90:76-81): block partials, summed in
    // block order by the last block
    const double tv = block_reduce_fast<false>(sv, sh);
    const double tw = block_reduce_fast<false>(sw, sh);
    const int b = blockIdx.x, nb = gridDim.x;
    double *rv = d.red, *rw = d.red + kRedSlot;
    if (threadIdx.x == 0) {
        rv[b] = tv;
        rw[b] = tw;
        __threadfence();
        last = (atomicAdd(d.count + 1, 1u) == static_cast<unsigned>(nb - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double av = 0.0, aw = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        av = av + __ldcg(rv + i);
        aw = aw + __ldcg(rw + i);
    }
    av = block_reduce_fast<false>(av, sh);
    aw = block_reduce_fast<false>(aw, sh);
    if (threadIdx.x == 0) {
        d.count[1] = 0u;
        d.scal[S_NBCV] = sqrt(av) / static_cast<double>(d.nlm);
        d.scal[S_NBCW] = sqrt(aw) / static_cast<double>(d.nlm);
    }
}

constexpr int kLoadFin = 128;   // markers per block of the finish
__global__ void __launch_bounds__(kLoadFin) k_loads_finish(Dev d) {
    FB_GRID_WAIT();
    loads_finish_body(d);
}

// ------------------------------------------------------------ rigid body

// rigid.F90:341-369 (modfn) for the uncoupled 3-DOF system
__device__ void modfn(double K[6], const double t[6], const double FF[6], const double Mi[3], const Dev &d) {
    for (int i = 0; i < 3; ++i) {
        const double cube = t[i] * t[i] * t[i];
        const double lin = -d.kk[i] * t[i] + -d.cc[i] * t[i + 3];
        const double rhs = lin + -d.kk3[i] * cube + FF[i + 3];
        K[i] = t[i + 3];
        K[i + 3] = Mi[i] * rhs;
    }
}

// rigid.F90:4-138 (rigid) with int_stress :373-464, kinem_RK4 :165-228 /
// kinem_RK4i :233-299, get_rotmat :142-161, createnorm :468-495; then the
// clock update of main.F90:92 and one history row.  Single block.
// mode RIGID_STEP: the reference's loose coupling (loads -> forces -> RK4 ->
// markers -> commit).  The strong coupling iteration splits it:
// RIGID_PLACE moves the markers to the state that the load fin[0..2] (Fy,
// Fz, M) gives, without committing; RIGID_FORCES integrates the loads of the
// markers at that new state (moment about the new centre) and evaluates the
// RK4 update they give into rigid[9..17] only; RIGID_COMMIT is RIGID_STEP
// with the load fin (markers restored to the start of the step first).
__device__ __forceinline__ void rigid_body(const Dev &d, int hist_rows, int mode, const double *fin,
                                           double *mbox = nullptr) {
    __shared__ double sh[32 * 5];
    __shared__ double cm[18];
    __shared__ double rot[4];
    __shared__ double xns[6];
    __shared__ double rs[18], kin[9];   // the body state and the prescribed kinematics, read once
    __shared__ int mcon[3];
    const int tid = threadIdx.x, nt = blockDim.x, nlm = d.nlm;
    double *R = d.rigid;
    const bool from_loads = (mode == RIGID_STEP || mode == RIGID_FORCES);
    if (tid < 18) rs[tid] = R[tid];
    else if (tid >= 32 && tid < 41) kin[tid - 32] = d.kinori[tid - 32];
    else if (tid >= 64 && tid < 67) mcon[tid - 64] = d.rbmcon[tid - 64];
    if (!from_loads) __syncthreads();   // (otherwise the block sums' barriers order them)
    double fyp = 0.0, fzp = 0.0, fyv = 0.0, fzv = 0.0, mom = 0.0;
    if (from_loads) {
        const double c0 = (mode == RIGID_FORCES) ? R[9] : R[0], c1 = (mode == RIGID_FORCES) ? R[10] : R[1];
        double f[5] = {0.0, 0.0, 0.0, 0.0, 0.0};   // fyp, fzp, fyv, fzv, mom
        for (int i = tid; i < nlm; i += nt) {
            const double p = d.press[i], A = d.lmA[i];
            const double Fp1 = -p * d.lmnor[2 * i] * A, Fp2 = -p * d.lmnor[2 * i + 1] * A;
            const double Fv1 = d.tau[2 * i] * A, Fv2 = d.tau[2 * i + 1] * A;
            f[0] = f[0] + Fp1;
            f[1] = f[1] + Fp2;
            f[2] = f[2] + Fv1;
            f[3] = f[3] + Fv2;
            const double r1 = d.lmcc[2 * i] - c0, r2 = d.lmcc[2 * i + 1] - c1;
            f[4] = f[4] + (r1 * (Fp2 + Fv2) - r2 * (Fp1 + Fv1));
        }
        block_sum_n<5>(f, sh);   // the five block sums (the same trees as one at a time)
        fyp = f[0];
        fzp = f[1];
        fyv = f[2];
        fzv = f[3];
        mom = f[4];
    }
    // the loads of the step (every thread forms the same values)
    const double time = d.scal[S_TIME], dt = d.dt;
    double Fy, Fz, M;
    if (from_loads) {
        const double fy = fyp + fyv, fz = fzp + fzv;
        const double g0 = (1.0 - 1.0 / d.rbden) * d.rba0 * d.rbgravF0;
        const double g1 = (1.0 - 1.0 / d.rbden) * d.rba0 * d.rbgravF1;
        Fy = fy + g0;
        Fz = fz + g1;
        M = mom;
    } else {
        Fy = fin[0];
        Fz = fin[1];
        M = fin[2];
    }
    if (tid == 0 && from_loads) {
        d.forces[0] = time;
        d.forces[1] = Fy;
        d.forces[2] = Fz;
        d.forces[3] = M;
        d.forces[4] = fyp;
        d.forces[5] = fzp;
        d.forces[6] = fyv;
        d.forces[7] = fzv;
    }
    // explicit RK4 with loads frozen over the stages: the three degrees of
    // freedom (y, z, rotation) are independent (modfn), one thread each
    if (tid < 3) {
        const int i = tid;
        const double csp = (i == 0) ? d.cmposi0 : (i == 1 ? d.cmposi1 : d.cmroti);
        double FFi, Mii;
        if (i == 0) {
            if (d.rtcoup) {
                FFi = Fy + M / d.rrr;
                Mii = 1.0 / ((d.rba1 / (d.rrr * d.rrr) + d.rba0) * d.rbden);
            } else {
                FFi = Fy;
                Mii = 1.0 / (d.rba0 * d.rbden);
            }
        } else if (i == 1) {
            FFi = Fz;
            Mii = 1.0 / (d.rba0 * d.rbden);
        } else {
            FFi = M;
            Mii = 1.0 / (d.rba1 * d.rbden);
        }
        const double kk = d.kk[i], cc = d.cc[i], kk3 = d.kk3[i];
        // modfn (rigid.F90) for component i: K_x = v, K_v = Mi (-kk x + -cc v + -kk3 x^3 + F)
        auto mod = [&](double x, double v, double &kx, double &kv) {
            const double cube = x * x * x;
            const double lin = -kk * x + -cc * v;
            const double rhs = lin + -kk3 * cube + FFi;
            kx = v;
            kv = Mii * rhs;
        };
        const double xo = rs[i] - csp, vo = rs[3 + i];
        double k1x, k1v, k2x, k2v, k3x, k3v, k4x, k4v;
        mod(xo, vo, k1x, k1v);
        mod(xo + k1x * dt / 2.0, vo + k1v * dt / 2.0, k2x, k2v);
        mod(xo + k2x * dt / 2.0, vo + k2v * dt / 2.0, k3x, k3v);
        mod(xo + k3x * dt, vo + k3v * dt, k4x, k4v);
        xns[i] = xo + dt * (k1x / 6.0 + k2x / 3.0 + k3x / 3.0 + k4x / 6.0);
        xns[3 + i] = vo + dt * (k1v / 6.0 + k2v / 3.0 + k3v / 3.0 + k4v / 6.0);
    }
    __syncthreads();
    if (tid == 0) {
        const double csp[3] = {d.cmposi0, d.cmposi1, d.cmroti};
        double xn[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) xn[i] = xns[i];
        // P1, V1, A1 (rigid[9..17]) formed in shared memory (cm), then stored
        for (int i = 0; i < 18; ++i) cm[i] = rs[i];
        double *P1 = cm + 9, *V1 = cm + 12, *A1 = cm + 15;
        if (!d.rtcoup) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                P1[i] = csp[i] + xn[i];
                V1[i] = xn[3 + i];
                A1[i] = (V1[i] - rs[3 + i]) / dt;
            }
        } else {
            P1[0] = csp[0] + xn[0];
            V1[0] = xn[3];
            A1[0] = (V1[0] - rs[3]) / dt;
            P1[1] = csp[1];
            V1[1] = 0.0;
            A1[1] = 0.0;
            P1[2] = csp[2] + xn[0] / d.rrr;
            V1[2] = V1[0] / d.rrr;
            A1[2] = A1[2] / d.rrr;  // as rigid.F90:296 (incoming value / rr)
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
            if (mcon[i] == 1) {
                P1[i] = kin[i];
                V1[i] = kin[3 + i];
                A1[i] = kin[6 + i];
            }
        const double cmrot = P1[2] - rs[2];
        rot[0] = cos(cmrot);
        rot[1] = -sin(cmrot);
        rot[2] = sin(cmrot);
        rot[3] = cos(cmrot);
        for (int i = 9; i < 18; ++i) R[i] = cm[i];
    }
    __syncthreads();
    if (mode == RIGID_FORCES) return;   // the update the loads give, markers untouched
    // Each loop reads all of a thread's kRgU entries before it stores any: the
    // stores could alias the next loads, so a load after a store would wait
    // for the store's round trip.
    constexpr int kRgU = 4;
    const double *P0 = cm, *P1 = cm + 9, *V1 = cm + 12, *A1 = cm + 15;
    for (int i0 = tid; i0 < nlm; i0 += kRgU * nt) {
        double y[kRgU], z[kRgU];
#pragma unroll
        for (int u = 0; u < kRgU; ++u) {
            const int i = min(i0 + u * nt, nlm - 1);
            y[u] = d.lmcc[2 * i];
            z[u] = d.lmcc[2 * i + 1];
        }
#pragma unroll
        for (int u = 0; u < kRgU; ++u) {
            const int i = i0 + u * nt;
            if (i >= nlm) break;
            const double rho0 = y[u] - P0[0], rho1 = z[u] - P0[1];
            const double c10 = -V1[2] * rho1, c11 = V1[2] * rho0;
            const double c20 = -A1[2] * rho1, c21 = A1[2] * rho0;
            const double c30 = -V1[2] * c11, c31 = V1[2] * c10;
            d.lmcc[2 * i] = P1[0] + (rot[0] * rho0 + rot[1] * rho1);
            d.lmcc[2 * i + 1] = P1[1] + (rot[2] * rho0 + rot[3] * rho1);
            d.lmvel[2 * i] = V1[0] + c10;
            d.lmvel[2 * i + 1] = V1[1] + c11;
            d.lmacc[2 * i] = A1[0] + c20 + c30;
            d.lmacc[2 * i + 1] = A1[1] + c21 + c31;
        }
    }
    // vertices rotate about the updated centre (rigid.F90:110-121)
    for (int i0 = tid; i0 <= nlm; i0 += kRgU * nt) {
        double y[kRgU], z[kRgU];
#pragma unroll
        for (int u = 0; u < kRgU; ++u) {
            const int i = min(i0 + u * nt, nlm);
            y[u] = d.vert[2 * i];
            z[u] = d.vert[2 * i + 1];
        }
#pragma unroll
        for (int u = 0; u < kRgU; ++u) {
            const int i = i0 + u * nt;
            if (i > nlm) break;
            const double rho0 = y[u] - P1[0], rho1 = z[u] - P1[1];
            d.vert[2 * i] = P1[0] + (rot[0] * rho0 + rot[1] * rho1);
            d.vert[2 * i + 1] = P1[1] + (rot[2] * rho0 + rot[3] * rho1);
        }
    }
    __syncthreads();
    for (int i0 = tid; i0 < nlm; i0 += kRgU * nt) {
        double va[kRgU][4];   // vertices i and i + 1
#pragma unroll
        for (int u = 0; u < kRgU; ++u) {
            const int i = min(i0 + u * nt, nlm - 1);
#pragma unroll
            for (int q = 0; q < 4; ++q) va[u][q] = d.vert[2 * i + q];
        }
#pragma unroll
        for (int u = 0; u < kRgU; ++u) {
            const int i = i0 + u * nt;
            if (i >= nlm) break;
            const double *a = va[u], *b = va[u] + 2;
            const double v1[3] = {0.0 - 0.0, b[0] - a[0], b[1] - a[1]};
            const double v2[3] = {-1.0 - 0.0, (a[0] + b[0]) * 0.5 - a[0], (a[1] + b[1]) * 0.5 - a[1]};
            const double c0 = v1[1] * v2[2] - v1[2] * v2[1];
            const double c1 = v1[2] * v2[0] - v1[0] * v2[2];
            const double c2 = v1[0] * v2[1] - v1[1] * v2[0];
            const double den = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
            d.lmnor[2 * i] = c1 / den;
            d.lmnor[2 * i + 1] = c2 / den;
        }
    }
    if (mode == RIGID_PLACE) return;     // markers at the trial state; nothing committed
    if (tid == 0) {
        // every value read before the first store (see above)
        const double t0 = d.scal[S_TIME], stepd = d.scal[S_STEP];
        const double nbcv = d.scal[S_NBCV], nbcw = d.scal[S_NBCW], cflm = d.scal[S_CFLM];
        double fv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) fv[i] = d.forces[i];
        const double solves = (mode == RIGID_COMMIT) ? fin[3] : 1.0;   // fluid solves this step
        for (int i = 0; i < 9; ++i) R[i] = cm[9 + i];
        const double t1 = t0 + d.dt;
        d.scal[S_TIME] = t1;
        const int row = static_cast<int>(stepd);
        if (hist_rows > 0) {
            double *h = d.hist + static_cast<size_t>(row % hist_rows) * FB_HIST_COLS;
#pragma unroll
            for (int i = 0; i < 8; ++i) h[i] = fv[i];
            h[8] = t1;
            for (int i = 0; i < 9; ++i) h[9 + i] = cm[9 + i];
            h[18] = nbcv;
            h[19] = nbcw;
            h[20] = cflm;
            h[21] = d.dt;
            for (int i = 22; i < FB_HIST_COLS; ++i) h[i] = 0.0;  // diagnostics, when enabled
            h[30] = solves;
        }
        d.scal[S_STEP] = static_cast<double>(row + 1);
        if (mbox) {   // the synchronous call's status and forcecomp row, into mapped host memory
            volatile double *m = mbox;
            m[0] = static_cast<double>(*d.status);
#pragma unroll
            for (int i = 0; i < 8; ++i) m[1 + i] = fv[i];
            __threadfence_system();
        }
    }
}

__global__ void __launch_bounds__(512) k_rigid(Dev d, int hist_rows, int mode, const double *fin, double *mbox) {
    FB_GRID_WAIT();
    rigid_body(d, hist_rows, mode, fin, mbox);
}

// ------------------------------------------------------------ diagnostics

// ttime.F90:24-147: diagnostics of the end-of-step field for the fluid report
// (fluid_rep.out) -- vmaxv/vminv (vcheck.F90:4-80), cfl (cfl.F90) times dt,
// divgck (divergence.F90:49-82), kinen (utils_proc.F90:474-515) and the line
// vorticity of getintvort (utils_proc.F90:582-632) at row indz.  Eight block
// reductions; the last block writes history columns 22..29 of the step.
__device__ __forceinline__ void diag_body(const Dev &d, int hist_rows) {
    __shared__ double sh[32];
    __shared__ bool last;
    constexpr int kV = 8, kStride = 2048;  // partial v of block b at red[v * kStride + b]
    const int t = threadIdx.x, nt = blockDim.x, b = blockIdx.x, nb = gridDim.x;
    const long cells = static_cast<long>(d.n2m) * d.n3m;
    double v[kV] = {-100.0, -100.0, -100.0, -100.0, 1.0e-8, -100.0, 0.0, 0.0};
    for (long idx = static_cast<long>(b) * nt + t; idx < cells; idx += static_cast<long>(nb) * nt) {
        const int j = static_cast<int>(idx % d.n2m) + 1, k = static_cast<int>(idx / d.n2m) + 1;
        const int jp = j + 1, kp = k + 1;
        const double q2c = Fv(d.q2, j, k), q3c = Fv(d.q3, j, k);
        const double q2j = Fv(d.q2, jp, k), q3k = Fv(d.q3, j, kp);
        v[0] = fmax(v[0], fabs(q2c));
        v[1] = fmax(v[1], fabs(q3c));
        v[2] = fmax(v[2], -q2c);
        v[3] = fmax(v[3], -q3c);
        v[4] = fmax(v[4], fabs((q2c + q2j) * 0.5 * d.udx2m[j]) + fabs((q3c + q3k) * 0.5 * d.udx3m[k]));
        v[5] = fmax(v[5], fabs((q2j - q2c) * d.udx2m[j] + (q3k - q3c) * d.udx3m[k]));
        const double vol = (d.zz[kp] - d.zz[k]) * (d.rc[jp] - d.rc[j]);
        const double vccv = (q2c + q2j) * 0.5, vccw = (q3c + q3k) * 0.5;
        v[6] = v[6] + (vccv * vccv + vccw * vccw) * vol;
        if (k == d.indz) {
            const double dz = d.zz[kp] - d.zz[k];
            const double dwdy = (Fv(d.q3, jp, k) - q3c) / (d.rc[jp] - d.rc[j]);
            const double dvdz = (Fv(d.q2, j, kp) - q2c) / dz;
            v[7] = v[7] + (dwdy - dvdz) * (d.rc[jp] - d.rc[j]);
        }
    }
#pragma unroll
    for (int i = 0; i < kV; ++i) {
        const double r = (i < 6) ? block_reduce_fast<true>(v[i], sh) : block_reduce_fast<false>(v[i], sh);
        if (t == 0) d.red[i * kStride + b] = r;
    }
    if (t == 0) {
        __threadfence();
        last = (atomicAdd(d.count + 3, 1u) == static_cast<unsigned>(nb - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a[kV];
#pragma unroll
    for (int i = 0; i < kV; ++i) {
        double x = (i < 6) ? -1.0e300 : 0.0;
        for (int q = t; q < nb; q += nt) {
            const double y = __ldcg(d.red + i * kStride + q);
            x = (i < 6) ? fmax(x, y) : x + y;
        }
        a[i] = (i < 6) ? block_reduce_fast<true>(x, sh) : block_reduce_fast<false>(x, sh);
    }
    if (t == 0) {
        d.count[3] = 0u;
        if (hist_rows > 0) {
            const int row = static_cast<int>(d.scal[S_STEP]) - 1;  // the step k_rigid closed
            double *h = d.hist + static_cast<size_t>((row + hist_rows) % hist_rows) * FB_HIST_COLS;
            h[22] = a[4] * d.dt;                                   // cflm at the end of the step
            h[23] = a[5];                                          // dmax
            h[24] = 0.5 * a[6] / (d.rext2 * d.alx3);               // ektot
            h[25] = a[7];                                          // vorti
            h[26] = a[0];                                          // vmax(1), vmax(2)
            h[27] = a[1];
            h[28] = -a[2];                                         // vmin(1), vmin(2)
            h[29] = -a[3];
        }
    }
}

__global__ void __launch_bounds__(256) k_diag(Dev d, int hist_rows) {
    FB_GRID_WAIT();
    diag_body(d, hist_rows);
}

// ------------------------------------------------------------ grouped launches

// The same kernels over a group of cases of one launch geometry: blockIdx.z
// selects the case; its view (and substep n's constants, n 0-based) are
// staged in shared memory from the group's device array (the single-case
// kernels take them by value).

__global__ void __launch_bounds__(256) kg_cfl(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    cfl_body(d);
}

__global__ void __launch_bounds__(1024) kg_boucdq(const GroupCase *__restrict__ g, int n) {
    __shared__ Dev d;
    __shared__ SubDev s;
    if (!stage_case(g, &d, &s, n)) return;
    boucdq_body(d, s.ga, s.ro);
}

__global__ void __launch_bounds__(256, kNlBlocksPerSM) kg_nl_rhs(const GroupCase *__restrict__ g, int n, int pend) {
    extern __shared__ __align__(16) unsigned char nl_smem[];
    __shared__ Dev d;
    __shared__ SubDev s;
    if (!stage_case(g, &d, &s, n)) return;
    nl_rhs_body(d, s.al, s.ga, s.ro, reinterpret_cast<NlTile *>(nl_smem), pend != 0);
}
__global__ void kg_lgrdist(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    lgrdist_body(d);
}

__global__ void kg_mls_setup(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    mls_setup_body(d);
}

__global__ void kg_spread_chains(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    spread_chains_body(d);
}

__global__ void kg_mls_interp(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    mls_interp_body(d);
}

__global__ void kg_mls_spread(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    mls_spread_body(d);
}

__global__ void kg_divg(const GroupCase *__restrict__ g, int n) {
    __shared__ Dev d;
    __shared__ SubDev s;
    if (!stage_case(g, &d, &s, n)) return;
    divg_body(d, s.usdtal);
}

__global__ void __launch_bounds__(256, kUpBlocksPerSM) kg_updvp_prcalc(const GroupCase *__restrict__ g, int n,
                                                                       int pend) {
    extern __shared__ __align__(16) unsigned char up_smem[];
    __shared__ Dev d;
    __shared__ SubDev s;
    if (!stage_case(g, &d, &s, n)) return;
    updvp_prcalc_body<false>(d, s.al, s.al * s.beta, reinterpret_cast<UpTile *>(up_smem), pend != 0);
}

__global__ void kg_submean_boucqt(const GroupCase *__restrict__ g, int deferred) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    submean_boucqt_body(d, deferred != 0);
}

// n: the next substep (0-based) whose boucdq runs here
__global__ void __launch_bounds__(1024) kg_substep_mid(const GroupCase *__restrict__ g, int n, int slot) {
    __shared__ Dev d;
    __shared__ SubDev s;
    if (!stage_case(g, &d, &s, n)) return;
    substep_mid_body(d, slot, s.ga, s.ro);
}

__global__ void __launch_bounds__(kLoadThreads, 5) kg_loads_probe(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    loads_probe_tan_body(d);
}

__global__ void __launch_bounds__(kLoadFin) kg_loads_finish(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d)) return;
    loads_finish_body(d);
}

// mode as k_rigid, with the case's trial load; the commit after a coupling
// iteration runs for every case (no gate)
__global__ void __launch_bounds__(512) kg_rigid(const GroupCase *__restrict__ g, int mode) {
    __shared__ Dev d;
    if (!stage_case(g, &d, nullptr, 0, mode == RIGID_PLACE || mode == RIGID_FORCES)) return;
    rigid_body(d, g[blockIdx.z].hist_rows, mode, g[blockIdx.z].fin);
}

__global__ void __launch_bounds__(256) kg_diag(const GroupCase *__restrict__ g) {
    __shared__ Dev d;
    if (!stage_case(g, &d, nullptr, 0, false)) return;
    diag_body(d, g[blockIdx.z].hist_rows);
}

// ------------------------------------------------------------ launchers

namespace {
inline dim3 grid2(int nx, int ny, dim3 b) { return dim3((nx + b.x - 1) / b.x, (ny + b.y - 1) / b.y); }
}  // namespace

int stride_blocks(const Dev &d) {
    const long cells = static_cast<long>(d.n2m) * d.n3m;
    return static_cast<int>(std::min<long>((cells + 255) / 256, 148L * 8));
}

// grid-stride reductions of a group: the cases fill the GPU together, so each
// case takes fewer blocks (about eight cells per thread) and the block and
// last-block reductions are paid less often
int group_stride_blocks(const Dev &d) {
    const long cells = static_cast<long>(d.n2m) * d.n3m;
    return static_cast<int>(std::max<long>(1, std::min<long>((cells + 2047) / 2048, 148L * 8)));
}
// two blocks per SM, each on pairs of rows: few partials for the last block
// to gather, and few arrivals on the grid's counter
void launch_cfl(const Dev &d, cudaStream_t s) { pdl(k_cfl, dim3(std::min(d.n3m, 148 * 2)), dim3(256), 0, s, d); }
void launch_boucdq(const Dev &d, double ga, double ro, cudaStream_t s) { pdl(k_boucdq, dim3(1), dim3(1024), 0, s, d, ga, ro); }
int nl_tiles(const Dev &d) { return ((d.n2m + kNlJ - 1) / kNlJ) * ((d.n3m + kNlK - 1) / kNlK); }

void launch_nl_rhs(const Dev &d, double al, double ga, double ro, cudaStream_t s, bool pend, const NlMaps *maps) {
    const int blocks = std::min(nl_tiles(d), 148 * kNlBlocksPerSM);
    if (maps) pdl(k_nl_rhs_tma, dim3(blocks), dim3(32, 8), kNlSmemT, s, d, *maps, al, ga, ro, pend ? 1 : 0);
    else pdl(k_nl_rhs, dim3(blocks), dim3(32, 8), kNlSmem, s, d, al, ga, ro, pend ? 1 : 0);
}

// q2, q3, pr, dph as 2-D FP64 tensors: x = j - 1 (j = 1 .. n2), y = k (0 .. n3),
// rows P doubles apart; a box is one tile with its halo (kNlTW x kNlTH)
int encode_nl_maps(NlMaps *m, const Dev &d) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return FB_ERR_CUDA;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const double *f[4] = {d.q2, d.q3, d.pr, d.dph};
    CUtensorMap *dst[4] = {&m->q2, &m->q3, &m->pr, &m->dph};
    for (int i = 0; i < 4; ++i) {
        if ((reinterpret_cast<uintptr_t>(f[i]) & 15u) || (static_cast<long>(d.P) * 8) % 16 || d.P < d.n2)
            return FB_ERR_STATE;
        const cuuint64_t dims[2] = {static_cast<cuuint64_t>(d.n2), static_cast<cuuint64_t>(d.n3) + 1u};
        const cuuint64_t strides[1] = {static_cast<cuuint64_t>(d.P) * 8u};
        const cuuint32_t box[2] = {static_cast<cuuint32_t>(kNlTW), static_cast<cuuint32_t>(kNlTH)};
        const cuuint32_t es[2] = {1, 1};
        const CUresult r = encode(dst[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(f[i]), dims,
                                  strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return FB_ERR_CUDA;
    }
    return FB_OK;
}
void launch_lgrdist(const Dev &d, cudaStream_t s) {
    if (d.nlm) pdl(k_lgrdist, dim3((d.nlm + 127) / 128), dim3(128), 0, s, d);
}
void launch_mls_setup(const Dev &d, cudaStream_t s) {
    if (d.nlm) pdl(k_mls_setup, dim3((2 * d.nlm * kNodeLanes + 255) / 256), dim3(256), 0, s, d);
}
void launch_mls_interp(const Dev &d, cudaStream_t s) {
    if (d.nlm) pdl(k_mls_interp, dim3((2 * d.nlm * kInterpLanes + 255) / 256), dim3(256), 0, s, d);
}
void launch_spread_chains(const Dev &d, cudaStream_t s) {
    const int n = 2 * d.nlm * kSD;
    if (n) pdl(k_spread_chains, dim3((n + 127) / 128), dim3(128), 0, s, d);
}
void launch_mls_spread(const Dev &d, cudaStream_t s) {
    const int n = 2 * d.nlm * kSD;
    if (n) pdl(k_mls_spread, dim3((n + 127) / 128), dim3(128), 0, s, d);
}
void launch_helsolve(const Dev &d, const SubDev &sd, cudaStream_t s) {
    pdl(k_tri_y2, dim3((d.n3m + 63) / 64), dim3(64), 0, s, d, sd);
    pdl(k_tri_z2, dim3((d.n2m + 63) / 64), dim3(64), 0, s, d, sd);
    pdl(k_tri_y3, dim3((d.n3m + 63) / 64), dim3(64), 0, s, d, sd);
    pdl(k_tri_z3, dim3((d.n2m + 63) / 64), dim3(64), 0, s, d, sd);
}
void launch_divg(const Dev &d, double usdtal, cudaStream_t s, double *rmax) {
    dim3 b(32, 8);   // the row maxima's reduction assumes these blocks
    pdl(k_divg, dim3(grid2(d.n2m, (d.n3m + kDivK - 1) / kDivK, b)), dim3(b), 0, s, d, usdtal, rmax);
}
void launch_updvp_prcalc(const Dev &d, double al, double be, cudaStream_t s, bool pend, const NlMaps *maps) {
    const int blocks = std::min(nl_tiles(d), 148 * kUpBlocksPerSM);
    if (maps) pdl(k_updvp_prcalc_tma, dim3(blocks), dim3(32, 8), kUpSmemT, s, d, *maps, al, be, pend ? 1 : 0);
    else pdl(k_updvp_prcalc, dim3(blocks), dim3(32, 8), kUpSmem, s, d, al, be, pend ? 1 : 0);
}
void launch_submean_boucqt(const Dev &d, cudaStream_t s, bool deferred) {
    dim3 b(32, 8);
    pdl(k_submean_boucqt, dim3(grid2(d.n2, d.n3 + 1, b)), dim3(b), 0, s, d, deferred ? 1 : 0);
}
void launch_substep_mid(const Dev &d, int slot, double ga, double ro, cudaStream_t s) {
    pdl(k_substep_mid, dim3(1), dim3(1024), 0, s, d, slot, ga, ro);
}
void launch_loads(const Dev &d, cudaStream_t s) {
    if (!d.nlm) return;
    pdl(k_loads_probe, dim3((d.nlm + kLoadMk - 1) / kLoadMk), dim3(kLoadThreads), 0, s, d);
    pdl(k_loads_finish, dim3((d.nlm + kLoadFin - 1) / kLoadFin), dim3(kLoadFin), 0, s, d);
}
void launch_diag(const Dev &d, int hist_rows, cudaStream_t s) {
    pdl(k_diag, dim3(std::min(stride_blocks(d), 2048)), dim3(256), 0, s, d, hist_rows);
}
// The end of a synchronous API call: the status word (and the forcecomp
// row) written by the GPU into mapped host memory, so that the host reads them
// after its stream synchronisation without a device-to-host copy
__global__ void k_publish(const int *status, const double *forces, double *mbox) {
    FB_GRID_WAIT();
    volatile double *m = mbox;
    m[0] = static_cast<double>(*status);
    if (forces)
        for (int i = 0; i < 8; ++i) m[1 + i] = forces[i];
    __threadfence_system();
}
void launch_publish(const Dev &d, bool forces, double *mbox, cudaStream_t s) {
    pdl(k_publish, dim3(1), dim3(1), 0, s, static_cast<const int *>(d.status),
        forces ? static_cast<const double *>(d.forces) : nullptr, mbox);
}

void launch_rigid(const Dev &d, int hist_rows, cudaStream_t s, int mode, const double *fin, double *mbox) {
    if (d.nlm) pdl(k_rigid, dim3(1), dim3(512), 0, s, d, hist_rows, mode, fin, mbox);
}


// grouped launchers: the geometry of the group's first case, gridDim.z = cases
namespace {
inline dim3 zgrid(dim3 g, const Group &gr) { return dim3(g.x, g.y, static_cast<unsigned>(gr.n)); }
}  // namespace

void glaunch_cfl(const Group &g, cudaStream_t s) {
    pdl(kg_cfl, zgrid(dim3(std::max(1, std::min(g.rep.n3m, (2 * 148 * 8 + g.n - 1) / g.n))), g), dim3(256), 0, s,
        g.cases);
}
void glaunch_boucdq(const Group &g, int n, cudaStream_t s) {
    pdl(kg_boucdq, zgrid(dim3(1), g), dim3(1024), 0, s, g.cases, n);
}
void glaunch_nl_rhs(const Group &g, int n, cudaStream_t s, bool pend) {
    // about two waves of resident blocks over the whole group
    const int per_case = std::max(1, std::min(nl_tiles(g.rep), (2 * 148 * kNlBlocksPerSM + g.n - 1) / g.n));
    pdl(kg_nl_rhs, zgrid(dim3(per_case), g), dim3(32, 8), kNlSmem, s, g.cases, n, pend ? 1 : 0);
}

cudaError_t kernels_configure() {
    cudaError_t e = cudaFuncSetAttribute(k_nl_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kNlSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_nl_rhs_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kNlSmemT));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_updvp_prcalc_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kUpSmemT));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kg_nl_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kNlSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_updvp_prcalc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kUpSmem));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kg_updvp_prcalc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(kUpSmem));
    return e;
}
void glaunch_marker_setup(const Group &g, cudaStream_t s) {
    const Dev &d = g.rep;
    if (!d.nlm) return;
    pdl(kg_lgrdist, zgrid(dim3((d.nlm + 127) / 128), g), dim3(128), 0, s, g.cases);
    pdl(kg_mls_setup, zgrid(dim3((2 * d.nlm * kNodeLanes + 255) / 256), g), dim3(256), 0, s, g.cases);
    pdl(kg_spread_chains, zgrid(dim3((2 * d.nlm * kSD + 127) / 128), g), dim3(128), 0, s, g.cases);
}
void glaunch_forcing(const Group &g, cudaStream_t s) {
    const Dev &d = g.rep;
    if (!d.nlm) return;
    pdl(kg_mls_interp, zgrid(dim3((2 * d.nlm * kInterpLanes + 255) / 256), g), dim3(256), 0, s, g.cases);
    pdl(kg_mls_spread, zgrid(dim3((2 * d.nlm * kSD + 127) / 128), g), dim3(128), 0, s, g.cases);
}
void glaunch_divg(const Group &g, int n, cudaStream_t s) {
    dim3 b(32, 8);
    pdl(kg_divg, zgrid(grid2(g.rep.n2m, (g.rep.n3m + kDivK - 1) / kDivK, b), g), dim3(b), 0, s, g.cases, n);
}
void glaunch_updvp_prcalc(const Group &g, int n, cudaStream_t s, bool pend) {
    const int per_case = std::max(1, std::min(nl_tiles(g.rep), (2 * 148 * kUpBlocksPerSM + g.n - 1) / g.n));
    pdl(kg_updvp_prcalc, zgrid(dim3(per_case), g), dim3(32, 8), kUpSmem, s, g.cases, n, pend ? 1 : 0);
}
void glaunch_submean_boucqt(const Group &g, cudaStream_t s, bool deferred) {
    dim3 b(32, 8);
    pdl(kg_submean_boucqt, zgrid(grid2(g.rep.n2, g.rep.n3 + 1, b), g), dim3(b), 0, s, g.cases, deferred ? 1 : 0);
}
void glaunch_substep_mid(const Group &g, int n_next, int slot, cudaStream_t s) {
    pdl(kg_substep_mid, zgrid(dim3(1), g), dim3(1024), 0, s, g.cases, n_next, slot);
}
void glaunch_loads(const Group &g, cudaStream_t s) {
    const Dev &d = g.rep;
    if (!d.nlm) return;
    pdl(kg_loads_probe, zgrid(dim3((d.nlm + kLoadMk - 1) / kLoadMk), g), dim3(kLoadThreads), 0, s, g.cases);
    pdl(kg_loads_finish, zgrid(dim3((d.nlm + kLoadFin - 1) / kLoadFin), g), dim3(kLoadFin), 0, s, g.cases);
}
void glaunch_rigid(const Group &g, cudaStream_t s, int mode) {
    if (g.rep.nlm) pdl(kg_rigid, zgrid(dim3(1), g), dim3(512), 0, s, g.cases, mode);
}
void glaunch_diag(const Group &g, cudaStream_t s) {
    pdl(kg_diag, zgrid(dim3(std::min(group_stride_blocks(g.rep), 2048)), g), dim3(256), 0, s, g.cases);
}

}  // namespace fb
