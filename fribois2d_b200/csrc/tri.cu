// Batched tridiagonal line solves (solve_fluid.F90 solq2j/solq2k/solq3j/
// solq3k and the per-mode y solves of phcalc_outflow.F90:34-56).
//
// Every system is factorised once on the host (DGTTRF without row
// interchanges, which these diagonally dominant systems never need); a
// line solve is then the two first-order recurrences of the LU
// substitution,
//     forward   y(i) = a(i) y(i-1) + b(i),        a(0)   = 0
//     backward  x(i) = e(i) x(i+1) + g(i) y(i),   e(n-1) = 0
// Each line is staged in shared memory with coalesced loads and solved by
// one warp: every lane owns a contiguous chunk, composes its chunk's affine
// map, a 5-step shuffle scan gives each lane its incoming value, and the
// lane then applies its chunk.  Depth is O(n/32 + log 32) instead of O(n).
#include <cuda_runtime.h>

#include "device.cuh"
#include "tri.h"

namespace fb {

#define Fv(a, j, k) (a)[fidx(d, (j), (k))]

namespace {

constexpr unsigned kFull = 0xffffffffu;

// y-direction coefficient sets: 1-D arrays shared by all lines
struct CoefShared {
    const double *a, *e, *g;
    __device__ double A(int i) const { return __ldg(a + i); }
    __device__ double E(int i) const { return __ldg(e + i); }
    __device__ double G(int i) const { return __ldg(g + i); }
};

// Poisson mode: only the reciprocal pivots depend on the mode; the
// multipliers follow from the operator's off-diagonals (1-based arrays)
struct CoefMode {
    const double *g;       // this mode's 1/d(i), i = 0..n-1
    const double *amphj, *apphj;
    int n;
    __device__ double A(int i) const { return i == 0 ? 0.0 : -(__ldg(amphj + i + 1) * __ldg(g + i - 1)); }
    __device__ double E(int i) const { return i == n - 1 ? 0.0 : -(__ldg(apphj + i + 1) * __ldg(g + i)); }
    __device__ double G(int i) const { return __ldg(g + i); }
};

template <class Co>
__device__ __forceinline__ void warp_solve(double *v, int n, const Co &co) {
    const int lane = threadIdx.x & 31;
    const int m = (n + 31) >> 5;
    const int i0 = min(lane * m, n), i1 = min(i0 + m, n);
    // forward substitution
    double A = 1.0, C = 0.0;
    for (int i = i0; i < i1; ++i) {
        const double a = co.A(i);
        C = fma(a, C, v[i]);
        A *= a;
    }
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
    for (int i = i0; i < i1; ++i) {
        y = fma(co.A(i), y, v[i]);
        v[i] = y;
    }
    // back substitution
    A = 1.0;
    C = 0.0;
    for (int i = i1 - 1; i >= i0; --i) {
        const double e = co.E(i);
        C = fma(e, C, co.G(i) * v[i]);
        A *= e;
    }
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
    for (int i = i1 - 1; i >= i0; --i) {
        x = fma(co.E(i), x, co.G(i) * v[i]);
        v[i] = x;
    }
}

inline __device__ int odd_ld(int n) { return n | 1; }

}  // namespace

// solq2j (solve_fluid.F90:135-157): lines k = 1..n3m of n2 unknowns, rows 1
// and n2 identity with zero right-hand side; result stays in rhs2.
__global__ void __launch_bounds__(kYLines * 32) k_scan_y2(Dev d, ScanSys s, const double *by) {
    extern __shared__ double sm[];
    const int n = d.n2, ld = odd_ld(n);
    const int k0 = blockIdx.x * kYLines + 1;
    for (int l = 0; l < kYLines; ++l) {
        const int k = k0 + l;
        if (k > d.n3m) break;
        const double *row = d.rhs2 + fidx(d, 1, k);
        for (int j = threadIdx.x + 1; j <= n; j += blockDim.x)
            sm[l * ld + j - 1] = (j >= 2 && j <= d.n2m) ? row[j - 1] * by[j] : 0.0;
    }
    __syncthreads();
    const int w = threadIdx.x >> 5;
    if (k0 + w <= d.n3m) warp_solve(sm + w * ld, n, CoefShared{s.a, s.e, s.g});
    __syncthreads();
    for (int l = 0; l < kYLines; ++l) {
        const int k = k0 + l;
        if (k > d.n3m) break;
        double *row = d.rhs2 + fidx(d, 1, k);
        for (int j = threadIdx.x; j < n; j += blockDim.x) row[j] = sm[l * ld + j];
    }
}

// solq3j (solve_fluid.F90:79-101): lines k = 2..n3m of n2m unknowns
__global__ void __launch_bounds__(kYLines * 32) k_scan_y3(Dev d, ScanSys s, const double *by) {
    extern __shared__ double sm[];
    const int n = d.n2m, ld = odd_ld(n);
    const int k0 = blockIdx.x * kYLines + 2;
    for (int l = 0; l < kYLines; ++l) {
        const int k = k0 + l;
        if (k > d.n3m) break;
        const double *row = d.rhs3 + fidx(d, 1, k);
        for (int j = threadIdx.x + 1; j <= n; j += blockDim.x) sm[l * ld + j - 1] = row[j - 1] * by[j];
    }
    __syncthreads();
    const int w = threadIdx.x >> 5;
    if (k0 + w <= d.n3m) warp_solve(sm + w * ld, n, CoefShared{s.a, s.e, s.g});
    __syncthreads();
    for (int l = 0; l < kYLines; ++l) {
        const int k = k0 + l;
        if (k > d.n3m) break;
        double *row = d.rhs3 + fidx(d, 1, k);
        for (int j = threadIdx.x; j < n; j += blockDim.x) row[j] = sm[l * ld + j];
    }
}

// solq2k (solve_fluid.F90:185-224) and helsolve.F90:32-33: lines j of n3m
// unknowns with the inflow/outflow terms; q2 += x; wall columns zeroed.
__global__ void __launch_bounds__(kZLines * 32) k_scan_z2(Dev d, ScanSys s, const double *bz, double ugkks,
                                                          double ugkkn) {
    extern __shared__ double sm[];
    const int n = d.n3m, ld = odd_ld(n);
    const int j0 = blockIdx.x * kZLines + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int t = tid; t < kZLines * n; t += nt) {
        const int l = t % kZLines, k = t / kZLines + 1, j = j0 + l;
        double v = 0.0;
        if (j <= d.n2m) {
            v = Fv(d.rhs2, j, k) * bz[k];
            if (k == 1) v = v + d.dqb2s[j] * ugkks;
            if (k == n) v = v + d.dqb2n[j] * ugkkn;
        }
        sm[l * ld + k - 1] = v;
    }
    __syncthreads();
    const int w = tid >> 5;
    if (j0 + w <= d.n2m && j0 + w >= 2) warp_solve(sm + w * ld, n, CoefShared{s.a, s.e, s.g});
    __syncthreads();
    for (int t = tid; t < kZLines * n; t += nt) {
        const int l = t % kZLines, k = t / kZLines + 1, j = j0 + l;
        if (j >= 2 && j <= d.n2m) Fv(d.q2, j, k) = Fv(d.q2, j, k) + sm[l * ld + k - 1];
    }
    if (j0 == 1) {
        for (int k = tid; k <= d.n3; k += nt) {
            Fv(d.q2, 1, k) = 0.0;
            Fv(d.q2, d.n2, k) = 0.0;
        }
    }
}

// solq3k (solve_fluid.F90:262-307): lines j of n3 unknowns with Dirichlet
// end rows; q3 += x, the outflow row advanced by dqb3n.
__global__ void __launch_bounds__(kZLines * 32) k_scan_z3(Dev d, ScanSys s, const double *bz) {
    extern __shared__ double sm[];
    const int n = d.n3, ld = odd_ld(n);
    const int j0 = blockIdx.x * kZLines + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int t = tid; t < kZLines * n; t += nt) {
        const int l = t % kZLines, k = t / kZLines + 1, j = j0 + l;
        double v = 0.0;
        if (j <= d.n2m) {
            if (k == 1) v = d.dqb3s[j];
            else if (k == n) v = d.dqb3n[j];
            else v = Fv(d.rhs3, j, k) * bz[k];
        }
        sm[l * ld + k - 1] = v;
    }
    __syncthreads();
    const int w = tid >> 5;
    if (j0 + w <= d.n2m) warp_solve(sm + w * ld, n, CoefShared{s.a, s.e, s.g});
    __syncthreads();
    for (int t = tid; t < kZLines * n; t += nt) {
        const int l = t % kZLines, k = t / kZLines + 1, j = j0 + l;
        if (j > d.n2m) continue;
        if (k < n) Fv(d.q3, j, k) = Fv(d.q3, j, k) + sm[l * ld + k - 1];
        else Fv(d.q3, j, k) = Fv(d.q3, j, k) + d.dqb3n[j];
    }
}

// phcalc_outflow.F90:34-56: one y system per z mode, in place in hmn
__global__ void __launch_bounds__(kYLines * 32) k_scan_poisson(Dev d) {
    extern __shared__ double sm[];
    const int n = d.n2m, ld = odd_ld(n);
    const int m0 = blockIdx.x * kYLines;
    for (int l = 0; l < kYLines; ++l) {
        const int m = m0 + l;
        if (m >= d.n3m) break;
        const double *row = d.hmn + static_cast<size_t>(m) * d.ldh;
        for (int j = threadIdx.x; j < n; j += blockDim.x) sm[l * ld + j] = row[j];
    }
    __syncthreads();
    const int w = threadIdx.x >> 5, m = m0 + w;
    if (m < d.n3m) warp_solve(sm + w * ld, n, CoefMode{d.pg + static_cast<size_t>(m) * d.ldh, d.amphj, d.apphj, n});
    __syncthreads();
    for (int l = 0; l < kYLines; ++l) {
        const int mm = m0 + l;
        if (mm >= d.n3m) break;
        double *row = d.hmn + static_cast<size_t>(mm) * d.ldh;
        for (int j = threadIdx.x; j < n; j += blockDim.x) row[j] = sm[l * ld + j];
    }
}

size_t scan_smem_y(int n) { return static_cast<size_t>(kYLines) * static_cast<size_t>(n | 1) * sizeof(double); }
size_t scan_smem_z(int n) { return static_cast<size_t>(kZLines) * static_cast<size_t>(n | 1) * sizeof(double); }

cudaError_t scan_configure() {
    const int big = 200 * 1024;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(k_scan_y2, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_scan_y3, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_scan_z2, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_scan_z3, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    if ((e = cudaFuncSetAttribute(k_scan_poisson, cudaFuncAttributeMaxDynamicSharedMemorySize, big))) return e;
    return cudaSuccess;
}

void launch_scan_helsolve(const Dev &d, const SubDev &s, cudaStream_t st) {
    k_scan_y2<<<(d.n3m + kYLines - 1) / kYLines, kYLines * 32, scan_smem_y(d.n2), st>>>(d, s.sy2, s.by2);
    k_scan_z2<<<(d.n2m + kZLines - 1) / kZLines, kZLines * 32, scan_smem_z(d.n3m), st>>>(d, s.sz2, s.bz2, s.ugkks,
                                                                                       s.ugkkn);
    k_scan_y3<<<(d.n3m - 1 + kYLines - 1) / kYLines, kYLines * 32, scan_smem_y(d.n2m), st>>>(d, s.sy3, s.by3);
    k_scan_z3<<<(d.n2m + kZLines - 1) / kZLines, kZLines * 32, scan_smem_z(d.n3), st>>>(d, s.sz3, s.bz3);
}

void launch_scan_poisson(const Dev &d, cudaStream_t st) {
    k_scan_poisson<<<(d.n3m + kYLines - 1) / kYLines, kYLines * 32, scan_smem_y(d.n2m), st>>>(d);
}

}  // namespace fb
