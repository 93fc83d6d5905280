// fb_cfl_noalloc: the CFL number and mean streamwise velocity of cfl.F90 for
// a caller that cannot allocate device memory.
//
// Who needs this: hosts whose device memory belongs to another runtime --
// a Fortran code whose arrays live in CUDA Fortran or OpenACC data regions,
// or an application that carves all GPU memory out of its own arena under a
// hard budget -- and that therefore must not let a library call cudaMalloc
// (which can fail, fragment the arena, or exceed the budget).  They hand us
// device pointers to their own velocity and grid arrays and get two numbers
// back; nothing is allocated here.
//
// How: the per-row partial results live in one file-scope __device__ array of
// fixed size, shared by every call on a device.  Its device address is looked
// up once per device with cudaGetSymbolAddress (host code must not use the
// symbol itself as a pointer).  Each call clears the completion counter in
// that array before its kernel starts; two calls whose kernels overlap on the
// GPU (different streams, no ordering between them) race on the array.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>

#include "../../include/fribois2d.h"

namespace {

constexpr int kThreads = 256;

// [0, 2*kMaxRows): per-row (max, sum) pairs; [2*kMaxRows]: completion counter
__device__ __align__(256) double g_cfl_scratch[2 * FB_NOALLOC_MAX_ROWS + 32];

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// one block per row k = 1..n3m (row-wise partials), the last block combines
// the rows in order; q fields are (j, k) at q[k*pitch + j-1]
__global__ void __launch_bounds__(kThreads) k_cfl_rows(double *scratch, const double *q2, const double *q3,
                                                       int pitch, int n2m, int n3m, const double *rc,
                                                       const double *zz, const double *udx2m,
                                                       const double *udx3m, double dt, double rext2,
                                                       double alx3, double *out) {
    __shared__ double shm[kThreads / 32], shs[kThreads / 32];
    __shared__ bool last;
    const int k = blockIdx.x + 1, t = threadIdx.x, w = t >> 5, lane = t & 31;
    double mx = 1.0e-8, sm = 0.0;
    const double udx3 = udx3m[k - 1];
    for (int j = t + 1; j <= n2m; j += kThreads) {
        const double a = (q2[static_cast<size_t>(k) * pitch + j - 1] + q2[static_cast<size_t>(k) * pitch + j]) * 0.5 * udx2m[j - 1];
        const double b = (q3[static_cast<size_t>(k) * pitch + j - 1] + q3[static_cast<size_t>(k + 1) * pitch + j - 1]) * 0.5 * udx3;
        const double q = fabs(a) + fabs(b);
        mx = fmax(mx, (q == q) ? q : INFINITY);   // a NaN velocity reads as +inf
        sm = sm + q3[static_cast<size_t>(k) * pitch + j - 1] * (zz[k] - zz[k - 1]) * (rc[j] - rc[j - 1]);
    }
    mx = warp_max(mx);
    sm = warp_sum(sm);
    if (lane == 0) {
        shm[w] = mx;
        shs[w] = sm;
    }
    __syncthreads();
    unsigned *counter = reinterpret_cast<unsigned *>(scratch + 2 * FB_NOALLOC_MAX_ROWS);
    if (t == 0) {
        double m2 = shm[0], s2 = shs[0];
        for (int q = 1; q < kThreads / 32; ++q) {
            m2 = fmax(m2, shm[q]);
            s2 = s2 + shs[q];
        }
        scratch[2 * (k - 1)] = m2;
        scratch[2 * (k - 1) + 1] = s2;
        __threadfence();
        last = (atomicAdd(counter, 1u) == static_cast<unsigned>(n3m - 1));
    }
    __syncthreads();
    if (!last || t != 0) return;
    __threadfence();
    double m3 = 1.0e-8, s3 = 0.0;
    for (int r = 0; r < n3m; ++r) {
        m3 = fmax(m3, __ldcg(scratch + 2 * r));
        s3 = s3 + __ldcg(scratch + 2 * r + 1);
    }
    out[0] = m3 * dt;
    out[1] = s3 / (rext2 * alx3);
    *counter = 0u;
}

double *scratch_for_device(int dev) {
    // device addresses of g_cfl_scratch, looked up on first use per device;
    // two host threads may both look it up the first time, and both store
    // the same address
    static std::atomic<double *> addr[64];
    if (dev < 0 || dev >= 64) return nullptr;
    double *a = addr[dev].load(std::memory_order_acquire);
    if (!a) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_cfl_scratch) != cudaSuccess) return nullptr;
        a = static_cast<double *>(p);
        addr[dev].store(a, std::memory_order_release);
    }
    return a;
}

}  // namespace

extern "C" int fb_cfl_noalloc(const double *q2, const double *q3, int pitch, int n2, int n3, const double *rc,
                              const double *zz, const double *udx2m, const double *udx3m, double dt,
                              double rext2, double alx3, double *out, void *stream) {
    if (!q2 || !q3 || !rc || !zz || !udx2m || !udx3m || !out || n2 < 2 || n3 < 2 || pitch < n2)
        return FB_ERR_STATE;
    const int n2m = n2 - 1, n3m = n3 - 1;
    if (n3m > FB_NOALLOC_MAX_ROWS) {
        std::fprintf(stderr,
                     "fribois2d: fb_cfl_noalloc: %d z cells exceed the fixed scratch capacity of %d rows\n",
                     n3m, FB_NOALLOC_MAX_ROWS);
        return FB_ERR_UNSUPPORTED;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FB_ERR_CUDA;
    double *scratch = scratch_for_device(dev);
    if (!scratch) return FB_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the counter keeps the previous call's value only if that call was cut
    // short; clear it so that this call's last block is found correctly
    if (cudaMemsetAsync(scratch + 2 * FB_NOALLOC_MAX_ROWS, 0, sizeof(unsigned), st) != cudaSuccess)
        return FB_ERR_CUDA;
    // the launch's own status (cudaGetLastError would also return, and clear,
    // an earlier error of the caller's); the runtime may still report an
    // earlier asynchronous error here
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(n3m));
    cfg.blockDim = dim3(kThreads);
    cfg.stream = st;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_cfl_rows, scratch, q2, q3, pitch, n2m, n3m, rc, zz, udx2m,
                                             udx3m, dt, rext2, alx3, out);
    return e == cudaSuccess ? FB_OK : FB_ERR_CUDA;
}
