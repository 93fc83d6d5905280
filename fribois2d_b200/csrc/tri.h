// Batched tridiagonal line solves (definitions in tri.cu).
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace fb {

constexpr int kYLines = 2;  // contiguous lines per block
constexpr int kYWarps = 2;  // warps per contiguous line
constexpr int kYPoissonWarps = 4;  // warps per line of the Poisson mode solves
constexpr int kZLines = 4;  // strided lines per block (one warp each)

constexpr int kWinMax = 24;  // longest truncation window of the windowed helsolve

cudaError_t scan_configure();
void launch_win_helsolve(const Dev &d, const SubDev &s, cudaStream_t st);
void launch_scan_helsolve(const Dev &d, const SubDev &s, cudaStream_t st);
// rmax (may be null): n2m row maxima of |hmn| (over the modes) accumulated for
// the INT8 digit cut
void launch_scan_poisson(const Dev &d, cudaStream_t st, double *rmax = nullptr);
void glaunch_win_helsolve(const Group &g, int n, cudaStream_t st);  // substep n (0-based)
void glaunch_scan_poisson(const Group &g, cudaStream_t st);

}  // namespace fb
