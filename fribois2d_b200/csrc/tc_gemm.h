// Split-precision (3xTF32) tensor-core GEMM (definitions in tc_gemm.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "device.cuh"

namespace fb {

struct SplitPlane {      // TF32 high/low parts of an FP64 matrix: rows x K floats, row stride ld
    float *hi, *lo;
    long ld;
};

struct GemmOut {         // out[col * ldo + row] = (base ? base[col * ldb + row] : 0) + C[row][col]
    double *out;
    long ldo;
    const double *base;
    long ldb;
    int M, N;
};

struct Tf32x3Plan {      // tensor maps of one C = A * B^T product
    CUtensorMap a_hi, a_lo, b_hi, b_lo;
    int M, N, K;
    int bn;              // tile width: 64 or 128 columns of C per CTA
};

int tf32x3_configure();
int tf32x3_plan(Tf32x3Plan &p, const SplitPlane &a, const SplitPlane &b, int M, int N, int K, int bn);
void launch_tf32x3(const Tf32x3Plan &p, double *out, long ldo, const double *base, long ldb, int *status,
                   cudaStream_t st);
void launch_split_t(const double *src, long lds, int R, int C, const SplitPlane &dst, cudaStream_t st);
void launch_poisson_residual(const Dev &d, const double *phi, const SplitPlane &dst, cudaStream_t st);

}  // namespace fb
