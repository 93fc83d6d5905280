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

struct GemmOut {         // out[col * ldo + row] = (base ? base[col * ldb + row] : 0) + cscale[col] C[row][col]
    double *out;
    long ldo;
    const double *base;
    long ldb;
    const double *cscale;  // per-column factor (null: 1)
    int M, N;
};

// tile codes: 64 or 128 = one CTA per 128 x code tile; kPairTile + w = a CTA
// pair (tcgen05 cta_group::2) per 256 x w tile, w = 128, 192 or 256
constexpr int kPairTile = 1000;

struct Tf32x3Plan {      // tensor maps of one C = A * B^T product
    CUtensorMap a_hi, a_lo, b_hi, b_lo;
    int M, N, K;
    int bn;              // tile code (kPairTile above)
};

// grouped launches (blockIdx.z = product or case), task arrays in device memory
// gate (all task kinds): the product or split runs only while *gate is
// non-zero (null: always) -- the case's strong-coupling iteration is active
struct GemmTask {        // one product: its tensor maps, output and status word
    Tf32x3Plan p;
    GemmOut o;
    int *status;
    const int *gate;
};
struct SplitTask {       // one transposed split: src (lds) -> hi, lo (ldd), column factors
    const double *src;
    long lds;
    float *hi, *lo;
    long ldd;
    const double *cscale;
    const int *gate;
};
struct ResidualTask {    // one Poisson residual: phi -> hi, lo (ldd), row factors
    const double *phi;
    float *hi, *lo;
    long ldd;
    const double *kscale;
};

// FP64 products C = A B^T on the INT8 tensor cores (kI8S digit slices per
// operand; tc_gemm.cu).  An operand: digit planes [slice][row][k] of
// rows_pad x ldk bytes (ldk a multiple of 128), 2^e per row, its tensor map.
constexpr int kI8S = 8;       // digit slices per operand
constexpr int kI8BK = 128;    // K bytes per k-block (one 128-byte swizzle row)
constexpr int kI8BN = 64;     // output tile width (the default; 48 is the other choice)
// Largest K of one product: weight class t = kI8S - 1 sums kI8S digit pairs
// of at most 127 * 127 per k into an int32 TMEM accumulator, so
// K * kI8S * 127^2 must stay below 2^31 (K <= 16642); i8_plan rejects more.
constexpr int kI8MaxK = 16384;

// The INT8 product's tile width for C[rows x cols] (one CTA per 128 x width
// tile): the width of 64, 48 or 32 that minimises (CTA waves on sms SMs) x
// width, ties to the wider tile.  A CTA's time grows with its width, so this
// is the product's time in units of one column of one wave.
inline int i8_tile_width(int rows, int cols, int sms = 148) {
    const int mt = (rows + 127) / 128;
    int best_w = 64;
    long best = -1;
    for (int w : {64, 48, 32}) {
        const long ctas = static_cast<long>(mt) * ((cols + w - 1) / w);
        const long cost = ((ctas + sms - 1) / sms) * w;
        if (best < 0 || cost < best) {
            best = cost;
            best_w = w;
        }
    }
    return best_w;
}
struct I8Plan {
    CUtensorMap map;
    int8_t *dig;
    double *scale;            // 2^e(row)
    long ldk;
    int rows_pad, rows, K;
    int box;                  // rows per TMA box: 128 (A) or the output tile width (B: 48 or 64)
};
struct I8Out {
    double *out;
    long ldo;
    const double *rowscale, *colscale;
    int M, N;
    int b_const = 0;   // B's digit planes and scales were written before the previous kernel ran
};
// grouped launches (blockIdx.z = case): per-case split sources and products
struct I8SplitTask {
    const double *src;
    long lds;
    int8_t *dig;
    long ldk;
    double *scale;
    int rows_pad;
    const int *gate;
};
struct I8Task {
    CUtensorMap a, b;
    I8Out o;
    int K;
    int *status;
    const int *gate;
};
int i8_configure();
// box_rows: 128 for the A operand, the output tile width (48 or 64) for B
int i8_plan(I8Plan &p, int rows, int K, int box_rows);
// digits of the column-major source A(r, k) = src[k * lds + r], r < R, k < K
void launch_i8_split(const double *src, long lds, int R, int K, const I8Plan &p, cudaStream_t st);
// the cut with the rows' maxima of |src| given in rmax (R entries); clear
// (R entries, may be null) is zeroed for the next producer's maxima
void launch_i8_cut_rows(const double *src, long lds, int R, int K, const I8Plan &p, const double *rmax,
                        double *clear, cudaStream_t st);
// rmax[r] = max(rmax[r], max_k |src(r, k)|); rmax must start at zero
void launch_i8_rowmax(const double *src, long lds, int R, int K, double *rmax, cudaStream_t st);
// out[c * ldo + r] = sum_k A(r, k) B(c, k)
// b_const: b's planes and scales were written before the previous kernel in
// the stream started (the constant eigenvector operand), so its first copies
// may be issued before waiting for that kernel
void launch_i8x8(const I8Plan &a, const I8Plan &b, double *out, long ldo, int *status, cudaStream_t st,
                 bool b_const = false);
// the same over n cases of one shape (rep: geometry of the split)
void launch_i8_split_group(const I8SplitTask *tasks, const I8Plan &rep, int R, int K, int n, cudaStream_t st);
void launch_i8x8_group(const I8Task *tasks, int M, int N, int n, int bn, cudaStream_t st);

int tf32x3_configure();
bool tf32x3_shape_ok(int bn);
int tf32x3_plan(Tf32x3Plan &p, const SplitPlane &a, const SplitPlane &b, int M, int N, int K, int bn);
void launch_tf32x3(const Tf32x3Plan &p, double *out, long ldo, const double *base, long ldb, int *status,
                   cudaStream_t st, const double *cscale = nullptr);
// cscale (may be null): factor of source column c before splitting
void launch_split_t(const double *src, long lds, int R, int C, const SplitPlane &dst, cudaStream_t st,
                    const double *cscale = nullptr);
void launch_poisson_residual(const Dev &d, const double *phi, const SplitPlane &dst, cudaStream_t st,
                             const double *kscale = nullptr);
// the same over n products / cases; every product has the shape and tile of p
void launch_tf32x3_group(const GemmTask *tasks, const Tf32x3Plan &p, int n, cudaStream_t st);
void launch_split_t_group(const SplitTask *tasks, int R, int C, int n, cudaStream_t st);
void launch_poisson_residual_group(const Group &g, const ResidualTask *tasks, cudaStream_t st);

}  // namespace fb
