// Split-precision (3xTF32) GEMM on the Blackwell tensor cores, for the
// eigen transforms of the Poisson solve (phcalc_outflow.F90:31,61) in the
// precision form of the time step.
//
//   C[M x N] = A[M x K] * B[N x K]^T,  A = Ahi + Alo, B = Bhi + Blo,
//   C ~ Alo*Bhi + Ahi*Blo + Ahi*Bhi      (FP32 accumulation in TMEM)
//
// Operands are FP32 planes holding TF32-rounded high and low parts of FP64
// values (k_split_t), K contiguous.  One CTA computes a 128 x BN tile:
// one thread issues TMA loads (128-byte swizzle, no multicast) into a
// shared-memory ring of 3 or 4 stages, one thread issues tcgen05.mma
// (kind::tf32, M = 128, N = BN, K = 8) into a TMEM accumulator, and the four warps read
// the accumulator back with tcgen05.ld and store FP64 results.  Every
// mbarrier wait gives up after one second, records FB_ERR_TIMEOUT and lets
// the CTA finish (waiting for its own copies and MMAs, freeing its TMEM).
#include <cooperative_groups.h>
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "../../include/fribois2d.h"
#include "device.cuh"
#include "pdl.h"
#include "tc_gemm.h"
#include "tma.cuh"

namespace fb {

namespace {

constexpr int kBM = 128, kBK = 32, kThreads = 128;
constexpr int kI8Threads = 256;   // the INT8 product: producer and MMA warps, eight epilogue warps

// tile width BN (64 or 128) sets the B tiles, the stage count (192 KB ring),
// the TMEM columns and the instruction descriptor
template <int BN>
struct TcCfg {
    static constexpr int kStages = (BN == 64) ? 4 : 3;
    static constexpr uint32_t kATile = kBM * kBK * 4;                  // 16 KB
    static constexpr uint32_t kBTile = BN * kBK * 4;                   // 8 or 16 KB
    static constexpr uint32_t kStageBytes = 2 * kATile + 2 * kBTile;   // A hi, A lo, B hi, B lo
    static constexpr uint32_t kTmemCols = BN;                          // FP32 accumulator: 128 lanes x BN
    static constexpr size_t kSmem = kStages * kStageBytes + 1024 + 256;
    // instruction descriptor: D FP32, A and B TF32, both K-major, N = BN, M = kBM
    static constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) |
                                       (static_cast<uint32_t>(BN >> 3) << 17) |
                                       (static_cast<uint32_t>(kBM >> 4) << 24);
    static_assert(BN == 64 || BN == 128, "tile widths built");
    static_assert(kStages * kStageBytes + 1024 + 256 <= 227 * 1024, "shared memory per CTA");
};

// tensor maps that the host copied into global memory: make the generic-proxy
// writes visible to the tensor-map proxy before the first TMA copy uses them
__device__ __forceinline__ void acquire_maps(const CUtensorMap *a, const CUtensorMap *b, const CUtensorMap *c,
                                             const CUtensorMap *d) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(a) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(b) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(c) : "memory");
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(d) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major operand, 128-byte swizzle atoms of
// 8 rows x 128 bytes (stride between atoms 1024 bytes), sm100 version bits
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    uint64_t d = static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(1u) << 16;           // leading byte offset (16 B; unused when swizzled)
    d |= static_cast<uint64_t>(1024u >> 4) << 32;   // stride byte offset
    d |= static_cast<uint64_t>(1u) << 46;           // descriptor version
    d |= static_cast<uint64_t>(2u) << 61;           // SWIZZLE_128B
    return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_load32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// the int32 in v as an FP64 value, exactly, with one FP64 subtraction instead
// of a conversion: 2^52 + 2^31 + v has v + 2^31 (v with its sign bit
// flipped) as the low 32 bits of its mantissa
__device__ __forceinline__ double i32_as_f64(uint32_t v) {
    return __hiloint2double(0x43300000, static_cast<int>(v ^ 0x80000000u)) - 4503601774854144.0;
}

// 8 columns of 32 lanes without waiting; tmem_wait8 waits for every load
// issued so far and ties the registers to the wait (their uses follow it),
// tmem_after8 ties further registers to the same point
__device__ __forceinline__ void tmem_load8_async(uint32_t taddr, uint32_t (&r)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait8(uint32_t (&r)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
                 :
                 : "memory");
}

__device__ __forceinline__ void tmem_after8(uint32_t (&r)[8]) {
    asm volatile(""
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7])
                 :
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// (the form without an output-lane mask: every lane of D is written)
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

}  // namespace

// The kernel bodies take the tensor maps by address: kernel parameters for a
// single product, a task array in global memory for grouped products (whose
// maps the producer thread acquires for the tensor-map proxy first).
template <int BN, bool kGlobalMaps>
__device__ __forceinline__ void gemm_body(const CUtensorMap *ma_hi, const CUtensorMap *ma_lo, const CUtensorMap *mb_hi,
                                          const CUtensorMap *mb_lo, const GemmOut &o, int K, int *status) {
    using Cfg = TcCfg<BN>;
    constexpr int kStages = Cfg::kStages;
    constexpr uint32_t kATile = Cfg::kATile, kBTile = Cfg::kBTile, kStageBytes = Cfg::kStageBytes;
    constexpr uint32_t kTmemCols = Cfg::kTmemCols, kIdesc = Cfg::kIdesc;
    constexpr int kBN = BN;
    extern __shared__ uint8_t smraw[];
    const uint32_t raw = smem_u32(smraw);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;  // swizzle atoms need 1024-byte alignment
    uint8_t *sm = smraw + pad;
    const uint32_t sbase = raw + pad;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kStages * kStageBytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 1);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages), done = smem_u32(bars + 2 * kStages);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
    const int nk = (K + kBK - 1) / kBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    if (warp == 0 && lane == 0) {
        // ---- TMA producer
        if (kGlobalMaps) acquire_maps(ma_hi, ma_lo, mb_hi, mb_lo);
        int issued = 0;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
            if (!mbar_wait(empty0 + 8 * s, ph ^ 1u)) {
                ok = false;
                break;
            }
            const uint32_t st = sbase + s * kStageBytes, fb = full0 + 8 * s;
            mbar_expect_tx(fb, kStageBytes);
            tma_load_2d(st, ma_hi, fb, kb * kBK, m0);
            tma_load_2d(st + kATile, ma_lo, fb, kb * kBK, m0);
            tma_load_2d(st + 2 * kATile, mb_hi, fb, kb * kBK, n0);
            tma_load_2d(st + 2 * kATile + kBTile, mb_lo, fb, kb * kBK, n0);
            issued = kb + 1;
        }
        // every copy issued has landed before the CTA may finish
        for (int kb = (issued > kStages ? issued - kStages : 0); kb < issued; ++kb)
            if (!mbar_wait(full0 + 8 * (kb % kStages), static_cast<uint32_t>(kb / kStages) & 1u)) ok = false;
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
            if (!mbar_wait(full0 + 8 * s, ph)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t st = sbase + s * kStageBytes;
#pragma unroll
            for (int k = 0; k < kBK / 8; ++k) {  // K = 8 per MMA: 32 bytes along the swizzled row
                const uint64_t ahi = sw128_desc(st + 32 * k), alo = sw128_desc(st + kATile + 32 * k);
                const uint64_t bhi = sw128_desc(st + 2 * kATile + 32 * k);
                const uint64_t blo = sw128_desc(st + 2 * kATile + kBTile + 32 * k);
                mma_tf32(tmem, alo, bhi, kIdesc, (kb > 0 || k > 0) ? 1u : 0u);
                mma_tf32(tmem, ahi, blo, kIdesc, 1u);
                mma_tf32(tmem, ahi, bhi, kIdesc, 1u);
            }
            mma_commit(empty0 + 8 * s);  // frees the stage once these MMAs have read it
        }
        mma_commit(done);  // arrives when every MMA issued above has completed
    }
    __syncwarp();

    // ---- epilogue: TMEM lane = tile row; warp w owns lanes 32w .. 32w+31
    if (!mbar_wait(done, 0)) ok = false;
    __syncwarp();
    tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    const bool rok = ok && row < o.M;
#pragma unroll 1
    for (int c = 0; c < kBN / 32; ++c) {
        uint32_t r[32];
        tmem_load32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c * 32), r);
        if (rok) {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int col = n0 + c * 32 + i;
                if (col < o.N) {
                    double v = static_cast<double>(__uint_as_float(r[i]));
                    if (o.cscale) v = o.cscale[col] * v;
                    if (o.base) v = o.base[static_cast<size_t>(col) * o.ldb + row] + v;
                    o.out[static_cast<size_t>(col) * o.ldo + row] = v;
                }
            }
        }
    }
    if (!ok) atomicCAS(status, 0, FB_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    k_tf32x3_gemm(const __grid_constant__ CUtensorMap ma_hi, const __grid_constant__ CUtensorMap ma_lo,
                  const __grid_constant__ CUtensorMap mb_hi, const __grid_constant__ CUtensorMap mb_lo,
                  GemmOut o, int K, int *status) {
    FB_GRID_WAIT();
    gemm_body<BN, false>(&ma_hi, &ma_lo, &mb_hi, &mb_lo, o, K, status);
}

// grouped: blockIdx.z selects the product
template <int BN>
__global__ void __launch_bounds__(kThreads, 1) kg_tf32x3_gemm(const GemmTask *__restrict__ t) {
    FB_GRID_WAIT();
    const GemmTask &tk = t[blockIdx.z];
    if (tk.gate && !*tk.gate) return;
    const GemmOut o = tk.o;
    gemm_body<BN, true>(&tk.p.a_hi, &tk.p.a_lo, &tk.p.b_hi, &tk.p.b_lo, o, tk.p.K, tk.status);
}

// ---- the same product on CTA pairs (tcgen05 cta_group::2) ------------------
// A cluster of two CTAs computes a 256 x BN tile: CTA r holds rows
// 128 r .. 128 r + 127 of A and half of B (BN/2 rows) in its shared memory,
// CTA 0's thread issues tcgen05.mma.cta_group::2 (M = 256, N = BN, K = 8)
// which reads both halves, and each CTA's TMEM receives its 128 rows.  Both
// CTAs' TMA loads (no multicast) complete on CTA 0's full barrier; the MMA
// commits arrive on both CTAs' empty and done barriers.  Per CTA and k-block
// this loads 32 KB of A and BN/4 KB of B for 12 MMAs: less operand traffic per
// tensor-core cycle than one CTA per 128 x 128 tile.
template <int BN>
struct TcCfg2 {
    static constexpr int kBH = BN / 2;                                 // B rows per CTA
    static constexpr uint32_t kATile = kBM * kBK * 4;                  // 16 KB
    static constexpr uint32_t kBTile = kBH * kBK * 4;
    static constexpr uint32_t kStageBytes = 2 * kATile + 2 * kBTile;
    static constexpr int kStages = (kStageBytes * 4 + 2048 <= 227 * 1024) ? 4 : 3;
    static constexpr uint32_t kTmemCols = BN <= 128 ? 128 : 256;      // power of two >= BN
    static constexpr size_t kSmem = kStages * kStageBytes + 1024 + 256;
    static constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) |
                                       (static_cast<uint32_t>(BN >> 3) << 17) |
                                       (static_cast<uint32_t>(256 >> 4) << 24);
    static_assert(BN % 32 == 0 && BN >= 64 && BN <= 256 && kBH % 8 == 0, "tile widths built");
    static_assert(kStages * kStageBytes + 1024 + 256 <= 227 * 1024, "shared memory per CTA");
};

namespace {

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t map_to_rank(uint32_t addr, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(rank));
    return out;
}

__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, uint32_t bar_cluster, int x,
                                                 int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void mma_tf32_pair(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                              uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8, %9, %10, %11, %12}, p;\n\t}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z), "r"(z),
        "r"(z), "r"(z)
        : "memory");
}

// arrives once on the barrier at this shared-memory offset in both CTAs of the pair
__device__ __forceinline__ void mma_commit_pair(uint32_t bar) {
    const uint16_t mask = 0x3;
    asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;"
                 ::"r"(bar), "h"(mask)
                 : "memory");
}

}  // namespace

template <int BN, bool kGlobalMaps>
__device__ __forceinline__ void gemm2_body(const CUtensorMap *ma_hi, const CUtensorMap *ma_lo, const CUtensorMap *mb_hi,
                                           const CUtensorMap *mb_lo, const GemmOut &o, int K, int *status) {
    using Cfg = TcCfg2<BN>;
    constexpr int kStages = Cfg::kStages;
    constexpr uint32_t kATile = Cfg::kATile, kBTile = Cfg::kBTile, kStageBytes = Cfg::kStageBytes;
    constexpr uint32_t kTmemCols = Cfg::kTmemCols, kIdesc = Cfg::kIdesc;
    extern __shared__ uint8_t smraw[];
    const uint32_t raw = smem_u32(smraw);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
    uint8_t *sm = smraw + pad;
    const uint32_t sbase = raw + pad;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kStages * kStageBytes);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 1);
    const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + kStages), done = smem_u32(bars + 2 * kStages);

    const uint32_t rank = cluster_rank();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair = blockIdx.x >> 1;
    const int m0 = pair * 2 * kBM + static_cast<int>(rank) * kBM;   // this CTA's rows of A and C
    const int n0 = blockIdx.y * BN;                                  // the pair's columns of C
    const int nb0 = n0 + static_cast<int>(rank) * Cfg::kBH;          // this CTA's rows of B
    const int nk = (K + kBK - 1) / kBK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    cluster_sync();   // both CTAs' barriers and TMEM exist before either signals the other
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    if (warp == 0 && lane == 0) {
        // ---- TMA producer of this CTA: its A rows and B half land on CTA 0's full barrier
        if (kGlobalMaps) acquire_maps(ma_hi, ma_lo, mb_hi, mb_lo);
        int issued = 0;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
            if (!mbar_wait(empty0 + 8 * s, ph ^ 1u)) {
                ok = false;
                break;
            }
            const uint32_t st = sbase + s * kStageBytes, fb_local = full0 + 8 * s;
            const uint32_t fb0 = map_to_rank(fb_local, 0);
            if (rank == 0) mbar_expect_tx(fb_local, 2 * kStageBytes);
            tma_load_2d_pair(st, ma_hi, fb0, kb * kBK, m0);
            tma_load_2d_pair(st + kATile, ma_lo, fb0, kb * kBK, m0);
            tma_load_2d_pair(st + 2 * kATile, mb_hi, fb0, kb * kBK, nb0);
            tma_load_2d_pair(st + 2 * kATile + kBTile, mb_lo, fb0, kb * kBK, nb0);
            issued = kb + 1;
        }
        // the copies in flight have been consumed (or landed) before the CTA may finish
        for (int kb = (issued > kStages ? issued - kStages : 0); kb < issued; ++kb)
            if (!mbar_wait(empty0 + 8 * (kb % kStages), static_cast<uint32_t>(kb / kStages) & 1u)) ok = false;
    } else if (warp == 1 && lane == 0 && rank == 0) {
        // ---- MMA issuer of the pair
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % kStages;
            const uint32_t ph = static_cast<uint32_t>(kb / kStages) & 1u;
            if (!mbar_wait(full0 + 8 * s, ph)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t st = sbase + s * kStageBytes;
#pragma unroll
            for (int k = 0; k < kBK / 8; ++k) {
                const uint64_t ahi = sw128_desc(st + 32 * k), alo = sw128_desc(st + kATile + 32 * k);
                const uint64_t bhi = sw128_desc(st + 2 * kATile + 32 * k);
                const uint64_t blo = sw128_desc(st + 2 * kATile + kBTile + 32 * k);
                mma_tf32_pair(tmem, alo, bhi, kIdesc, (kb > 0 || k > 0) ? 1u : 0u);
                mma_tf32_pair(tmem, ahi, blo, kIdesc, 1u);
                mma_tf32_pair(tmem, ahi, bhi, kIdesc, 1u);
            }
            mma_commit_pair(empty0 + 8 * s);
        }
        mma_commit_pair(done);
    }
    __syncwarp();

    // ---- epilogue: this CTA's 128 rows of the pair's tile
    if (!mbar_wait(done, 0)) ok = false;
    __syncwarp();
    tc_fence_after();
    const int row = m0 + warp * 32 + lane;
    const bool rok = ok && row < o.M;
#pragma unroll 1
    for (int c = 0; c < BN / 32; ++c) {
        uint32_t r[32];
        tmem_load32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c * 32), r);
        if (rok) {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int col = n0 + c * 32 + i;
                if (col < o.N) {
                    double v = static_cast<double>(__uint_as_float(r[i]));
                    if (o.cscale) v = o.cscale[col] * v;
                    if (o.base) v = o.base[static_cast<size_t>(col) * o.ldb + row] + v;
                    o.out[static_cast<size_t>(col) * o.ldo + row] = v;
                }
            }
        }
    }
    if (!ok) atomicCAS(status, 0, FB_ERR_TIMEOUT);
    tc_fence_before();
    cluster_sync();   // neither CTA frees its TMEM or leaves while the pair still uses it
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                     : "memory");
    }
}

template <int BN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1)
    k_tf32x3_gemm2(const __grid_constant__ CUtensorMap ma_hi, const __grid_constant__ CUtensorMap ma_lo,
                   const __grid_constant__ CUtensorMap mb_hi, const __grid_constant__ CUtensorMap mb_lo,
                   GemmOut o, int K, int *status) {
    FB_GRID_WAIT();
    gemm2_body<BN, false>(&ma_hi, &ma_lo, &mb_hi, &mb_lo, o, K, status);
}

// grouped: blockIdx.z selects the product (a cluster never spans two)
template <int BN>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kThreads, 1) kg_tf32x3_gemm2(const GemmTask *__restrict__ t) {
    FB_GRID_WAIT();
    const GemmTask &tk = t[blockIdx.z];
    if (tk.gate && !*tk.gate) return;   // both CTAs of the pair: one case
    const GemmOut o = tk.o;
    gemm2_body<BN, true>(&tk.p.a_hi, &tk.p.a_lo, &tk.p.b_hi, &tk.p.b_lo, o, tk.p.K, tk.status);
}

// dst[r * ldd + c] = (hi, lo) TF32 parts of src[c * lds + r], r < R, c < C:
// the transposed split of a column-major FP64 matrix (32 x 32 tiles)
__device__ __forceinline__ void split_t_body(const double *__restrict__ src, long lds, int R, int C,
                                             float *__restrict__ hi, float *__restrict__ lo, long ldd,
                                             const double *__restrict__ cscale) {
    __shared__ double t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows of 32
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int c = c0 + ty + 8 * i, r = r0 + tx;
        double v = (r < R && c < C) ? src[static_cast<size_t>(c) * lds + r] : 0.0;
        if (cscale && c < C) v = cscale[c] * v;
        t[ty + 8 * i][tx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = r0 + ty + 8 * i, c = c0 + tx;
        if (r < R && c < C) {
            const double x = t[tx][ty + 8 * i];
            const float h = tf32_round(static_cast<float>(x));
            const float l = tf32_round(static_cast<float>(x - static_cast<double>(h)));
            hi[static_cast<size_t>(r) * ldd + c] = h;
            lo[static_cast<size_t>(r) * ldd + c] = l;
        }
    }
}

__global__ void __launch_bounds__(256) k_split_t(const double *__restrict__ src, long lds, int R, int C,
                                                  float *__restrict__ hi, float *__restrict__ lo, long ldd,
                                                  const double *__restrict__ cscale) {
    FB_GRID_WAIT();
    split_t_body(src, lds, R, C, hi, lo, ldd, cscale);
}

// grouped: blockIdx.z selects the matrix (the task array is host-written)
__global__ void __launch_bounds__(256) kg_split_t(const SplitTask *__restrict__ tk, int R, int C) {
    const SplitTask t = tk[blockIdx.z];
    FB_GRID_WAIT();
    if (t.gate && !*t.gate) return;
    split_t_body(t.src, t.lds, R, C, t.hi, t.lo, t.ldd, t.cscale);
}

// FP64 residual of the Poisson equation that phcalc solves,
//   r = dph - (A_yy + A_zz) phi,
// with A_yy = tridiag(amphj, acphj, apphj) along j and A_zz = tridiag(amphk,
// acphk, apphk) along k (the operators of phcalc_outflow.F90:36-45 and
// phini.F90:59-65), written as the transposed TF32 split [j][k] that the
// forward transform reads.  One 32 x 32 tile per block.
__device__ __forceinline__ void poisson_residual_body(const Dev &d, const double *__restrict__ phi,
                                                      float *__restrict__ hi, float *__restrict__ lo, long ldd,
                                                      const double *__restrict__ kscale) {
    __shared__ double t[32][33];
    const int j0 = 1 + blockIdx.x * 32, k0 = 1 + blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int j = j0 + tx;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int k = k0 + ty + 8 * i;
        double r = 0.0;
        if (j <= d.n2m && k <= d.n3m) {
            const double pc = phi[fidx(d, j, k)];
            double lp = (d.acphj[j] + d.acphk[k]) * pc;
            if (j > 1) lp = fma(d.amphj[j], phi[fidx(d, j - 1, k)], lp);
            if (j < d.n2m) lp = fma(d.apphj[j], phi[fidx(d, j + 1, k)], lp);
            if (k > 1) lp = fma(d.amphk[k], phi[fidx(d, j, k - 1)], lp);
            if (k < d.n3m) lp = fma(d.apphk[k], phi[fidx(d, j, k + 1)], lp);
            r = d.dph[fidx(d, j, k)] - lp;
            if (kscale) r = kscale[k - 1] * r;
        }
        t[ty + 8 * i][tx] = r;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int jj = j0 + ty + 8 * i, kk = k0 + tx;
        if (jj <= d.n2m && kk <= d.n3m) {
            const double x = t[tx][ty + 8 * i];
            const float h = tf32_round(static_cast<float>(x));
            const float l = tf32_round(static_cast<float>(x - static_cast<double>(h)));
            hi[static_cast<size_t>(jj - 1) * ldd + (kk - 1)] = h;
            lo[static_cast<size_t>(jj - 1) * ldd + (kk - 1)] = l;
        }
    }
}

__global__ void __launch_bounds__(256) k_poisson_residual(Dev d, const double *__restrict__ phi, float *__restrict__ hi,
                                                           float *__restrict__ lo, long ldd,
                                                           const double *__restrict__ kscale) {
    FB_GRID_WAIT();
    poisson_residual_body(d, phi, hi, lo, ldd, kscale);
}

__global__ void __launch_bounds__(256) kg_poisson_residual(const GroupCase *__restrict__ g,
                                                            const ResidualTask *__restrict__ tk) {
    __shared__ Dev d;
    const ResidualTask t = tk[blockIdx.z];
    if (!stage_case(g, &d)) return;
    poisson_residual_body(d, t.phi, t.hi, t.lo, t.ldd, t.kscale);
}

// ---- FP64 products on the INT8 tensor cores -------------------------------
// C = A B^T to FP64 accuracy from exact integer products (the Ozaki scheme
// with power-of-two row scaling, Ozaki, Ogita, Oishi and Rump): every row r
// of A is scaled by 2^-e(r) (|A(r,k)| < 2^e(r)) and cut into kI8S signed
// 8-bit digits, a = sum_i d_i 128^-(i+1), likewise the rows of B with f(c).
// Then
//   C(r,c) = 2^(e(r)+f(c)) sum_t 128^-(t+2) G_t(r,c),  G_t = sum_{i+j=t} D_i E_j^T,
// keeping the digit pairs with i + j < kI8S.  Each G_t is an exact int32
// sum of tcgen05.mma kind::i8 products accumulated in its own TMEM columns
// (exact while K <= kI8MaxK); the epilogue adds the G_t in FP64 from the
// smallest weight up and applies the power-of-two scales (exact).  The
// error is absolute, relative to the row and column maxima: the digit
// truncation and the dropped pairs leave at most about
// K 2^-55 max|A(r,:)| max|B(c,:)| (each operand is cut to 56 bits of its
// row maximum), plus the rounding of the FP64 additions.  For rows of
// moderate dynamic range that is ~2e-16 of sum |a||b| at K = 1024, as FP64
// DGEMM; a row whose entries span many decades is reproduced only to
// 2^-55 of its largest entry.

// Two forms of the digit cut.  k_i8_cut_rows (the time step, the public
// product) takes each row's maximum from an array that the operand's producer
// (or k_i8_rowmax) accumulated, so its blocks are independent.  k_i8_cut (the
// eigenvector operands at set-up, the batched launches) finds the maxima
// itself: a cluster of kCutCl CTAs per 32 rows, each CTA over its own range of
// 8 V columns.  Thread (lane, warp w) holds V
// consecutive columns of row lane in registers, all its loads in flight at
// once (each load coalesced over the 32 rows); the CTA's row maxima go to the
// cluster through distributed shared memory, so every CTA derives each row's
// exponent from the whole row; then each thread turns its values into 56-bit
// integers (one conversion each), takes the digits from them with shifts,
// four columns to a 32-bit word, and stores each slice's V digit bytes of its
// row with 16-byte stores.  The operand is read once.
// Columns past K and rows past R get zero digits, up to ldk and rows_pad.
constexpr int kCutCl = 8;

// the digits of a thread's V values a of row r (columns c0 ..) at the row's
// scale s = 2^-e into the kI8S slices
template <int V>
__device__ __forceinline__ void i8_cut_emit(const double (&a)[V / 4][4], double s, int r, int c0, int8_t *dig,
                                            long ldk, long plane) {
    constexpr int kP = V / 4;   // 32-bit words (four columns) per thread and slice
    // |a s| < 1, so a s 2^(7 kI8S) (exact: powers of two) truncated toward
    // zero is an integer below 2^(7 kI8S) whose base-128 digits, carrying the
    // sign of a, are the kI8S digits: d_i = sign(a) floor(|a s| 128^(i+1)) mod 128
    unsigned long long u[kP][4];
    uint32_t neg[kP];
#pragma unroll
    for (int p = 0; p < kP; ++p) {
        neg[p] = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const long long v = __double2ll_rz((a[p][q] * s) * 72057594037927936.0);   // 2^56
            u[p][q] = static_cast<unsigned long long>(v < 0 ? -v : v);
            neg[p] |= (v < 0 ? 0xFFu : 0u) << (8 * q);
        }
    }
    static_assert(kI8S == 8, "2^56 = 128^kI8S");
    // each slice's V digits of row r are V consecutive bytes: the thread
    // stores them itself (a whole 32-byte sector between neighbouring warps),
    // no shared-memory transpose; rows up to rows_pad get digits (zero past R)
    const bool live = c0 < ldk;   // ldk is a multiple of 128, so a run is inside or wholly past it
    int8_t *out = dig + static_cast<size_t>(r) * ldk + c0;
    constexpr int kUnroll = (V <= 32) ? kI8S : 1;   // constant shifts where registers allow
#pragma unroll kUnroll
    for (int i = 0; i < kI8S; ++i) {
        const int sh = 7 * (kI8S - 1 - i);
        uint32_t word[kP];
#pragma unroll
        for (int p = 0; p < kP; ++p) {
            uint32_t mag = 0;
#pragma unroll
            for (int q = 0; q < 4; ++q) mag |= static_cast<uint32_t>((u[p][q] >> sh) & 127u) << (8 * q);
            // the negative values' bytes negated (bytewise, no carries between bytes)
            const uint32_t mk = neg[p];
            word[p] = (mag & ~mk) | (__vsub4(0u, mag) & mk);
        }
        if (live) {
            int8_t *o = out + static_cast<size_t>(i) * plane;
#pragma unroll
            for (int v4 = 0; v4 < V / 16; ++v4)
                reinterpret_cast<uint4 *>(o)[v4] =
                    make_uint4(word[4 * v4], word[4 * v4 + 1], word[4 * v4 + 2], word[4 * v4 + 3]);
        }
    }
}

template <int V>
__device__ __forceinline__ void i8_cut_body(const double *__restrict__ src, long lds, int R, int K, int8_t *dig,
                                            long ldk, long plane, double *rowscale) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    constexpr int kP = V / 4;   // 32-bit words (four columns) per thread and slice
    static_assert(V % 16 == 0, "a thread's run of columns is whole 16-byte stores");
    __shared__ double part[32];
    __shared__ double mx[8][32];
    __shared__ double sc[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int rank = static_cast<int>(cl.block_rank());
    const int r0 = (blockIdx.x / kCutCl) * 32, r = r0 + lane;
    const int c0 = rank * 8 * V + V * w;   // this thread's V consecutive columns of row r
    double a[kP][4];
    double m = 0.0;
#pragma unroll
    for (int p = 0; p < kP; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = c0 + 4 * p + q;   // each load coalesced over the warp's 32 rows
            a[p][q] = (r < R && k < K) ? src[static_cast<size_t>(k) * lds + r] : 0.0;
        }
#pragma unroll
    for (int p = 0; p < kP; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) m = fmax(m, fabs(a[p][q]));
    mx[w][lane] = m;
    __syncthreads();
    if (w == 0) {
        for (int q = 1; q < 8; ++q) m = fmax(m, mx[q][lane]);
        part[lane] = m;
    }
    cl.sync();   // every CTA's maxima are written
    if (w == 0) {
        double mm = 0.0;
        for (int q = 0; q < kCutCl; ++q) mm = fmax(mm, *cl.map_shared_rank(&part[lane], q));
        int e = 0;
        if (mm > 0.0) frexp(mm, &e);   // mm < 2^e
        sc[lane] = ldexp(1.0, -e);
        if (rank == 0 && r < R) rowscale[r] = ldexp(1.0, e);
    }
    cl.sync();   // no CTA leaves while another still reads its maxima
    i8_cut_emit<V>(a, sc[lane], r, c0, dig, ldk, plane);
}

// The cut with the rows' maxima of |a| given (accumulated by the operand's
// producer, or by k_i8_rowmax): no exchange between blocks.  Block (x, y):
// rows 32 x .. 32 x + 31 (lane = row), columns 8 V y + V w .. (warp w), the
// layout of the cluster form.  Column group 0 stores the row scales and, for
// the next producer, clears its maxima (clear, may be null).
template <int V>
__global__ void __launch_bounds__(256)
    k_i8_cut_rows(const double *__restrict__ src, long lds, int R, int K, int8_t *dig, long ldk, long plane,
                  double *rowscale, const double *__restrict__ rmax, double *clear) {
    FB_GRID_WAIT();
    constexpr int kP = V / 4;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int r = blockIdx.x * 32 + lane;
    const int c0 = blockIdx.y * 8 * V + V * w;
    double a[kP][4];
#pragma unroll
    for (int p = 0; p < kP; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = c0 + 4 * p + q;   // each load coalesced over the warp's 32 rows
            a[p][q] = (r < R && k < K) ? src[static_cast<size_t>(k) * lds + r] : 0.0;
        }
    const double mm = (r < R) ? rmax[r] : 0.0;
    int e = 0;
    if (mm > 0.0) frexp(mm, &e);   // mm < 2^e
    if (blockIdx.y == 0 && w == 0 && r < R) {
        rowscale[r] = ldexp(1.0, e);
        if (clear) clear[r] = 0.0;
    }
    i8_cut_emit<V>(a, ldexp(1.0, -e), r, c0, dig, ldk, plane);
}

// rmax[r] = max(rmax[r], max_k |src[k lds + r]|) for rows r < R, columns k < K
// (NaN dropped, as fmax does); blocks of 32 rows x 8 column strides
__global__ void __launch_bounds__(256) k_i8_rowmax(const double *__restrict__ src, long lds, int R, int K,
                                                   double *rmax) {
    __shared__ double part[8][32];
    FB_GRID_WAIT();
    const int r = blockIdx.x * 32 + threadIdx.x;
    double m = 0.0;
    if (r < R)
        for (int k = blockIdx.y * 8 + threadIdx.y; k < K; k += gridDim.y * 8)
            m = fmax(m, fabs(src[static_cast<size_t>(k) * lds + r]));
    part[threadIdx.y][threadIdx.x] = m;
    __syncthreads();
    if (threadIdx.y == 0 && r < R) {
        for (int q = 1; q < 8; ++q) m = fmax(m, part[q][threadIdx.x]);
        atomic_max_nonneg(rmax + r, m);
    }
}

template <int V>
__global__ void __cluster_dims__(kCutCl, 1, 1) __launch_bounds__(256)
    k_i8_cut(const double *__restrict__ src, long lds, int R, int K, int8_t *dig, long ldk, long plane,
             double *rowscale) {
    FB_GRID_WAIT();
    i8_cut_body<V>(src, lds, R, K, dig, ldk, plane, rowscale);
}

// grouped (blockIdx.z = case; a cluster never spans two cases)
template <int V>
__global__ void __cluster_dims__(kCutCl, 1, 1) __launch_bounds__(256)
    kg_i8_cut(const I8SplitTask *__restrict__ tk, int R, int K) {
    const I8SplitTask t = tk[blockIdx.z];
    FB_GRID_WAIT();
    if (t.gate && !*t.gate) return;   // the whole cluster: one case
    i8_cut_body<V>(t.src, t.lds, R, K, t.dig, t.ldk, t.ldk * static_cast<long>(t.rows_pad), t.scale);
}

// columns per thread: the CTA's share of ldk over its 8 warps
inline int cut_values(long ldk) {
    const long per = (ldk + 8 * kCutCl - 1) / (8 * kCutCl);
    // at least 16: whole 16-byte stores per slice and thread
    return per <= 16 ? 16 : per <= 32 ? 32 : 64;
}

// BN: output tile width, 64, 48 or 32 (a 128 x 48 tile puts 132 CTAs on a
// 768 x 1024 product where 128 x 64 tiles leave a third of the 148 SMs idle;
// 32 spreads small products over more SMs, one MMA of N = 32 (8 - i) per A slice)
template <int BN>
struct I8Cfg {
    static constexpr uint32_t kATile = 128 * kI8BK;                 // one A digit slice: 128 rows x 128 B
    static constexpr uint32_t kBSlice = BN * kI8BK;                 // one B digit slice
    static constexpr uint32_t kBStage = kI8S * BN * kI8BK;          // all B slices of a k-block
    // as many A slots as the shared memory holds beside two B stages
    static constexpr int kASlots = static_cast<int>((227u * 1024u - 1280u - 2u * kBStage) / kATile);
    static constexpr size_t kSmem = 2 * kBStage + kASlots * kATile + 1024 + 256;
    static constexpr uint32_t kTmemCols = 512;                      // kI8S class accumulators of BN columns
    // D s32 (2), A and B signed 8-bit (1), both K-major, M = 128; N set per MMA
    static constexpr uint32_t kIdescBase = (2u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(128 >> 4) << 24);
    static_assert(kI8S * BN <= 512, "TMEM columns");
    static_assert(BN % 16 == 0 && BN <= 256, "MMA N: a multiple of 16, at most 256");
    static_assert(kASlots >= 2 && kSmem <= 227 * 1024, "shared memory per CTA");
};

// One CTA per 128 x BN tile of C.  Per k-block of 128: the producer
// thread loads all B slices (one barrier) and streams the A slices through
// a ring, two slices per barrier; the MMA thread multiplies A slice i with B
// slices j < kI8S - i into accumulators i + j (MMAs of K = 32 over up to
// 256 / BN slices at once); eight warps drain the accumulators.  Every wait
// gives up after one second with FB_ERR_TIMEOUT.
template <int BN, bool kGlobalMaps>
__device__ __forceinline__ void i8x8_body(const CUtensorMap *ma, const CUtensorMap *mb, const I8Out &o, int K,
                                          int *status) {
    using Cfg = I8Cfg<BN>;
    constexpr int kS = kI8S, kAS = Cfg::kASlots, kAP = kAS / 2;   // A slots, in pairs of slices
    static_assert(kAS % 2 == 0 && kS % 2 == 0, "A slices move in pairs");
    extern __shared__ uint8_t smraw[];
    const uint32_t raw = smem_u32(smraw);
    const uint32_t pad = (1024u - (raw & 1023u)) & 1023u;
    uint8_t *sm = smraw + pad;
    const uint32_t sbase = raw + pad;
    const uint32_t sB = sbase, sA = sbase + 2 * Cfg::kBStage;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + 2 * Cfg::kBStage + kAS * Cfg::kATile);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * 2 + 2 * kAS + 1);
    const uint32_t bfull0 = smem_u32(bars), bempty0 = smem_u32(bars + 2);
    const uint32_t afull0 = smem_u32(bars + 4), aempty0 = smem_u32(bars + 4 + kAS), done = smem_u32(bars + 4 + 2 * kAS);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * BN;
    const int nk = (K + kI8BK - 1) / kI8BK;

    if (threadIdx.x == 0) {
        for (int q = 0; q < 2; ++q) {
            mbar_init(bfull0 + 8 * q, 1);
            mbar_init(bempty0 + 8 * q, 1);
        }
        for (int q = 0; q < kAP; ++q) {
            mbar_init(afull0 + 8 * q, 1);
            mbar_init(aempty0 + 8 * q, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(Cfg::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // The set-up above touches no global memory: under programmatic dependent
    // launch it overlaps the previous kernel's tail.  Every thread but the
    // producer waits for that kernel here; the producer first issues the copies
    // of a B operand that was in place before it (the eigenvector planes), so
    // that they are in flight while the previous kernel drains.
    const bool producer = (warp == 0 && lane == 0);
    if (!kGlobalMaps && !producer) FB_GRID_WAIT();
    // the epilogue's scales: this row's, and columns n0 + lane, n0 + 32 + lane
    const int quarter = warp & 3;
    const int row = m0 + quarter * 32 + lane;
    double rs = 0.0, cs0 = 0.0, cs1 = 0.0;
    auto load_scales = [&]() {
        if (row < o.M) rs = o.rowscale[row];
        if (n0 + lane < o.N) cs0 = o.colscale[n0 + lane];
        if (BN > 32 && lane + 32 < BN && n0 + 32 + lane < o.N) cs1 = o.colscale[n0 + 32 + lane];
    };
    if (!producer) load_scales();

    bool ok = true;
    if (producer) {
        // ---- TMA producer
        if (kGlobalMaps) acquire_maps(ma, ma, mb, mb);
        int pre = 0;   // B stages issued before the wait (both buffers start empty)
        if (!kGlobalMaps && o.b_const) {
            for (; pre < 2 && pre < nk; ++pre) {
                mbar_expect_tx(bfull0 + 8 * pre, Cfg::kBStage);
                for (int j = 0; j < kS; ++j)
                    tma_load_3d(sB + pre * Cfg::kBStage + j * Cfg::kBSlice, mb, bfull0 + 8 * pre, pre * kI8BK, n0, j);
            }
        }
        if (!kGlobalMaps) FB_GRID_WAIT();
        load_scales();
        int ip = 0, nb = pre, ps = 0;   // A slice pairs issued, B stages issued, pair slot
        uint32_t aph = 0;
        for (int kb = 0; kb < nk && ok; ++kb) {
            const int sb = kb & 1;
            if (kb >= pre) {
                if (!mbar_wait(bempty0 + 8 * sb, (static_cast<uint32_t>(kb >> 1) & 1u) ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(bfull0 + 8 * sb, Cfg::kBStage);
                for (int j = 0; j < kS; ++j)
                    tma_load_3d(sB + sb * Cfg::kBStage + j * Cfg::kBSlice, mb, bfull0 + 8 * sb, kb * kI8BK, n0, j);
                nb = kb + 1;
            }
#pragma unroll
            for (int i = 0; i < kS; i += 2) {   // slices i, i + 1 on one barrier
                if (!mbar_wait(aempty0 + 8 * ps, aph ^ 1u)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(afull0 + 8 * ps, 2 * Cfg::kATile);
                tma_load_3d(sA + (2 * ps) * Cfg::kATile, ma, afull0 + 8 * ps, kb * kI8BK, m0, i);
                tma_load_3d(sA + (2 * ps + 1) * Cfg::kATile, ma, afull0 + 8 * ps, kb * kI8BK, m0, i + 1);
                ++ip;
                if (++ps == kAP) {
                    ps = 0;
                    aph ^= 1u;
                }
            }
        }
        // every copy issued has landed before the CTA may finish
        for (int q = (ip > kAP ? ip - kAP : 0); q < ip; ++q)
            if (!mbar_wait(afull0 + 8 * (q % kAP), static_cast<uint32_t>(q / kAP) & 1u)) ok = false;
        for (int q = (nb > 2 ? nb - 2 : 0); q < nb; ++q)
            if (!mbar_wait(bfull0 + 8 * (q & 1), static_cast<uint32_t>(q >> 1) & 1u)) ok = false;
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer.  One thread issues every MMA, so its loop is kept
        // lean: descriptors advance by constants (the 14-bit address field
        // holds byte address / 16), the digit loops are unrolled, and one MMA
        // covers up to 256 / BN B slices (N <= 256).
        constexpr int kG = 256 / BN;
        const uint64_t adesc = sw128_desc(sA), bdesc = sw128_desc(sB);
        int ps = 0;
        uint32_t aph = 0;
        for (int kb = 0; kb < nk && ok; ++kb) {
            const int sb = kb & 1;
            if (!mbar_wait(bfull0 + 8 * sb, static_cast<uint32_t>(kb >> 1) & 1u)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint64_t bst = bdesc + static_cast<uint64_t>((sb * Cfg::kBStage) >> 4);
#pragma unroll
            for (int i2 = 0; i2 < kS; i2 += 2) {   // A slices i2, i2 + 1: one wait, one commit
                if (!mbar_wait(afull0 + 8 * ps, aph)) {
                    ok = false;
                    break;
                }
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int i = i2 + e;
                    const uint64_t ast = adesc + static_cast<uint64_t>(((2 * ps + e) * Cfg::kATile) >> 4);
                    // B slices j0 .. j0+nsl-1 are consecutive rows in shared memory and
                    // their classes i+j0 .. consecutive TMEM column blocks: one MMA of
                    // N = nsl * BN covers nsl digit pairs
#pragma unroll
                    for (int j0 = 0; j0 < kS - i; j0 += kG) {
                        const int nsl = (kS - i - j0 < kG) ? kS - i - j0 : kG;
                        const uint32_t idesc = Cfg::kIdescBase | (static_cast<uint32_t>((nsl * BN) >> 3) << 17);
                        const uint32_t acc_t = tmem + static_cast<uint32_t>((i + j0) * BN);
                        const uint64_t bj = bst + static_cast<uint64_t>((j0 * Cfg::kBSlice) >> 4);
#pragma unroll
                        for (int kk = 0; kk < kI8BK / 32; ++kk)   // K = 32 bytes per MMA: +2 in the address field
                            mma_i8(acc_t, ast + 2 * kk, bj + 2 * kk, idesc, (kb > 0 || i > 0 || kk > 0) ? 1u : 0u);
                    }
                }
                mma_commit(aempty0 + 8 * ps);   // frees the two A slots once these MMAs have read them
                if (++ps == kAP) {
                    ps = 0;
                    aph ^= 1u;
                }
            }
            if (!ok) break;
            mma_commit(bempty0 + 8 * sb);
        }
        mma_commit(done);
    }
    __syncwarp();

    // ---- epilogue: TMEM lane = tile row; accumulators summed in FP64 from the
    // smallest weight up.  Eight warps: warp w reads TMEM lanes 32 (w % 4) ..
    // (its rows) and every other 8-column chunk, starting at chunk w / 4.
    if (!mbar_wait_idle(done, 0)) ok = false;
    __syncwarp();
    tc_fence_after();
    const bool rok = ok && row < o.M;
#pragma unroll 1
    for (int c = warp >> 2; c < BN / 8; c += kI8Threads / 128) {
        uint32_t v[kS][8];
#pragma unroll
        for (int t = 0; t < kS; ++t)
            tmem_load8_async(tmem + (static_cast<uint32_t>(quarter * 32) << 16) + static_cast<uint32_t>(t * BN + c * 8),
                             v[t]);
        tmem_wait8(v[0]);
#pragma unroll
        for (int t = 1; t < kS; ++t) tmem_after8(v[t]);
        double acc[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = 0.0;
#pragma unroll
        for (int t = kS - 1; t >= 0; --t) {
            const double wgt = ldexp(1.0, -7 * (t + 2));
#pragma unroll
            for (int q = 0; q < 8; ++q) acc[q] = acc[q] + i32_as_f64(v[t][q]) * wgt;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int cc = c * 8 + q, col = n0 + cc;   // cc is the same on every lane
            const double cs = __shfl_sync(0xffffffffu, cc < 32 ? cs0 : cs1, cc & 31);
            if (rok && col < o.N) o.out[static_cast<size_t>(col) * o.ldo + row] = acc[q] * rs * cs;
        }
    }
    if (!ok) atomicCAS(status, 0, FB_ERR_TIMEOUT);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::kTmemCols)
                     : "memory");
    }
}

template <int BN>
__global__ void __launch_bounds__(kI8Threads, 1)
    k_i8x8_gemm(const __grid_constant__ CUtensorMap ma, const __grid_constant__ CUtensorMap mb, I8Out o, int K,
                int *status) {
    i8x8_body<BN, false>(&ma, &mb, o, K, status);   // waits for the previous kernel after its set-up
}

// grouped: blockIdx.z selects the product
template <int BN>
__global__ void __launch_bounds__(kI8Threads, 1) kg_i8x8_gemm(const I8Task *__restrict__ t) {
    FB_GRID_WAIT();
    const I8Task &tk = t[blockIdx.z];
    if (tk.gate && !*tk.gate) return;
    const I8Out o = tk.o;
    i8x8_body<BN, true>(&tk.a, &tk.b, o, tk.K, tk.status);
}

void launch_poisson_residual(const Dev &d, const double *phi, const SplitPlane &dst, cudaStream_t st,
                             const double *kscale) {
    const dim3 grid((d.n2m + 31) / 32, (d.n3m + 31) / 32);
    pdl(k_poisson_residual, dim3(grid), dim3(256), 0, st, d, phi, dst.hi, dst.lo, dst.ld, kscale);
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int encode_plane(CUtensorMap *m, const float *p, int rows, int K, long ld, int box_rows) {
    if (!g_encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return FB_ERR_CUDA;
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if ((reinterpret_cast<uintptr_t>(p) & 15u) || (ld % 4) || ld < K) return FB_ERR_STATE;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 4u};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kBK), static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(p), dims, strides, box, es,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? FB_OK : FB_ERR_CUDA;
}

}  // namespace

int tf32x3_configure() {
    const bool ok =
        cudaFuncSetAttribute(k_tf32x3_gemm<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg<64>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(k_tf32x3_gemm<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg<128>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(k_tf32x3_gemm2<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg2<128>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(k_tf32x3_gemm2<192>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg2<192>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(k_tf32x3_gemm2<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg2<256>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(kg_tf32x3_gemm<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg<64>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(kg_tf32x3_gemm<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg<128>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(kg_tf32x3_gemm2<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg2<128>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(kg_tf32x3_gemm2<192>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg2<192>::kSmem)) == cudaSuccess &&
        cudaFuncSetAttribute(kg_tf32x3_gemm2<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(TcCfg2<256>::kSmem)) == cudaSuccess;
    return ok ? FB_OK : FB_ERR_CUDA;
}

bool tf32x3_shape_ok(int bn) {
    return bn == 64 || bn == 128 || bn == kPairTile + 128 || bn == kPairTile + 192 || bn == kPairTile + 256;
}

int tf32x3_plan(Tf32x3Plan &p, const SplitPlane &a, const SplitPlane &b, int M, int N, int K, int bn) {
    if (!tf32x3_shape_ok(bn)) return FB_ERR_STATE;
    // B boxes: a CTA's tile width, or half the pair's width for CTA pairs
    const int brows = (bn > kPairTile) ? (bn - kPairTile) / 2 : bn;
    int st;
    if ((st = encode_plane(&p.a_hi, a.hi, M, K, a.ld, kBM))) return st;
    if ((st = encode_plane(&p.a_lo, a.lo, M, K, a.ld, kBM))) return st;
    if ((st = encode_plane(&p.b_hi, b.hi, N, K, b.ld, brows))) return st;
    if ((st = encode_plane(&p.b_lo, b.lo, N, K, b.ld, brows))) return st;
    p.M = M;
    p.N = N;
    p.K = K;
    p.bn = bn;
    return FB_OK;
}

void launch_tf32x3(const Tf32x3Plan &p, double *out, long ldo, const double *base, long ldb, int *status,
                   cudaStream_t st, const double *cscale) {
    GemmOut o{out, ldo, base, ldb, cscale, p.M, p.N};
    if (p.bn > kPairTile) {   // CTA pairs: 256 rows per cluster of two
        const int bn = p.bn - kPairTile;
        const dim3 g2(2 * ((p.M + 2 * kBM - 1) / (2 * kBM)), (p.N + bn - 1) / bn);
        if (bn == 128)
            pdl(k_tf32x3_gemm2<128>, g2, dim3(kThreads), TcCfg2<128>::kSmem, st, p.a_hi, p.a_lo, p.b_hi, p.b_lo, o,
                p.K, status);
        else if (bn == 192)
            pdl(k_tf32x3_gemm2<192>, g2, dim3(kThreads), TcCfg2<192>::kSmem, st, p.a_hi, p.a_lo, p.b_hi, p.b_lo, o,
                p.K, status);
        else
            pdl(k_tf32x3_gemm2<256>, g2, dim3(kThreads), TcCfg2<256>::kSmem, st, p.a_hi, p.a_lo, p.b_hi, p.b_lo, o,
                p.K, status);
        return;
    }
    const dim3 grid((p.M + kBM - 1) / kBM, (p.N + p.bn - 1) / p.bn);
    if (p.bn == 64)
        pdl(k_tf32x3_gemm<64>, dim3(grid), dim3(kThreads), TcCfg<64>::kSmem, st, p.a_hi, p.a_lo, p.b_hi, p.b_lo, o, p.K, status);
    else
        pdl(k_tf32x3_gemm<128>, dim3(grid), dim3(kThreads), TcCfg<128>::kSmem, st, p.a_hi, p.a_lo, p.b_hi, p.b_lo, o, p.K, status);
}

void launch_tf32x3_group(const GemmTask *tasks, const Tf32x3Plan &p, int n, cudaStream_t st) {
    if (p.bn > kPairTile) {
        const int bn = p.bn - kPairTile;
        const dim3 g2(2 * ((p.M + 2 * kBM - 1) / (2 * kBM)), (p.N + bn - 1) / bn, n);
        if (bn == 128) pdl(kg_tf32x3_gemm2<128>, g2, dim3(kThreads), TcCfg2<128>::kSmem, st, tasks);
        else if (bn == 192) pdl(kg_tf32x3_gemm2<192>, g2, dim3(kThreads), TcCfg2<192>::kSmem, st, tasks);
        else pdl(kg_tf32x3_gemm2<256>, g2, dim3(kThreads), TcCfg2<256>::kSmem, st, tasks);
        return;
    }
    const dim3 grid((p.M + kBM - 1) / kBM, (p.N + p.bn - 1) / p.bn, n);
    if (p.bn == 64) pdl(kg_tf32x3_gemm<64>, grid, dim3(kThreads), TcCfg<64>::kSmem, st, tasks);
    else pdl(kg_tf32x3_gemm<128>, grid, dim3(kThreads), TcCfg<128>::kSmem, st, tasks);
}

void launch_split_t_group(const SplitTask *tasks, int R, int C, int n, cudaStream_t st) {
    const dim3 grid((R + 31) / 32, (C + 31) / 32, n);
    pdl(kg_split_t, grid, dim3(256), 0, st, tasks, R, C);
}

void launch_poisson_residual_group(const Group &g, const ResidualTask *tasks, cudaStream_t st) {
    const dim3 grid((g.rep.n2m + 31) / 32, (g.rep.n3m + 31) / 32, g.n);
    pdl(kg_poisson_residual, grid, dim3(256), 0, st, g.cases, tasks);
}

void launch_split_t(const double *src, long lds, int R, int C, const SplitPlane &dst, cudaStream_t st,
                    const double *cscale) {
    const dim3 grid((R + 31) / 32, (C + 31) / 32);
    pdl(k_split_t, dim3(grid), dim3(256), 0, st, src, lds, R, C, dst.hi, dst.lo, dst.ld, cscale);
}


// ---- INT8 FP64 products: buffers, maps, launches
int i8_plan(I8Plan &p, int rows, int K, int box_rows) {
    if (K > kI8MaxK) return FB_ERR_UNSUPPORTED;   // the int32 class sums would overflow
    if (box_rows != 128 && box_rows != 64 && box_rows != 48 && box_rows != 32) return FB_ERR_STATE;
    if (!p.dig || (p.ldk % 128) || p.rows_pad < rows) return FB_ERR_STATE;
    if (!g_encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return FB_ERR_CUDA;
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if (reinterpret_cast<uintptr_t>(p.dig) & 15u) return FB_ERR_STATE;
    const cuuint64_t dims[3] = {static_cast<cuuint64_t>(p.ldk), static_cast<cuuint64_t>(p.rows_pad),
                                static_cast<cuuint64_t>(kI8S)};
    const cuuint64_t strides[2] = {static_cast<cuuint64_t>(p.ldk),
                                   static_cast<cuuint64_t>(p.ldk) * static_cast<cuuint64_t>(p.rows_pad)};
    const cuuint32_t box[3] = {static_cast<cuuint32_t>(kI8BK), static_cast<cuuint32_t>(box_rows), 1};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUresult r = g_encode(&p.map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, p.dig, dims, strides, box, es,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    p.rows = rows;
    p.K = K;
    p.box = box_rows;
    return r == CUDA_SUCCESS ? FB_OK : FB_ERR_CUDA;
}

int i8_configure() {
    const bool ok = cudaFuncSetAttribute(k_i8x8_gemm<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(I8Cfg<64>::kSmem)) == cudaSuccess &&
                    cudaFuncSetAttribute(kg_i8x8_gemm<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(I8Cfg<64>::kSmem)) == cudaSuccess &&
                    cudaFuncSetAttribute(k_i8x8_gemm<48>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(I8Cfg<48>::kSmem)) == cudaSuccess &&
                    cudaFuncSetAttribute(kg_i8x8_gemm<48>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(I8Cfg<48>::kSmem)) == cudaSuccess &&
                    cudaFuncSetAttribute(k_i8x8_gemm<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(I8Cfg<32>::kSmem)) == cudaSuccess &&
                    cudaFuncSetAttribute(kg_i8x8_gemm<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(I8Cfg<32>::kSmem)) == cudaSuccess;
    return ok ? FB_OK : FB_ERR_CUDA;
}

void launch_i8_split_group(const I8SplitTask *tasks, const I8Plan &rep, int R, int K, int n, cudaStream_t st) {
    const dim3 grid(rep.rows_pad / 32 * kCutCl, 1, n);
    switch (cut_values(rep.ldk)) {
#define FB_CUT_CASE(V) \
    case V: pdl(kg_i8_cut<V>, grid, dim3(256), 0, st, tasks, R, K); break;
        FB_CUT_CASE(16) FB_CUT_CASE(32)
#undef FB_CUT_CASE
    default: pdl(kg_i8_cut<64>, grid, dim3(256), 0, st, tasks, R, K); break;
    }
}

void launch_i8x8_group(const I8Task *tasks, int M, int N, int n, int bn, cudaStream_t st) {
    const dim3 grid((M + 127) / 128, (N + bn - 1) / bn, n);
    if (bn == 48) pdl(kg_i8x8_gemm<48>, grid, dim3(kI8Threads), I8Cfg<48>::kSmem, st, tasks);
    else if (bn == 32) pdl(kg_i8x8_gemm<32>, grid, dim3(kI8Threads), I8Cfg<32>::kSmem, st, tasks);
    else pdl(kg_i8x8_gemm<64>, grid, dim3(kI8Threads), I8Cfg<64>::kSmem, st, tasks);
}

void launch_i8_split(const double *src, long lds, int R, int K, const I8Plan &p, cudaStream_t st) {
    const dim3 grid(p.rows_pad / 32 * kCutCl);
    const long plane = p.ldk * static_cast<long>(p.rows_pad);
    switch (cut_values(p.ldk)) {
#define FB_CUT_CASE(V) \
    case V: pdl(k_i8_cut<V>, grid, dim3(256), 0, st, src, lds, R, K, p.dig, p.ldk, plane, p.scale); break;
        FB_CUT_CASE(16) FB_CUT_CASE(32)
#undef FB_CUT_CASE
    default: pdl(k_i8_cut<64>, grid, dim3(256), 0, st, src, lds, R, K, p.dig, p.ldk, plane, p.scale); break;
    }
}

void launch_i8_cut_rows(const double *src, long lds, int R, int K, const I8Plan &p, const double *rmax,
                        double *clear, cudaStream_t st) {
    const dim3 grid(p.rows_pad / 32, kCutCl);
    const long plane = p.ldk * static_cast<long>(p.rows_pad);
    switch (cut_values(p.ldk)) {
#define FB_CUT_CASE(V)                                                                                           \
    case V:                                                                                                      \
        pdl(k_i8_cut_rows<V>, grid, dim3(256), 0, st, src, lds, R, K, p.dig, p.ldk, plane, p.scale, rmax, clear); \
        break;
        FB_CUT_CASE(16) FB_CUT_CASE(32)
#undef FB_CUT_CASE
    default:
        pdl(k_i8_cut_rows<64>, grid, dim3(256), 0, st, src, lds, R, K, p.dig, p.ldk, plane, p.scale, rmax, clear);
        break;
    }
}

void launch_i8_rowmax(const double *src, long lds, int R, int K, double *rmax, cudaStream_t st) {
    const dim3 grid((R + 31) / 32, std::max(1, std::min((K + 7) / 8, 16)));
    pdl(k_i8_rowmax, grid, dim3(32, 8), 0, st, src, lds, R, K, rmax);
}

// the tile width is the B operand's box height (i8_plan)
void launch_i8x8(const I8Plan &a, const I8Plan &b, double *out, long ldo, int *status, cudaStream_t st,
                 bool b_const) {
    I8Out o{out, ldo, a.scale, b.scale, a.rows, b.rows, b_const ? 1 : 0};
    const dim3 grid((a.rows + 127) / 128, (b.rows + b.box - 1) / b.box);
    if (b.box == 48) pdl(k_i8x8_gemm<48>, grid, dim3(kI8Threads), I8Cfg<48>::kSmem, st, a.map, b.map, o, a.K, status);
    else if (b.box == 32) pdl(k_i8x8_gemm<32>, grid, dim3(kI8Threads), I8Cfg<32>::kSmem, st, a.map, b.map, o, a.K, status);
    else pdl(k_i8x8_gemm<64>, grid, dim3(kI8Threads), I8Cfg<64>::kSmem, st, a.map, b.map, o, a.K, status);
}

}  // namespace fb
