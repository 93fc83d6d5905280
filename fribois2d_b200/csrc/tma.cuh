// mbarrier and TMA helpers shared by the tensor-core products and the
// TMA-staged stencil tiles (inline PTX, sm_100a).  Every wait gives up after
// one second and reports it, so that no kernel spins without a bound.
#pragma once
#include <cuda.h>

#include <cstdint>

namespace fb {
namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// has the phase with the given parity completed?  (never suspends the thread)
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// wait for the phase with the given parity; false after one second.  The
// waits poll with test_wait: a try_wait that suspends the thread resumes
// late (a pipeline with its loads and MMAs removed took 2-2.5 us per
// k-block of producer/consumer hand-offs with suspending waits), and each
// waiting thread here is alone on its warp scheduler
__device__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_test_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t i = 1;; ++i) {
        if (mbar_test_wait(bar, parity)) return true;
        if ((i & 255u) == 0 && global_ns() - t0 > 1000000000ull) return false;
    }
}

// the same wait for threads that only wait (the epilogue's): they sleep
// between polls and leave the issue slots to the producer and MMA threads
__device__ bool mbar_wait_idle(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    while (!mbar_test_wait(bar, parity)) {
        __nanosleep(128);
        if (global_ns() - t0 > 1000000000ull) return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
        : "memory");
}

}  // namespace
}  // namespace fb
