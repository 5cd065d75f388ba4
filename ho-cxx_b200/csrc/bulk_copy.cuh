// bulk_copy.cuh -- one-dimensional bulk copies global -> shared through the Tensor Memory
// Accelerator (cp.async.bulk, sm_90+), completed on a shared-memory mbarrier.
//
// The copies are plain (no cluster multicast) and read this GPU's own memory: source and
// destination 16-byte aligned, size a multiple of 16 bytes. A waiting thread polls the
// barrier a bounded number of times; a wait that runs out reports false, and the caller
// records the failure for the host instead of spinning on.
#pragma once

#include <cstdint>

namespace ho2d {

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Initialise a barrier that completes when one arrival and the expected bytes are in, and
// make the initialisation visible to the copy engine.
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// The one arrival, announcing `bytes` of copies that will complete on this barrier.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst[0, bytes) = src[0, bytes), completing on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of bar to complete; false if it has not after `polls` polls
// (about polls x 64 ns).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned polls) {
    for (unsigned i = 0; i < polls; ++i) {
        if (mbar_test(bar, parity)) return true;
        __nanosleep(64);
    }
    return false;
}

// Polls of a first wait (about a quarter of a second) and of the second wait a kernel
// makes, after recording a timeout, for copies it still has in flight.
constexpr unsigned kBulkWaitPolls = 1u << 22;

}  // namespace ho2d
