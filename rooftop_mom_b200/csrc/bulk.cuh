// Bulk asynchronous copies global -> shared memory (cp.async.bulk, the untiled TMA form) completed on
// an mbarrier, with bounded waits. Device code only.
//
// One thread arms a barrier with the bytes it expects (mbarrier.arrive.expect_tx) and issues the copies;
// every thread that reads the data waits for the barrier's phase to flip. Each copy needs 16-byte
// aligned source and destination and a size that is a multiple of 16 bytes. No multicast is used: every
// CTA copies only for itself, from this GPU's own memory.
//
// A wait gives up after kBulkWaitTries polls (each poll may suspend the thread for a short, hardware
// chosen time; the bound is far above any real copy time). It then records RTM_ERR_TIMEOUT in the
// fault word passed to it, and the caller returns without using the data; the host reads the word
// after its next synchronisation (device_fault_check) and reports the timeout instead of a result.
#pragma once

#include <stdint.h>

#include "internal.h"

namespace rtm {

constexpr unsigned kBulkWaitTries = 1u << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes initialised barriers visible to the asynchronous (TMA) proxy before the first copy uses them.
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bytes of global memory at src into shared memory at dst, completing on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits until the barrier's phase with the given parity has completed. Returns false, after recording
// RTM_ERR_TIMEOUT in *fault, if it did not within kBulkWaitTries polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* fault) {
    for (unsigned i = 0; i < kBulkWaitTries; ++i)
        if (mbar_test(bar, parity)) return true;
    if (fault) atomicExch(fault, (int)RTM_ERR_TIMEOUT);
    return false;
}

}  // namespace rtm
