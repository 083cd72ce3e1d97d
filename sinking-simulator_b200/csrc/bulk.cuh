// bulk.cuh -- bulk asynchronous copies global -> shared memory on sm_100a, completed on
// an mbarrier, with a bounded wait.
//
// One thread arms a CTA-local mbarrier with the byte count it expects and issues
// cp.async.bulk copies (the TMA unit's untiled form: 16-byte aligned addresses, sizes
// a multiple of 16).  The copies land in the CTA's own shared memory and count their
// bytes against the barrier; the barrier's phase flips when all have arrived.  No
// multicast: every copy reads this GPU's own global memory into one CTA.
#pragma once

#include <stdint.h>

namespace fs {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async proxy (the copy engine)
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once and announce `bytes` more bytes of transactions for this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Arrive once with no transactions (a phase with nothing to copy).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Copy `bytes` (a multiple of 16) from 16-byte aligned global `src` to 16-byte aligned
// shared `dst`; completion counts against `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for phase `parity` of `bar` to complete, giving up after `limit` polls (each
// poll may itself suspend the thread for a while).  Returns whether it completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_test(bar, parity)) return true;
    return false;
}

}  // namespace fs
