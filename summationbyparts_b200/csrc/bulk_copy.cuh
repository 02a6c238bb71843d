// Bulk (TMA-engine) copies of contiguous global rows into shared memory, completed on an
// mbarrier, and the bounded wait for them (sm_90+ PTX, used on sm_100a).
//
// cp.async.bulk moves `bytes` (a multiple of 16) from a 16-byte aligned global address to a
// 16-byte aligned shared address without occupying the issuing threads; the copy signals the
// mbarrier with its byte count (complete_tx), and the phase completes once the arrival that
// announced the expected byte total (arrive.expect_tx) and all the announced bytes are in.
// No multicast form is used: every copy reads this GPU's own memory into this CTA.
#pragma once

#include <cstdint>

namespace sbp {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bulk_mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once on the barrier and announce `bytes` still to come from bulk copies.
__device__ __forceinline__ void bulk_expect(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
}

// Global -> shared copy of `bytes` bytes (16-byte aligned ends, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(mbar))
        : "memory");
}

// Wait for the barrier's phase `parity` to complete, polling at most `limit` times; false if it
// did not complete (the caller then skips the work that needed the data).
__device__ __forceinline__ bool bulk_wait(uint64_t* mbar, uint32_t parity, int limit) {
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred q;\nmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\nselp.b32 %0, 1, 0, q;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(mbar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace sbp
