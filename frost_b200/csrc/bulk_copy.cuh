// 1-D bulk asynchronous copies (cp.async.bulk, global -> this CTA's shared
// memory, no multicast) completing on shared-memory mbarriers, with bounded
// waits. Used by the pipelined FDMT level kernel and the search kernel.
//
// Rules the callers keep: source and destination 16-byte aligned, size a
// multiple of 16 bytes, one elected thread arms a barrier (expect_tx) and
// issues the copies that complete on it, and a buffer is refilled only after
// a __syncthreads that follows every thread's last read of it.
#pragma once

#include <cstdint>

namespace fb::bulk {

/** Iterations of mbarrier.try_wait before a wait gives up (each try may
 * suspend the thread for a hardware-defined interval). */
constexpr long kSpinLimit = 1L << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

/** Initialises `bar` for one arrival per phase; call from one thread, then
 * __syncthreads before any use. */
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    return done != 0;
}

/** Waits for phase `phase` of `bar` to complete; false if it did not within
 * `limit` tries (kSpinLimit by default). */
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit = kSpinLimit) {
    const uint32_t b = smem_addr(bar);
    for (long long it = 0; it < limit; ++it)
        if (mbar_try(b, phase))
            return true;
    return false;
}

/** Arms `bar` for `bytes` of copies (the elected thread's arrival). */
__device__ __forceinline__ void mbar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

/** dst[0..bytes) <- src[0..bytes), completing on `bar`. */
__device__ __forceinline__ void load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

/** Starts fetching global [src, src + bytes) into L2 (no shared memory, no
 * completion to wait for): a later bulk copy of the range then waits for
 * L2, not HBM. 16-byte aligned, a multiple of 16 bytes. */
__device__ __forceinline__ void prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

} // namespace fb::bulk
