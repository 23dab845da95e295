// Time-ordered streaming of a block's channel columns through shared memory.
//
// The order-exact statistics kernels give each thread one channel and walk
// it in time order (their double sums must follow the reference's order).
// Read straight from HBM, each step is one byte (or word) per thread with
// a row stride between steps: few bytes in flight and latency-bound. Here
// the block's threads instead copy whole row segments (the block's
// channels, 16-byte cp.async copies, coalesced) a stage of rows at a time,
// two to eight stages deep, and then every thread walks its column in
// shared memory.
//
// Requirements (the launchers check them and otherwise use the direct
// kernels): the row pitch and the segment's byte offset are multiples of
// 16 bytes.
#pragma once

#include <cstdint>

namespace fb::rfi::stage {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }

template <int N> __device__ __forceinline__ void wait_pending() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

/** Copies the first `copy_bytes` of rows [r0, r0 + nr) of a segment (row r
 * at src + r * pitch) to dst[nr][seg_bytes]; every thread commits one
 * group. */
__device__ __forceinline__ void stage_rows(uint8_t* dst, const uint8_t* src, uint64_t pitch,
                                           uint64_t r0, int nr, int seg_bytes, int copy_bytes) {
    const int per_row = copy_bytes >> 4;
    const int total   = nr * per_row;
    for (int i = static_cast<int>(threadIdx.x); i < total; i += static_cast<int>(blockDim.x)) {
        const int r = i / per_row, v = i - r * per_row;
        cp_async16(dst + r * seg_bytes + v * 16, src + (r0 + static_cast<uint64_t>(r)) * pitch + v * 16);
    }
    commit();
}

/** Staging of rows [b, e) of one column segment through S buffers (S - 1
 * stages in flight while one is read). Every thread of the block calls
 * start(), then for k = 0 .. nblk-1: wait(k), reads rows_of(k) rows at
 * buf(k) (row r is time t0(k) + r), release(k). `smem` holds
 * S * rows * seg_bytes bytes; `copy_bytes` (<= seg_bytes, a multiple of 16)
 * of each row are fetched (a row's last segment can be short). */
template <int S> struct StagerN {
    static_assert(S >= 2 && S <= 8, "2 to 8 stages");
    uint8_t* smem;
    const uint8_t* src;
    uint64_t pitch;
    int seg_bytes, copy_bytes, rows;
    uint64_t b, n;
    int nblk;

    __device__ StagerN(uint8_t* smem_, const uint8_t* src_, uint64_t pitch_, int seg_bytes_,
                       int copy_bytes_, int rows_, uint64_t b_, uint64_t e_)
        : smem(smem_), src(src_), pitch(pitch_), seg_bytes(seg_bytes_), copy_bytes(copy_bytes_),
          rows(rows_), b(b_), n(e_ > b_ ? e_ - b_ : 0) {
        nblk = static_cast<int>((n + rows - 1) / rows);
    }
    __device__ __forceinline__ int rows_of(int k) const {
        const uint64_t left = n - static_cast<uint64_t>(k) * rows;
        return static_cast<int>(left < static_cast<uint64_t>(rows) ? left : rows);
    }
    __device__ __forceinline__ uint64_t t0(int k) const { return b + static_cast<uint64_t>(k) * rows; }
    __device__ __forceinline__ int slot(int k) const { return k % S; }
    __device__ __forceinline__ const uint8_t* buf(int k) const {
        return smem + slot(k) * rows * seg_bytes;
    }
    __device__ __forceinline__ void issue(int k) {
        stage_rows(smem + slot(k) * rows * seg_bytes, src, pitch, t0(k), rows_of(k), seg_bytes, copy_bytes);
    }
    __device__ __forceinline__ void start() {
        for (int k = 0; k < S && k < nblk; ++k)
            issue(k);
    }
    /** Waits for stage k's copies (this thread's, then the block's): the
     * groups committed after stage k's may stay pending. */
    __device__ __forceinline__ void wait(int k) {
        const int later = nblk - 1 - k; // stages issued after k (at most S - 1)
        if (later >= S - 1) {
            wait_pending<S - 1>();
        } else {
            switch (later) {
            case 0: wait_pending<0>(); break;
            case 1: wait_pending<1>(); break;
            case 2: wait_pending<2>(); break;
            case 3: wait_pending<3>(); break;
            case 4: wait_pending<4>(); break;
            case 5: wait_pending<5>(); break;
            default: wait_pending<6>(); break;
            }
        }
        __syncthreads();
    }
    /** Every thread is done with stage k's buffer: refill it with k + S. */
    __device__ __forceinline__ void release(int k) {
        __syncthreads();
        if (k + S < nblk)
            issue(k + S);
    }
};

/** The double-buffered form. */
using Stager = StagerN<2>;

} // namespace fb::rfi::stage
