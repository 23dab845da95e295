// FDMT level kernels for sm_100a.
//
// Every level is one streaming pass: read two child rows, write one parent
// row, HBM-bound. Level 1 is fused with the leaf initialisation (each
// thread slides the per-channel window sums over the node's rows in
// shared memory), so the ~C * (1 + d) leaf rows are never materialised. Rows live in level
// buffers with a per-level history prefix (see LevelView), so a shifted read
// t - d_lo before the tile start lands in the history columns without a
// branch. The shifted (high-child) row segment of each CTA is staged in
// shared memory with aligned 16-byte loads; the unshifted row is read
// directly, coalesced. Storage is float or __half; arithmetic is float.

#include <algorithm>
#include <type_traits>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bulk_copy.cuh"
#include "common.hpp"
#include "fdmt_kernels.hpp"

namespace fb::fdmt {

namespace {

constexpr int kThreads = 256;
constexpr int kPer     = kTimePerCta / kThreads; // 8 samples per thread

template <class S> __device__ __forceinline__ float ld(const S* p);
template <> __device__ __forceinline__ float ld<float>(const float* p) { return *p; }
template <> __device__ __forceinline__ float ld<__half>(const __half* p) { return __half2float(*p); }

// Two sums of finite fp16 level values (at most four of them, so finite
// floats) rounded to an fp16 pair, lo in the low half: the saturating
// convert gives clamp-to-+-65504-then-round bit for bit for finite inputs
// (a magnitude past 65504 becomes 65504), in one instruction.
__device__ __forceinline__ uint32_t pack_sat(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.satfinite.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// Stores a level value. FP16 storage saturates at the largest finite half
// instead of overflowing to infinity (a strong unexcised burst must not
// poison a whole DM row): one saturating convert, which for finite values
// gives clamp-then-round bit for bit (as pack_sat does for pairs).
template <class S> __device__ __forceinline__ void st_sat(S* p, float v);
template <> __device__ __forceinline__ void st_sat<float>(float* p, float v) { *p = v; }
template <> __device__ __forceinline__ void st_sat<__half>(__half* p, float v) {
    unsigned short h;
    asm("cvt.rn.satfinite.f16.f32 %0, %1;" : "=h"(h) : "f"(v));
    *reinterpret_cast<unsigned short*>(p) = h;
}

// Level 1 with the leaf initialisation: row (d_lo, d_hi) of a two-channel
// node at time t is sum_{s=0..d_lo} a[t - s] + sum_{s=0..d_hi} b[t - d_lo - s]
// (one channel: the first term). The node's rows have non-decreasing d_lo
// and d_hi (ascending delays), so each thread walks them in order and moves
// its two windows by the samples that enter or leave them. FP32 storage
// accumulates in double (every window sum is then its exact value to ~1e-16
// relative, however long the tile, and rounds once to float); FP16 storage
// in float, the precision variant's FP32 accumulation (a window of a few
// tens of unit-variance samples moved a few tens of times carries an error
// some 1e-5 of an fp16 step). The two channels' tile segments, with the H
// samples before the tile, sit in shared memory in the accumulator's type
// (converted once); thread t owns samples t, t + 256, ... of the tile.
constexpr int kFill = 8; // tile elements each thread loads at once (the H + 1 more follow)

// acc[j] += x[i + j * kThreads] (SIGN = 1) or -= (SIGN = -1) for j < kPer:
// float accumulators two lanes per instruction (add/sub.rn.f32x2: each lane
// rounds as the scalar operation), doubles one at a time.
// a[j] += b[j], two lanes per instruction.
template <int N> __device__ __forceinline__ void slide_regs(float (&a)[N], const float (&b)[N]) {
#pragma unroll
    for (int j = 0; j < N; j += 2)
        asm("{\n .reg .b64 p, q;\n mov.b64 p, {%0, %1};\n mov.b64 q, {%2, %3};\n"
            " add.rn.f32x2 p, p, q;\n mov.b64 {%0, %1}, p;\n}"
            : "+f"(a[j]), "+f"(a[j + 1])
            : "f"(b[j]), "f"(b[j + 1]));
}

template <int SIGN, class Acc, int N>
__device__ __forceinline__ void slide(Acc (&acc)[N], const Acc* x, int i) {
    if constexpr (sizeof(Acc) == 4) {
#pragma unroll
        for (int j = 0; j < N; j += 2) {
            const float a = x[i + j * kThreads], b = x[i + (j + 1) * kThreads];
            if constexpr (SIGN > 0)
                asm("{\n .reg .b64 p, q;\n mov.b64 p, {%0, %1};\n mov.b64 q, {%2, %3};\n"
                    " add.rn.f32x2 p, p, q;\n mov.b64 {%0, %1}, p;\n}"
                    : "+f"(acc[j]), "+f"(acc[j + 1])
                    : "f"(a), "f"(b));
            else
                asm("{\n .reg .b64 p, q;\n mov.b64 p, {%0, %1};\n mov.b64 q, {%2, %3};\n"
                    " sub.rn.f32x2 p, p, q;\n mov.b64 {%0, %1}, p;\n}"
                    : "+f"(acc[j]), "+f"(acc[j + 1])
                    : "f"(a), "f"(b));
        }
    } else {
#pragma unroll
        for (int j = 0; j < N; ++j) {
            if constexpr (SIGN > 0)
                acc[j] += x[i + j * kThreads];
            else
                acc[j] -= x[i + j * kThreads];
        }
    }
}

template <class S> using Level1Acc = std::conditional_t<sizeof(S) == 2, float, double>;

template <class S>
__global__ void __launch_bounds__(kThreads, sizeof(S) == 2 ? 6 : 5)
    k_level1(const LeafOp* __restrict__ ops, const int32_t* __restrict__ node_first_op, int32_t nnodes,
             int32_t ntiles, int32_t H, const float* __restrict__ wf, int64_t wpitch, int64_t t0,
             int32_t n_valid, const float* __restrict__ hist, int32_t hist_len, S* __restrict__ out,
             int64_t pitch, int32_t base) {
    using Acc = Level1Acc<S>;
    extern __shared__ __align__(16) unsigned char smem_l1[];
    const int32_t N = kTimePerCta + H + 1;
    Acc* Xa         = reinterpret_cast<Acc*>(smem_l1);
    Acc* Xb         = Xa + N;
    // Work items (node, tile), nodes fastest; a CTA takes items blockIdx.x,
    // blockIdx.x + gridDim.x, ...
    const int64_t nitems = static_cast<int64_t>(nnodes) * ntiles;
    for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int32_t node = static_cast<int32_t>(item % nnodes);
        const int32_t op0 = node_first_op[node], op1 = node_first_op[node + 1];
        const int32_t ca  = ops[op0].chan_lo;
        const int32_t cb  = ops[op0].chan_hi;
        const int32_t k0  = static_cast<int32_t>(item / nnodes) * kTimePerCta;
        // x(i) for tile-relative time t = k0 + i - H - 1 (index 0 unused):
        // the first kFill elements of each thread are all loaded before any
        // is stored, so a fill waits for one round trip, not one per element
        auto fetch = [&](int i, float& a, float& b) {
            const int64_t t = static_cast<int64_t>(k0) + i - H - 1;
            a = 0.0F;
            b = 0.0F;
            if (i > 0 && i < N) {
                if (t < 0) {
                    a = hist[static_cast<int64_t>(ca) * hist_len + hist_len + t];
                    if (cb >= 0)
                        b = hist[static_cast<int64_t>(cb) * hist_len + hist_len + t];
                } else if (t < n_valid) {
                    a = wf[static_cast<int64_t>(ca) * wpitch + t0 + t];
                    if (cb >= 0)
                        b = wf[static_cast<int64_t>(cb) * wpitch + t0 + t];
                }
            }
        };
        {
            float ra[kFill], rb[kFill];
#pragma unroll
            for (int u = 0; u < kFill; ++u)
                fetch(threadIdx.x + u * kThreads, ra[u], rb[u]);
#pragma unroll
            for (int u = 0; u < kFill; ++u) {
                const int i = threadIdx.x + u * kThreads;
                if (i < N) {
                    Xa[i] = static_cast<Acc>(ra[u]);
                    Xb[i] = static_cast<Acc>(rb[u]);
                }
            }
            for (int i = threadIdx.x + kFill * kThreads; i < N; i += kThreads) {
                float a, b;
                fetch(i, a, b);
                Xa[i] = static_cast<Acc>(a);
                Xb[i] = static_cast<Acc>(b);
            }
        }
        __syncthreads();
        // window state per owned sample: A = sum a[t - dl .. t],
        // B = sum b[t - dl - dh .. t - dl]; (dl, dh) = (-1, -1): both empty
        Acc A[kPer], B[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            A[j] = 0;
            B[j] = 0;
        }
        int32_t dl = -1, dh = -1;
        const int i0 = threadIdx.x + H + 1; // index of the thread's first sample
        for (int32_t r = op0; r < op1; ++r) {
            const LeafOp op = ops[r];
            S* row          = out + static_cast<int64_t>(r) * pitch + base + k0 + threadIdx.x;
            // A's window grows from dl to op.d_lo samples back (restarts if
            // the rows ever went backwards)
            int32_t from = dl + 1;
            if (op.d_lo < dl) {
#pragma unroll
                for (int j = 0; j < kPer; ++j)
                    A[j] = 0;
                from = 0;
            }
            for (int32_t q = from; q <= op.d_lo; ++q)
                slide<1>(A, Xa, i0 - q);
            if (cb >= 0) {
                // B's window moves from back offsets [dl, dl + dh] to
                // [op.d_lo, op.d_lo + op.d_hi]: drop the top, add the bottom,
                // or start afresh when the two do not overlap
                const int32_t ob = dl + dh, nb = op.d_lo + op.d_hi;
                if (dh < 0 || op.d_lo > ob || nb < ob || op.d_lo < dl) {
#pragma unroll
                    for (int j = 0; j < kPer; ++j)
                        B[j] = 0;
                    for (int32_t q = op.d_lo; q <= nb; ++q)
                        slide<1>(B, Xb, i0 - q);
                } else {
                    for (int32_t q = dl; q < op.d_lo; ++q)
                        slide<-1>(B, Xb, i0 - q);
                    for (int32_t q = ob + 1; q <= nb; ++q)
                        slide<1>(B, Xb, i0 - q);
                }
            }
            if constexpr (sizeof(Acc) == 4) {
                float sum[kPer];
#pragma unroll
                for (int j = 0; j < kPer; ++j)
                    sum[j] = A[j];
                slide_regs(sum, B);
#pragma unroll
                for (int j = 0; j < kPer; ++j)
                    st_sat<S>(row + j * kThreads, sum[j]);
            } else {
#pragma unroll
                for (int j = 0; j < kPer; ++j)
                    st_sat<S>(row + j * kThreads, static_cast<float>(A[j] + B[j]));
            }
            dl = op.d_lo;
            dh = op.d_hi;
        }
        __syncthreads(); // every thread is done with Xa / Xb
    }
}

// dst[0..8) = lo[0..8) + stage[off + e .. off + e + 8): `lo` and `dst` are
// 16-byte aligned (global or shared), `stage` is the 16-byte aligned staged
// high-child segment, e = 8 * thread.
template <class S>
__device__ __forceinline__ void merge8(const S* lo, const S* stage, int e, int off, S* dst) {
    if constexpr (sizeof(S) == 4) {
        const float4* l4 = reinterpret_cast<const float4*>(lo);
        const float4 a0 = l4[0], a1 = l4[1];
        const float4* h4 = reinterpret_cast<const float4*>(stage) + e / 4;
        const float4 b0 = h4[0], b1 = h4[1], b2 = h4[2]; // b2 unused when off == 0
        const float h[12] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w};
        float g[8];
        switch (off) {
#define FB_PICK(O)                                                                                \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 8; ++i) g[i] = h[O + i];                             \
        break;
            FB_PICK(0) FB_PICK(1) FB_PICK(2) FB_PICK(3)
#undef FB_PICK
        }
        float4* d4 = reinterpret_cast<float4*>(dst);
        d4[0]      = make_float4(a0.x + g[0], a0.y + g[1], a0.z + g[2], a0.w + g[3]);
        d4[1]      = make_float4(a1.x + g[4], a1.y + g[5], a1.z + g[6], a1.w + g[7]);
    } else {
        const uint4 a   = *reinterpret_cast<const uint4*>(lo);
        const uint4* sv = reinterpret_cast<const uint4*>(stage) + e / 8;
        const uint4 b0 = sv[0], b1 = sv[1]; // b1 unused when off == 0
        const uint32_t w[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        uint32_t g[4];
        switch (off) {
#define FB_PICK_EVEN(O)                                                                           \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 4; ++i) g[i] = w[O / 2 + i];                         \
        break;
#define FB_PICK_ODD(O)                                                                            \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 4; ++i) g[i] =                                      \
            __byte_perm(w[O / 2 + i], w[O / 2 + i + 1], 0x5432);                                  \
        break;
            FB_PICK_EVEN(0) FB_PICK_ODD(1) FB_PICK_EVEN(2) FB_PICK_ODD(3)
            FB_PICK_EVEN(4) FB_PICK_ODD(5) FB_PICK_EVEN(6) FB_PICK_ODD(7)
#undef FB_PICK_EVEN
#undef FB_PICK_ODD
        }
        const uint32_t av[4] = {a.x, a.y, a.z, a.w};
        uint32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 x = __half22float2(*reinterpret_cast<const __half2*>(&av[i]));
            const float2 y = __half22float2(*reinterpret_cast<const __half2*>(&g[i]));
            r[i]           = pack_sat(x.x + y.x, x.y + y.y);
        }
        *reinterpret_cast<uint4*>(dst) = make_uint4(r[0], r[1], r[2], r[3]);
    }
}

// ---- TMA-pipelined level kernel ------------------------------------------
//
// One CTA per (output row, run of `tpc` time tiles). Thread 0 keeps
// kStages tiles in flight with 1-D bulk async copies (cp.async.bulk, local
// global memory only, no multicast) of the unshifted child segment and the
// 16-byte-aligned superset of the shifted one, each stage completing on its
// own mbarrier; all threads combine a landed stage from shared memory and
// store 16-byte vectors. Every wait is bounded: a wait that runs out sets
// *err and the CTA drains its copies (again bounded) and returns.

constexpr int kStages      = 4;
using bulk::mbar_wait;

template <class S, int K>
__global__ void __launch_bounds__(kThreads)
    k_level_pipe(const __grid_constant__ LevelSegTable<K> tab, long long wait_limit) {
    constexpr int VEC       = 16 / static_cast<int>(sizeof(S));
    constexpr int kLoBytes  = kTimePerCta * static_cast<int>(sizeof(S));
    constexpr int kHiBytes  = kLoBytes + 16;
    constexpr int kStageBytes = kLoBytes + kHiBytes;
    extern __shared__ __align__(128) unsigned char pipe_smem[];
    __shared__ __align__(8) uint64_t bar[kStages];
    __shared__ int abort_flag;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < kStages; ++s)
            bulk::mbar_init(&bar[s]);
    }
    __syncthreads();
    // Work items (segment, row, run of tpc tiles), rows fastest within a
    // segment; a CTA takes items blockIdx.x, blockIdx.x + gridDim.x, ... and
    // its tiles use the stages in turn across items and segments (the CTA's
    // tile n: stage n % kStages, barrier phase (n / kStages) % 2, kept as
    // running counters).
    const int64_t nitems = tab.s[tab.n - 1].item_end;
    const int e          = 8 * threadIdx.x;
    int cs      = 0;  // stage of the CTA's next tile
    uint32_t cp = 0U; // and its barrier's phase parity
    int sg       = 0;  // the segment of the CTA's current item
    int64_t sbeg = 0;  // and its first item
    for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
        while (item >= tab.s[sg].item_end) {
            sbeg = tab.s[sg].item_end;
            ++sg;
        }
        const LevelSeg& G      = tab.s[sg];
        const RowOp* ops       = static_cast<const RowOp*>(G.ops);
        const S* in            = static_cast<const S*>(G.in);
        S* out                 = static_cast<S*>(G.out);
        const int64_t in_pitch = G.in_pitch, out_pitch = G.out_pitch;
        const int32_t in_base = G.in_base, out_base = G.out_base;
        unsigned* err          = G.err;
        const int64_t local    = item - sbeg;
        const int64_t r        = G.rows != nullptr ? G.rows[local % G.nrows] : local % G.nrows;
        const RowOp op         = ops[r];
        const int tile0        = static_cast<int>(local / G.nrows) * G.tpc;
        const int nt           = min(G.tpc, G.ntiles - tile0);
        const bool has_hi = op.hi_row >= 0;
        const S* lo_row   = in + static_cast<int64_t>(op.lo_row) * in_pitch + in_base;
        const S* hi_base  = in + static_cast<int64_t>(has_hi ? op.hi_row : op.lo_row) * in_pitch;
        S* dst_row        = out + r * out_pitch + out_base;
        // the shifted segment's offset inside its aligned superset is the same
        // for every tile (tiles start at multiples of kTimePerCta)
        const int64_t e_first = static_cast<int64_t>(in_base) - op.shift;
        const int off         = static_cast<int>(((e_first % VEC) + VEC) % VEC);
        const uint32_t hi_bytes = has_hi ? static_cast<uint32_t>((kTimePerCta / VEC + (off > 0 ? 1 : 0)) * 16) : 0U;

        auto issue = [&](int i, int s) {
            const int64_t k0  = static_cast<int64_t>(tile0 + i) * kTimePerCta;
            unsigned char* st = pipe_smem + s * kStageBytes;
            bulk::mbar_expect(&bar[s], static_cast<uint32_t>(kLoBytes) + hi_bytes);
            bulk::load(st, lo_row + k0, static_cast<uint32_t>(kLoBytes), &bar[s]);
            if (has_hi) {
                const int64_t v0 = (e_first + k0 - off) / VEC; // aligned start, in vectors
                bulk::load(st + kLoBytes, hi_base + v0 * VEC, hi_bytes, &bar[s]);
            }
        };

        if (threadIdx.x == 0)
            for (int i = 0, s = cs; i < min(kStages, nt); ++i, s = s + 1 == kStages ? 0 : s + 1)
                issue(i, s);
        int i = 0;
        for (; i < nt; ++i) {
            const int s = cs;
            if (!mbar_wait(&bar[s], cp, wait_limit))
                atomicExch(&abort_flag, 1);
            __syncthreads();
            if (abort_flag)
                break;
            const S* lo_s = reinterpret_cast<const S*>(pipe_smem + s * kStageBytes);
            const S* hi_s = reinterpret_cast<const S*>(pipe_smem + s * kStageBytes + kLoBytes);
            S* dst        = dst_row + static_cast<int64_t>(tile0 + i) * kTimePerCta + e;
            if (has_hi) {
                merge8<S>(lo_s + e, hi_s, e, off, dst);
            } else {
                const uint4* s4 = reinterpret_cast<const uint4*>(lo_s + e);
                uint4* d4       = reinterpret_cast<uint4*>(dst);
                for (int v = 0; v < 8 / VEC; ++v)
                    d4[v] = s4[v];
            }
            __syncthreads(); // every thread is done with stage s
            if (threadIdx.x == 0 && i + kStages < nt)
                issue(i + kStages, s);
            if (++cs == kStages) {
                cs = 0;
                cp ^= 1U;
            }
        }
        if (i < nt) {
            if (threadIdx.x == 0) {
                // a wait ran out: report it, then let the copies still in flight land
                atomicOr(err, 1U);
                for (int j = i, s = cs, p = static_cast<int>(cp); j < min(nt, i + kStages); ++j) {
                    (void)mbar_wait(&bar[s], static_cast<uint32_t>(p));
                    if (++s == kStages) {
                        s = 0;
                        p ^= 1;
                    }
                }
            }
            return;
        }
    }
}

// ---- two levels in one pass ---------------------------------------------
//
// A row of level h+1 is a row of level h plus a shifted one, and each of
// those is a row of level h-1 plus a shifted one, so it is the sum of up to
// four level h-1 rows read at shifts 0, s1, s2, s3 (FusedOp). Computing
// (x0 + x1) + (x2 + x3) is what the two single levels compute, bit for bit
// (float storage: float adds; fp16 storage: each sum rounded to fp16 with
// saturation, as a stored middle level would be), and level h is never
// written or read back. Staging as in
// k_level_pipe: one unshifted segment and up to three 16-byte-aligned
// supersets of the shifted ones per tile, kStages2 tiles in flight.

// The 8 fp16 values starting at element off + e of a staged aligned
// segment (off < 8), as packed pairs (value 2i in the low half of g[i]).
__device__ __forceinline__ void pick8h(const __half* stage, int e, int off, uint32_t (&g)[4]) {
    const uint4* sv = reinterpret_cast<const uint4*>(stage) + e / 8;
    const uint4 b0 = sv[0], b1 = sv[1]; // b1 unused when off == 0
    const uint32_t w[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
    switch (off) {
#define FB_PICK_EVEN(O)                                                                           \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 4; ++i) g[i] = w[O / 2 + i];                         \
        break;
#define FB_PICK_ODD(O)                                                                            \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 4; ++i) g[i] =                                      \
            __byte_perm(w[O / 2 + i], w[O / 2 + i + 1], 0x5432);                                  \
        break;
        FB_PICK_EVEN(0) FB_PICK_ODD(1) FB_PICK_EVEN(2) FB_PICK_ODD(3)
        FB_PICK_EVEN(4) FB_PICK_ODD(5) FB_PICK_EVEN(6) FB_PICK_ODD(7)
#undef FB_PICK_EVEN
#undef FB_PICK_ODD
    }
}

// 8 consecutive floats starting at element off + e of a staged aligned
// segment (off < 4).
__device__ __forceinline__ void load8(const float* stage, int e, int off, float (&x)[8]) {
    const float4* h4 = reinterpret_cast<const float4*>(stage) + e / 4;
    const float4 b0 = h4[0], b1 = h4[1], b2 = h4[2]; // b2 unused when off == 0
    const float h[12] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w};
    switch (off) {
#define FB_PICK(O)                                                                                \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 8; ++i) x[i] = h[O + i];                             \
        break;
        FB_PICK(0) FB_PICK(1) FB_PICK(2) FB_PICK(3)
#undef FB_PICK
    }
}

// acc[q] = acc[q] + (value q of load8).
__device__ __forceinline__ void add8(const float* stage, int e, int off, float (&acc)[8]) {
    float x[8];
    load8(stage, e, off, x);
#pragma unroll
    for (int q = 0; q < 8; ++q)
        acc[q] = acc[q] + x[q];
}

// a[i] = a[i] + b[i] for four packed fp16 pairs as the single-level kernel
// rounds it: the float sum of two fp16 values is exact when their exponents
// differ by at most 12 and otherwise rounds to the larger one, as the fp16
// add does; the clamp to +-65504 is the saturating convert's (sums past it
// round to infinity).
__device__ __forceinline__ void add_sat4(uint32_t (&a)[4], const uint32_t (&b)[4]) {
    const __half2 top = __float2half2_rn(65504.0F);
    const __half2 bot = __float2half2_rn(-65504.0F);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const __half2 x = __hadd2(*reinterpret_cast<const __half2*>(&a[i]), *reinterpret_cast<const __half2*>(&b[i]));
        const __half2 c = __hmin2(__hmax2(x, bot), top);
        a[i]            = *reinterpret_cast<const uint32_t*>(&c);
    }
}

template <class S> constexpr int kStages2 = sizeof(S) == 2 ? 4 : 3;

template <class S, int NS, int K>
__global__ void __launch_bounds__(kThreads)
    k_level2_pipe(const __grid_constant__ LevelSegTable<K> tab, long long wait_limit) {
    constexpr int VEC       = 16 / static_cast<int>(sizeof(S));
    constexpr int kLoBytes  = kTimePerCta * static_cast<int>(sizeof(S));
    constexpr int kHiBytes  = kLoBytes + 16;
    constexpr int kStageBytes = kLoBytes + 3 * kHiBytes;
    extern __shared__ __align__(128) unsigned char pipe2_smem[];
    __shared__ __align__(8) uint64_t bar[NS];
    __shared__ int abort_flag;

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int st = 0; st < NS; ++st)
            bulk::mbar_init(&bar[st]);
    }
    __syncthreads();
    // Work items (segment, row, run of tpc tiles) as in k_level_pipe.
    const int64_t nitems = tab.s[tab.n - 1].item_end;
    const int e          = 8 * threadIdx.x;
    int cs      = 0;  // stage of the CTA's next tile
    uint32_t cp = 0U; // and its barrier's phase parity
    int sg       = 0;
    int64_t sbeg = 0;
    for (int64_t item = blockIdx.x; item < nitems; item += gridDim.x) {
        while (item >= tab.s[sg].item_end) {
            sbeg = tab.s[sg].item_end;
            ++sg;
        }
        const LevelSeg& G      = tab.s[sg];
        const FusedOp* ops     = static_cast<const FusedOp*>(G.ops);
        const S* in            = static_cast<const S*>(G.in);
        S* out                 = static_cast<S*>(G.out);
        const int64_t in_pitch = G.in_pitch, out_pitch = G.out_pitch;
        const int32_t in_base = G.in_base, out_base = G.out_base;
        unsigned* err          = G.err;
        const int64_t local    = item - sbeg;
        const int64_t r        = local % G.nrows;
        const FusedOp op       = ops[r];
        const int tile0        = static_cast<int>(local / G.nrows) * G.tpc;
        const int nt           = min(G.tpc, G.ntiles - tile0);
        const S* rows[4];
        int off[4];
        uint32_t bytes[4];
        int64_t first[4];
        uint32_t total = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool has = op.row[j] >= 0;
            rows[j]        = in + static_cast<int64_t>(has ? op.row[j] : op.row[0]) * in_pitch;
            first[j]       = static_cast<int64_t>(in_base) - op.shift[j];
            off[j]         = static_cast<int>(((first[j] % VEC) + VEC) % VEC);
            bytes[j]       = !has ? 0U
                             : j == 0 ? static_cast<uint32_t>(kLoBytes)
                                      : static_cast<uint32_t>((kTimePerCta / VEC + (off[j] > 0 ? 1 : 0)) * 16);
            total += bytes[j];
        }
        S* dst_row = out + r * out_pitch + out_base;

        auto issue = [&](int i, int st) {
            const int64_t k0  = static_cast<int64_t>(tile0 + i) * kTimePerCta;
            unsigned char* sb = pipe2_smem + st * kStageBytes;
            bulk::mbar_expect(&bar[st], total);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (bytes[j] == 0U)
                    continue;
                const int64_t v0 = (first[j] + k0 - off[j]) / VEC; // aligned start, in vectors
                bulk::load(sb + (j == 0 ? 0 : kLoBytes + (j - 1) * kHiBytes), rows[j] + v0 * VEC, bytes[j],
                           &bar[st]);
            }
        };

        if (threadIdx.x == 0)
            for (int i = 0, st = cs; i < min(NS, nt); ++i, st = st + 1 == NS ? 0 : st + 1)
                issue(i, st);
        int i = 0;
        for (; i < nt; ++i) {
            const int st = cs;
            if (!mbar_wait(&bar[st], cp, wait_limit))
                atomicExch(&abort_flag, 1);
            __syncthreads();
            if (abort_flag)
                break;
            const unsigned char* sb = pipe2_smem + st * kStageBytes;
            S* dst = dst_row + static_cast<int64_t>(tile0 + i) * kTimePerCta + e;
            if constexpr (sizeof(S) == 4) {
                float a[8];
                load8(reinterpret_cast<const float*>(sb), e, 0, a);
                if (bytes[1] != 0U)
                    add8(reinterpret_cast<const float*>(sb + kLoBytes), e, off[1], a);
                if (bytes[2] != 0U) {
                    float b[8];
                    load8(reinterpret_cast<const float*>(sb + kLoBytes + kHiBytes), e, off[2], b);
                    if (bytes[3] != 0U)
                        add8(reinterpret_cast<const float*>(sb + kLoBytes + 2 * kHiBytes), e, off[3], b);
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        a[q] = a[q] + b[q];
                }
                float4* d4 = reinterpret_cast<float4*>(dst);
                d4[0]      = make_float4(a[0], a[1], a[2], a[3]);
                d4[1]      = make_float4(a[4], a[5], a[6], a[7]);
            } else {
                // fp16 storage: each of the three sums is the single-level
                // kernel's (the float sum of two fp16 values rounded with
                // saturation), as fp16 adds clamped to +-65504, so two levels
                // in one pass give the bits of two single steps
                uint32_t a[4], b[4];
                {
                    const uint4 u = *reinterpret_cast<const uint4*>(reinterpret_cast<const S*>(sb) + e);
                    a[0] = u.x, a[1] = u.y, a[2] = u.z, a[3] = u.w;
                }
                if (bytes[1] != 0U) {
                    pick8h(reinterpret_cast<const __half*>(sb + kLoBytes), e, off[1], b);
                    add_sat4(a, b);
                }
                if (bytes[2] != 0U) {
                    pick8h(reinterpret_cast<const __half*>(sb + kLoBytes + kHiBytes), e, off[2], b);
                    if (bytes[3] != 0U) {
                        uint32_t c[4];
                        pick8h(reinterpret_cast<const __half*>(sb + kLoBytes + 2 * kHiBytes), e, off[3], c);
                        add_sat4(b, c);
                    }
                    add_sat4(a, b);
                }
                *reinterpret_cast<uint4*>(dst) = make_uint4(a[0], a[1], a[2], a[3]);
            }
            __syncthreads(); // every thread is done with stage st
            if (threadIdx.x == 0 && i + NS < nt)
                issue(i + NS, st);
            if (++cs == NS) {
                cs = 0;
                cp ^= 1U;
            }
        }
        if (i < nt) {
            if (threadIdx.x == 0) {
                // a wait ran out: report it, then let the copies still in flight land
                atomicOr(err, 1U);
                for (int j = i, st = cs, p = static_cast<int>(cp); j < min(nt, i + NS); ++j) {
                    (void)mbar_wait(&bar[st], static_cast<uint32_t>(p));
                    if (++st == NS) {
                        st = 0;
                        p ^= 1;
                    }
                }
            }
            return;
        }
    }
}

template <class S>
__global__ void __launch_bounds__(kThreads)
    k_level(const RowOp* __restrict__ ops, const S* __restrict__ in, int64_t in_pitch,
            int32_t in_base, S* __restrict__ out, int64_t out_pitch, int32_t out_base) {
    constexpr int VEC = 16 / sizeof(S);
    __shared__ __align__(16) S stage[kTimePerCta + VEC];
    const RowOp op = ops[blockIdx.x];
    const int32_t k0 = blockIdx.y * kTimePerCta;
    const S* lo = in + static_cast<int64_t>(op.lo_row) * in_pitch + in_base + k0;
    S* dst      = out + static_cast<int64_t>(blockIdx.x) * out_pitch + out_base + k0;
    // Each thread owns 8 consecutive samples: one 16-byte (fp16) or two
    // 16-byte (fp32) vectors of the unshifted row and of the output.
    const int e = 8 * threadIdx.x;
    if (op.hi_row < 0) {
        const uint4* s4 = reinterpret_cast<const uint4*>(lo + e);
        uint4* d4       = reinterpret_cast<uint4*>(dst + e);
        for (int v = 0; v < 8 / VEC; ++v)
            d4[v] = s4[v];
        return;
    }
    // Stage hi[k0 - shift, k0 - shift + kTimePerCta) with aligned vectors;
    // element k of the segment is stage[off + k].
    const S* hrow    = in + static_cast<int64_t>(op.hi_row) * in_pitch;
    const int64_t e0 = static_cast<int64_t>(in_base) + k0 - op.shift;
    const int64_t v0 = e0 / VEC;
    const int off    = static_cast<int>(e0 - v0 * VEC);
    const int nvec   = kTimePerCta / VEC + (off > 0 ? 1 : 0);
    const uint4* src = reinterpret_cast<const uint4*>(hrow) + v0;
    uint4* sv        = reinterpret_cast<uint4*>(stage);
    for (int i = threadIdx.x; i < nvec; i += kThreads)
        sv[i] = src[i];
    __syncthreads();
    if constexpr (sizeof(S) == 4) {
        const float4* l4 = reinterpret_cast<const float4*>(lo + e);
        const float4 a0 = l4[0], a1 = l4[1];
        const float4* h4 = reinterpret_cast<const float4*>(stage) + e / 4;
        const float4 b0 = h4[0], b1 = h4[1], b2 = h4[2]; // b2 unused when off == 0
        const float h[12] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w, b2.x, b2.y, b2.z, b2.w};
        float g[8];
        switch (off) {
#define FB_PICK(O)                                                                                \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 8; ++i) g[i] = h[O + i];                             \
        break;
            FB_PICK(0) FB_PICK(1) FB_PICK(2) FB_PICK(3)
#undef FB_PICK
        }
        float4* d4 = reinterpret_cast<float4*>(dst + e);
        d4[0]      = make_float4(a0.x + g[0], a0.y + g[1], a0.z + g[2], a0.w + g[3]);
        d4[1]      = make_float4(a1.x + g[4], a1.y + g[5], a1.z + g[6], a1.w + g[7]);
    } else {
        const uint4 a  = *reinterpret_cast<const uint4*>(lo + e);
        const uint4 b0 = sv[threadIdx.x], b1 = sv[threadIdx.x + 1]; // b1 unused when off == 0
        const uint32_t w[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
        uint32_t g[4];
        // 8 halves starting at half `off` of the 16 in w[]
        switch (off) {
#define FB_PICK_EVEN(O)                                                                           \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 4; ++i) g[i] = w[O / 2 + i];                         \
        break;
#define FB_PICK_ODD(O)                                                                            \
    case O:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < 4; ++i) g[i] =                                      \
            __byte_perm(w[O / 2 + i], w[O / 2 + i + 1], 0x5432);                                  \
        break;
            FB_PICK_EVEN(0) FB_PICK_ODD(1) FB_PICK_EVEN(2) FB_PICK_ODD(3)
            FB_PICK_EVEN(4) FB_PICK_ODD(5) FB_PICK_EVEN(6) FB_PICK_ODD(7)
#undef FB_PICK_EVEN
#undef FB_PICK_ODD
        }
        const uint32_t av[4] = {a.x, a.y, a.z, a.w};
        uint32_t r[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 x = __half22float2(*reinterpret_cast<const __half2*>(&av[i]));
            const float2 y = __half22float2(*reinterpret_cast<const __half2*>(&g[i]));
            r[i]           = pack_sat(x.x + y.x, x.y + y.y);
        }
        *reinterpret_cast<uint4*>(dst + e) = make_uint4(r[0], r[1], r[2], r[3]);
    }
}

template <class S>
__global__ void k_capture(const S* __restrict__ in, int64_t pitch, int32_t base,
                          const int64_t* __restrict__ rows, float* __restrict__ out,
                          int64_t out_pitch, int64_t t_off, int32_t n_valid) {
    const int64_t r = blockIdx.y;
    const S* src    = in + rows[r] * pitch + base;
    for (int64_t k = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; k < n_valid;
         k += static_cast<int64_t>(gridDim.x) * blockDim.x)
        out[r * out_pitch + t_off + k] = ld<S>(src + k);
}

} // namespace

void launch_capture_rows(LevelView v, const int64_t* rows, int64_t nrows, float* out,
                         int64_t out_pitch, int64_t t_off, int32_t n_valid, cudaStream_t s) {
    if (nrows == 0 || n_valid <= 0)
        return;
    const dim3 grid(static_cast<unsigned>(std::min<int64_t>((n_valid + 255) / 256, 64)),
                    static_cast<unsigned>(nrows));
    if (v.fp16)
        k_capture<__half><<<grid, 256, 0, s>>>(static_cast<const __half*>(v.data), v.pitch, v.base,
                                               rows, out, out_pitch, t_off, n_valid);
    else
        k_capture<float><<<grid, 256, 0, s>>>(static_cast<const float*>(v.data), v.pitch, v.base,
                                              rows, out, out_pitch, t_off, n_valid);
    FB_LAUNCH_CHECK();
}

namespace {
// One CTA per work item, or at most `ctas` CTAs looping over the items.
unsigned grid_for(int64_t items, int32_t ctas) {
    const int64_t g = ctas > 0 ? std::min<int64_t>(items, ctas) : items;
    if (g > 0x7FFFFFFF)
        throw Error(FROST_ERR_INTERNAL, "level: too many work items for one launch");
    return static_cast<unsigned>(g);
}
} // namespace

void launch_level1(const LeafOp* ops, const int32_t* node_first_op, int32_t nnodes,
                   int32_t max_node_delay, const float* waterfall, int64_t waterfall_pitch,
                   int64_t t0, int32_t n_valid, const float* input_hist, int32_t hist_len,
                   LevelView out, int32_t ncols, cudaStream_t s, int32_t ctas) {
    if (ncols % kTimePerCta != 0 || max_node_delay > hist_len)
        throw Error(FROST_ERR_INTERNAL, "level1: bad geometry");
    const int32_t ntiles = ncols / kTimePerCta;
    const dim3 grid(grid_for(static_cast<int64_t>(nnodes) * ntiles, ctas));
    const size_t acc  = out.fp16 ? sizeof(float) : sizeof(double); // Level1Acc
    const size_t smem = 2 * acc * (kTimePerCta + max_node_delay + 1);
    if (smem > 200 * 1024)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "level1: leaf windows too long for shared memory");
    if (out.fp16) {
        allow_large_smem(reinterpret_cast<const void*>(&k_level1<__half>));
        k_level1<__half><<<grid, kThreads, smem, s>>>(
            ops, node_first_op, nnodes, ntiles, max_node_delay, waterfall, waterfall_pitch, t0, n_valid,
            input_hist, hist_len, static_cast<__half*>(out.data), out.pitch, out.base);
    } else {
        allow_large_smem(reinterpret_cast<const void*>(&k_level1<float>));
        k_level1<float><<<grid, kThreads, smem, s>>>(
            ops, node_first_op, nnodes, ntiles, max_node_delay, waterfall, waterfall_pitch, t0, n_valid,
            input_hist, hist_len, static_cast<float*>(out.data), out.pitch, out.base);
    }
    FB_LAUNCH_CHECK();
}

void launch_level(const RowOp* ops, int64_t nrows, LevelView in, LevelView out, int32_t ncols,
                  unsigned* err, cudaStream_t s, int32_t tpc, int32_t ctas, long long wait_limit,
                  const int32_t* row_map) {
    if (nrows == 0)
        return;
    if (ncols % kTimePerCta != 0 || in.base % 8 != 0 || in.pitch % 8 != 0 || out.base % 8 != 0 ||
        out.pitch % 8 != 0 || in.fp16 != out.fp16)
        throw Error(FROST_ERR_INTERNAL, "level: bad geometry");
    const int ntiles = ncols / kTimePerCta;
    if (tpc < 1 || tpc > 128)
        throw Error(FROST_ERR_INTERNAL, "level: tiles per CTA must be in [1, 128]");
    if (err == nullptr && row_map != nullptr)
        throw Error(FROST_ERR_INTERNAL, "level: a row map needs the pipelined kernel");
    if (err == nullptr) {
        // direct form (no bulk copies): one CTA per (row, tile)
        const dim3 grid(static_cast<unsigned>(nrows), static_cast<unsigned>(ntiles));
        if (out.fp16)
            k_level<__half><<<grid, kThreads, 0, s>>>(ops, static_cast<const __half*>(in.data), in.pitch,
                                                      in.base, static_cast<__half*>(out.data),
                                                      out.pitch, out.base);
        else
            k_level<float><<<grid, kThreads, 0, s>>>(ops, static_cast<const float*>(in.data), in.pitch,
                                                     in.base, static_cast<float*>(out.data), out.pitch,
                                                     out.base);
        FB_LAUNCH_CHECK();
        return;
    }
    LevelSeg g{ops, in.data, out.data, in.pitch, out.pitch, in.base, out.base, ntiles, tpc, nrows, 0, err, row_map};
    launch_level_segs(&g, 1, false, out.fp16 != 0, 0, s, ctas, wait_limit);
}

namespace {

template <int K>
LevelSegTable<K> seg_table(LevelSeg* segs, int n, int64_t* total, bool fused) {
    LevelSegTable<K> t{};
    t.n       = n;
    int64_t e = 0;
    for (int i = 0; i < n; ++i) {
        LevelSeg& g = segs[i];
        if (g.tpc < 1 || g.tpc > 128 || g.ntiles < 1 || g.nrows < 1 || g.err == nullptr || (fused && g.rows) ||
            g.in_base % 8 != 0 || g.in_pitch % 8 != 0 || g.out_base % 8 != 0 || g.out_pitch % 8 != 0)
            throw Error(FROST_ERR_INTERNAL, "level: bad segment geometry");
        e += g.nrows * ((g.ntiles + g.tpc - 1) / g.tpc);
        g.item_end = e;
        t.s[i]     = g;
    }
    *total = e;
    return t;
}

template <class S, int NS, int K>
void level2_go(const LevelSegTable<K>& t, int64_t total, cudaStream_t s, int32_t ctas, long long wait_limit) {
    const size_t smem = NS * (4 * kTimePerCta * sizeof(S) + 48);
    allow_large_smem(reinterpret_cast<const void*>(&k_level2_pipe<S, NS, K>));
    k_level2_pipe<S, NS, K><<<grid_for(total, ctas), kThreads, smem, s>>>(t, wait_limit);
}

template <class S, int K>
void level_go(const LevelSegTable<K>& t, int64_t total, bool fused, int32_t stages, cudaStream_t s, int32_t ctas,
              long long wait_limit) {
    if (!fused) {
        const size_t smem = kStages * (2 * kTimePerCta * sizeof(S) + 16);
        allow_large_smem(reinterpret_cast<const void*>(&k_level_pipe<S, K>));
        k_level_pipe<S, K><<<grid_for(total, ctas), kThreads, smem, s>>>(t, wait_limit);
        return;
    }
    switch (stages == 0 ? kStages2<S> : stages) {
    case 2: level2_go<S, 2, K>(t, total, s, ctas, wait_limit); break;
    case 3: level2_go<S, 3, K>(t, total, s, ctas, wait_limit); break;
    case 4:
        if constexpr (sizeof(S) == 2)
            level2_go<S, 4, K>(t, total, s, ctas, wait_limit);
        else
            throw Error(FROST_ERR_INTERNAL, "level2: 4 float stages exceed the shared memory of a CTA");
        break;
    default: throw Error(FROST_ERR_INTERNAL, "level2: stages must be 2, 3 or 4");
    }
}

template <int K>
void launch_table(LevelSeg* segs, int n, bool fused, bool fp16, int32_t stages, cudaStream_t s, int32_t ctas,
                  long long wait_limit) {
    int64_t total = 0;
    const LevelSegTable<K> t = seg_table<K>(segs, n, &total, fused);
    if (fp16)
        level_go<__half, K>(t, total, fused, stages, s, ctas, wait_limit);
    else
        level_go<float, K>(t, total, fused, stages, s, ctas, wait_limit);
    FB_LAUNCH_CHECK();
}

} // namespace

void launch_level_segs(LevelSeg* segs, int n, bool fused, bool fp16, int32_t stages, cudaStream_t s, int32_t ctas,
                       long long wait_limit) {
    if (wait_limit < 0)
        throw Error(FROST_ERR_INTERNAL, "level: wait limit must be >= 0");
    if (n == 1) {
        launch_table<1>(segs, 1, fused, fp16, stages, s, ctas, wait_limit);
        return;
    }
    for (int i = 0; i < n; i += kMaxLevelSegs)
        launch_table<kMaxLevelSegs>(segs + i, std::min(kMaxLevelSegs, n - i), fused, fp16, stages, s, ctas,
                                    wait_limit);
}

void launch_level2(const FusedOp* ops, int64_t nrows, LevelView in, LevelView out, int32_t ncols,
                   unsigned* err, cudaStream_t s, int32_t tpc, int32_t stages, int32_t ctas,
                   long long wait_limit) {
    if (nrows == 0)
        return;
    if (ncols % kTimePerCta != 0 || in.base % 8 != 0 || in.pitch % 8 != 0 || out.base % 8 != 0 ||
        out.pitch % 8 != 0 || in.fp16 != out.fp16 || err == nullptr)
        throw Error(FROST_ERR_INTERNAL, "level2: bad geometry");
    if (tpc < 1 || tpc > 128)
        throw Error(FROST_ERR_INTERNAL, "level2: tiles per CTA must be in [1, 128]");
    if (stages == 4 && !out.fp16)
        throw Error(FROST_ERR_INTERNAL, "level2: 4 float stages exceed the shared memory of a CTA");
    const int ntiles = ncols / kTimePerCta;
    LevelSeg g{ops, in.data, out.data, in.pitch, out.pitch, in.base, out.base, ntiles, tpc, nrows, 0, err};
    launch_level_segs(&g, 1, true, out.fp16 != 0, stages, s, ctas, wait_limit);
}

namespace {
// dst[r][0 .. w) = src[r][0 .. w) in 16-byte vectors, w vectors a row.
__global__ void __launch_bounds__(256)
    k_copy_rows16(uint4* __restrict__ dst, int64_t dpitch, const uint4* __restrict__ src, int64_t spitch,
                  uint32_t w, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t r = i / w, c = i - r * w;
        dst[r * dpitch + c] = src[r * spitch + c];
    }
}
} // namespace

void copy_rows(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows,
               cudaStream_t s) {
    if (rows == 0 || width == 0)
        return;
    const uintptr_t bits = reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src) | dpitch | spitch | width;
    const size_t n = rows * (width / 16);
    if (bits % 16 != 0 || n > 0x7FFFFFFFU) {
        FB_CUDA(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToDevice, s));
        return;
    }
    int dev = 0, sms = 0;
    FB_CUDA(cudaGetDevice(&dev));
    FB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t blocks = std::min<size_t>((n + 255) / 256, static_cast<size_t>(sms) * 8);
    k_copy_rows16<<<static_cast<unsigned>(blocks), 256, 0, s>>>(
        static_cast<uint4*>(dst), static_cast<int64_t>(dpitch / 16), static_cast<const uint4*>(src),
        static_cast<int64_t>(spitch / 16), static_cast<uint32_t>(width / 16), static_cast<uint32_t>(n));
    FB_LAUNCH_CHECK();
}

void launch_save_history(LevelView v, int64_t rows, int32_t hist, int32_t n_valid, void* hist_buf,
                         cudaStream_t s) {
    if (rows == 0 || hist == 0)
        return;
    const size_t es  = v.fp16 ? 2 : 4;
    const char* src  = static_cast<const char*>(v.data) + (v.base + n_valid - hist) * es;
    copy_rows(hist_buf, hist * es, src, v.pitch * es, hist * es, static_cast<size_t>(rows), s);
}

void launch_load_history(LevelView v, int64_t rows, int32_t hist, const void* hist_buf,
                         cudaStream_t s) {
    if (rows == 0 || hist == 0)
        return;
    const size_t es = v.fp16 ? 2 : 4;
    char* dst       = static_cast<char*>(v.data) + (v.base - hist) * es;
    copy_rows(dst, v.pitch * es, hist_buf, hist * es, hist * es, static_cast<size_t>(rows), s);
}

void launch_save_input_history(const float* wf, int64_t pitch, int64_t t0, int32_t n_valid,
                               int32_t nchans, float* hist, float* scratch, int32_t hist_len,
                               cudaStream_t s) {
    if (hist_len == 0)
        return;
    const size_t es = sizeof(float);
    if (n_valid >= hist_len) {
        FB_CUDA(cudaMemcpy2DAsync(hist, hist_len * es, wf + t0 + n_valid - hist_len, pitch * es,
                                  hist_len * es, nchans, cudaMemcpyDeviceToDevice, s));
        return;
    }
    // Keep the newest hist_len - n_valid old samples, then append the tile.
    const int32_t keep = hist_len - n_valid;
    FB_CUDA(cudaMemcpy2DAsync(scratch, hist_len * es, hist + n_valid, hist_len * es, keep * es,
                              nchans, cudaMemcpyDeviceToDevice, s));
    if (n_valid > 0)
        FB_CUDA(cudaMemcpy2DAsync(scratch + keep, hist_len * es, wf + t0, pitch * es, n_valid * es,
                                  nchans, cudaMemcpyDeviceToDevice, s));
    FB_CUDA(cudaMemcpyAsync(hist, scratch, static_cast<size_t>(nchans) * hist_len * es,
                            cudaMemcpyDeviceToDevice, s));
}

} // namespace fb::fdmt
