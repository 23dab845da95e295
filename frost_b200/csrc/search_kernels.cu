// Boxcar/trapezoid matched filter, exact noise and peak finding on sm_100a.
//
// One CTA per searched (plane, DM) row walks the tile in chunks of 2048 or
// 4096 samples (a launch-shape choice), the raw row segment bulk-copied into
// shared memory one chunk ahead. Each thread owns P = chunk / 256
// consecutive samples and keeps their prefix sums in registers (serial sum,
// warp shuffles, one offset per warp); the prefix origin is the chunk's
// first column, and the halo before it (the widest boxcar, rounded to 256
// columns) is the previous chunk's last columns rebased to that origin, so
// only a tile's first chunk scans its halo. Every width's window sum is a
// difference of two (four for the trapezoid) prefix values. In the steady
// state (no cold prefix, no mask change in the chunk) a sample is above
// threshold when its window sum exceeds thresh * sigma, precomputed per
// width, and nothing is written to shared memory but the least prefix value
// of each 4-sample group and of each thread's samples: widths 1 and 2 take
// the exact sums in registers, wider boxcars a bound (the greatest prefix
// value of a set of samples minus the least one their windows start from),
// per thread first for wide boxcars, then per group. A chunk where nothing
// may fire costs one block vote. Only otherwise are the prefix sums stored
// and the exact test run on the groups a bound did not clear, writing the
// per-width bit masks of the samples that fired. The first chunks of a
// stream or after a mask change (cold prefix, OR-mask variance) build the
// bit masks from the general S/N. For every width that fired, one lane
// (widths spread over the warps) walks its set bits in time order,
// extending or closing the run carried from the previous chunk (and tile,
// and gulp) and emitting each closed run's peak. The DM-time rows are never
// re-read and the run state is the only thing carried between calls.
//
// When the FDMT step into the searched level is a single level step, the
// same kernel also performs it for its rows (the fused level step): each
// chunk stages the row's two children from the level below instead of the
// row, adds them as the level kernel would, writes the row back for the
// next levels and the history, and searches it; the level kernel then
// computes only the rows no plane searches.
//
// Results are ordered on the device afterwards (k_cand_range, k_cand_keys,
// a radix sort of packed keys, k_cand_gather), so the candidates of one
// call come back in (level, sub-band, DM row, peak, width) order whatever
// order the CTAs appended them in.

#include <algorithm>

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "bulk_copy.cuh"
#include "common.hpp"
#include "search_kernels.hpp"

namespace fb::fdmt {

namespace {

constexpr int kThreads   = 256;
static_assert(kThreads == 256, "the warp offsets read the 8 warp totals as two float4");
constexpr int kMaxWidths = 32;
// widths 1, 2, ..., 2^15 take the unrolled steady-state tests
constexpr int kMaxPow2Widths = 16;
#define FB_NEG_INF (-__int_as_float(0x7f800000))
#define FB_POS_INF (__int_as_float(0x7f800000))

template <class S> __device__ __forceinline__ float ldf(const S* p);
template <> __device__ __forceinline__ float ldf<float>(const float* p) { return *p; }
template <> __device__ __forceinline__ float ldf<__half>(const __half* p) { return __half2float(*p); }

// Three-operand max / min (one sm_100 instruction; the same values as two
// fmaxf / fminf: no rounding, NaN operands ignored).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// max over e of q[e] - q[e - S] (S = 1 or 2) for e = S .. P - 1, folded into
// `m`, two differences per instruction.
template <int P, int S>
__device__ __forceinline__ float max_diffs(const float (&q)[P], float m) {
#pragma unroll
    for (int e = S; e < P; e += 2) {
        if (e + 1 < P)
            m = fmax3(m, q[e] - q[e - S], q[e + 1] - q[e + 1 - S]);
        else
            m = fmaxf(m, q[e] - q[e - S]);
    }
    return m;
}

__device__ void scan_inplace(float* a, int n) {
    __shared__ __align__(16) float warp_tot[kThreads / 32];
    const int per = (n + kThreads - 1) / kThreads;
    const int beg = threadIdx.x * per;
    const int end = min(beg + per, n);
    float run     = 0.0F;
    for (int i = beg; i < end; ++i) {
        run += a[i];
        a[i] = run;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float v        = run;
    for (int o = 1; o < 32; o <<= 1) {
        const float u = __shfl_up_sync(0xFFFFFFFFU, v, o);
        if (lane >= o)
            v += u;
    }
    if (lane == 31)
        warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        float w = lane < kThreads / 32 ? warp_tot[lane] : 0.0F;
        for (int o = 1; o < 32; o <<= 1) {
            const float u = __shfl_up_sync(0xFFFFFFFFU, w, o);
            if (lane >= o)
                w += u;
        }
        if (lane < kThreads / 32)
            warp_tot[lane] = w;
    }
    __syncthreads();
    const float offset = (v - run) + (warp > 0 ? warp_tot[warp - 1] : 0.0F);
    for (int i = beg; i < end; ++i)
        a[i] += offset;
    __syncthreads();
}

/** Per-row constants, in shared memory. */
struct RowConst {
    int64_t tile_t0;  // absolute sample of tile column 0
    int64_t gulp_t0;  // absolute sample of the gulp's first column
    int32_t or_active;
    int W[kMaxWidths];
    int E[kMaxWidths];      // trapezoid half-weight edge, 0 for a boxcar
    float inv[kMaxWidths];  // 1/sigma
    float inv_or[kMaxWidths];
    float thr[kMaxWidths];  // window-sum threshold thresh * sigma
};

// Window sum of width W (trapezoid edge E, 0 for a boxcar) ending at chunk
// sample k; Q[k] is the prefix sum through sample k.
// The steady-state pre-test evaluates the same expression, so the trapezoid
// correction is written with non-contractible intrinsics (no FMA) to give
// bit-identical sums in both places.
__device__ __forceinline__ float trap_sum(float qk, float qw, float qe, float qwe) {
    return __fsub_rn(qk - qw, __fmul_rn(0.5F, (qk - qe) + (qwe - qw)));
}

__device__ __forceinline__ float wsum(const float* Q, int k, int W, int E) {
    const float qk = Q[k], qw = Q[k - W];
    return E > 0 ? trap_sum(qk, qw, Q[k - E], Q[k - W + E]) : qk - qw;
}

// General S/N of chunk sample k at width wi: -inf past the valid columns or
// in the cold prefix; the OR-mask variance right after a mask change.
__device__ __forceinline__ float snr_general(const SearchParams& p, const RowConst& rc,
                                             const float* Q, int64_t c0, int k, int wi,
                                             int32_t delay) {
    const int64_t col = c0 + k;
    if (col >= p.n_valid)
        return FB_NEG_INF;
    const int W     = rc.W[wi];
    const int64_t t = rc.tile_t0 + col;
    if (p.skip_cold && t < static_cast<int64_t>(delay) + W - 1)
        return FB_NEG_INF;
    const bool use_or = rc.or_active && (t - rc.gulp_t0) < static_cast<int64_t>(delay) + W - 1;
    const float inv   = use_or ? rc.inv_or[wi] : rc.inv[wi];
    if (inv == 0.0F)
        return FB_NEG_INF;
    return wsum(Q, k, W, rc.E[wi]) * inv;
}

// Q[idx .. idx + 4) with idx mod 4 the same across the warp: one or two
// aligned 16-byte shared-memory loads (Q itself is 16-byte aligned).
__device__ __forceinline__ float4 ld4(const float* Q, int idx) {
    const int r     = idx & 3;
    const float4* v = reinterpret_cast<const float4*>(Q + (idx - r));
    const float4 a  = v[0];
    if (r == 0)
        return a;
    const float4 b = v[1];
    if (r == 1)
        return make_float4(a.y, a.z, a.w, b.x);
    if (r == 2)
        return make_float4(a.z, a.w, b.x, b.y);
    return make_float4(a.w, b.x, b.y, b.z);
}

// Eight consecutive staged samples (16-byte aligned) as float.
template <class S> __device__ __forceinline__ void ld8s(const S* p, float (&x)[8]) {
    if constexpr (sizeof(S) == 4) {
        const float4 a = reinterpret_cast<const float4*>(p)[0];
        const float4 b = reinterpret_cast<const float4*>(p)[1];
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    } else {
        const uint4 u       = *reinterpret_cast<const uint4*>(p);
        const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[i]));
            x[2 * i]       = f.x;
            x[2 * i + 1]   = f.y;
        }
    }
}

// `count` (shared or global) is the row's emitted total this call.
__device__ void emit(const SearchParams& p, const SearchRow& row, const RunState& r,
                     uint32_t* count) {
    const uint32_t before = atomicAdd(count, 1U);
    if (p.max_per_dm != 0 && before >= p.max_per_dm) {
        atomicAdd(&p.dropped[1], 1ULL);
        return;
    }
    const unsigned long long idx = atomicAdd(p.ncands, 1ULL);
    if (idx >= p.max_cands) {
        atomicAdd(&p.dropped[0], 1ULL);
        return;
    }
    const PlaneInfo& pl = p.planes[row.plane];
    frost_candidate c;
    c.peak_sample   = static_cast<uint64_t>(r.best_t);
    c.begin_sample  = static_cast<uint64_t>(r.start);
    c.end_sample    = static_cast<uint64_t>(r.last_t);
    c.snr           = r.best;
    c.dm            = row.dm;
    c.f_low_mhz     = pl.f_low;
    c.f_high_mhz    = pl.f_high;
    c.filter_idx    = static_cast<uint32_t>(r.best_w);
    c.width         = static_cast<uint32_t>(p.widths[r.best_w]);
    c.dm_idx        = static_cast<uint32_t>(row.prow);
    c.chan_begin    = pl.chan_begin;
    c.chan_end      = pl.chan_end;
    c.beam_idx      = 0;
    c.subband_level = pl.subband_level;
    c.subband_idx   = pl.subband_idx;
    p.cands[idx]    = c;
}

// A maximal run of set bits inside one lane's share of a chunk's mask: its
// first and last chunk sample and its first maximum.
struct Seg {
    int32_t first_k, last_k, best_k, best_w;
    float best;
};

// S/N of set bit k for width wi, or the best over widths (first maximum)
// for wi < 0.
__device__ __forceinline__ float bit_snr(const SearchParams& p, const RowConst& rc, const float* Q, int64_t c0,
                                         int k, int wi, int32_t delay, int& bw) {
    if (wi >= 0) {
        bw = wi;
        return snr_general(p, rc, Q, c0, k, wi, delay);
    }
    float best = FB_NEG_INF;
    bw         = 0;
    for (int w = 0; w < p.nwidths; ++w) {
        const float s = snr_general(p, rc, Q, c0, k, w, delay);
        if (s > best) {
            best = s;
            bw   = w;
        }
    }
    return best;
}

__device__ __forceinline__ RunState run_of(const RowConst& rc, int64_t c0, const Seg& g) {
    RunState r{};
    r.open   = 1;
    r.start  = rc.tile_t0 + c0 + g.first_k;
    r.best   = g.best;
    r.best_t = rc.tile_t0 + c0 + g.best_k;
    r.best_w = g.best_w;
    r.last_t = rc.tile_t0 + c0 + g.last_k;
    return r;
}

__device__ __forceinline__ Seg shfl_seg(const Seg& g, int src) {
    Seg r;
    r.first_k = __shfl_sync(0xFFFFFFFFU, g.first_k, src);
    r.last_k  = __shfl_sync(0xFFFFFFFFU, g.last_k, src);
    r.best_k  = __shfl_sync(0xFFFFFFFFU, g.best_k, src);
    r.best_w  = __shfl_sync(0xFFFFFFFFU, g.best_w, src);
    r.best    = __shfl_sync(0xFFFFFFFFU, g.best, src);
    return r;
}

// The runs of one chunk's mask for one width (or across widths, wi < 0), by
// a whole warp: lane L takes the chunk's samples [L CH / 32, (L + 1) CH / 32)
// (cut at the last valid sample) and finds its maximal runs in time order
// (S/N of each set bit, first maximum); runs that touch neither end of the
// lane's share are complete and emitted at once. Lane 0 then joins, in time order, the runs that do
// touch a share's end with each other and with the run carried from the
// previous chunk, exactly as a sequential walk over the bits would (the
// strict comparison keeps the earliest maximum), emits the closed ones and
// leaves `run` open when it reaches the chunk's last valid sample.
template <int CH>
__device__ __forceinline__ void walk_runs_warp(const SearchParams& p, const RowConst& rc, const float* Q, int64_t c0,
                               int32_t delay, const uint32_t* bits, int wi, RunState& run,
                               const SearchRow& row, uint32_t* count) {
    constexpr int kPerLane = CH / 32 / 32; // mask words per lane
    const int lane = threadIdx.x & 31;
    // the lane's share ends at its last sample or at the chunk's last valid one
    const int64_t valid = static_cast<int64_t>(p.n_valid) - c0;
    const int kbeg = lane * kPerLane * 32;
    const int kend = static_cast<int>(min(static_cast<int64_t>(kbeg + kPerLane * 32), valid));
    Seg left{}, right{}, cur{};
    bool has_left = false, has_right = false, whole = false, open = false;
    int prev = -2;
    auto finish = [&](const Seg& g) {
        if (g.first_k == kbeg) {
            left     = g;
            has_left = true;
        } else {
            emit(p, row, run_of(rc, c0, g), count);
        }
    };
#pragma unroll
    for (int wd = 0; wd < kPerLane; ++wd) {
        uint32_t b = bits[lane * kPerLane + wd];
        while (b) {
            const int k = (lane * kPerLane + wd) * 32 + __ffs(b) - 1;
            b &= b - 1;
            int bw;
            const float sn = bit_snr(p, rc, Q, c0, k, wi, delay, bw);
            if (open && k == prev + 1) {
                if (sn > cur.best) {
                    cur.best   = sn;
                    cur.best_k = k;
                    cur.best_w = bw;
                }
                cur.last_k = k;
            } else {
                if (open)
                    finish(cur);
                cur  = Seg{k, k, k, bw, sn};
                open = true;
            }
            prev = k;
        }
    }
    if (open) {
        if (cur.last_k == kend - 1) {
            has_right = true;
            right     = cur;
            if (cur.first_k == kbeg) {
                whole    = true;
                left     = cur;
                has_left = true;
            }
        } else {
            finish(cur);
        }
    }
    // lane 0 joins the share-end runs in time order
    uint32_t ev = __ballot_sync(0xFFFFFFFFU, has_left || has_right);
    RunState r    = run;
    int64_t last  = r.open ? c0 - 1 : -2; // tile column of the run's last sample
    while (ev) {
        const int L = __ffs(static_cast<int>(ev)) - 1;
        ev &= ev - 1;
        const bool hl = __shfl_sync(0xFFFFFFFFU, has_left, L);
        const bool hr = __shfl_sync(0xFFFFFFFFU, has_right, L);
        const bool wh = __shfl_sync(0xFFFFFFFFU, whole, L);
        const Seg gl  = shfl_seg(left, L);
        const Seg gr  = shfl_seg(right, L);
        if (lane != 0)
            continue;
        const int64_t lstart = c0 + L * kPerLane * 32;
        if (hl) {
            if (r.open && last == lstart - 1) {
                if (gl.best > r.best) {
                    r.best   = gl.best;
                    r.best_t = rc.tile_t0 + c0 + gl.best_k;
                    r.best_w = gl.best_w;
                }
                r.last_t = rc.tile_t0 + c0 + gl.last_k;
            } else {
                if (r.open)
                    emit(p, row, r, count);
                r = run_of(rc, c0, gl);
            }
            last = c0 + gl.last_k;
            if (!wh) {
                emit(p, row, r, count);
                r.open = 0;
            }
        }
        if (hr && !wh) {
            if (r.open)
                emit(p, row, r, count);
            r    = run_of(rc, c0, gr);
            last = c0 + gr.last_k;
        }
    }
    if (lane == 0) {
        // a run that does not reach the chunk's last valid column has closed
        const int64_t chunk_end = min(c0 + CH, static_cast<int64_t>(p.n_valid));
        if (r.open && last != chunk_end - 1) {
            emit(p, row, r, count);
            r.open = 0;
        }
        run = r;
    }
}

// Words of the per-width bit masks [nw][chunk / 32].
__host__ __device__ constexpr int search_bits_words(int nw, int chunk) { return nw * (chunk / 32); }

// How the steady-state pass clears a width before any exact test.
enum : int {
    kTestExact = 0, // boxcar of 1 or 2 samples: the exact window sums, in registers
    kTestGroup = 1, // per 4-sample group: group max minus the least prefix a window starts from
    kTestBlock = 2, // per thread's columns first (wide boxcars), then per group
    kTestAll   = 3, // trapezoid: the exact test on every group
};

/** Per-width constants of the steady-state pass, built once per CTA. For a
 * thread t owning chunk columns [P t, P t + P): gmin index of its first
 * group's first window start = NG t + gconst, tmin index of its first
 * window start = t + bconst; `two` / `btwo`: the starts straddle two
 * groups / blocks. */
struct WidthTest {
    int kind;
    int W;
    int gconst;
    int two;
    int bconst;
    int btwo;
    float T;
    int pad;
};

// Loads P staged samples (16-byte aligned) as float.
template <class S, int P> __device__ __forceinline__ void ld_cols(const S* p, float (&x)[P]) {
#pragma unroll
    for (int i = 0; i < P / 8; ++i) {
        float y[8];
        ld8s<S>(p + 8 * i, y);
#pragma unroll
        for (int e = 0; e < 8; ++e)
            x[8 * i + e] = y[e];
    }
}

// q[e] = x[0] + ... + x[e] (left to right, float) of P samples already in
// q; xmax = the largest of them.
template <int P> __device__ __forceinline__ void scan_floats(float (&q)[P], float& xmax) {
    float m = q[0];
#pragma unroll
    for (int e = 1; e + 1 < P; e += 2)
        m = fmax3(m, q[e], q[e + 1]);
    if constexpr (P % 2 == 0)
        m = fmaxf(m, q[P - 1]);
    xmax = m;
#pragma unroll
    for (int e = 1; e < P; ++e)
        q[e] += q[e - 1];
}

// The same for P fp16 samples packed in pairs (sample 2i in the low half of
// w[i]), added with mixed-precision adds (`add.rn.f32.f16`: the widening is
// exact, so the same bits as widening first).
template <int P>
__device__ __forceinline__ void scan_halves(const uint32_t (&w)[P / 2], float (&q)[P], float& xmax) {
    // the largest sample: packed fp16 maxima (exact), then one widening
    __half2 hm = *reinterpret_cast<const __half2*>(&w[0]);
#pragma unroll
    for (int i = 1; i < P / 2; ++i)
        hm = __hmax2(hm, *reinterpret_cast<const __half2*>(&w[i]));
    xmax = fmaxf(__low2float(hm), __high2float(hm));
    q[0] = __half2float(__ushort_as_half(static_cast<unsigned short>(w[0] & 0xFFFFU)));
#pragma unroll
    for (int e = 1; e < P; ++e) {
        const uint16_t h = static_cast<uint16_t>((e & 1) ? (w[e / 2] >> 16) : (w[e / 2] & 0xFFFFU));
        asm("add.rn.f32.f16 %0, %1, %2;" : "=f"(q[e]) : "h"(h), "f"(q[e - 1]));
    }
}

// Prefix sums of the P staged samples at `p` (16-byte aligned).
template <class S, int P> __device__ __forceinline__ void scan_cols(const S* p, float (&q)[P], float& xmax) {
    if constexpr (sizeof(S) == 4) {
        ld_cols<S, P>(p, q);
        scan_floats<P>(q, xmax);
    } else {
        uint32_t w[P / 2];
#pragma unroll
        for (int i = 0; i < P / 8; ++i) {
            const uint4 u = reinterpret_cast<const uint4*>(p)[i];
            w[4 * i] = u.x, w[4 * i + 1] = u.y, w[4 * i + 2] = u.z, w[4 * i + 3] = u.w;
        }
        scan_halves<P>(w, q, xmax);
    }
}

// Fused level step: this thread's P columns of a searched row computed from
// the level below, out = lo + hi shifted, bit for bit as the single-level
// kernel computes them, stored to the row in global memory and
// prefix-summed. `lo` is the staged unshifted child segment at the thread's
// first column and `hi` the staged 16-byte-aligned superset of the shifted
// child at the same place, the thread's first shifted sample `hoff`
// elements in (hi == nullptr: the row copies its low child); both buffers
// hold at least 16 bytes past the thread's P columns.
// fp16: the level kernel rounds the float sum of two fp16 values with the
// saturating convert. That float sum is exact when their exponents differ
// by at most 12 (11-bit significands: the sum needs at most 24 bits), and
// otherwise the smaller operand is below a quarter of the larger one's fp16
// spacing, so that both roundings return the larger operand; the fp16 add
// (round to nearest even of the exact sum) gives the same bits, with a
// clamp to +-65504 for the saturation (sums past it round to infinity).
template <class S, int P>
__device__ __forceinline__ void merge_scan(const S* lo, const S* hi, int hoff, S* dst, float (&q)[P],
                                           float& xmax) {
    if constexpr (sizeof(S) == 4) {
        ld_cols<S, P>(lo, q);
        if (hi != nullptr) {
            float h[P + 4];
#pragma unroll
            for (int i = 0; i < P / 4 + 1; ++i) {
                const float4 v = reinterpret_cast<const float4*>(hi)[i];
                h[4 * i] = v.x, h[4 * i + 1] = v.y, h[4 * i + 2] = v.z, h[4 * i + 3] = v.w;
            }
            switch (hoff) {
#define FB_SHIFTED(O)                                                                             \
    case O:                                                                                       \
        _Pragma("unroll") for (int e = 0; e < P; ++e) q[e] = q[e] + h[O + e];                      \
        break;
                FB_SHIFTED(0) FB_SHIFTED(1) FB_SHIFTED(2) FB_SHIFTED(3)
#undef FB_SHIFTED
            }
        }
#pragma unroll
        for (int i = 0; i < P / 4; ++i)
            reinterpret_cast<float4*>(dst)[i] = make_float4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
        scan_floats<P>(q, xmax);
    } else {
        uint32_t w[P / 2];
#pragma unroll
        for (int i = 0; i < P / 8; ++i) {
            const uint4 u = reinterpret_cast<const uint4*>(lo)[i];
            w[4 * i] = u.x, w[4 * i + 1] = u.y, w[4 * i + 2] = u.z, w[4 * i + 3] = u.w;
        }
        if (hi != nullptr) {
            uint32_t W[P / 2 + 4];
#pragma unroll
            for (int i = 0; i < P / 8 + 1; ++i) {
                const uint4 u = reinterpret_cast<const uint4*>(hi)[i];
                W[4 * i] = u.x, W[4 * i + 1] = u.y, W[4 * i + 2] = u.z, W[4 * i + 3] = u.w;
            }
            // the shifted pairs: whole words hoff / 2 on, shifted by a half
            // when hoff is odd
            const uint32_t sh = (hoff & 1) * 16U;
            uint32_t g[P / 2];
            switch (hoff >> 1) {
#define FB_SHIFTED(K)                                                                             \
    case K:                                                                                       \
        _Pragma("unroll") for (int i = 0; i < P / 2; ++i) g[i] = __funnelshift_r(W[K + i], W[K + i + 1], sh); \
        break;
                FB_SHIFTED(0) FB_SHIFTED(1) FB_SHIFTED(2) FB_SHIFTED(3)
#undef FB_SHIFTED
            }
            const __half2 top = __float2half2_rn(65504.0F);
            const __half2 bot = __float2half2_rn(-65504.0F);
#pragma unroll
            for (int i = 0; i < P / 2; ++i) {
                const __half2 x = __hadd2(*reinterpret_cast<const __half2*>(&w[i]),
                                          *reinterpret_cast<const __half2*>(&g[i]));
                const __half2 c = __hmin2(__hmax2(x, bot), top);
                w[i]            = *reinterpret_cast<const uint32_t*>(&c);
            }
        }
#pragma unroll
        for (int i = 0; i < P / 8; ++i)
            reinterpret_cast<uint4*>(dst)[i] = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
        scan_halves<P>(w, q, xmax);
    }
}

// q[e] += off for every e, two lanes per instruction (add.rn.f32x2: each
// lane rounds as a scalar add).
template <int P> __device__ __forceinline__ void add_offset(float (&q)[P], float off) {
#pragma unroll
    for (int e = 0; e + 1 < P; e += 2)
        asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%0, %1};\n mov.b64 b, {%2, %2};\n"
            " add.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
            : "+f"(q[e]), "+f"(q[e + 1])
            : "f"(off));
    if constexpr (P % 2 != 0)
        q[P - 1] += off;
}

template <int R, int NG, int N>
__device__ __forceinline__ void pick_lows(const float (&e)[N], bool two, float (&lo)[NG]) {
#pragma unroll
    for (int g = 0; g < NG; ++g)
        lo[g] = two ? fminf(e[R + g], e[R + g + 1]) : e[R + g];
}

// lo[g] = gmin[i0 + g], or the lesser of gmin[i0 + g] and gmin[i0 + g + 1]
// when the window starts straddle two groups: the least prefix value a
// window of the thread's group g starts from. i0 mod NG is the same for
// every thread of the block, so the values come from aligned vector loads
// (gmin is padded by 4 floats for the second one).
template <int NG>
__device__ __forceinline__ void group_lows(const float* gmin, int i0, bool two, float (&lo)[NG]) {
    if constexpr (NG == 4) {
        const int r     = i0 & 3;
        const float4* v = reinterpret_cast<const float4*>(gmin + (i0 - r));
        const float4 a  = v[0];
        const float4 b  = (r != 0 || two) ? v[1] : a;
        const float e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        switch (r) {
        case 0: pick_lows<0, 4, 8>(e, two, lo); break;
        case 1: pick_lows<1, 4, 8>(e, two, lo); break;
        case 2: pick_lows<2, 4, 8>(e, two, lo); break;
        default: pick_lows<3, 4, 8>(e, two, lo); break;
        }
    } else {
        const int r     = i0 & 1;
        const float2* v = reinterpret_cast<const float2*>(gmin + (i0 - r));
        const float2 a  = v[0];
        const float2 b  = (r != 0 || two) ? v[1] : a;
        const float e[4] = {a.x, a.y, b.x, b.y};
        if (r == 0)
            pick_lows<0, 2, 4>(e, two, lo);
        else
            pick_lows<1, 2, 4>(e, two, lo);
    }
}

// The steady-state test of width 2^WI for the widths 1, 2, 4, ... (no
// trapezoid): the same tests as the per-width table, with every offset and
// alignment a compile-time constant (the halo is a multiple of 256, so the
// window starts' group and block offsets depend on W alone).
template <int P, int NG, int WI>
__device__ __forceinline__ bool pow2_maybe(const float (&q)[P], float pm1, float pm2, const float (&gmx)[NG],
                                           float bmax, const float* gmin, const float* tmin, int halo, float T,
                                           float& m1) {
    constexpr int W = 1 << WI;
    if constexpr (W == 1) {
        // m1 arrives as an upper bound of every width-1 sum of the thread's
        // samples (see the caller)
        return m1 > T;
    } else if constexpr (W == 2) {
        // Every width-2 window sum is, before rounding, the sum of two of the
        // thread's width-1 sums (or of its first one and the one ending just
        // before it). With M the largest of them as rounded, each is at most
        // M (1 + 2^-23) when M > 0 and at most 0 otherwise (a rounded
        // difference is 0 only when exact), so no width-2 sum rounds above
        // 2 M (1 + 2^-22): skip the exact test when that cannot exceed T
        // (NaN M or T <= 0: test).
        const float d = fmaxf(m1, pm1 - pm2);
        if (T > 0.0F && 2.0F * d * (1.0F + 0x1p-20F) <= T)
            return false;
        const float m = max_diffs<P, 2>(q, fmaxf(q[0] - pm2, q[1] - pm1));
        return m > T;
    } else {
        if constexpr (W >= 4 * P) {
            // the thread's window starts are exactly block t - W / P
            if (!(bmax - tmin[static_cast<int>(threadIdx.x) + halo / P - W / P] > T))
                return false;
        }
        // own group g starts in group NG t + g + halo / 4 - W / 4, whose
        // vector alignment R is fixed by W
        constexpr int R = (NG - (W / 4) % NG) % NG;
        const int i0    = NG * static_cast<int>(threadIdx.x) + halo / 4 - W / 4;
        float lo[NG];
        if constexpr (NG == 4) {
            const float4* v = reinterpret_cast<const float4*>(gmin + (i0 - R));
            const float4 a  = v[0];
            const float4 b  = R != 0 ? v[1] : a;
            const float e[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
            pick_lows<R, 4, 8>(e, false, lo);
        } else {
            const float2* v = reinterpret_cast<const float2*>(gmin + (i0 - R));
            const float2 a  = v[0];
            const float2 b  = R != 0 ? v[1] : a;
            const float e[4] = {a.x, a.y, b.x, b.y};
            pick_lows<R, 2, 4>(e, false, lo);
        }
        float m;
        if constexpr (NG == 4)
            m = fmaxf(fmax3(gmx[0] - lo[0], gmx[1] - lo[1], gmx[2] - lo[2]), gmx[3] - lo[3]);
        else
            m = fmaxf(gmx[0] - lo[0], gmx[1] - lo[1]);
        return m > T;
    }
}

// The steady-state tests of the widths 2^WI .. 2^(WI1 - 1) that are below nw
// (one by one: a test of a set of widths against its smallest threshold,
// bounded by the set's least window start, measured slower).
template <int P, int NG, int WI, int WI1>
__device__ __forceinline__ void pow2_range(uint32_t& cand, const float (&q)[P], float pm1, float pm2,
                                           const float (&gmx)[NG], float bmax, const float* gmin,
                                           const float* tmin, int halo, const WidthTest* wt, int nw, float& m1) {
    if constexpr (WI < WI1) {
        if (WI < nw) {
            if (pow2_maybe<P, NG, WI>(q, pm1, pm2, gmx, bmax, gmin, tmin, halo, wt[WI].T, m1))
                cand |= 1U << WI;
            pow2_range<P, NG, WI + 1, WI1>(cand, q, pm1, pm2, gmx, bmax, gmin, tmin, halo, wt, nw, m1);
        }
    }
}

// Q[-halo .. -1] straight from the staged halo columns: a prefix sum from
// the first column a window can reach (earlier columns count 0), rebased so
// that Q[-1] = 0, and the halo's entries of gmin (per 4 columns) and tmin
// (per P columns). Rounding is monotonic, so the least rebased value of a
// group is its least prefix value, rebased.
template <class S, int P>
__device__ void scan_halo(const S* seg, int halo, int jmin, float* Q, float* gmin, float* tmin) {
    float* H = Q - halo;
    for (int i = threadIdx.x; i < halo; i += kThreads)
        H[i] = i < jmin ? 0.0F : ldf<S>(seg + i);
    __syncthreads();
    scan_inplace(H, halo);
    const float last = H[halo - 1];
    for (int j = threadIdx.x; j < halo / 4; j += kThreads)
        gmin[j] = fminf(fminf(H[4 * j], H[4 * j + 1]), fminf(H[4 * j + 2], H[4 * j + 3])) - last;
    for (int j = threadIdx.x; j < halo / P; j += kThreads) {
        float m = H[P * j];
        for (int e = 1; e < P; ++e)
            m = fminf(m, H[P * j + e]);
        tmin[j] = m - last;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < halo; i += kThreads)
        H[i] -= last;
}

template <class S, int CH, bool POW2, int FSB, int K>
__global__ void __launch_bounds__(kThreads, FSB == 2 ? (CH == 2048 ? 4 : 3) : (CH == 2048 ? 5 : 4))
    k_search(const __grid_constant__ SearchSegTable<K> tab) {
    constexpr bool FS = FSB > 0; // fused level step, FSB chunks staged at once
    // The search shape (widths, halo, peak mode, valid columns) is the same
    // in every segment; the rows, tables and outputs are each segment's.
    const SearchParams& p = tab.s[0].p;
    constexpr int P  = CH / kThreads; // chunk columns per thread
    constexpr int NG = P / 4;         // 4-column groups per thread
    // Dynamic shared memory (floats unless noted):
    //   Ps     4 pad + halo + CH + 4 pad: Q = Ps + 4 + halo holds the chunk's
    //          prefix sums from its first column (Q[-1] = 0) and, before it,
    //          the halo's, rebased to the same origin; Q is written only in
    //          chunks where some test may fire
    //   gmin   (halo + CH) / 4 + 4 pad: least Q of each aligned 4-column group
    //   tmin   (halo + CH) / P: least Q of each thread's P columns
    //   nh     2 x nh_len: the next chunk's halo (Q, gmin, tmin and this
    //          chunk's last Q, not yet rebased), by chunk parity
    //   bits   uint32 [nw][CH / 32]: per-width masks of the samples that fired
    //   stage  S [2][halo + CH]: the raw row segment, bulk-copied one chunk
    //          ahead (the halo columns only for the first chunk)
    // With the level step fused (FS), the stage instead holds the row's
    // halo columns (first chunk) and, for each of the FSB chunks in flight
    // (one or two), the chunk's unshifted child segment and the aligned
    // superset of its shifted one: S [halo] + [FSB][CH + CH + 16 / es]. With
    // one, the next chunk's copies start once every thread has merged this
    // one (no more shared memory than the two raw buffers).
    extern __shared__ __align__(16) float Ps[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int abort_flag;
    __shared__ uint32_t any_bits[(CH / 32)];
    __shared__ RunState runs[kMaxWidths];
    __shared__ RowConst rc;
    __shared__ WidthTest wt[kMaxWidths];
    __shared__ uint32_t local_count;
    __shared__ uint32_t fired_w; // widths with a set bit in this chunk
    __shared__ float warp_tot[kThreads / 32];
    __shared__ float wtail[kThreads / 32][2]; // each warp's last two prefix values

    const int nw        = p.nwidths;
    const int wmax      = p.wmax;
    const int halo      = p.halo;
    const bool across   = p.peak_mode == FROST_PEAK_ACROSS_WIDTHS;
    const bool all      = p.peak_mode == FROST_PEAK_ALL;
    const int nruns     = across ? 1 : nw;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg_cols   = halo + CH;
    float* const Q       = Ps + 4 + halo;
    float* const gmin    = Ps + 4 + seg_cols + 4;
    float* const tmin    = gmin + seg_cols / 4 + 4;
    const int nh_len     = halo + halo / 4 + halo / P + 4;
    float* const nh0     = tmin + seg_cols / P;
    uint32_t* const bits = reinterpret_cast<uint32_t*>(nh0 + 2 * nh_len);
    S* const stage0      = reinterpret_cast<S*>(bits + search_bits_words(nw, CH)); // buffer b at stage0 + b * seg_cols
    // A chunk's halo is the previous chunk's last `halo` columns, whose prefix
    // sums that chunk has: only the first chunk (or every chunk, for a halo
    // wider than a chunk) stages and scans its halo.
    const bool carry_halo = halo <= CH;
    const int nchunks     = (p.n_valid + CH - 1) / CH;
    if (threadIdx.x == 0) {
        abort_flag = 0;
        bulk::mbar_init(&bar[0]);
        bulk::mbar_init(&bar[1]);
    }
    __syncthreads();
    // Rows blockIdx.x, blockIdx.x + gridDim.x, ...; the staging buffers and
    // barriers alternate over the CTA's chunks across rows.
    int64_t cc = 0; // chunks this CTA has consumed
    const int64_t nrows_all = tab.s[tab.n - 1].row_end;
    int sg       = 0; // the segment of the CTA's current row
    int64_t sbeg = 0; // and its first row
    for (int64_t gi = blockIdx.x; gi < nrows_all; gi += gridDim.x) {
        while (gi >= tab.s[sg].row_end) {
            sbeg = tab.s[sg].row_end;
            ++sg;
        }
        const SearchSeg& SG   = tab.s[sg];
        const SearchParams& p = SG.p;
        const S* level        = static_cast<const S*>(SG.level);
        const int64_t pitch   = SG.pitch;
        const int32_t base    = SG.base;
        const int64_t g       = SG.g0 + (gi - sbeg);
        const SearchRow row = p.rows[g];
        if (threadIdx.x == 0) {
            local_count  = p.row_counts[g];
            const GulpClock ck = *p.clock;
            rc.gulp_t0   = ck.gulp_t0;
            rc.tile_t0   = ck.gulp_t0 + p.tile_off;
            rc.or_active = ck.or_active;
        }
        if (threadIdx.x < nw) {
            const int w    = threadIdx.x;
            const int W    = p.widths[w];
            const int E    = (p.trapezoid && W >= 3) ? (W + 1) / 4 : 0;
            rc.W[w]        = W;
            rc.E[w]        = E;
            const float iv = p.inv_sigma[g * nw + w];
            rc.inv[w]      = iv;
            rc.inv_or[w]   = p.inv_sigma_or[g * nw + w];
            const float T  = iv > 0.0F ? p.thresh / iv : FB_POS_INF;
            rc.thr[w]      = T;
            WidthTest t;
            t.kind   = E > 0 ? kTestAll : W <= 2 ? kTestExact : W < 4 * P ? kTestGroup : kTestBlock;
            t.W      = W;
            t.gconst = (halo - W) >> 2;
            t.two    = ((halo - W) & 3) != 0 ? 1 : 0;
            t.bconst = (halo - W) / P;
            t.btwo   = ((halo - W) % P) != 0 ? 1 : 0;
            t.T      = T;
            t.pad    = 0;
            wt[w]    = t;
        }
        if (threadIdx.x < nruns && !all)
            runs[threadIdx.x] = p.carry[g * nruns + threadIdx.x];
        __syncthreads();

        const S* src = level + row.level_row * pitch + base;
        // fused level step: the row's op, its children's segments and the
        // offset of the shifted one inside its 16-byte-aligned superset
        constexpr int VEC  = 16 / static_cast<int>(sizeof(S));
        S* const fs_halo   = stage0;
        auto fs_lo         = [&](int b) { return stage0 + halo + b * (2 * CH + VEC); };
        auto fs_hi         = [&](int b) { return stage0 + halo + b * (2 * CH + VEC) + CH; };
        const S* lo_src    = nullptr;
        const S* hi_src    = nullptr;
        int hoff           = 0;
        uint32_t hi_bytes  = 0;
        if constexpr (FS) {
            const RowOp op      = SG.ops[g];
            const S* in         = static_cast<const S*>(SG.in);
            lo_src              = in + static_cast<int64_t>(op.lo_row) * SG.in_pitch + SG.in_base;
            const int64_t first = static_cast<int64_t>(SG.in_base) - op.shift;
            hoff                = static_cast<int>(((first % VEC) + VEC) % VEC);
            if (op.hi_row >= 0) {
                hi_src   = in + static_cast<int64_t>(op.hi_row) * SG.in_pitch + (first - hoff);
                hi_bytes = static_cast<uint32_t>((CH / VEC + (hoff > 0 ? 1 : 0)) * 16);
            }
        }
        auto issue_fs = [&](int ci) {
            const int b    = static_cast<int>((cc + ci) & 1); // barrier
            const int sb   = FSB == 2 ? b : 0;                  // staging buffers
            uint32_t bytes = static_cast<uint32_t>(CH * sizeof(S)) + hi_bytes;
            if (ci == 0)
                bytes += static_cast<uint32_t>(halo * sizeof(S));
            bulk::mbar_expect(&bar[b], bytes);
            if (ci == 0)
                bulk::load(fs_halo, src - halo, static_cast<uint32_t>(halo * sizeof(S)), &bar[b]);
            bulk::load(fs_lo(sb), lo_src + static_cast<int64_t>(ci) * CH, static_cast<uint32_t>(CH * sizeof(S)),
                       &bar[b]);
            if (hi_bytes != 0)
                bulk::load(fs_hi(sb), hi_src + static_cast<int64_t>(ci) * CH, hi_bytes, &bar[b]);
            // the chunk staged next after those in flight is fetched into L2 meanwhile
            if (ci + FSB < nchunks) {
                bulk::prefetch_l2(lo_src + static_cast<int64_t>(ci + FSB) * CH, static_cast<uint32_t>(CH * sizeof(S)));
                if (hi_bytes != 0)
                    bulk::prefetch_l2(hi_src + static_cast<int64_t>(ci + FSB) * CH, hi_bytes);
            }
        };
        auto issue = [&](int ci) {
            const int b          = static_cast<int>((cc + ci) & 1);
            const int off        = (ci == 0 || !carry_halo) ? 0 : halo;
            const uint32_t bytes = static_cast<uint32_t>((seg_cols - off) * sizeof(S));
            bulk::mbar_expect(&bar[b], bytes);
            bulk::load(stage0 + b * seg_cols + off, src + static_cast<int64_t>(ci) * CH - halo + off, bytes, &bar[b]);
            // two buffers hold one chunk in flight: the chunk staged two
            // issues later is fetched into L2 meanwhile (the same columns its
            // copy reads), so that copy waits for L2, not HBM
            if (ci + 2 < nchunks)
                bulk::prefetch_l2(src + static_cast<int64_t>(ci + 2) * CH, static_cast<uint32_t>(CH * sizeof(S)));
        };
        if (threadIdx.x == 0) {
            if constexpr (FS) {
                for (int ci = 0; ci < min(FSB, nchunks); ++ci)
                    issue_fs(ci);
            } else {
                for (int ci = 0; ci < min(2, nchunks); ++ci)
                    issue(ci);
            }
        }
        const int jmin     = halo - wmax + 1; // earlier columns never enter a window
        const int64_t warm = static_cast<int64_t>(row.delay) + wmax - 1;
        auto close_runs = [&]() {
            // nothing fired: runs open at the chunk start close here
            if (!all && threadIdx.x < nruns && runs[threadIdx.x].open) {
                emit(p, row, runs[threadIdx.x], &local_count);
                runs[threadIdx.x].open = 0;
            }
        };
        int ci = 0;
        for (int64_t c0 = 0; c0 < p.n_valid; c0 += CH, ++ci) {
            // ---- wait for the chunk's segment (bounded; a timeout ends the row)
            if (!bulk::mbar_wait(&bar[(cc + ci) & 1], static_cast<uint32_t>(((cc + ci) >> 1) & 1), p.wait_limit))
                atomicExch(&abort_flag, 1);
            __syncthreads();
            if (abort_flag)
                break;
            const S* seg           = FS ? fs_halo : stage0 + ((cc + ci) & 1) * seg_cols;
            const bool direct_halo = ci == 0 || !carry_halo;
            if (direct_halo)
                scan_halo<S, P>(seg, halo, jmin, Q, gmin, tmin);
            // ---- prefix sums of the thread's P columns: serial, then across the
            // warp (shuffles), then across warps (one offset per warp)
            float q[P];
            float xmax; // the thread's largest sample
            if constexpr (FS) {
                const int b = FSB == 2 ? static_cast<int>((cc + ci) & 1) : 0;
                merge_scan<S, P>(fs_lo(b) + P * threadIdx.x, hi_bytes != 0 ? fs_hi(b) + P * threadIdx.x : nullptr,
                                 hoff, const_cast<S*>(src) + c0 + P * threadIdx.x, q, xmax);
            }
            else
                scan_cols<S, P>(seg + halo + P * threadIdx.x, q, xmax);
            float incl = q[P - 1];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const float u = __shfl_up_sync(0xFFFFFFFFU, incl, o);
                if (lane >= o)
                    incl += u;
            }
            float excl = __shfl_up_sync(0xFFFFFFFFU, incl, 1);
            if (lane == 0)
                excl = 0.0F;
            if (lane == 31)
                warp_tot[warp] = incl;
            __syncthreads();
            // every thread has read this chunk's staging buffer: refill it
            if constexpr (FS) {
                if (threadIdx.x == 0 && ci + FSB < nchunks)
                    issue_fs(ci + FSB);
            } else {
                if (threadIdx.x == 0 && ci + 2 < nchunks)
                    issue(ci + 2);
            }
            // the totals of the warps before this one, in warp order (the
            // later terms add +0, which leaves the sum's bits unchanged)
            const float4 ta = reinterpret_cast<const float4*>(warp_tot)[0];
            const float4 tb = reinterpret_cast<const float4*>(warp_tot)[1];
            const float tw[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
            float woff        = 0.0F;
#pragma unroll
            for (int w = 0; w < kThreads / 32 - 1; ++w)
                woff += w < warp ? tw[w] : 0.0F;
            const float off = excl + woff;
            add_offset<P>(q, off);
            // ---- group and block extremes (registers; the minima to shared memory)
            float gmx[NG], gmn[NG];
#pragma unroll
            for (int gq = 0; gq < NG; ++gq) {
                gmx[gq] = fmaxf(fmax3(q[4 * gq], q[4 * gq + 1], q[4 * gq + 2]), q[4 * gq + 3]);
                gmn[gq] = fminf(fmin3(q[4 * gq], q[4 * gq + 1], q[4 * gq + 2]), q[4 * gq + 3]);
            }
            float bmax, bmin;
            if constexpr (NG == 4) {
                bmax = fmaxf(fmax3(gmx[0], gmx[1], gmx[2]), gmx[3]);
                bmin = fminf(fmin3(gmn[0], gmn[1], gmn[2]), gmn[3]);
            } else {
                bmax = fmaxf(gmx[0], gmx[1]);
                bmin = fminf(gmn[0], gmn[1]);
            }
            if constexpr (NG == 4)
                reinterpret_cast<float4*>(gmin + halo / 4)[threadIdx.x] = make_float4(gmn[0], gmn[1], gmn[2], gmn[3]);
            else
                reinterpret_cast<float2*>(gmin + halo / 4)[threadIdx.x] = make_float2(gmn[0], gmn[1]);
            tmin[halo / P + threadIdx.x] = bmin;
            if (lane == 31) {
                wtail[warp][0] = q[P - 2];
                wtail[warp][1] = q[P - 1];
            }
            if (carry_halo) {
                // the next chunk's halo: this chunk's last `halo` columns
                float* nh    = nh0 + (ci & 1) * nh_len;
                const int tt = static_cast<int>(threadIdx.x) - (kThreads - halo / P);
                if (tt >= 0) {
                    float4* d = reinterpret_cast<float4*>(nh + P * tt);
#pragma unroll
                    for (int i = 0; i < P / 4; ++i)
                        d[i] = make_float4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
#pragma unroll
                    for (int gq = 0; gq < NG; ++gq)
                        nh[halo + NG * tt + gq] = gmn[gq];
                    nh[halo + halo / 4 + tt] = bmin;
                    if (threadIdx.x == kThreads - 1)
                        nh[halo + halo / 4 + halo / P] = q[P - 1];
                }
                if (!direct_halo) {
                    // this chunk's halo from the previous chunk's, rebased so
                    // that Q[-1] = 0: the group and thread minima and Q[-2],
                    // Q[-1] now (the bound tests read them); the halo's other
                    // prefix sums only when Q is stored (store_q)
                    const float* ph  = nh0 + ((ci - 1) & 1) * nh_len;
                    const int n      = halo / 4 + halo / P;
                    const float last = ph[halo + n];
                    for (int i = threadIdx.x; i < n + 2; i += kThreads) {
                        if (i < halo / 4)
                            gmin[i] = ph[halo + i] - last;
                        else if (i < n)
                            tmin[i - halo / 4] = ph[halo + i] - last;
                        else
                            Q[i - n - 2] = ph[halo + i - n - 2] - last;
                    }
                }
            }
            __syncthreads();

            auto store_q = [&]() {
                float4* d = reinterpret_cast<float4*>(Q + P * threadIdx.x);
#pragma unroll
                for (int i = 0; i < P / 4; ++i)
                    d[i] = make_float4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
                if (carry_halo && !direct_halo) {
                    // the rest of the halo's prefix sums, rebased (Q[-2], Q[-1] are)
                    const float* ph  = nh0 + ((ci - 1) & 1) * nh_len;
                    const float last = ph[halo + halo / 4 + halo / P];
                    for (int i = threadIdx.x; i < halo - 2; i += kThreads)
                        Q[i - halo] = ph[i] - last;
                }
                for (int i = threadIdx.x; i < nw * (CH / 32); i += kThreads)
                    bits[i] = 0U;
                if (threadIdx.x == 0)
                    fired_w = 0U;
            };
            const bool fast = c0 + CH <= p.n_valid && (!p.skip_cold || rc.tile_t0 + c0 >= warm) &&
                              (!rc.or_active || rc.tile_t0 + c0 - rc.gulp_t0 >= warm);
            if (fast) {
                // ---- steady state. A window sum Q[k] - Q[k - W] of a set of
                // samples is at most their greatest Q minus the least Q their
                // windows start from (rounding is monotonic), so a set the bound
                // clears cannot fire. Widths 1 and 2 take the exact sums in
                // registers, the others a bound per 4-sample group (wide boxcars
                // first one per thread); only a chunk where some test may fire
                // stores Q and runs the exact tests.
                float pm1 = __shfl_up_sync(0xFFFFFFFFU, q[P - 1], 1); // Q[P t - 1]
                float pm2 = __shfl_up_sync(0xFFFFFFFFU, q[P - 2], 1); // Q[P t - 2]
                if (lane == 0) {
                    pm1 = warp == 0 ? Q[-1] : wtail[warp - 1][1];
                    pm2 = warp == 0 ? Q[-2] : wtail[warp - 1][0];
                }
                uint32_t cand = 0U;
                if constexpr (POW2) {
                    // A width-1 window sum Q[k] - Q[k-1] inside the thread's
                    // samples (k >= 1) differs from the sample x[k] by four
                    // roundings (the local prefix, the offset twice, the
                    // difference), each at most 2^-24 of a magnitude below
                    // max|Q| + |off| (Q within [bmin, bmax]): 2^-20 of that
                    // bounds their sum. The first sample's sum reaches back
                    // into the previous thread's prefix (the block scan's own
                    // rounding) and is taken exactly.
                    const float qmag = fmaxf(fabsf(bmax), fabsf(bmin)) + fabsf(off);
                    float m1         = fmaxf(xmax + qmag * 0x1p-20F, q[0] - pm1);
                    pow2_range<P, NG, 0, kMaxPow2Widths>(cand, q, pm1, pm2, gmx, bmax, gmin, tmin, halo, wt, nw, m1);
                }
                else {
                    for (int wi = 0; wi < nw; ++wi) {
                        const WidthTest t = wt[wi];
                        bool maybe        = true;
                        if (t.kind == kTestExact) {
                            float m;
                            if (t.W == 1) {
                                m = q[0] - pm1;
#pragma unroll
                                for (int e = 1; e < P; ++e)
                                    m = fmaxf(m, q[e] - q[e - 1]);
                            } else {
                                m = fmaxf(q[0] - pm2, q[1] - pm1);
#pragma unroll
                                for (int e = 2; e < P; ++e)
                                    m = fmaxf(m, q[e] - q[e - 2]);
                            }
                            maybe = m > t.T;
                        } else if (t.kind != kTestAll) {
                            if (t.kind == kTestBlock) {
                                const int b = static_cast<int>(threadIdx.x) + t.bconst;
                                float lo    = tmin[b];
                                if (t.btwo)
                                    lo = fminf(lo, tmin[b + 1]);
                                maybe = bmax - lo > t.T;
                            }
                            if (maybe) {
                                float lo[NG];
                                group_lows<NG>(gmin, NG * static_cast<int>(threadIdx.x) + t.gconst, t.two != 0, lo);
                                float m = gmx[0] - lo[0];
#pragma unroll
                                for (int gq = 1; gq < NG; ++gq)
                                    m = fmaxf(m, gmx[gq] - lo[gq]);
                                maybe = m > t.T;
                            }
                        }
                        if (maybe)
                            cand |= 1U << wi;
                    }
                }
                if (!__syncthreads_or(cand != 0U)) {
                    close_runs();
                    continue; // shared memory is rewritten only after every thread passed the barrier
                }
                store_q();
                __syncthreads();
                bool up = false;
                // the exact test of group gi at width wi (sets the fired bits)
                auto exact = [&](int gi, int wi, int W, int E, float T) {
                    const int k    = 4 * gi;
                    const float4 a = *reinterpret_cast<const float4*>(Q + k);
                    const float4 b = ld4(Q, k - W);
                    float s0, s1, s2, s3;
                    if (E > 0) {
                        const float4 c = ld4(Q, k - E);
                        const float4 d = ld4(Q, k - W + E);
                        s0 = trap_sum(a.x, b.x, c.x, d.x);
                        s1 = trap_sum(a.y, b.y, c.y, d.y);
                        s2 = trap_sum(a.z, b.z, c.z, d.z);
                        s3 = trap_sum(a.w, b.w, c.w, d.w);
                    } else {
                        s0 = a.x - b.x;
                        s1 = a.y - b.y;
                        s2 = a.z - b.z;
                        s3 = a.w - b.w;
                    }
                    const uint32_t nib = (s0 > T ? 1U : 0U) | (s1 > T ? 2U : 0U) | (s2 > T ? 4U : 0U) |
                                         (s3 > T ? 8U : 0U);
                    if (nib != 0U) {
                        // samples 4 gi .. 4 gi + 3: word gi / 8, nibble gi % 8
                        atomicOr(&bits[wi * (CH / 32) + (gi >> 3)], nib << ((gi & 7) * 4));
                        atomicOr(&fired_w, 1U << wi);
                        up = true;
                    }
                };
                for (uint32_t c = cand; c != 0U; c &= c - 1U) {
                    const int wi      = __ffs(static_cast<int>(c)) - 1;
                    const WidthTest t = wt[wi];
                    const int E       = rc.E[wi];
                    if (t.kind == kTestGroup || t.kind == kTestBlock) {
                        float lo[NG];
                        group_lows<NG>(gmin, NG * static_cast<int>(threadIdx.x) + t.gconst, t.two != 0, lo);
#pragma unroll
                        for (int gq = 0; gq < NG; ++gq)
                            if (gmx[gq] - lo[gq] > t.T)
                                exact(NG * static_cast<int>(threadIdx.x) + gq, wi, t.W, E, t.T);
                    } else {
#pragma unroll
                        for (int gq = 0; gq < NG; ++gq)
                            exact(NG * static_cast<int>(threadIdx.x) + gq, wi, t.W, E, t.T);
                    }
                }
                if (!__syncthreads_or(up)) {
                    close_runs();
                    continue;
                }
            } else {
                // ---- not steady (cold prefix, mask change, partial chunk): the
                // bit masks from the general S/N
                store_q();
                __syncthreads();
                for (int j = 0; j < (CH / kThreads); ++j) {
                    const int k = threadIdx.x + j * kThreads;
                    for (int wi = 0; wi < nw; ++wi) {
                        const bool hit   = snr_general(p, rc, Q, c0, k, wi, row.delay) > p.thresh;
                        const uint32_t m = __ballot_sync(0xFFFFFFFFU, hit);
                        if (lane == 0) {
                            bits[wi * (CH / 32) + j * (kThreads / 32) + warp] = m;
                            if (m != 0U)
                                atomicOr(&fired_w, 1U << wi);
                        }
                    }
                }
                __syncthreads();
            }
            // bits now hold exactly the above-threshold samples of every width
            const uint32_t fw = fired_w;
            if (across) {
                for (int wd = threadIdx.x; wd < (CH / 32); wd += kThreads) {
                    uint32_t m = 0;
                    for (int wi = 0; wi < nw; ++wi)
                        if ((fw >> wi) & 1U)
                            m |= bits[wi * (CH / 32) + wd];
                    any_bits[wd] = m;
                }
                __syncthreads();
            }
            // Widths are independent (each has its own run state): warp w
            // walks widths w, w + 8, ..., its lanes over the chunk's samples.
            // Candidates may therefore reach the output in any order (results
            // are sorted afterwards; only which ones a per-DM cap drops can
            // vary).
            if (all) {
                for (int wi = warp; wi < nw; wi += kThreads / 32) {
                    if (((fw >> wi) & 1U) == 0U)
                        continue;
                    for (int wd = lane; wd < (CH / 32); wd += 32) {
                        uint32_t m = bits[wi * (CH / 32) + wd];
                        while (m) {
                            const int k = wd * 32 + __ffs(m) - 1;
                            m &= m - 1;
                            RunState r{};
                            r.best   = snr_general(p, rc, Q, c0, k, wi, row.delay);
                            r.best_w = wi;
                            r.start = r.best_t = r.last_t = rc.tile_t0 + c0 + k;
                            emit(p, row, r, &local_count);
                        }
                    }
                }
            } else if (!across) {
                for (int wi = warp; wi < nw; wi += kThreads / 32)
                    if (((fw >> wi) & 1U) != 0U || runs[wi].open)
                        walk_runs_warp<CH>(p, rc, Q, c0, row.delay, bits + wi * (CH / 32), wi, runs[wi], row,
                                           &local_count);
            }
            if (across && warp == 0 && (fw != 0U || runs[0].open))
                walk_runs_warp<CH>(p, rc, Q, c0, row.delay, any_bits, -1, runs[0], row, &local_count);
            __syncthreads();
        }
        if (abort_flag) {
            // a segment never landed: report it and let the copies in flight end
            if (threadIdx.x == 0) {
                atomicOr(p.err, 1U);
                for (int j = ci; j < min(ci + (FSB == 1 ? 1 : 2), nchunks); ++j)
                    (void)bulk::mbar_wait(&bar[(cc + j) & 1], static_cast<uint32_t>(((cc + j) >> 1) & 1));
            }
            return;
        }
        if (threadIdx.x < nruns && !all)
            p.carry[g * nruns + threadIdx.x] = runs[threadIdx.x];
        if (threadIdx.x == 0)
            p.row_counts[g] = local_count;
        cc += nchunks;
        __syncthreads(); // the next row rewrites the row constants and run states
    }
}

__global__ void k_flush(SearchParams p, int64_t nrows) {
    const int64_t g = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (g >= nrows)
        return;
    const int nruns     = p.peak_mode == FROST_PEAK_ACROSS_WIDTHS ? 1 : p.nwidths;
    const SearchRow row = p.rows[g];
    for (int i = 0; i < nruns; ++i) {
        RunState& r = p.carry[g * nruns + i];
        if (r.open) {
            emit(p, row, r, &p.row_counts[g]);
            r.open = 0;
        }
    }
}

// Noise tables: for every searched row and width, the sum over the row's
// channels of the boxcar variance of a channel's leaf run (masked and
// OR-masked). A warp per row: the lanes take every 32nd channel, each
// accumulates its share of the sums of eight widths at a time, and the warp
// adds the lanes' sums by a butterfly (the same terms as a sequential sum in
// another order: within a few ulp of it).
__global__ void __launch_bounds__(256)
    k_variance_warp(const SearchRow* __restrict__ rows, const PlaneInfo* __restrict__ planes,
                    const int64_t* __restrict__ leaf_offset, const uint16_t* __restrict__ leaf_len, int64_t nrows,
                    const double* __restrict__ gtab, int32_t max_len, int32_t nw,
                    const uint8_t* __restrict__ mask, const uint8_t* __restrict__ mask_or,
                    double* __restrict__ var, float* __restrict__ inv, float* __restrict__ inv_or) {
    const int lane  = threadIdx.x & 31;
    const int64_t g = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (g >= nrows)
        return; // the whole warp
    const SearchRow r   = rows[g];
    const PlaneInfo pl  = planes[r.plane];
    const int32_t nch   = static_cast<int32_t>(pl.chan_end - pl.chan_begin);
    const uint16_t* len = leaf_len + leaf_offset[g];
    constexpr int kW = 8;
    for (int w0 = 0; w0 < nw; w0 += kW) {
        double v[kW], vo[kW];
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            v[j]  = 0.0;
            vo[j] = 0.0;
        }
        for (int32_t c = lane; c < nch; c += 32) {
            const bool on   = mask[pl.chan_begin + c] != 0;
            const bool on_o = mask_or[pl.chan_begin + c] != 0;
            if (!on && !on_o)
                continue;
            const int L      = min(static_cast<int>(len[c]), max_len);
            const double* gt = gtab + static_cast<int64_t>(L) * nw + w0;
#pragma unroll
            for (int j = 0; j < kW; ++j) {
                if (w0 + j < nw) {
                    const double x = gt[j];
                    if (on)
                        v[j] += x;
                    if (on_o)
                        vo[j] += x;
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            for (int o = 16; o > 0; o >>= 1) {
                v[j] += __shfl_xor_sync(0xFFFFFFFFU, v[j], o);
                vo[j] += __shfl_xor_sync(0xFFFFFFFFU, vo[j], o);
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < kW; ++j) {
                const int w = w0 + j;
                if (w < nw) {
                    var[g * nw + w]    = v[j];
                    inv[g * nw + w]    = v[j] > 0.0 ? static_cast<float>(1.0 / sqrt(v[j])) : 0.0F;
                    inv_or[g * nw + w] = vo[j] > 0.0 ? static_cast<float>(1.0 / sqrt(vo[j])) : 0.0F;
                }
            }
        }
    }
}

} // namespace

namespace {

void check_search(const SearchParams& p, int64_t pitch, int32_t base, int32_t chunk) {
    if (p.nwidths > kMaxWidths)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "search: more than 32 boxcar widths");
    if (p.halo != search_halo(p.wmax) || base < p.halo)
        throw Error(FROST_ERR_INTERNAL, "search: level history shorter than the search halo");
    if (pitch - base < ((p.n_valid + chunk - 1) / chunk) * chunk)
        throw Error(FROST_ERR_INTERNAL, "search: tile columns are not a whole number of chunks");
    if (p.err == nullptr)
        throw Error(FROST_ERR_INTERNAL, "search: no error flag");
    if (p.wait_limit < 0)
        throw Error(FROST_ERR_INTERNAL, "search: wait limit must be >= 0");
}

bool same_shape(const SearchParams& a, const SearchParams& b) {
    return a.nwidths == b.nwidths && a.wmax == b.wmax && a.halo == b.halo && a.peak_mode == b.peak_mode &&
           a.trapezoid == b.trapezoid && a.skip_cold == b.skip_cold && a.pow2_widths == b.pow2_widths &&
           a.n_valid == b.n_valid;
}

template <int K>
void search_table(SearchSeg* segs, int n, cudaStream_t s, int32_t chunk, int32_t ctas) {
    SearchSegTable<K> t{};
    t.n            = n;
    int64_t rows   = 0;
    const auto& p0 = segs[0].p;
    const bool fs  = segs[0].in != nullptr;
    const int fsb  = segs[0].fs_buffers;
    for (int i = 0; i < n; ++i) {
        SearchSeg& g = segs[i];
        check_search(g.p, g.pitch, g.base, chunk);
        if (!same_shape(g.p, p0) || g.fp16 != segs[0].fp16 || (g.in != nullptr) != fs || g.fs_buffers != fsb)
            throw Error(FROST_ERR_INTERNAL, "search: segments of one launch differ in shape");
        if (fs && (K != 1 || g.ops == nullptr || (fsb != 1 && fsb != 2) || g.p.halo > chunk || g.in_base % 8 != 0 || g.in_pitch % 8 != 0 ||
                   g.base % 8 != 0 || g.pitch % 8 != 0))
            throw Error(FROST_ERR_INTERNAL, "search: bad fused level step geometry");
        rows += g.nrows;
        g.row_end = rows;
        t.s[i]    = g;
    }
    const size_t es   = segs[0].fp16 ? 2 : 4;
    const size_t seg  = static_cast<size_t>(p0.halo) + chunk;
    // Ps, gmin (+4 padding), tmin, the next chunk's halo by parity, the bit
    // masks and the staging buffers (the kernel's layout)
    const size_t per  = static_cast<size_t>(chunk) / kThreads; // columns per thread
    const size_t nh   = static_cast<size_t>(p0.halo) + p0.halo / 4 + p0.halo / per + 4;
    // staging: two raw row segments, or (fused level step) the halo and
    // two pairs of child segments
    const size_t stage_elems = fs ? p0.halo + fsb * (2 * static_cast<size_t>(chunk) + 16 / es) : 2 * seg;
    const size_t smem = sizeof(float) * ((4 + seg + 4) + (seg / 4 + 4) + seg / per + 2 * nh) +
                        sizeof(uint32_t) * search_bits_words(p0.nwidths, chunk) + es * stage_elems;
    const dim3 grid(static_cast<unsigned>(ctas > 0 ? std::min<int64_t>(rows, ctas) : rows));
    auto go = [&](auto kernel) {
        allow_large_smem(reinterpret_cast<const void*>(kernel));
        kernel<<<grid, kThreads, smem, s>>>(t);
    };
    // widths 1, 2, 4, ... (no trapezoid): the unrolled steady-state tests
    const bool pow2 = p0.pow2_widths != 0 && !p0.trapezoid && p0.nwidths <= kMaxPow2Widths;
    auto typed = [&](auto tag) {
        using S = decltype(tag);
        if constexpr (K == 1) {
            if (fs && fsb == 1) {
                if (chunk == 2048)
                    pow2 ? go(k_search<S, 2048, true, 1, K>) : go(k_search<S, 2048, false, 1, K>);
                else
                    pow2 ? go(k_search<S, 4096, true, 1, K>) : go(k_search<S, 4096, false, 1, K>);
                return;
            }
            if (fs) {
                if (chunk == 2048)
                    pow2 ? go(k_search<S, 2048, true, 2, K>) : go(k_search<S, 2048, false, 2, K>);
                else
                    pow2 ? go(k_search<S, 4096, true, 2, K>) : go(k_search<S, 4096, false, 2, K>);
                return;
            }
        }
        if (chunk == 2048)
            pow2 ? go(k_search<S, 2048, true, 0, K>) : go(k_search<S, 2048, false, 0, K>);
        else
            pow2 ? go(k_search<S, 4096, true, 0, K>) : go(k_search<S, 4096, false, 0, K>);
    };
    if (segs[0].fp16)
        typed(__half{});
    else
        typed(float{});
    FB_LAUNCH_CHECK();
}

} // namespace

void launch_search_segs(SearchSeg* segs, int n, cudaStream_t s, int32_t chunk, int32_t ctas) {
    if (chunk != 2048 && chunk != 4096)
        throw Error(FROST_ERR_INTERNAL, "search: chunk must be 2048 or 4096 samples");
    // segments without rows or valid columns launch nothing
    int m = 0;
    for (int i = 0; i < n; ++i)
        if (segs[i].nrows > 0 && segs[i].p.n_valid > 0)
            segs[m++] = segs[i];
    if (m == 0)
        return;
    if (m == 1) {
        search_table<1>(segs, 1, s, chunk, ctas);
        return;
    }
    for (int i = 0; i < m; i += kMaxSearchSegs)
        search_table<kMaxSearchSegs>(segs + i, std::min(kMaxSearchSegs, m - i), s, chunk, ctas);
}

void launch_search(const SearchParams& p, LevelView level, int64_t g0, int64_t g1, cudaStream_t s,
                   int32_t chunk, int32_t ctas) {
    if (g1 <= g0 || p.n_valid <= 0)
        return;
    SearchSeg g{};
    g.p     = p;
    g.level = level.data;
    g.pitch = level.pitch;
    g.base  = level.base;
    g.fp16  = level.fp16;
    g.g0    = g0;
    g.nrows = g1 - g0;
    launch_search_segs(&g, 1, s, chunk, ctas);
}

void launch_search_fused(const SearchParams& p, LevelView in, LevelView level, const RowOp* ops, int64_t g0,
                         int64_t g1, cudaStream_t s, int32_t chunk, int32_t ctas, int32_t buffers) {
    if (g1 <= g0 || p.n_valid <= 0)
        return;
    if (in.fp16 != level.fp16)
        throw Error(FROST_ERR_INTERNAL, "search: fused level step between storage types");
    SearchSeg g{};
    g.p        = p;
    g.level    = level.data;
    g.pitch    = level.pitch;
    g.base     = level.base;
    g.fp16     = level.fp16;
    g.g0       = g0;
    g.nrows    = g1 - g0;
    g.in       = in.data;
    g.in_pitch = in.pitch;
    g.in_base  = in.base;
    g.ops        = ops;
    g.fs_buffers = buffers;
    launch_search_segs(&g, 1, s, chunk, ctas);
}

void launch_variance(const SearchRow* rows, const PlaneInfo* planes, const int64_t* leaf_offset,
                     const uint16_t* leaf_len, int64_t nrows, const double* gtab, int32_t max_len,
                     int32_t nwidths, const uint8_t* mask, const uint8_t* mask_or, double* var,
                     float* inv_sigma, float* inv_sigma_or, cudaStream_t s) {
    if (nrows == 0)
        return;
    if (nwidths > kMaxWidths)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "variance: more than 32 boxcar widths");
    k_variance_warp<<<static_cast<unsigned>((nrows + 7) / 8), 256, 0, s>>>(
        rows, planes, leaf_offset, leaf_len, nrows, gtab, max_len, nwidths, mask, mask_or, var,
        inv_sigma, inv_sigma_or);
    FB_LAUNCH_CHECK();
}

void launch_flush_runs(const SearchParams& p, int64_t nrows, cudaStream_t s) {
    if (nrows == 0 || p.peak_mode == FROST_PEAK_ALL)
        return;
    k_flush<<<static_cast<unsigned>((nrows + 127) / 128), 128, 0, s>>>(p, nrows);
    FB_LAUNCH_CHECK();
}

// ---- candidate ordering ------------------------------------------------------
//
// The search kernels append detections in whatever order their CTAs reach
// them; results are returned sorted by (sub-band level, sub-band, DM row,
// peak sample, width). The five fields pack into one 64-bit key (field
// widths from the plan, the peak relative to the smallest peak of the
// call), so the order is a stable radix sort of the keys followed by a
// gather.

namespace {

__global__ void __launch_bounds__(256)
    k_cand_range(const frost_candidate* __restrict__ c, const unsigned long long* __restrict__ count,
                 uint64_t cap, unsigned long long* __restrict__ range) {
    const uint64_t n = min(static_cast<uint64_t>(*count), cap);
    unsigned long long lo = ~0ULL, hi = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const unsigned long long p = c[i].peak_sample;
        lo = p < lo ? p : lo;
        hi = p > hi ? p : hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long l2 = __shfl_xor_sync(0xFFFFFFFFU, lo, o);
        const unsigned long long h2 = __shfl_xor_sync(0xFFFFFFFFU, hi, o);
        lo = l2 < lo ? l2 : lo;
        hi = h2 > hi ? h2 : hi;
    }
    __shared__ unsigned long long s_lo[8], s_hi[8];
    const int warp = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_lo[warp] = lo;
        s_hi[warp] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) {
            lo = s_lo[w] < lo ? s_lo[w] : lo;
            hi = s_hi[w] > hi ? s_hi[w] : hi;
        }
        if (lo <= hi) {
            atomicMin(&range[0], lo);
            atomicMax(&range[1], hi);
        }
    }
}

__global__ void k_cand_keys(const frost_candidate* __restrict__ c, uint64_t n, CandKeySpec k,
                            uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= n)
        return;
    const frost_candidate& x = c[i];
    uint64_t key             = x.subband_level;
    key                      = (key << k.idx_bits) | x.subband_idx;
    key                      = (key << k.dm_bits) | x.dm_idx;
    key                      = (key << k.peak_bits) | (x.peak_sample - k.peak_base);
    key                      = (key << k.filter_bits) | x.filter_idx;
    keys[i]                  = key;
    idx[i]                   = static_cast<uint32_t>(i);
}

__global__ void k_cand_gather(const frost_candidate* __restrict__ c, const uint32_t* __restrict__ perm,
                              uint64_t n, frost_candidate* __restrict__ out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        out[i] = c[perm[i]];
}

unsigned blocks256(uint64_t n) { return static_cast<unsigned>((n + 255) / 256); }

} // namespace

void launch_cand_range(const frost_candidate* c, const unsigned long long* count, uint64_t cap,
                       unsigned long long* range, cudaStream_t s) {
    FB_CUDA(cudaMemsetAsync(range, 0xFF, sizeof(unsigned long long), s));
    FB_CUDA(cudaMemsetAsync(range + 1, 0, sizeof(unsigned long long), s));
    const uint64_t grid = std::min<uint64_t>(blocks256(cap), 4 * 148);
    k_cand_range<<<static_cast<unsigned>(grid), 256, 0, s>>>(c, count, cap, range);
    FB_LAUNCH_CHECK();
}

void launch_cand_keys(const frost_candidate* c, uint64_t n, const CandKeySpec& k, uint64_t* keys,
                      uint32_t* idx, cudaStream_t s) {
    if (n == 0)
        return;
    k_cand_keys<<<blocks256(n), 256, 0, s>>>(c, n, k, keys, idx);
    FB_LAUNCH_CHECK();
}

void launch_cand_gather(const frost_candidate* c, const uint32_t* perm, uint64_t n, frost_candidate* out,
                        cudaStream_t s) {
    if (n == 0)
        return;
    k_cand_gather<<<blocks256(n), 256, 0, s>>>(c, perm, n, out);
    FB_LAUNCH_CHECK();
}

} // namespace fb::fdmt
