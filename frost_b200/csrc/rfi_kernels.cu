// RFI excision kernels for sm_100a.
//
// The cleaner's decisions (masks, time flags, cell states) must agree bit for
// bit with frost's CPU cleaner, so every threshold-deciding sum keeps the
// reference's summation order: per (window, channel) over time for the
// bandpass refinement, moments and Welford statistics; per row over channels
// for the detection series; per (chunk, channel) over time for zdot and
// Kadane-along-time. Parallelism comes from the many independent
// (window, channel), row and (chunk, channel) sequences instead of from
// splitting any one of them. This file is compiled with --fmad=false so no
// multiply-add is contracted and each float/double operation rounds exactly
// as the IEEE host build does.
//
// Packed samples are decoded on the fly from the raw time-major block (LSB
// first below 8 bits, lib/prepare/sample_codec.hpp:18-109), so the 1/4-byte
// raw block is what every statistics pass reads from HBM.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cstdint>
#include <cstring>
#include <type_traits>

#include <cuda_runtime.h>

#include "common.hpp"
#include "rfi_kernels.hpp"
#include "rfi_stage.cuh"

namespace fb::rfi {

namespace {

// ---- sample decoding --------------------------------------------------

template <int D> __device__ __forceinline__ float rd(const uint8_t* __restrict__ row, uint64_t c) {
    if constexpr (D == FROST_UINT8) {
        return static_cast<float>(row[c]);
    } else if constexpr (D == FROST_UINT16) {
        return static_cast<float>(reinterpret_cast<const uint16_t*>(row)[c]);
    } else if constexpr (D == FROST_UINT32) {
        return static_cast<float>(reinterpret_cast<const uint32_t*>(row)[c]);
    } else if constexpr (D == FROST_FLOAT32) {
        return reinterpret_cast<const float*>(row)[c];
    } else {
        constexpr unsigned kBits = D == FROST_UINT1 ? 1U : D == FROST_UINT2 ? 2U : 4U;
        constexpr unsigned kMask = (1U << kBits) - 1U;
        const uint64_t bit       = c * kBits;
        return static_cast<float>((row[bit >> 3U] >> (bit & 7U)) & kMask);
    }
}

// The integer code of sample c of an integer dtype D (rd<D> is its float).
template <int D> __device__ __forceinline__ uint32_t rdi(const uint8_t* __restrict__ row, uint64_t c) {
    if constexpr (D == FROST_UINT8) {
        return row[c];
    } else if constexpr (D == FROST_UINT16) {
        return reinterpret_cast<const uint16_t*>(row)[c];
    } else if constexpr (D == FROST_UINT32) {
        return reinterpret_cast<const uint32_t*>(row)[c];
    } else {
        static_assert(D != FROST_FLOAT32, "rdi: integer dtypes only");
        constexpr unsigned kBits = D == FROST_UINT1 ? 1U : D == FROST_UINT2 ? 2U : 4U;
        constexpr unsigned kMask = (1U << kBits) - 1U;
        const uint64_t bit       = c * kBits;
        return (row[bit >> 3U] >> (bit & 7U)) & kMask;
    }
}

// Bits per packed sample of dtype D (usable in device code).
template <int D>
constexpr uint64_t kBitsOf = D == FROST_UINT1 ? 1 : D == FROST_UINT2 ? 2 : D == FROST_UINT4 ? 4
                           : D == FROST_UINT8 ? 8 : D == FROST_UINT16 ? 16 : 32;

#define FB_DTYPE_CASE(DT, ...)                                                                    \
    case DT: {                                                                                    \
        constexpr int D = DT;                                                                     \
        __VA_ARGS__;                                                                              \
    } break;

#define FB_DISPATCH(dtype, ...)                                                                   \
    switch (dtype) {                                                                              \
        FB_DTYPE_CASE(FROST_UINT1, __VA_ARGS__)                                                   \
        FB_DTYPE_CASE(FROST_UINT2, __VA_ARGS__)                                                   \
        FB_DTYPE_CASE(FROST_UINT4, __VA_ARGS__)                                                   \
        FB_DTYPE_CASE(FROST_UINT8, __VA_ARGS__)                                                   \
        FB_DTYPE_CASE(FROST_UINT16, __VA_ARGS__)                                                  \
        FB_DTYPE_CASE(FROST_UINT32, __VA_ARGS__)                                                  \
        FB_DTYPE_CASE(FROST_FLOAT32, __VA_ARGS__)                                                 \
    default: throw ::fb::Error(FROST_ERR_INVALID_ARGUMENT, "unsupported dtype");                 \
    }

// Rows fetched ahead per thread in the time-ordered (window or chunk,
// channel) loops: the loads are independent, only the sums are sequential.
constexpr int kBlock = 16;

// Buffers of the per-window sequence kernels' staging: with one or two CTAs
// per SM, three stages in flight keep enough bytes moving for the chains.
constexpr int kDeepStages = 4;

// ---- order-exact helpers ------------------------------------------------

// std::min / std::max semantics (first argument kept on ties), which the
// remedian's median network relies on for bit-identical results.
template <class T> __device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }

__device__ __forceinline__ float median3(float a, float b, float c) {
    return a < b ? (b < c ? b : (a < c ? c : a)) : (a < c ? a : (b < c ? c : b));
}

// Median of five: drop the extremes of the first four, then the median of
// the remaining pair and the fifth value.
__device__ __forceinline__ float median5(float a, float b, float c, float d, float e) {
    const float f = smax(smin(a, b), smin(c, d));
    const float g = smin(smax(a, b), smax(c, d));
    return median3(e, f, g);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
    return (v < lo) ? lo : (hi < v) ? hi : v;
}

__device__ __forceinline__ uint64_t window_of(uint64_t t, uint64_t window, uint64_t nwin) {
    // a 32-bit division when both fit (a 64-bit one is a long software
    // sequence, paid per thread and row in the row-parallel kernels)
    const uint64_t w = (t | window) < (uint64_t{1} << 32)
                           ? static_cast<uint64_t>(static_cast<uint32_t>(t) / static_cast<uint32_t>(window))
                           : t / window;
    return w < nwin - 1 ? w : nwin - 1;
}

__device__ __forceinline__ uint64_t window_begin(uint64_t w, uint64_t window) { return w * window; }
__device__ __forceinline__ uint64_t window_end(uint64_t w, const Dims& d) {
    return w + 1 == d.nwin ? d.nsamps : (w + 1) * d.window;
}

__device__ __forceinline__ float normal_deviate(uint64_t h) {
    constexpr double kTwoPi = 6.283185307179586;
    const double u1         = uniform_open(h);
    const double u2         = uniform_open(splitmix64(h));
    return static_cast<float>(sqrt(-2.0 * log(u1)) * cos(kTwoPi * u2));
}

__device__ __forceinline__ uint64_t draw(const ApplyParams& p, uint64_t stream, uint64_t t,
                                         uint64_t c, uint64_t attempt) {
    return hash5(p.seed, p.block_index, (stream << 56U) ^ t, c, attempt);
}

// ---- finite check ---------------------------------------------------------

__global__ void k_check_finite(const uint32_t* __restrict__ w, uint64_t n,
                               unsigned long long* first_bad) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += stride) {
        if ((w[i] & 0x7F800000U) == 0x7F800000U)
            atomicMin(first_bad, static_cast<unsigned long long>(i));
    }
}

// ---- bandpass -------------------------------------------------------------

// The evenly spaced sample rows of each window (row i of window w is block
// row b + i * len / m, lib/cpu/spectra_cpu.cpp:96-104), decoded to float:
// one CTA per (row, window), its threads across the channels.
template <int D>
__global__ void k_sample_rows(Dims d, const uint8_t* __restrict__ raw, float* __restrict__ out) {
    const uint64_t i   = blockIdx.x;
    const uint64_t w   = blockIdx.y;
    const uint64_t b   = window_begin(w, d.window);
    const uint64_t len = window_end(w, d) - b;
    const uint64_t m   = largest_power_of_five_leq(len < kMaxBandpassRows ? len : kMaxBandpassRows);
    if (i >= m)
        return;
    const uint64_t t  = b + (i * len) / m;
    const uint8_t* in = raw + t * d.row_bytes;
    float* dst        = out + (w * kMaxBandpassRows + i) * d.nchans;
    for (uint64_t c = threadIdx.x; c < d.nchans; c += blockDim.x)
        dst[c] = rd<D>(in, c);
}

// Recursive median-of-5 over m = 5^k values streamed in order: the same
// groups of five, level by level, as the batch remedian in
// lib/cpu/spectra_cpu.cpp:43-69.
struct Remedian {
    float buf[5][5];
    int cnt[5];
    int depth;
    float result;

    __device__ void init(int levels) {
        depth = levels;
        for (int l = 0; l < 5; ++l)
            cnt[l] = 0;
        result = 0.0F;
    }
    __device__ void push(float x) {
        int l = 0;
        while (true) {
            if (l == depth) {
                result = x;
                return;
            }
            buf[l][cnt[l]++] = x;
            if (cnt[l] < 5)
                return;
            cnt[l] = 0;
            x      = median5(buf[l][0], buf[l][1], buf[l][2], buf[l][3], buf[l][4]);
            ++l;
        }
    }
};

__global__ void k_bandpass(Dims d, const float* __restrict__ samples, float* __restrict__ loc_out,
                           float* __restrict__ scale_out, float* __restrict__ inv_out,
                           uint32_t* __restrict__ unmeasured) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t w = blockIdx.y;
    if (c >= d.nchans)
        return;
    const uint64_t b   = window_begin(w, d.window);
    const uint64_t len = window_end(w, d) - b;
    const uint64_t m   = largest_power_of_five_leq(len < kMaxBandpassRows ? len : kMaxBandpassRows);
    int levels         = 0;
    for (uint64_t p = m; p > 1; p /= 5)
        ++levels;
    const uint64_t n = d.nchans;
    const float* v   = samples + w * kMaxBandpassRows * n + c;

    // Level: remedian over the sampled rows; scale: remedian of |x - level|
    // times 1.4826 (lib/cpu/spectra_cpu.cpp:73-130).
    Remedian r;
    r.init(levels);
    for (uint64_t i = 0; i < m; ++i)
        r.push(v[i * n]);
    const float level = r.result;
    r.init(levels);
    for (uint64_t i = 0; i < m; ++i)
        r.push(fabsf(v[i * n] - level));
    const float rms = r.result * kMadToStd;

    // Clipped refinement in double (lib/cpu/bandpass_kernels.hpp:17-76).
    float lo = v[0], hi = v[0];
    for (uint64_t i = 1; i < m; ++i) {
        lo = smin(lo, v[i * n]);
        hi = smax(hi, v[i * n]);
    }
    const uint64_t o = w * n + c;
    if (!(hi > lo)) {
        loc_out[o]   = lo;
        scale_out[o] = 0.0F;
        inv_out[o]   = 0.0F;
        atomicAdd(&unmeasured[c], 1U);
        return;
    }
    double centre = level;
    double s      = rms;
    const double dm = static_cast<double>(m);
    if (!(s > 0.0)) {
        double mean = 0.0;
        for (uint64_t i = 0; i < m; ++i)
            mean += v[i * n];
        mean /= dm;
        double ss = 0.0;
        for (uint64_t i = 0; i < m; ++i)
            ss += (v[i * n] - mean) * (v[i * n] - mean);
        s = sqrt(ss / dm);
    }
    for (int it = 0; it < kClipIterations; ++it) {
        const double cut = kClipSigma * s;
        double count = 0.0, sum = 0.0;
        for (uint64_t i = 0; i < m; ++i) {
            const double dv = v[i * n] - centre;
            if (fabs(dv) <= cut) {
                count += 1.0;
                sum += dv;
            }
        }
        if (count < 2.0)
            break;
        const double shift = sum / count;
        double ss          = 0.0;
        for (uint64_t i = 0; i < m; ++i) {
            const double dv = v[i * n] - centre;
            if (fabs(dv) <= cut)
                ss += (dv - shift) * (dv - shift);
        }
        const double clipped = sqrt(ss / count);
        if (!(clipped > 0.0))
            break;
        centre += shift;
        s = clipped;
    }
    const float fl = static_cast<float>(centre);
    const float fs = static_cast<float>(s);
    loc_out[o]     = fl;
    scale_out[o]   = fs;
    inv_out[o]     = 1.0F / fs;
}

// The remedian is a fixed tree (medians of five consecutive values, level by
// level), so its groups are independent: k_remedian evaluates it in
// parallel. One CTA covers 32 channels (a lane each) of one window; each
// warp reduces 125-row blocks (three tree levels in registers) to one value
// per channel, and warp 0 finishes the tree over the <= 25 block values.
// Pass 1 (ABS false) writes the level to loc and a flat flag (every sampled
// value of the channel compares equal) to inv; pass 2 (ABS true) the scale,
// remedian(|x - level|) x 1.4826, to scale (lib/cpu/spectra_cpu.cpp:73-130).
constexpr int kRemedianWarps = 8;

// The remedian of 25 values p[0], p[stride], ... (medians of five
// consecutive values, then their median): the 25 loads are issued together
// before any is used, then lo / hi track the range of the raw values.
template <bool ABS>
__device__ __forceinline__ float remedian25(const float* __restrict__ p, uint64_t stride, float level, float& lo,
                                            float& hi) {
    float x[25];
#pragma unroll
    for (int i = 0; i < 25; ++i)
        x[i] = p[i * stride];
    float v[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        float y[5];
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            const float r = x[5 * j + i];
            if constexpr (ABS) {
                y[i] = fabsf(r - level);
            } else {
                lo   = fminf(lo, r);
                hi   = fmaxf(hi, r);
                y[i] = r;
            }
        }
        v[j] = median5(y[0], y[1], y[2], y[3], y[4]);
    }
    return median5(v[0], v[1], v[2], v[3], v[4]);
}

template <bool ABS>
__device__ __forceinline__ float remedian5(const float* __restrict__ p, uint64_t stride, float level, float& lo,
                                           float& hi) {
    float y[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const float r = p[i * stride];
        if constexpr (ABS) {
            y[i] = fabsf(r - level);
        } else {
            lo   = fminf(lo, r);
            hi   = fmaxf(hi, r);
            y[i] = r;
        }
    }
    return median5(y[0], y[1], y[2], y[3], y[4]);
}

// 125 values: five 25-value subtrees in turn (25 loads in flight per lane),
// their results shifted through registers in order.
template <bool ABS>
__device__ __forceinline__ float remedian125(const float* __restrict__ p, uint64_t stride, float level, float& lo,
                                             float& hi) {
    float a = 0.0F, b = 0.0F, c = 0.0F, d = 0.0F, e = 0.0F;
#pragma unroll 1
    for (int j = 0; j < 5; ++j) {
        const float t = remedian25<ABS>(p + 25 * j * stride, stride, level, lo, hi);
        a = b;
        b = c;
        c = d;
        d = e;
        e = t;
    }
    return median5(a, b, c, d, e);
}

template <bool ABS>
__global__ void __launch_bounds__(32 * kRemedianWarps)
    k_remedian(Dims d, const float* __restrict__ samples, float* __restrict__ loc, float* __restrict__ scale,
               float* __restrict__ flat_out) {
    __shared__ float part[25][32];
    __shared__ float plo[kRemedianWarps][32], phi[kRemedianWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t n = d.nchans;
    const uint64_t c = static_cast<uint64_t>(blockIdx.x) * 32 + lane;
    const uint64_t w = blockIdx.y;
    const bool in    = c < n;
    const uint64_t len = window_end(w, d) - window_begin(w, d.window);
    const uint64_t m   = largest_power_of_five_leq(len < kMaxBandpassRows ? len : kMaxBandpassRows);
    int levels = 0;
    for (uint64_t q = m; q > 1; q /= 5)
        ++levels;
    const int kb       = levels < 3 ? levels : 3; // tree levels inside a block
    const int up       = levels - kb;             // levels over the blocks (0..2)
    const int nblk     = up == 0 ? 1 : up == 1 ? 5 : 25;
    const uint64_t blk = kb == 1 ? 5 : kb == 2 ? 25 : 125;
    const uint64_t o   = w * n + c;
    const float level  = (ABS && in) ? loc[o] : 0.0F;
    const float* src   = samples + w * kMaxBandpassRows * n + (in ? c : 0);
    float lo = FLT_MAX, hi = -FLT_MAX;
    for (int b = warp; b < nblk; b += kRemedianWarps) {
        const float* p = src + static_cast<uint64_t>(b) * blk * n;
        float v        = 0.0F;
        if (in) {
            switch (kb) {
            case 1: v = remedian5<ABS>(p, n, level, lo, hi); break;
            case 2: v = remedian25<ABS>(p, n, level, lo, hi); break;
            default: v = remedian125<ABS>(p, n, level, lo, hi); break;
            }
        }
        part[b][lane] = v;
    }
    if constexpr (!ABS) {
        plo[warp][lane] = lo;
        phi[warp][lane] = hi;
    }
    __syncthreads();
    if (warp != 0 || !in)
        return;
    float r;
    if (up == 0) {
        r = part[0][lane];
    } else if (up == 1) {
        r = median5(part[0][lane], part[1][lane], part[2][lane], part[3][lane], part[4][lane]);
    } else {
        float v[5];
#pragma unroll
        for (int j = 0; j < 5; ++j)
            v[j] = median5(part[5 * j][lane], part[5 * j + 1][lane], part[5 * j + 2][lane],
                           part[5 * j + 3][lane], part[5 * j + 4][lane]);
        r = median5(v[0], v[1], v[2], v[3], v[4]);
    }
    if constexpr (ABS) {
        scale[o] = r * kMadToStd;
    } else {
        float a = plo[0][lane], z = phi[0][lane];
#pragma unroll
        for (int k = 1; k < kRemedianWarps; ++k) {
            a = fminf(a, plo[k][lane]);
            z = fmaxf(z, phi[k][lane]);
        }
        loc[o]      = r;
        flat_out[o] = z > a ? 0.0F : 1.0F;
    }
}

// The clipped refinement of the bandpass (lib/cpu/bandpass_kernels.hpp:17-76)
// after the two remedian passes, with the sampled rows streamed through
// shared memory (rfi_stage.cuh), one thread per channel of a 128-channel
// segment. Every pass over the rows is one staged sweep; the block runs the
// optional passes (mean fallback, clip iterations) when any of its channels
// needs them, and each channel updates only while its own sequence of steps
// is still running, so every channel takes exactly the steps of the direct
// kernel above. A flat channel (every sampled value equal) keeps its first
// sampled value as its level, as the sequential minimum does.
constexpr int kBandChans = 128;

__global__ void __launch_bounds__(kBandChans)
    k_bandpass_staged(Dims d, const float* __restrict__ samples, float* __restrict__ loc_out,
                      float* __restrict__ scale_out, float* __restrict__ inv_out,
                      uint32_t* __restrict__ unmeasured, int seg_bytes, int rows) {
    extern __shared__ __align__(16) uint8_t stage_buf[];
    const uint64_t c0  = static_cast<uint64_t>(blockIdx.x) * kBandChans;
    const uint64_t c   = c0 + threadIdx.x;
    const uint64_t w   = blockIdx.y;
    const bool in      = c < d.nchans;
    const uint64_t b   = window_begin(w, d.window);
    const uint64_t len = window_end(w, d) - b;
    const uint64_t m   = largest_power_of_five_leq(len < kMaxBandpassRows ? len : kMaxBandpassRows);
    const uint64_t n     = d.nchans;
    const uint64_t pitch = n * sizeof(float);
    const uint64_t left  = pitch - c0 * sizeof(float);
    const int copy       = static_cast<int>(left < static_cast<uint64_t>(seg_bytes) ? left : seg_bytes);
    const int stride     = seg_bytes / static_cast<int>(sizeof(float));
    const uint8_t* src   = reinterpret_cast<const uint8_t*>(samples + w * kMaxBandpassRows * n + c0);
    // one sweep over rows 0 .. m-1: f(x, i) per row, in order
    auto sweep = [&](auto&& f) {
        stage::StagerN<kDeepStages> st(stage_buf, src, pitch, seg_bytes, copy, rows, 0, m);
        st.start();
        for (int k = 0; k < st.nblk; ++k) {
            st.wait(k);
            const float* buf = reinterpret_cast<const float*>(st.buf(k));
            const int nr     = st.rows_of(k);
            const uint64_t i0 = st.t0(k);
            if (in)
                for (int r = 0; r < nr; ++r)
                    f(buf[r * stride + threadIdx.x], i0 + r);
            st.release(k);
        }
    };

    const uint64_t o   = w * n + c;
    const float level  = in ? loc_out[o] : 0.0F;
    const float rms    = in ? scale_out[o] : 0.0F;
    const bool flat    = in && inv_out[o] != 0.0F;
    if (in && flat) {
        loc_out[o]   = samples[w * kMaxBandpassRows * n + c];
        scale_out[o] = 0.0F;
        inv_out[o]   = 0.0F;
        atomicAdd(&unmeasured[c], 1U);
    }
    bool live       = in && !flat;
    double centre   = level;
    double sd       = rms;
    const double dm = static_cast<double>(m);
    const bool need_mean = live && !(sd > 0.0);
    if (__syncthreads_or(need_mean)) {
        double mean = 0.0;
        sweep([&](float x, uint64_t) {
            if (need_mean)
                mean += x;
        });
        mean /= dm;
        double ss = 0.0;
        sweep([&](float x, uint64_t) {
            if (need_mean)
                ss += (x - mean) * (x - mean);
        });
        if (need_mean)
            sd = sqrt(ss / dm);
    }
    for (int it = 0; it < kClipIterations; ++it) {
        if (!__syncthreads_or(live))
            break;
        const double cut = kClipSigma * sd;
        uint32_t kept    = 0; // the count of kept samples (exact as a double)
        double sum       = 0.0;
        sweep([&](float x, uint64_t) {
            if (live) {
                const double dv = x - centre;
                if (fabs(dv) <= cut) {
                    ++kept;
                    sum += dv;
                }
            }
        });
        const double count = static_cast<double>(kept);
        if (live && count < 2.0)
            live = false;
        const double shift = live ? sum / count : 0.0;
        if (!__syncthreads_or(live))
            break;
        double ss = 0.0;
        sweep([&](float x, uint64_t) {
            if (live) {
                const double dv = x - centre;
                if (fabs(dv) <= cut)
                    ss += (dv - shift) * (dv - shift);
            }
        });
        if (live) {
            const double clipped = sqrt(ss / count);
            if (!(clipped > 0.0)) {
                live = false;
            } else {
                centre += shift;
                sd = clipped;
            }
        }
    }
    if (in && !flat) {
        const float fl = static_cast<float>(centre);
        const float fs = static_cast<float>(sd);
        loc_out[o]     = fl;
        scale_out[o]   = fs;
        inv_out[o]     = 1.0F / fs;
    }
}

// ---- moments --------------------------------------------------------------

// One (window, channel) sequence of the moments pass, fed in time order
// (lib/cpu/rfi_cpu_measure.cpp:91-138).
struct MomentsAcc {
    MomentSums s{0, 0, 0, 0, 0, 0, 0, 0, 0};
    uint32_t n = 0, nc = 0; // the counts s.n and s.nc, kept as integers (exact)
    double prev = 0.0;
    float l, iv;
    double clip;
    uint64_t b;
    __device__ __forceinline__ void step(float x, uint64_t t) {
        const double z  = (x - l) * iv;
        const double z2 = z * z;
        ++n;
        s.s1 += z;
        s.s2 += z2;
        s.s3 += z2 * z;
        s.s4 += z2 * z2;
        if (t > b)
            s.lag += z * prev;
        prev = z;
        if (fabs(z) <= clip) {
            ++nc;
            s.c1 += z;
            s.c2 += z2;
        }
    }
    __device__ __forceinline__ MomentSums sums() const {
        MomentSums r = s;
        r.n          = static_cast<double>(n);
        r.nc         = static_cast<double>(nc);
        return r;
    }
};

template <int D>
__global__ void k_moments(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                          const float* __restrict__ inv, const uint8_t* __restrict__ static_mask,
                          float clip, MomentSums* __restrict__ out) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t w = blockIdx.y;
    if (c >= d.nchans)
        return;
    const uint64_t o = w * d.nchans + c;
    const uint64_t b = window_begin(w, d.window), e = window_end(w, d);
    MomentsAcc acc;
    acc.l    = loc[o];
    acc.iv   = inv[o];
    acc.clip = clip;
    acc.b    = b;
    if (static_mask[c] != 0 && acc.iv != 0.0F) {
        // Rows are fetched kBlock at a time (independent loads in flight),
        // then consumed strictly in time order.
        for (uint64_t t0 = b; t0 < e; t0 += kBlock) {
            float xs[kBlock];
#pragma unroll
            for (int j = 0; j < kBlock; ++j)
                xs[j] = t0 + j < e ? rd<D>(raw + (t0 + j) * d.row_bytes, c) : 0.0F;
#pragma unroll
            for (int j = 0; j < kBlock; ++j) {
                if (t0 + j >= e)
                    break;
                acc.step(xs[j], t0 + j);
            }
        }
    }
    out[o] = acc.sums();
}

// The same sequences with the block's channel columns streamed through
// shared memory (rfi_stage.cuh): one thread per channel of a
// kStageChans-channel segment.
constexpr int kStageChans = 128;

template <int D>
__global__ void __launch_bounds__(kStageChans)
    k_moments_staged(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                     const float* __restrict__ inv, const uint8_t* __restrict__ static_mask,
                     float clip, MomentSums* __restrict__ out, int seg_bytes, int rows) {
    extern __shared__ __align__(16) uint8_t stage_buf[];
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kStageChans;
    const uint64_t c  = c0 + threadIdx.x;
    const uint64_t w  = blockIdx.y;
    const bool in     = c < d.nchans;
    const uint64_t o  = w * d.nchans + c;
    const uint64_t b = window_begin(w, d.window), e = window_end(w, d);
    MomentsAcc acc;
    acc.l    = in ? loc[o] : 0.0F;
    acc.iv   = in ? inv[o] : 0.0F;
    acc.clip = clip;
    acc.b    = b;
    const bool active   = in && static_mask[c] != 0 && acc.iv != 0.0F;
    const uint64_t off  = c0 * kBitsOf<D> / 8;
    const uint64_t left = d.row_bytes - off;
    const int copy      = static_cast<int>(left < static_cast<uint64_t>(seg_bytes) ? left : seg_bytes);
    stage::StagerN<kDeepStages> st(stage_buf, raw + off, d.row_bytes, seg_bytes, copy, rows, b, e);
    st.start();
    for (int k = 0; k < st.nblk; ++k) {
        st.wait(k);
        const uint8_t* buf = st.buf(k);
        const int nr       = st.rows_of(k);
        const uint64_t t0  = st.t0(k);
        if (active) {
#pragma unroll 8
            for (int r = 0; r < nr; ++r)
                acc.step(rd<D>(buf + r * seg_bytes, threadIdx.x), t0 + r);
        }
        st.release(k);
    }
    if (in)
        out[o] = acc.sums();
}

// ---- row scan ---------------------------------------------------------------

constexpr int kScanRows  = 128; // rows per CTA (one thread each)
constexpr int kScanChans = 64;  // channel tile staged in shared memory

template <int D> constexpr bool kIntRow = D != FROST_FLOAT32 && kBitsOf<D> <= 16;

// One row of the row scan (lib/cpu/rfi_cpu_measure.cpp:305-446), fed its
// channels in ascending order: the detection series sums and the Kadane
// states across frequency.
// With integer samples of at most 16 bits (INT) the row's sum and sum of
// squares are kept as integers: every partial double sum of such values is
// an integer below 2^53, so the reference's double sums are exact and equal
// the integer ones whatever the order.
template <bool INT, bool W32 = false>
struct ScanRowAcc {
    double sum_det = 0.0, sum_keep = 0.0, sx = 0.0, sxx = 0.0;
    uint64_t isx = 0, isxx = 0;
    uint32_t tsx = 0, tsxx = 0;      // W32: the current tile's integer sums
    uint32_t n_keep = 0, n_meas = 0; // counts (exact as doubles when used)
    KadaneBest sp, sn; // rows are scanned whole: only the best runs are needed
    // xi: the sample's integer code (INT: x == xi exactly)
    __device__ __forceinline__ void step(uint64_t c, float x, uint32_t xi, float l, float ic, float clip,
                                         int kspec) {
        ++n_meas;
        const float zc = (x - l) * ic;
        const float cl = clampf(zc, -clip, clip);
        sum_det += cl;
        if (fabsf(zc) <= clip) {
            sum_keep += zc;
            ++n_keep;
        }
        if constexpr (INT && W32) {
            tsx += xi;
            tsxx += xi * xi;
        } else if constexpr (INT) {
            isx += xi;
            isxx += static_cast<uint64_t>(xi) * xi;
        } else {
            sx += x;
            sxx += static_cast<double>(x) * x;
        }
        if (kspec) {
            sp.append(static_cast<int32_t>(c), cl);
            sn.append(static_cast<int32_t>(c), -cl);
        }
    }
    __device__ __forceinline__ void step(uint64_t c, float x, float l, float ic, float clip, int kspec) {
        step(c, x, INT ? static_cast<uint32_t>(x) : 0U, l, ic, clip, kspec);
    }
    // W32: moves the tile's integer sums into the 64-bit ones (exact: a tile
    // of at most 128 8-bit samples sums below 2^32 even squared)
    __device__ __forceinline__ void flush() {
        isx += tsx;
        isxx += tsxx;
        tsx  = 0;
        tsxx = 0;
    }
    __device__ void finish(const Dims& d, uint64_t t, const KspecParams& kp,
                           const uint64_t* __restrict__ good_prefix, float* __restrict__ s_det,
                           double* __restrict__ s_keep_d, float* __restrict__ s_keep_f,
                           float* __restrict__ row_std, Span32* __restrict__ kspec_pos,
                           Span32* __restrict__ kspec_neg, uint8_t* __restrict__ kspec_whole,
                           uint8_t* __restrict__ row_clip) const {
        const double dn     = n_meas > 1 ? static_cast<double>(n_meas) : 1.0;
        const double s_keep = n_keep > 0 ? sum_keep / static_cast<double>(n_keep) : 0.0;
        const double sx     = INT ? static_cast<double>(isx + tsx) : this->sx;
        const double sxx    = INT ? static_cast<double>(isxx + tsxx) : this->sxx;
        s_det[t]            = static_cast<float>(sum_det / dn);
        s_keep_f[t]         = static_cast<float>(s_keep);
        s_keep_d[t]         = s_keep;
        // a measured cell of this row is past the clip (a narrow-band cell
        // for the apply pass, which computes the same z from the same row,
        // constants and clip)
        row_clip[t] = n_keep != n_meas ? 1 : 0;
        const double mx     = sx / dn;
        const double var    = (sxx / dn) - (mx * mx);
        row_std[t]          = static_cast<float>(sqrt(var < 0.0 ? 0.0 : var));
        if (kp.enabled) {
            // accept_span (lib/cpu/rfi_cpu_measure.cpp:335-349)
            auto accept = [&](const Run& r, Span32& out) -> bool {
                out = {-1, -1};
                if (r.length() <= 0)
                    return false;
                const uint64_t lo    = static_cast<uint64_t>(r.start);
                const uint64_t hi    = static_cast<uint64_t>(r.end);
                const uint64_t count = good_prefix[hi + 1] - good_prefix[lo];
                const double nspan   = static_cast<double>(hi - lo + 1);
                const double snr     = r.sum / sqrt(static_cast<double>(count));
                if (snr > kp.threshold && nspan >= kp.min_bw_chans) {
                    out = {static_cast<int32_t>(lo), static_cast<int32_t>(hi)};
                    return nspan > kp.whole_chans;
                }
                return false;
            };
            Span32 a, b;
            bool whole     = accept(sp.best(), a);
            whole          = accept(sn.best(), b) || whole;
            kspec_pos[t]   = a;
            kspec_neg[t]   = b;
            kspec_whole[t] = whole ? 1 : 0;
        }
    }
};

template <int D>
__global__ void __launch_bounds__(kScanRows)
    k_scan_rows(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                const float* __restrict__ inv, const uint8_t* __restrict__ mask, float clip,
                KspecParams kp, const uint64_t* __restrict__ good_prefix, float* __restrict__ s_det,
                double* __restrict__ s_keep_d, float* __restrict__ s_keep_f,
                float* __restrict__ row_std, Span32* __restrict__ kspec_pos,
                Span32* __restrict__ kspec_neg, uint8_t* __restrict__ kspec_whole, uint8_t* __restrict__ row_clip) {
    __shared__ float tile[kScanRows][kScanChans + 1];
    const uint64_t t0    = static_cast<uint64_t>(blockIdx.x) * kScanRows;
    const uint64_t t     = t0 + threadIdx.x;
    const bool active    = t < d.nsamps;
    const uint64_t n     = d.nchans;
    const uint64_t w     = active ? window_of(t, d.window, d.nwin) : 0;
    const float* lw      = loc + w * n;
    const float* iw      = inv + w * n;
    ScanRowAcc<kIntRow<D>> acc;
    for (uint64_t c0 = 0; c0 < n; c0 += kScanChans) {
        const unsigned cl_ = threadIdx.x % kScanChans;
        const uint64_t cc  = c0 + cl_;
        __syncthreads();
        for (int r = threadIdx.x / kScanChans; r < kScanRows; r += kScanRows / kScanChans) {
            const uint64_t tr = t0 + r;
            tile[r][cl_] = (tr < d.nsamps && cc < n) ? rd<D>(raw + tr * d.row_bytes, cc) : 0.0F;
        }
        __syncthreads();
        if (!active)
            continue;
        const uint64_t cend = (c0 + kScanChans < n) ? c0 + kScanChans : n;
        for (uint64_t c = c0; c < cend; ++c) {
            if (mask[c] == 0)
                continue;
            const float ic = iw[c];
            if (ic == 0.0F)
                continue;
            acc.step(c, tile[threadIdx.x][c - c0], lw[c], ic, clip, kp.enabled);
        }
    }
    if (active)
        acc.finish(d, t, kp, good_prefix, s_det, s_keep_d, s_keep_f, row_std, kspec_pos, kspec_neg,
                   kspec_whole, row_clip);
}

// The same rows with 128-byte column tiles of all 128 rows bulk-copied
// into shared memory (cp.async, two tiles deep; rows padded to 144 bytes so
// that each thread's 16-byte reads of its own row are conflict-free).
constexpr int kRowTileBytes  = 128;
constexpr int kRowTileStride = kRowTileBytes + 16;

template <int D>
__global__ void __launch_bounds__(kScanRows)
    k_scan_rows_staged(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                       const float* __restrict__ inv, const uint8_t* __restrict__ mask, float clip,
                       KspecParams kp, const uint64_t* __restrict__ good_prefix,
                       float* __restrict__ s_det, double* __restrict__ s_keep_d,
                       float* __restrict__ s_keep_f, float* __restrict__ row_std,
                       Span32* __restrict__ kspec_pos, Span32* __restrict__ kspec_neg,
                       uint8_t* __restrict__ kspec_whole, uint8_t* __restrict__ row_clip) {
    extern __shared__ __align__(16) uint8_t tiles[]; // [2][kScanRows][kRowTileStride]
    constexpr int kPerChunk = static_cast<int>(128 / kBitsOf<D>); // channels per 16 bytes
    constexpr int kTileCh   = static_cast<int>(kRowTileBytes * 8 / kBitsOf<D>);
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kScanRows;
    const uint64_t t  = t0 + threadIdx.x;
    const bool active = t < d.nsamps;
    const uint64_t n  = d.nchans;
    const uint64_t w  = active ? window_of(t, d.window, d.nwin) : 0;
    const float* lw   = loc + w * n;
    const float* iw   = inv + w * n;
    // 16-byte loads of the window constants and mask need 16-byte aligned rows
    const bool vec_consts = (reinterpret_cast<uintptr_t>(lw) | reinterpret_cast<uintptr_t>(iw) |
                             reinterpret_cast<uintptr_t>(mask)) % 16 == 0;
    const int nrows   = static_cast<int>(d.nsamps - t0 < kScanRows ? d.nsamps - t0 : kScanRows);
    const int ntiles  = static_cast<int>((d.row_bytes + kRowTileBytes - 1) / kRowTileBytes);
    auto issue = [&](int j) {
        const uint64_t b0  = static_cast<uint64_t>(j) * kRowTileBytes;
        const int chunks   = static_cast<int>((d.row_bytes - b0 < kRowTileBytes ? d.row_bytes - b0 : kRowTileBytes) / 16);
        uint8_t* dst       = tiles + (j & 1) * kScanRows * kRowTileStride;
        for (int i = threadIdx.x; i < nrows * chunks; i += kScanRows) {
            const int r = i / chunks, v = i - r * chunks;
            stage::cp_async16(dst + r * kRowTileStride + v * 16, raw + (t0 + r) * d.row_bytes + b0 + v * 16);
        }
        stage::commit();
    };
    issue(0);
    if (ntiles > 1)
        issue(1);
    // 8-bit and narrower samples: the integer sums of a tile in 32 bits
    constexpr bool kW32 = kIntRow<D> && kBitsOf<D> <= 8;
    ScanRowAcc<kIntRow<D>, kW32> acc;
    for (int j = 0; j < ntiles; ++j) {
        if (j + 1 < ntiles)
            stage::wait_pending<1>();
        else
            stage::wait_pending<0>();
        __syncthreads();
        if (active) {
            const uint8_t* row = tiles + (j & 1) * kScanRows * kRowTileStride + threadIdx.x * kRowTileStride;
            const uint32_t cb  = static_cast<uint32_t>(j) * kTileCh; // channel indices fit 32 bits
            const uint32_t ce  = cb + kTileCh < n ? cb + kTileCh : static_cast<uint32_t>(n);
            for (uint32_t q = cb; q < ce; q += kPerChunk) {
                union {
                    uint4 v;
                    uint8_t b[16];
                } u;
                u.v = *reinterpret_cast<const uint4*>(row + (q - cb) * kBitsOf<D> / 8);
                if constexpr (kPerChunk == 16) {
                    if (vec_consts && q + kPerChunk <= ce) {
                        // a whole chunk: its mask bytes and window constants
                        // as 16-byte loads (the same for every row of the CTA)
                        union {
                            uint4 v;
                            uint8_t b[16];
                        } mk;
                        mk.v = *reinterpret_cast<const uint4*>(mask + q);
                        float ls[16], is[16];
#pragma unroll
                        for (int v4 = 0; v4 < 4; ++v4) {
                            const float4 a = reinterpret_cast<const float4*>(lw + q)[v4];
                            const float4 b = reinterpret_cast<const float4*>(iw + q)[v4];
                            ls[4 * v4] = a.x, ls[4 * v4 + 1] = a.y, ls[4 * v4 + 2] = a.z, ls[4 * v4 + 3] = a.w;
                            is[4 * v4] = b.x, is[4 * v4 + 1] = b.y, is[4 * v4 + 2] = b.z, is[4 * v4 + 3] = b.w;
                        }
#pragma unroll
                        for (int e = 0; e < 16; ++e)
                            if (mk.b[e] != 0 && is[e] != 0.0F) {
                                const uint32_t xi = rdi<D>(u.b, static_cast<uint64_t>(e));
                                acc.step(q + e, static_cast<float>(xi), xi, ls[e], is[e], clip, kp.enabled);
                            }
                        continue;
                    }
                }
#pragma unroll
                for (int e = 0; e < kPerChunk; ++e) {
                    const uint32_t c = q + e;
                    if (c >= ce)
                        break;
                    if (mask[c] == 0)
                        continue;
                    const float ic = iw[c];
                    if (ic == 0.0F)
                        continue;
                    acc.step(c, rd<D>(u.b, static_cast<uint64_t>(e)), lw[c], ic, clip, kp.enabled);
                }
            }
            if constexpr (kW32)
                acc.flush();
        }
        __syncthreads(); // every thread is done with this tile's buffer
        if (j + 2 < ntiles)
            issue(j + 2);
    }
    if (active)
        acc.finish(d, t, kp, good_prefix, s_det, s_keep_d, s_keep_f, row_std, kspec_pos, kspec_neg,
                   kspec_whole, row_clip);
}

// One (chunk, channel) sequence of the column scan
// (lib/cpu/rfi_cpu_measure.cpp:305-446): the block min/max of unmeasured
// cells, zdot sums and Kadane-along-time states. The per-(window, channel)
// constants are reloaded only when the window changes.
struct ScanColAcc {
    const Dims* d;
    const float* loc;
    const float* inv;
    const float* clip_mean;
    const float* clip_inv_std;
    const double* s_keep_d;
    uint64_t c;
    float clip;
    int zdot, kchan;
    uint64_t w = 0, wend = 0; // current window and its end (0: none yet)
    float l = 0.0F, iv = 0.0F, cm = 0.0F, ci = 0.0F;
    float cmin = FLT_MAX, cmax = -FLT_MAX;
    ZdotSums zs{0, 0, 0, 0, 0};
    uint32_t zn = 0;
    KadanePair32 kk; // Kadane along time of u and -u, widened when stored
    // the first sample of an active channel's chunk (every later sample of
    // the chunk follows in order)
    __device__ __forceinline__ void begin(uint64_t t0) {
        if (kchan)
            kk.begin(static_cast<int32_t>(t0));
    }
    __device__ __forceinline__ void step(float x, uint64_t t) {
        if (t >= wend) {
            w                = window_of(t, d->window, d->nwin);
            wend             = window_end(w, *d);
            const uint64_t o = w * d->nchans + c;
            l                = loc[o];
            iv               = inv[o];
            if (kchan) {
                cm = clip_mean[o];
                ci = clip_inv_std[o];
            }
        }
        float z = 0.0F;
        if (iv == 0.0F) {
            cmin = smin(cmin, x);
            cmax = smax(cmax, x);
        } else {
            z = (x - l) * iv;
        }
        const bool outlier = fabsf(z) > clip;
        if (zdot && !outlier && iv != 0.0F) {
            const double sk = s_keep_d[t];
            ++zn; // the count, exact as an integer (stored as a double)
            zs.sz += z;
            zs.ss += sk;
            zs.sss += sk * sk;
            zs.szs += z * sk;
        }
        if (kchan) {
            const double u = outlier ? 0.0 : static_cast<double>((z - cm) * ci);
            kk.append(static_cast<int32_t>(t), u);
        }
    }
    __device__ __forceinline__ void store(uint64_t k, float* cmin_out, float* cmax_out,
                                          ZdotSums* zs_out, KadaneState* kp_out,
                                          KadaneState* kn_out) const {
        const uint64_t o = k * d->nchans + c;
        cmin_out[o]      = cmin;
        cmax_out[o]      = cmax;
        if (zdot) {
            ZdotSums z = zs;
            z.n        = static_cast<double>(zn);
            zs_out[o]  = z;
        }
        if (kchan) {
            // an active channel appended every sample of the chunk
            const uint64_t t1   = (k + 1) * d->chunk < d->nsamps ? (k + 1) * d->chunk : d->nsamps;
            const int32_t last  = static_cast<int32_t>(t1) - 1;
            kp_out[o] = kk.widen_pos(last);
            kn_out[o] = kk.widen_neg(last);
        }
    }
};

template <int D>
__global__ void k_scan_cols(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                            const float* __restrict__ inv, const uint8_t* __restrict__ mask,
                            float clip, const double* __restrict__ s_keep_d, int zdot, int kchan,
                            const float* __restrict__ clip_mean,
                            const float* __restrict__ clip_inv_std, float* __restrict__ cmin_out,
                            float* __restrict__ cmax_out, ZdotSums* __restrict__ zs_out,
                            KadaneState* __restrict__ kp_out, KadaneState* __restrict__ kn_out) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t k = blockIdx.y;
    if (c >= d.nchans)
        return;
    ScanColAcc acc{&d, loc, inv, clip_mean, clip_inv_std, s_keep_d, c, clip, zdot, kchan};
    if (mask[c] != 0) {
        const uint64_t t0 = k * d.chunk;
        const uint64_t t1 = (t0 + d.chunk < d.nsamps) ? t0 + d.chunk : d.nsamps;
        if (t0 < t1)
            acc.begin(t0);
        for (uint64_t tb = t0; tb < t1; tb += kBlock) {
            // fetch kBlock rows ahead of their sequential use
            float xs[kBlock];
#pragma unroll
            for (int q = 0; q < kBlock; ++q)
                xs[q] = tb + q < t1 ? rd<D>(raw + (tb + q) * d.row_bytes, c) : 0.0F;
#pragma unroll
            for (int q = 0; q < kBlock; ++q) {
                if (tb + q >= t1)
                    break;
                acc.step(xs[q], tb + q);
            }
        }
    }
    acc.store(k, cmin_out, cmax_out, zs_out, kp_out, kn_out);
}

template <int D>
__global__ void __launch_bounds__(kStageChans)
    k_scan_cols_staged(Dims d, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                       const float* __restrict__ inv, const uint8_t* __restrict__ mask, float clip,
                       const double* __restrict__ s_keep_d, int zdot, int kchan,
                       const float* __restrict__ clip_mean, const float* __restrict__ clip_inv_std,
                       float* __restrict__ cmin_out, float* __restrict__ cmax_out,
                       ZdotSums* __restrict__ zs_out, KadaneState* __restrict__ kp_out,
                       KadaneState* __restrict__ kn_out, int seg_bytes, int rows) {
    extern __shared__ __align__(16) uint8_t stage_buf[];
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kStageChans;
    const uint64_t c  = c0 + threadIdx.x;
    const uint64_t k  = blockIdx.y;
    const bool in     = c < d.nchans;
    const bool active = in && mask[c] != 0;
    ScanColAcc acc{&d, loc, inv, clip_mean, clip_inv_std, s_keep_d, c, clip, zdot, kchan};
    const uint64_t t0   = k * d.chunk;
    const uint64_t t1   = (t0 + d.chunk < d.nsamps) ? t0 + d.chunk : d.nsamps;
    const uint64_t off  = c0 * kBitsOf<D> / 8;
    const uint64_t left = d.row_bytes - off;
    const int copy      = static_cast<int>(left < static_cast<uint64_t>(seg_bytes) ? left : seg_bytes);
    stage::Stager st(stage_buf, raw + off, d.row_bytes, seg_bytes, copy, rows, t0, t1);
    if (active && t0 < t1)
        acc.begin(t0);
    st.start();
    for (int kb = 0; kb < st.nblk; ++kb) {
        st.wait(kb);
        const uint8_t* buf = st.buf(kb);
        const int nr       = st.rows_of(kb);
        const uint64_t tb  = st.t0(kb);
        if (active) {
#pragma unroll 4
            for (int r = 0; r < nr; ++r)
                acc.step(rd<D>(buf + r * seg_bytes, threadIdx.x), tb + r);
        }
        st.release(kb);
    }
    if (in)
        acc.store(k, cmin_out, cmax_out, zs_out, kp_out, kn_out);
}

// Per channel, in chunk order: the block min/max of unmeasured cells, the
// zdot sums and the combined Kadane-along-time states
// (lib/cpu/rfi_cpu.cpp:352-366, 413-466).
__global__ void k_combine_chunks(Dims d, int zdot, int kchan, const float* __restrict__ cmin,
                                 const float* __restrict__ cmax, const ZdotSums* __restrict__ zs,
                                 const KadaneState* __restrict__ kp,
                                 const KadaneState* __restrict__ kn, float* __restrict__ lo_out,
                                 float* __restrict__ hi_out, ZdotSums* __restrict__ zs_out,
                                 Run* __restrict__ kp_best, Run* __restrict__ kn_best) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= d.nchans)
        return;
    const uint64_t n = d.nchans;
    float lo = FLT_MAX, hi = -FLT_MAX;
    ZdotSums s{0, 0, 0, 0, 0};
    KadaneState pos = KadaneState::make(), neg = KadaneState::make();
    for (uint64_t k = 0; k < d.nchunks; ++k) {
        lo = smin(lo, cmin[k * n + c]);
        hi = smax(hi, cmax[k * n + c]);
        if (zdot) {
            const ZdotSums& p = zs[k * n + c];
            s.n += p.n;
            s.sz += p.sz;
            s.ss += p.ss;
            s.sss += p.sss;
            s.szs += p.szs;
        }
        if (kchan) {
            pos = KadaneState::combine(pos, kp[k * n + c]);
            neg = KadaneState::combine(neg, kn[k * n + c]);
        }
    }
    lo_out[c] = lo;
    hi_out[c] = hi;
    if (zdot)
        zs_out[c] = s;
    if (kchan) {
        kp_best[c] = pos.best;
        kn_best[c] = neg.best;
    }
}

// ---- apply ------------------------------------------------------------------

__device__ __forceinline__ float level_of(const ApplyParams& p, float loc, float scale, float v) {
    return p.equalize ? p.eq_loc + (p.eq_scale * v) : loc + (scale * v);
}

// Unflagged rows (lib/cpu/rfi_cpu.cpp:537-624) in two kernels. Every
// measured cell of a row is clean when the row has no span across
// frequency, no cell past the clip (the row scan computed the same z of
// every measured cell from the same row, constants and clip; masks only
// grow after it, so a cell it did not clip is never clipped here) and no
// Kadane-along-time segment covering it. k_apply_clean writes those rows'
// clean values (a CTA per row, no cell states, few registers) and lists
// the others; k_apply_unflagged classifies the listed rows' cells, writes
// their values and, where a cell needs one, the fills: a row's samples and
// cell states are staged in shared memory so neighbour draws read them
// without touching HBM again. Masked cells are not written: the normalized
// output zeroes them, so their fill values are never observed.
template <int D, int V>
__global__ void __launch_bounds__(256)
    k_apply_clean(Dims d, ApplyParams p, const uint8_t* __restrict__ raw, const float* __restrict__ loc,
                  const float* __restrict__ scale, const float* __restrict__ inv,
                  const uint8_t* __restrict__ mask, const uint8_t* __restrict__ time_flags,
                  const Span32* __restrict__ kspec_pos, const Span32* __restrict__ kspec_neg,
                  const float* __restrict__ s_keep_f, const float* __restrict__ zdot_a,
                  const float* __restrict__ zdot_b, const uint8_t* __restrict__ row_clip,
                  const uint8_t* __restrict__ row_kchan, float* __restrict__ work,
                  uint32_t* __restrict__ slow_rows, unsigned int* __restrict__ nslow) {
    const uint64_t t = blockIdx.x;
    if (t >= d.nsamps || time_flags[t] != 0)
        return;
    const bool row_kspec = p.kspec && (kspec_pos[t].lo >= 0 || kspec_neg[t].lo >= 0);
    if (row_kspec || (p.narrow_active && row_clip[t] != 0) || (p.kchan && row_kchan[t] != 0)) {
        if (threadIdx.x == 0)
            slow_rows[atomicAdd(nslow, 1U)] = static_cast<uint32_t>(t);
        return;
    }
    const uint64_t n   = d.nchans;
    const uint32_t n32 = static_cast<uint32_t>(n);
    const uint64_t w   = window_of(t, d.window, d.nwin);
    const float* lw    = loc + w * n;
    const float* sw    = scale + w * n;
    const float* iw    = inv + w * n;
    const uint8_t* in  = raw + t * d.row_bytes;
    float* out         = work + t * n;
    const float sk     = s_keep_f[t];
    for (uint32_t cb = threadIdx.x * V; cb < n32; cb += blockDim.x * V) {
        float xs[V], ls[V], ss[V], is[V], outv[V];
        uint8_t ms[V];
        if constexpr (V == 4) {
            const float4 l4 = *reinterpret_cast<const float4*>(lw + cb);
            const float4 s4 = *reinterpret_cast<const float4*>(sw + cb);
            const float4 i4 = *reinterpret_cast<const float4*>(iw + cb);
            const uchar4 m4 = *reinterpret_cast<const uchar4*>(mask + cb);
            ls[0] = l4.x; ls[1] = l4.y; ls[2] = l4.z; ls[3] = l4.w;
            ss[0] = s4.x; ss[1] = s4.y; ss[2] = s4.z; ss[3] = s4.w;
            is[0] = i4.x; is[1] = i4.y; is[2] = i4.z; is[3] = i4.w;
            ms[0] = m4.x; ms[1] = m4.y; ms[2] = m4.z; ms[3] = m4.w;
            if constexpr (D == FROST_UINT8) {
                const uchar4 x4 = *reinterpret_cast<const uchar4*>(in + cb);
                xs[0] = static_cast<float>(x4.x); xs[1] = static_cast<float>(x4.y);
                xs[2] = static_cast<float>(x4.z); xs[3] = static_cast<float>(x4.w);
            } else {
#pragma unroll
                for (int e = 0; e < V; ++e)
                    xs[e] = rd<D>(in, cb + e);
            }
        } else {
            ls[0] = lw[cb];
            ss[0] = sw[cb];
            is[0] = iw[cb];
            ms[0] = mask[cb];
            xs[0] = rd<D>(in, cb);
        }
#pragma unroll
        for (int e = 0; e < V; ++e) {
            const uint32_t c = cb + e;
            const float x    = xs[e];
            if (ms[e] == 0) {
                outv[e] = 0.0F;
            } else if (is[e] == 0.0F) {
                outv[e] = x;
            } else {
                const float z = (x - ls[e]) * is[e];
                float term    = 0.0F;
                if (p.zero_dm == FROST_ZERO_DM_SUBTRACT)
                    term = sk;
                else if (p.zero_dm == FROST_ZERO_DM_ZDOT)
                    term = (zdot_a[c] * sk) + zdot_b[c];
                const float v = z - term;
                outv[e]       = p.transform ? level_of(p, ls[e], ss[e], v) : x;
            }
        }
        if constexpr (V == 4)
            *reinterpret_cast<float4*>(out + cb) = make_float4(outv[0], outv[1], outv[2], outv[3]);
        else
            out[cb] = outv[0];
    }
}

template <int D, int V>
__global__ void k_apply_unflagged(Dims d, ApplyParams p, const uint8_t* __restrict__ raw,
                                  const float* __restrict__ loc, const float* __restrict__ scale,
                                  const float* __restrict__ inv, const uint8_t* __restrict__ mask,
                                  const uint8_t* __restrict__ time_flags,
                                  const Span32* __restrict__ kspec_pos,
                                  const Span32* __restrict__ kspec_neg,
                                  const Segment* __restrict__ kchan_pos,
                                  const Segment* __restrict__ kchan_neg,
                                  const uint8_t* __restrict__ kchan_any,
                                  const float* __restrict__ s_keep_f,
                                  const float* __restrict__ zdot_a,
                                  const float* __restrict__ zdot_b, const uint32_t* __restrict__ slow_rows,
                                  const unsigned int* __restrict__ nslow, float* __restrict__ work,
                                  unsigned long long* __restrict__ counters) {
    extern __shared__ unsigned char smem[];
    const uint64_t n = d.nchans;
    float* sv        = reinterpret_cast<float*>(smem);           // v = z - zero-DM term
    uint8_t* state   = reinterpret_cast<uint8_t*>(sv + n);
    __shared__ unsigned long long cnt[kCountSlots];
    if (threadIdx.x < kCountSlots)
        cnt[threadIdx.x] = 0;
    unsigned long long narrow = 0, nks = 0, nkc = 0, fallbacks = 0;
    const unsigned int nrows = *nslow;
    for (unsigned int i = blockIdx.x; i < nrows; i += gridDim.x) {
        const uint64_t t = slow_rows[i];
        const uint64_t w  = window_of(t, d.window, d.nwin);
        const float* lw   = loc + w * n;
        const float* sw   = scale + w * n;
        const float* iw   = inv + w * n;
        const uint8_t* in = raw + t * d.row_bytes;
        float* out        = work + t * n;
        const float sk    = s_keep_f[t];
        const Span32 ksp  = p.kspec ? kspec_pos[t] : Span32{-1, -1};
        const Span32 ksn  = p.kspec ? kspec_neg[t] : Span32{-1, -1};
        // a row with no Kadane span across frequency (almost every row)
        // skips the per-cell span tests
        const bool row_kspec = ksp.lo >= 0 || ksn.lo >= 0;
        auto span_has     = [](const Span32& s, uint64_t c) {
            return s.lo >= 0 && static_cast<int32_t>(c) >= s.lo && static_cast<int32_t>(c) <= s.hi;
        };
        auto seg_has = [](const Segment& s, uint64_t tt) {
            const int64_t i = static_cast<int64_t>(tt);
            return i >= s.start && i <= s.end;
        };

        // V consecutive channels per thread (V = 4: 16-byte loads of the
        // per-window constants and stores of the row, when nchans % 4 == 0);
        // channel indices fit 32 bits (the launcher checks)
        const uint32_t n32 = static_cast<uint32_t>(n);
        // One pass over the thread's cells: classify each, then either write
        // the row's values (STATES false: every row) or the cell states and
        // zero-DM-corrected values the fills draw from (STATES true: only a
        // row with a cell to fill, recomputed the same way).
        auto cells = [&](auto states_tag) -> bool {
        constexpr bool STATES = decltype(states_tag)::value;
        bool dirty = false; // a cell of this thread's needs a fill
        for (uint32_t cb = threadIdx.x * V; cb < n32; cb += blockDim.x * V) {
            float xs[V], ls[V], ss[V], is[V], outv[V];
            uint8_t ms[V], ka[V];
            if constexpr (V == 4) {
                const float4 l4 = *reinterpret_cast<const float4*>(lw + cb);
                const float4 s4 = *reinterpret_cast<const float4*>(sw + cb);
                const float4 i4 = *reinterpret_cast<const float4*>(iw + cb);
                const uchar4 m4 = *reinterpret_cast<const uchar4*>(mask + cb);
                ls[0] = l4.x; ls[1] = l4.y; ls[2] = l4.z; ls[3] = l4.w;
                ss[0] = s4.x; ss[1] = s4.y; ss[2] = s4.z; ss[3] = s4.w;
                is[0] = i4.x; is[1] = i4.y; is[2] = i4.z; is[3] = i4.w;
                ms[0] = m4.x; ms[1] = m4.y; ms[2] = m4.z; ms[3] = m4.w;
                if (p.kchan) {
                    const uchar4 k4 = *reinterpret_cast<const uchar4*>(kchan_any + cb);
                    ka[0] = k4.x; ka[1] = k4.y; ka[2] = k4.z; ka[3] = k4.w;
                } else {
                    ka[0] = ka[1] = ka[2] = ka[3] = 0;
                }
                if constexpr (D == FROST_UINT8) {
                    const uchar4 x4 = *reinterpret_cast<const uchar4*>(in + cb);
                    xs[0] = static_cast<float>(x4.x); xs[1] = static_cast<float>(x4.y);
                    xs[2] = static_cast<float>(x4.z); xs[3] = static_cast<float>(x4.w);
                } else {
    #pragma unroll
                    for (int e = 0; e < V; ++e)
                        xs[e] = rd<D>(in, cb + e);
                }
            } else {
                ls[0] = lw[cb];
                ss[0] = sw[cb];
                is[0] = iw[cb];
                ms[0] = mask[cb];
                ka[0] = p.kchan ? kchan_any[cb] : 0;
                xs[0] = rd<D>(in, cb);
            }
    #pragma unroll
            for (int e = 0; e < V; ++e) {
                const uint32_t c = cb + e;
                const float x    = xs[e];
                uint8_t st;
                float v = 0.0F;
                outv[e] = 0.0F;
                if (ms[e] == 0) {
                    st = kMasked;
                } else if (is[e] == 0.0F) {
                    st      = kUnmeasured;
                    outv[e] = x;
                } else {
                    const float z = (x - ls[e]) * is[e];
                    if (p.narrow_active && fabsf(z) > p.clip) {
                        st = kNarrow;
                    } else if (row_kspec && (span_has(ksp, c) || span_has(ksn, c))) {
                        st = kKadaneSpectrum;
                    } else if (ka[e] != 0 && (seg_has(kchan_pos[c], t) || seg_has(kchan_neg[c], t))) {
                        st = kKadaneChannel;
                    } else {
                        st = kClean;
                        float term = 0.0F;
                        if (p.zero_dm == FROST_ZERO_DM_SUBTRACT)
                            term = sk;
                        else if (p.zero_dm == FROST_ZERO_DM_ZDOT)
                            term = (zdot_a[c] * sk) + zdot_b[c];
                        v       = z - term;
                        outv[e] = p.transform ? level_of(p, ls[e], ss[e], v) : x;
                    }
                }
                if constexpr (STATES) {
                    state[c] = st;
                    sv[c]    = v;
                }
                dirty = dirty || st == kNarrow || st == kKadaneSpectrum || st == kKadaneChannel;
            }
            // masked and flagged cells are (re)written below or never read
            if constexpr (!STATES) {
                if constexpr (V == 4)
                    *reinterpret_cast<float4*>(out + cb) = make_float4(outv[0], outv[1], outv[2], outv[3]);
                else
                    out[cb] = outv[0];
            }
        }
        return dirty;
        };
        // a row with no cell to fill (almost every row) is done
        if (!__syncthreads_or(cells(std::false_type{})))
            continue;
        cells(std::true_type{});
        __syncthreads(); // every cell state is written before the fills read them

        for (uint32_t c = threadIdx.x; c < n32; c += blockDim.x) {
            const uint8_t st = state[c];
            if (st == kClean || st == kUnmeasured || st == kMasked)
                continue;
            if (st == kNarrow)
                ++narrow;
            else if (st == kKadaneSpectrum)
                ++nks;
            else
                ++nkc;
            if (!p.neighbour) {
                const float v = p.noise ? normal_deviate(draw(p, kStreamNoise, t, c, 0)) : 0.0F;
                out[c]        = level_of(p, lw[c], sw[c], v);
                continue;
            }
            const uint64_t r  = p.chan_fill_radius;
            const uint64_t lo = c > r ? c - r : 0;
            const uint64_t hi = (c + r < n - 1) ? c + r : n - 1;
            float value       = 0.0F;
            bool found        = false;
            for (int a = 0; a < kMaxDraws && !found; ++a) {
                const uint64_t src = uniform_index(draw(p, kStreamCell, t, c, a), lo, hi);
                if (state[src] == kClean) {
                    value = sv[src];
                    found = true;
                }
            }
            fallbacks += found ? 0 : 1;
            out[c] = level_of(p, lw[c], sw[c], value);
        }
        __syncthreads(); // the fills read this row's states before the next row rewrites them
    }
    if (narrow | nks | nkc | fallbacks) {
        atomicAdd(&cnt[kCountNarrow], narrow);
        atomicAdd(&cnt[kCountKspec], nks);
        atomicAdd(&cnt[kCountKchan], nkc);
        atomicAdd(&cnt[kCountFallback], fallbacks);
    }
    __syncthreads();
    if (threadIdx.x < kCountSlots && cnt[threadIdx.x] != 0)
        atomicAdd(&counters[threadIdx.x], cnt[threadIdx.x]);
}

// Flagged rows (lib/cpu/rfi_cpu.cpp:626-715): each copies, per channel,
// from a random unflagged row within the time-fill radius (already final),
// or rebuilds the spectrum in noise units and removes its band mean when a
// zero-DM transform is on. The band-mean sum keeps channel order.
__device__ void apply_flagged_row(const Dims& d, const ApplyParams& p, uint64_t t, const float* __restrict__ loc,
                                  const float* __restrict__ scale, const float* __restrict__ inv,
                                  const uint8_t* __restrict__ mask, const uint8_t* __restrict__ time_flags,
                                  float* __restrict__ work, unsigned long long* __restrict__ counters,
                                  float* sv, uint8_t* contrib, float& s_mean, unsigned long long& s_fallbacks) {
    const uint64_t n = d.nchans;
    if (threadIdx.x == 0)
        s_fallbacks = 0;
    __syncthreads();
    const uint64_t w  = window_of(t, d.window, d.nwin);
    const uint64_t r  = p.time_fill_radius;
    const uint64_t lo = t > r ? t - r : 0;
    const uint64_t hi = (t + r < d.nsamps - 1) ? t + r : d.nsamps - 1;
    const bool rezero = p.zero_dm != FROST_ZERO_DM_OFF;
    float* out        = work + t * n;
    unsigned long long fallbacks = 0;

    for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
        contrib[c] = 0;
        sv[c]      = 0.0F;
        if (mask[c] == 0)
            continue;
        float v = 0.0F;
        if (!p.neighbour) {
            v = p.noise ? normal_deviate(draw(p, kStreamNoise, t, c, 0)) : 0.0F;
        } else {
            bool found = false;
            for (int a = 0; a < kMaxDraws && !found; ++a) {
                const uint64_t src = uniform_index(draw(p, kStreamTime, t, c, a), lo, hi);
                if (time_flags[src] != 0)
                    continue;
                found = true;
                const float sval = work[src * n + c];
                if (rezero) {
                    const uint64_t ws = window_of(src, d.window, d.nwin);
                    v = p.equalize ? (sval - p.eq_loc) / p.eq_scale
                                   : (sval - loc[ws * n + c]) * inv[ws * n + c];
                } else {
                    out[c] = sval;
                }
            }
            if (!found)
                ++fallbacks;
            if (found && !rezero)
                continue;
        }
        sv[c] = v;
        if (rezero) {
            contrib[c] = inv[w * n + c] != 0.0F ? 1 : 0;
        } else {
            out[c] = level_of(p, loc[w * n + c], scale[w * n + c], v);
        }
    }
    if (fallbacks)
        atomicAdd(&s_fallbacks, fallbacks);
    __syncthreads();
    if (rezero) {
        if (threadIdx.x == 0) {
            double sum = 0.0, count = 0.0;
            for (uint64_t c = 0; c < n; ++c) {
                if (contrib[c]) {
                    sum += sv[c];
                    count += 1.0;
                }
            }
            s_mean = static_cast<float>(count > 0.0 ? sum / count : 0.0);
        }
        __syncthreads();
        // Float samples: quantisation is the identity, so the carried
        // rounding error of lib/cpu/rfi_cpu.cpp:704-713 stays +0.
        for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
            if (mask[c] == 0)
                continue;
            out[c] = level_of(p, loc[w * n + c], scale[w * n + c], sv[c] - s_mean) + 0.0F;
        }
    }
    if (threadIdx.x == 0 && s_fallbacks)
        atomicAdd(&counters[kCountFallback], s_fallbacks);
    __syncthreads();
}

// The flagged rows listed in flagged[0 .. *count), a row per CTA at a time
// (the count is known only on the device).
__global__ void k_apply_flagged(Dims d, ApplyParams p, const uint64_t* __restrict__ flagged,
                                const unsigned long long* __restrict__ count, const float* __restrict__ loc,
                                const float* __restrict__ scale, const float* __restrict__ inv,
                                const uint8_t* __restrict__ mask, const uint8_t* __restrict__ time_flags,
                                float* __restrict__ work, unsigned long long* __restrict__ counters) {
    extern __shared__ unsigned char smem[];
    float* sv        = reinterpret_cast<float*>(smem);
    uint8_t* contrib = reinterpret_cast<uint8_t*>(sv + d.nchans);
    __shared__ float s_mean;
    __shared__ unsigned long long s_fallbacks;
    const unsigned long long rows = *count;
    for (unsigned long long i = blockIdx.x; i < rows; i += gridDim.x)
        apply_flagged_row(d, p, flagged[i], loc, scale, inv, mask, time_flags, work, counters, sv, contrib, s_mean,
                          s_fallbacks);
}

// ---- re-measure and normalise ---------------------------------------------

template <int D>
__global__ void k_unpack(Dims d, const uint8_t* __restrict__ raw, float* __restrict__ work) {
    const uint64_t i      = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t total  = d.nsamps * d.nchans;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t j = i; j < total; j += stride) {
        const uint64_t t = j / d.nchans, c = j % d.nchans;
        work[j]          = rd<D>(raw + t * d.row_bytes, c);
    }
}

// Division in the Welford re-measure. The reference updates
// mean += (x - mean) / n in double. A dependent double division costs
// ~400 cycles on sm_100; the division by the count is instead
// q = RN(delta * y_hi + RN(delta * y_lo)) (one multiply, one fused
// multiply-add), with y_hi = RN(1/n) and y_lo = RN((1 - n y_hi) / n) from
// the host (1 - n y_hi is exact in double). y_hi + y_lo is within 2^-105 / n
// of 1/n and the product's rounding adds at most 2^-105 |delta| / n, so the
// value rounded is within 2^-104 relative of delta / n; delta / n is never a
// rounding midpoint (n delta-midpoint products need more than 53 bits) and
// lies at least 2^-54 / n relative from every midpoint, far more than
// 2^-104 for n < 2^40, so q is the correctly rounded quotient, as
// Markstein-style corrections argue (P. Markstein, IBM J. Res. Develop. 34,
// 1990; Muller et al., Handbook of Floating-Point Arithmetic, ch. 4). Tiny
// nonzero |delta| (where delta * y_lo could lose bits) takes the plain
// division. The plain division as a call, so the compiler keeps it off the
// common path instead of computing it alongside (if-converting the branch).
__device__ __noinline__ double div_plain(double a, double n) { return a / n; }

// One (window, channel) Welford sequence of the re-measure after a
// transform (lib/cpu/rfi_cpu.cpp:219-238). The mean never becomes -0 (it
// starts at +0 and a rounded sum is -0 only when both terms are), so a zero
// quotient (delta = +-0) leaves it unchanged without a select.
struct WelfordAcc {
    double mean = 0.0, var = 0.0;
    uint64_t b;
    const double* recip; // recip[2n], recip[2n + 1] = y_hi, y_lo of 1/n, or null for the plain division
    __device__ __forceinline__ void step(float xf, uint64_t t) {
        const uint64_t n = t - b + 1;
        if (recip != nullptr)
            step_recip(xf, static_cast<double>(n), recip[2 * n], recip[2 * n + 1]);
        else
            step_plain(xf, static_cast<double>(n));
    }
    __device__ __forceinline__ void step_plain(float xf, double n) {
        const double x     = xf;
        const double delta = x - mean;
        mean += div_plain(delta, n);
        var += delta * (x - mean);
    }
    /** step_recip without the tiny-numerator branch: `bad` records that
     * the step needed it (the caller then redoes the steps with it). */
    __device__ __forceinline__ void step_fast(float xf, double yh, double yl, bool& bad) {
        const double x     = xf;
        const double delta = x - mean;
        bad |= !(fabs(delta) > 0x1p-900) && delta != 0.0;
        mean += fma(delta, yh, delta * yl);
        var += delta * (x - mean);
    }
    /** The update for the n-th sample given the two-term reciprocal of n. */
    __device__ __forceinline__ void step_recip(float xf, double n, double yh, double yl) {
        const double x     = xf;
        const double delta = x - mean;
        double q           = fma(delta, yh, delta * yl);
        if (!(fabs(delta) > 0x1p-900) && delta != 0.0)
            q = div_plain(delta, n);
        mean += q;
        var += delta * (x - mean);
    }
};

__global__ void k_welford(Dims d, const float* __restrict__ work, const double* __restrict__ recip,
                          float* __restrict__ loc, float* __restrict__ scale) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t w = blockIdx.y;
    if (c >= d.nchans)
        return;
    const uint64_t b = window_begin(w, d.window), e = window_end(w, d);
    WelfordAcc acc{0.0, 0.0, b, recip};
    for (uint64_t tb = b; tb < e; tb += kBlock) {
        float xs[kBlock];
#pragma unroll
        for (int q = 0; q < kBlock; ++q)
            xs[q] = tb + q < e ? work[(tb + q) * d.nchans + c] : 0.0F;
#pragma unroll
        for (int q = 0; q < kBlock; ++q) {
            if (tb + q >= e)
                break;
            acc.step(xs[q], tb + q);
        }
    }
    loc[w * d.nchans + c]   = static_cast<float>(acc.mean);
    scale[w * d.nchans + c] = e > b ? static_cast<float>(sqrt(acc.var / static_cast<double>(e - b))) : 0.0F;
}

__global__ void __launch_bounds__(kStageChans)
    k_welford_staged(Dims d, const float* __restrict__ work, const double* __restrict__ recip,
                     float* __restrict__ loc, float* __restrict__ scale, int seg_bytes, int rows) {
    extern __shared__ __align__(16) uint8_t stage_buf[];
    __shared__ double2 ys[kDeepStages][kStageChans]; // two-term reciprocals of each stage's rows
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * kStageChans;
    const uint64_t c  = c0 + threadIdx.x;
    const uint64_t w  = blockIdx.y;
    const bool in     = c < d.nchans;
    const uint64_t b = window_begin(w, d.window), e = window_end(w, d);
    WelfordAcc acc{0.0, 0.0, b, recip};
    const uint64_t pitch = d.nchans * sizeof(float);
    const uint64_t left  = pitch - c0 * sizeof(float);
    const int copy       = static_cast<int>(left < static_cast<uint64_t>(seg_bytes) ? left : seg_bytes);
    const int stride     = seg_bytes / static_cast<int>(sizeof(float));
    stage::StagerN<kDeepStages> st(stage_buf, reinterpret_cast<const uint8_t*>(work + c0), pitch, seg_bytes,
                                   copy, rows, b, e);
    // The reciprocals of a stage's counts are read into shared memory with
    // the stage, so no load sits on the sequential update chain.
    auto load_recip = [&](int k) {
        if (k < st.nblk && static_cast<int>(threadIdx.x) < st.rows_of(k)) {
            const uint64_t n = st.t0(k) - b + 1 + threadIdx.x;
            ys[k % kDeepStages][threadIdx.x] = recip != nullptr ? make_double2(recip[2 * n], recip[2 * n + 1])
                                                                : make_double2(0.0, 0.0);
        }
    };
    for (int k = 0; k < kDeepStages; ++k)
        load_recip(k);
    st.start();
    for (int k = 0; k < st.nblk; ++k) {
        st.wait(k);
        const float* buf  = reinterpret_cast<const float*>(st.buf(k));
        const int nr      = st.rows_of(k);
        double nd         = static_cast<double>(st.t0(k) - b); // exact below 2^53
        if (in) {
            if (recip != nullptr) {
                // Eight steps at a time without a branch on the update chain;
                // the rare eight with a tiny nonzero numerator are redone with
                // the plain division where it is needed.
                const double2* yk = ys[k % kDeepStages];
                for (int r0 = 0; r0 < nr; r0 += 8) {
                    const double m0 = acc.mean, v0 = acc.var;
                    bool bad        = false;
                    if (r0 + 8 <= nr) {
#pragma unroll
                        for (int r = r0; r < r0 + 8; ++r)
                            acc.step_fast(buf[r * stride + threadIdx.x], yk[r].x, yk[r].y, bad);
                    } else {
                        for (int r = r0; r < nr; ++r)
                            acc.step_fast(buf[r * stride + threadIdx.x], yk[r].x, yk[r].y, bad);
                    }
                    if (bad) {
                        acc.mean = m0;
                        acc.var  = v0;
                        for (int r = r0; r < min(r0 + 8, nr); ++r)
                            acc.step_recip(buf[r * stride + threadIdx.x], nd + (r + 1), yk[r].x, yk[r].y);
                    }
                }
            } else {
                for (int r = 0; r < nr; ++r) {
                    nd += 1.0;
                    acc.step_plain(buf[r * stride + threadIdx.x], nd);
                }
            }
        }
        st.release(k);
        load_recip(k + kDeepStages);
    }
    if (in) {
        loc[w * d.nchans + c] = static_cast<float>(acc.mean);
        scale[w * d.nchans + c] =
            e > b ? static_cast<float>(sqrt(acc.var / static_cast<double>(e - b))) : 0.0F;
    }
}

constexpr int kTile = 32;

// Normalise + transpose (lib/cpu/rfi_cpu.cpp:242-255): out[c][t] =
// (work[t][c] - loc) * (scale > 0 ? 1 / scale : 1) per (window, channel),
// masked channels zero. A block covers 32 channels and kNormSpan samples
// in 32 x 32 tiles through shared memory; each thread keeps its channel's
// window constants and reloads them only when its rows cross into the next
// window.
constexpr int kNormSpan = 256;

__global__ void k_normalize(Dims d, const float* __restrict__ work, const float* __restrict__ loc,
                            const float* __restrict__ scale, const uint8_t* __restrict__ mask,
                            int flip, uint64_t capacity, float* __restrict__ out) {
    __shared__ float tile[kTile][kTile + 1];
    const uint64_t n  = d.nchans;
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.y) * kTile;
    const uint64_t c  = c0 + threadIdx.x;
    const bool on     = c < n && mask[c] != 0;
    uint64_t wend     = 0;
    float l = 0.0F, is = 1.0F;
    const uint64_t span0 = static_cast<uint64_t>(blockIdx.x) * kNormSpan;
    for (uint64_t t0 = span0; t0 < span0 + kNormSpan && t0 < capacity; t0 += kTile) {
        for (int k = threadIdx.y; k < kTile; k += blockDim.y) {
            const uint64_t t = t0 + k;
            float v          = 0.0F;
            if (t < d.nsamps && on) {
                if (t >= wend) {
                    const uint64_t w = window_of(t, d.window, d.nwin);
                    wend             = window_end(w, d);
                    l                = loc[w * n + c];
                    const float sc   = scale[w * n + c];
                    is               = sc > 0.0F ? 1.0F / sc : 1.0F;
                }
                v = (work[t * n + c] - l) * is;
            }
            tile[k][threadIdx.x] = v;
        }
        __syncthreads();
        const uint64_t t = t0 + threadIdx.x;
        if (t < capacity) {
            for (int k = threadIdx.y; k < kTile; k += blockDim.y) {
                const uint64_t cc = c0 + k;
                if (cc < n) {
                    const uint64_t dst      = flip ? n - 1 - cc : cc;
                    out[dst * capacity + t] = tile[threadIdx.x][k];
                }
            }
        }
        __syncthreads();
    }
}

// The same with 64 x 64 tiles and 16-byte loads and stores (nchans and the
// output capacity multiples of 4): a thread reads 4 channels of a row and
// writes 4 samples of a channel.
constexpr int kNT = 64;

__global__ void __launch_bounds__(256)
    k_normalize4(Dims d, const float* __restrict__ work, const float* __restrict__ loc,
                 const float* __restrict__ scale, const uint8_t* __restrict__ mask, int flip,
                 uint64_t capacity, float* __restrict__ out) {
    __shared__ float tile[kNT][kNT + 1]; // [channel][time]
    const uint64_t n  = d.nchans;
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.y) * kNT;
    const int q       = threadIdx.x % 16; // channel quad (load) / sample quad (store)
    const int r       = threadIdx.x / 16; // row (load) / channel (store) offset, 0..15
    const uint64_t c  = c0 + 4 * q;
    bool on[4];
#pragma unroll
    for (int e = 0; e < 4; ++e)
        on[e] = c + e < n && mask[c + e] != 0;
    uint64_t wend = 0;
    float l[4] = {0, 0, 0, 0}, is[4] = {1, 1, 1, 1};
    const uint64_t span0 = static_cast<uint64_t>(blockIdx.x) * kNormSpan;
    for (uint64_t t0 = span0; t0 < span0 + kNormSpan && t0 < capacity; t0 += kNT) {
#pragma unroll
        for (int pass = 0; pass < kNT / 16; ++pass) {
            const int tl     = r + 16 * pass;
            const uint64_t t = t0 + tl;
            float v[4]       = {0, 0, 0, 0};
            if (t < d.nsamps && c < n) {
                if (t >= wend) {
                    const uint64_t w = window_of(t, d.window, d.nwin);
                    wend             = window_end(w, d);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        l[e]           = loc[w * n + c + e];
                        const float sc = scale[w * n + c + e];
                        is[e]          = sc > 0.0F ? 1.0F / sc : 1.0F;
                    }
                }
                const float4 x = *reinterpret_cast<const float4*>(work + t * n + c);
                const float xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    v[e] = on[e] ? (xs[e] - l[e]) * is[e] : 0.0F;
            }
#pragma unroll
            for (int e = 0; e < 4; ++e)
                tile[4 * q + e][tl] = v[e];
        }
        __syncthreads();
        const uint64_t t = t0 + 4 * q;
        if (t < capacity) {
#pragma unroll
            for (int pass = 0; pass < kNT / 16; ++pass) {
                const int cl      = r + 16 * pass;
                const uint64_t cc = c0 + cl;
                if (cc < n) {
                    const uint64_t dst = flip ? n - 1 - cc : cc;
                    const float4 o = make_float4(tile[cl][4 * q], tile[cl][4 * q + 1], tile[cl][4 * q + 2],
                                                 tile[cl][4 * q + 3]);
                    *reinterpret_cast<float4*>(out + dst * capacity + t) = o;
                }
            }
        }
        __syncthreads();
    }
}

__global__ void k_normalize_short(Dims d, ApplyParams p, const float* __restrict__ work,
                                  const float* __restrict__ tl, const float* __restrict__ ts,
                                  const float* __restrict__ tol, const float* __restrict__ tos,
                                  const uint8_t* __restrict__ mask, const float* __restrict__ za,
                                  const float* __restrict__ zb, int flip, uint64_t capacity,
                                  float* __restrict__ out) {
    extern __shared__ unsigned char smem[];
    const uint64_t n = d.nchans;
    float* z         = reinterpret_cast<float*>(smem);
    __shared__ float band_mean;
    const uint64_t t = blockIdx.x;
    for (uint64_t c = threadIdx.x; c < n; c += blockDim.x)
        z[c] = (work[t * n + c] - tl[c]) * (ts[c] > 0.0F ? 1.0F / ts[c] : 1.0F);
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum     = 0.0;
        uint64_t count = 0;
        for (uint64_t c = 0; c < n; ++c) {
            if (mask[c] && ts[c] > 0.0F && fabsf(z[c]) <= p.clip) {
                sum += z[c];
                ++count;
            }
        }
        band_mean = count ? static_cast<float>(sum / static_cast<double>(count)) : 0.0F;
    }
    __syncthreads();
    for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
        if (!mask[c])
            continue;
        float term = 0.0F;
        if (p.zero_dm == FROST_ZERO_DM_SUBTRACT)
            term = band_mean;
        else if (p.zero_dm == FROST_ZERO_DM_ZDOT)
            term = za[c] * band_mean + zb[c];
        const float x = work[t * n + c];
        const float transformed = ts[c] <= 0.0F ? x
                                  : p.equalize  ? p.eq_loc + p.eq_scale * (z[c] - term)
                                  : p.transform ? tl[c] + ts[c] * (z[c] - term)
                                                : x;
        const float s      = tos[c] > 0.0F ? 1.0F / tos[c] : 1.0F;
        const uint64_t dst = flip ? n - 1 - c : c;
        out[dst * capacity + t] = (transformed - tol[c]) * s;
    }
}

unsigned grid1(uint64_t n, unsigned block) { return static_cast<unsigned>((n + block - 1) / block); }

std::atomic<uint64_t> g_launches{0};

} // namespace

#define FB_COUNT_LAUNCH()                                                                         \
    do {                                                                                          \
        FB_LAUNCH_CHECK();                                                                        \
        g_launches.fetch_add(1, std::memory_order_relaxed);                                       \
    } while (0)

uint64_t launch_counter() { return g_launches.load(std::memory_order_relaxed); }

// ---- launchers ----------------------------------------------------------------

static void set_smem(const void* fn, size_t bytes) {
    if (bytes > 48 * 1024)
        allow_large_smem(fn);
}

void launch_check_finite(const uint8_t* raw, uint64_t nwords, unsigned long long* first_bad,
                         cudaStream_t s) {
    if (nwords == 0)
        return;
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((nwords + 255) / 256, 148 * 16));
    k_check_finite<<<blocks, 256, 0, s>>>(reinterpret_cast<const uint32_t*>(raw), nwords, first_bad);
    FB_COUNT_LAUNCH();
}

void launch_sample_rows(const Dims& d, const uint8_t* raw, float* samples, cudaStream_t s) {
    const dim3 grid(kMaxBandpassRows, static_cast<unsigned>(d.nwin));
    FB_DISPATCH(d.dtype, k_sample_rows<D><<<grid, 256, 0, s>>>(d, raw, samples));
    FB_COUNT_LAUNCH();
}

void launch_bandpass(const Dims& d, const float* samples, float* loc, float* scale, float* inv,
                     uint32_t* unmeasured, cudaStream_t s) {
    const uint64_t pitch = d.nchans * sizeof(float);
    if (pitch % 16 != 0 || reinterpret_cast<uintptr_t>(samples) % 16 != 0) {
        const dim3 grid(grid1(d.nchans, 64), static_cast<unsigned>(d.nwin));
        k_bandpass<<<grid, 64, 0, s>>>(d, samples, loc, scale, inv, unmeasured);
    } else {
        // level and flat flag, then the scale, then the clipped refinement
        const dim3 rgrid(grid1(d.nchans, 32), static_cast<unsigned>(d.nwin));
        k_remedian<false><<<rgrid, 32 * kRemedianWarps, 0, s>>>(d, samples, loc, scale, inv);
        FB_COUNT_LAUNCH();
        k_remedian<true><<<rgrid, 32 * kRemedianWarps, 0, s>>>(d, samples, loc, scale, inv);
        FB_COUNT_LAUNCH();
        const int seg     = static_cast<int>(std::min<uint64_t>(kBandChans * sizeof(float), pitch));
        const int rows    = std::max(8, 16384 / seg);
        const size_t smem = kDeepStages * static_cast<size_t>(seg) * rows;
        const dim3 grid(grid1(d.nchans, kBandChans), static_cast<unsigned>(d.nwin));
        set_smem(reinterpret_cast<const void*>(&k_bandpass_staged), smem);
        k_bandpass_staged<<<grid, kBandChans, smem, s>>>(d, samples, loc, scale, inv, unmeasured, seg, rows);
    }
    FB_COUNT_LAUNCH();
}

// Staging geometry of a kStageChans-channel column segment: bytes per row
// and rows per stage (about kStageBytes per buffer), or seg_bytes = 0 when
// the layout cannot be staged with 16-byte copies.
constexpr int kStageBytes = 16 * 1024;

struct StageGeom {
    int seg_bytes = 0, rows = 0;
    size_t smem() const { return 2 * static_cast<size_t>(seg_bytes) * rows; }
    size_t smem_deep() const { return kDeepStages * static_cast<size_t>(seg_bytes) * rows; }
};

bool aligned16(const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

StageGeom stage_geom(const void* base, uint64_t row_bytes, int bits) {
    StageGeom g;
    const uint64_t full = static_cast<uint64_t>(kStageChans) * bits / 8;
    if (!aligned16(base) || row_bytes % 16 != 0 || full % 16 != 0)
        return g;
    // every segment starts on a 16-byte boundary; the last may be shorter
    g.seg_bytes = static_cast<int>(std::min<uint64_t>(full, row_bytes));
    g.rows      = std::max(8, std::min(256, kStageBytes / g.seg_bytes));
    return g;
}

void launch_moments(const Dims& d, const uint8_t* raw, const float* loc, const float* inv,
                    const uint8_t* static_mask, float clip, MomentSums* out, cudaStream_t s) {
    const StageGeom g = stage_geom(raw, d.row_bytes, bits_of(d.dtype));
    if (g.seg_bytes == 0) {
        const dim3 grid(grid1(d.nchans, 64), static_cast<unsigned>(d.nwin));
        FB_DISPATCH(d.dtype, k_moments<D><<<grid, 64, 0, s>>>(d, raw, loc, inv, static_mask, clip, out));
    } else {
        const dim3 grid(grid1(d.nchans, kStageChans), static_cast<unsigned>(d.nwin));
        FB_DISPATCH(d.dtype, {
            set_smem(reinterpret_cast<const void*>(&k_moments_staged<D>), g.smem_deep());
            k_moments_staged<D><<<grid, kStageChans, g.smem_deep(), s>>>(d, raw, loc, inv, static_mask, clip, out,
                                                                        g.seg_bytes, g.rows);
        });
    }
    FB_COUNT_LAUNCH();
}

void launch_scan_rows(const Dims& d, const uint8_t* raw, const float* loc, const float* inv,
                      const uint8_t* mask, float clip, const KspecParams& kp,
                      const uint64_t* good_prefix, float* s_det, double* s_keep_d, float* s_keep_f,
                      float* row_std, Span32* kspec_pos, Span32* kspec_neg, uint8_t* kspec_whole,
                      uint8_t* row_clip, cudaStream_t s) {
    if (d.nchans >= (uint64_t{1} << 31))
        throw Error(FROST_ERR_INVALID_ARGUMENT, "scan: too many channels for 32-bit channel indices");
    const unsigned grid = grid1(d.nsamps, kScanRows);
    if (d.row_bytes % 16 != 0 || reinterpret_cast<uintptr_t>(raw) % 16 != 0) {
        FB_DISPATCH(d.dtype, k_scan_rows<D><<<grid, kScanRows, 0, s>>>(
                                 d, raw, loc, inv, mask, clip, kp, good_prefix, s_det, s_keep_d,
                                 s_keep_f, row_std, kspec_pos, kspec_neg, kspec_whole, row_clip));
    } else {
        const size_t smem = 2 * static_cast<size_t>(kScanRows) * kRowTileStride;
        FB_DISPATCH(d.dtype, {
            set_smem(reinterpret_cast<const void*>(&k_scan_rows_staged<D>), smem);
            k_scan_rows_staged<D><<<grid, kScanRows, smem, s>>>(
                d, raw, loc, inv, mask, clip, kp, good_prefix, s_det, s_keep_d, s_keep_f, row_std,
                kspec_pos, kspec_neg, kspec_whole, row_clip);
        });
    }
    FB_COUNT_LAUNCH();
}

void launch_scan_cols(const Dims& d, const uint8_t* raw, const float* loc, const float* inv,
                      const uint8_t* mask, float clip, const double* s_keep_d, int zdot, int kchan,
                      const float* clip_mean, const float* clip_inv_std, float* chunk_min,
                      float* chunk_max, ZdotSums* chunk_zdot, KadaneState* chunk_kpos,
                      KadaneState* chunk_kneg, float* lo, float* hi, ZdotSums* zdot_sum,
                      Run* kpos_best, Run* kneg_best, cudaStream_t s) {
    if (d.nsamps >= (uint64_t{1} << 31))
        throw Error(FROST_ERR_INVALID_ARGUMENT, "scan: too many samples for 32-bit time indices");
    const StageGeom g = stage_geom(raw, d.row_bytes, bits_of(d.dtype));
    if (g.seg_bytes == 0) {
        const dim3 grid(grid1(d.nchans, 64), static_cast<unsigned>(d.nchunks));
        FB_DISPATCH(d.dtype, k_scan_cols<D><<<grid, 64, 0, s>>>(
                                 d, raw, loc, inv, mask, clip, s_keep_d, zdot, kchan, clip_mean,
                                 clip_inv_std, chunk_min, chunk_max, chunk_zdot, chunk_kpos,
                                 chunk_kneg));
    } else {
        const dim3 grid(grid1(d.nchans, kStageChans), static_cast<unsigned>(d.nchunks));
        FB_DISPATCH(d.dtype, k_scan_cols_staged<D><<<grid, kStageChans, g.smem(), s>>>(
                                 d, raw, loc, inv, mask, clip, s_keep_d, zdot, kchan, clip_mean,
                                 clip_inv_std, chunk_min, chunk_max, chunk_zdot, chunk_kpos,
                                 chunk_kneg, g.seg_bytes, g.rows));
    }
    FB_COUNT_LAUNCH();
    k_combine_chunks<<<grid1(d.nchans, 128), 128, 0, s>>>(d, zdot, kchan, chunk_min, chunk_max,
                                                          chunk_zdot, chunk_kpos, chunk_kneg, lo,
                                                          hi, zdot_sum, kpos_best, kneg_best);
    FB_COUNT_LAUNCH();
}


namespace {
// row_kchan[t] = 1 for the rows a channel's Kadane-along-time segment
// covers (the caller zeroes it): CTA 2c + k takes channel c's positive
// (k = 0) or negative segment.
__global__ void __launch_bounds__(256)
    k_kchan_rows(uint64_t nchans, uint64_t nsamps, const Segment* __restrict__ kchan_pos,
                 const Segment* __restrict__ kchan_neg, const uint8_t* __restrict__ kchan_any,
                 uint8_t* __restrict__ row_kchan) {
    const uint64_t c = blockIdx.x >> 1;
    if (c >= nchans || kchan_any[c] == 0)
        return;
    const Segment g  = (blockIdx.x & 1) == 0 ? kchan_pos[c] : kchan_neg[c];
    const int64_t lo = g.start < 0 ? 0 : g.start;
    const int64_t hi = g.end < static_cast<int64_t>(nsamps) ? g.end : static_cast<int64_t>(nsamps) - 1;
    for (int64_t t = lo + threadIdx.x; t <= hi; t += blockDim.x)
        row_kchan[t] = 1;
}
} // namespace

void launch_kchan_rows(const Dims& d, const Segment* kchan_pos, const Segment* kchan_neg,
                       const uint8_t* kchan_any, uint8_t* row_kchan, cudaStream_t s) {
    FB_CUDA(cudaMemsetAsync(row_kchan, 0, d.nsamps, s));
    if (d.nsamps == 0 || d.nchans == 0)
        return;
    k_kchan_rows<<<static_cast<unsigned>(2 * d.nchans), 256, 0, s>>>(d.nchans, d.nsamps, kchan_pos, kchan_neg,
                                                                     kchan_any, row_kchan);
    FB_COUNT_LAUNCH();
}

void launch_apply_unflagged(const Dims& d, const ApplyParams& p, const uint8_t* raw,
                            const float* loc, const float* scale, const float* inv,
                            const uint8_t* mask, const uint8_t* time_flags, const Span32* kspec_pos,
                            const Span32* kspec_neg, const Segment* kchan_pos,
                            const Segment* kchan_neg, const uint8_t* kchan_any,
                            const float* s_keep_f, const float* zdot_a,
                            const float* zdot_b, const uint8_t* row_clip, const uint8_t* row_kchan,
                            uint32_t* slow_rows, unsigned int* nslow, float* work,
                            unsigned long long* counters, cudaStream_t s) {
    const size_t smem = d.nchans * (sizeof(float) + 1);
    if (d.nsamps == 0)
        return;
    if (d.nchans >= (uint64_t{1} << 31) || d.nsamps >= (uint64_t{1} << 31))
        throw Error(FROST_ERR_INVALID_ARGUMENT, "apply: too many channels or samples for one block");
    FB_CUDA(cudaMemsetAsync(nslow, 0, sizeof(unsigned int), s));
    // 4-channel vectors need nchans % 4 == 0 and, for the byte loads of the
    // raw row, a 4-byte aligned block
    const bool vec = d.nchans % 4 == 0 && reinterpret_cast<uintptr_t>(raw) % 4 == 0;
    int dev = 0, sms = 0;
    FB_CUDA(cudaGetDevice(&dev));
    FB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // the listed rows: a few CTAs an SM loop over them (the count is read on the device)
    const unsigned slow_grid = static_cast<unsigned>(std::min<uint64_t>(d.nsamps, static_cast<uint64_t>(sms) * 4));
    FB_DISPATCH(d.dtype, {
        if (vec) {
            k_apply_clean<D, 4><<<static_cast<unsigned>(d.nsamps), 256, 0, s>>>(
                d, p, raw, loc, scale, inv, mask, time_flags, kspec_pos, kspec_neg, s_keep_f, zdot_a, zdot_b,
                row_clip, row_kchan, work, slow_rows, nslow);
            set_smem(reinterpret_cast<const void*>(&k_apply_unflagged<D, 4>), smem);
            k_apply_unflagged<D, 4><<<slow_grid, 256, smem, s>>>(
                d, p, raw, loc, scale, inv, mask, time_flags, kspec_pos, kspec_neg, kchan_pos,
                kchan_neg, kchan_any, s_keep_f, zdot_a, zdot_b, slow_rows, nslow, work, counters);
        } else {
            k_apply_clean<D, 1><<<static_cast<unsigned>(d.nsamps), 256, 0, s>>>(
                d, p, raw, loc, scale, inv, mask, time_flags, kspec_pos, kspec_neg, s_keep_f, zdot_a, zdot_b,
                row_clip, row_kchan, work, slow_rows, nslow);
            set_smem(reinterpret_cast<const void*>(&k_apply_unflagged<D, 1>), smem);
            k_apply_unflagged<D, 1><<<slow_grid, 256, smem, s>>>(
                d, p, raw, loc, scale, inv, mask, time_flags, kspec_pos, kspec_neg, kchan_pos,
                kchan_neg, kchan_any, s_keep_f, zdot_a, zdot_b, slow_rows, nslow, work, counters);
        }
    });
    FB_COUNT_LAUNCH();
    FB_COUNT_LAUNCH();
}

void launch_apply_flagged(const Dims& d, const ApplyParams& p, const uint64_t* flagged,
                          const unsigned long long* nflagged, const float* loc, const float* scale,
                          const float* inv, const uint8_t* mask, const uint8_t* time_flags,
                          float* work, unsigned long long* counters, cudaStream_t s) {
    if (d.nsamps == 0)
        return;
    const size_t smem     = d.nchans * (sizeof(float) + 1);
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>(d.nsamps, 148 * 8));
    set_smem(reinterpret_cast<const void*>(&k_apply_flagged), smem);
    k_apply_flagged<<<blocks, 256, smem, s>>>(d, p, flagged, nflagged, loc, scale, inv, mask, time_flags, work,
                                              counters);
    FB_COUNT_LAUNCH();
}

void launch_unpack(const Dims& d, const uint8_t* raw, float* work, cudaStream_t s) {
    const uint64_t total = d.nsamps * d.nchans;
    if (total == 0)
        return;
    const unsigned blocks = static_cast<unsigned>(std::min<uint64_t>((total + 255) / 256, 148 * 32));
    FB_DISPATCH(d.dtype, k_unpack<D><<<blocks, 256, 0, s>>>(d, raw, work));
    FB_COUNT_LAUNCH();
}

void launch_welford(const Dims& d, const float* work, const double* recip, float* loc, float* scale,
                    cudaStream_t s) {
    const StageGeom g = stage_geom(work, d.nchans * sizeof(float), 32);
    if (g.seg_bytes == 0) {
        const dim3 grid(grid1(d.nchans, 64), static_cast<unsigned>(d.nwin));
        k_welford<<<grid, 64, 0, s>>>(d, work, recip, loc, scale);
    } else {
        const dim3 grid(grid1(d.nchans, kStageChans), static_cast<unsigned>(d.nwin));
        // a stage's reciprocals are loaded one per thread
        const int rows    = std::min(g.rows, kStageChans);
        const size_t smem = kDeepStages * static_cast<size_t>(g.seg_bytes) * rows;
        set_smem(reinterpret_cast<const void*>(&k_welford_staged), smem);
        k_welford_staged<<<grid, kStageChans, smem, s>>>(d, work, recip, loc, scale, g.seg_bytes, rows);
    }
    FB_COUNT_LAUNCH();
}

void launch_normalize(const Dims& d, const float* work, const float* loc, const float* scale,
                      const uint8_t* mask, int flip, uint64_t capacity, float* out, cudaStream_t s) {
    if (d.nchans % 4 == 0 && capacity % 4 == 0) {
        const dim3 grid(grid1(capacity, kNormSpan), grid1(d.nchans, kNT));
        k_normalize4<<<grid, 256, 0, s>>>(d, work, loc, scale, mask, flip, capacity, out);
    } else {
        const dim3 grid(grid1(capacity, kNormSpan), grid1(d.nchans, kTile));
        k_normalize<<<grid, dim3(kTile, 8), 0, s>>>(d, work, loc, scale, mask, flip, capacity, out);
    }
    FB_COUNT_LAUNCH();
}

void launch_normalize_short(const Dims& d, const ApplyParams& p, const float* work,
                            const float* tail_loc, const float* tail_scale,
                            const float* tail_out_loc, const float* tail_out_scale,
                            const uint8_t* mask, const float* zdot_a, const float* zdot_b,
                            int flip, uint64_t capacity, float* out, cudaStream_t s) {
    if (d.nsamps == 0)
        return;
    const size_t smem = d.nchans * sizeof(float);
    set_smem(reinterpret_cast<const void*>(&k_normalize_short), smem);
    k_normalize_short<<<static_cast<unsigned>(d.nsamps), 256, smem, s>>>(
        d, p, work, tail_loc, tail_scale, tail_out_loc, tail_out_scale, mask, zdot_a, zdot_b, flip,
        capacity, out);
    FB_COUNT_LAUNCH();
}

} // namespace fb::rfi
