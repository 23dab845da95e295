// Per-gulp RFI decisions on the device (see rfi_decide.hpp).
//
// Layout of the work:
//  * channel mask: one thread per channel folds the window moment sums into
//    the five moment statistics and the IQRM statistic; then one CTA per
//    sort job — each enabled moment statistic, and each (lag, sign) of IQRM
//    — sorts its values (bitonic network in shared memory, or in global
//    scratch for very wide bands) and takes the interpolated quartiles;
//    finally one CTA combines the outlier flags, resolves the IQRM votes,
//    grows the mask and writes mask and prefix counts.
//  * time flags: the broad-band detector's baseline resampling and
//    subtraction run as grid-wide passes of sizes planned on the host from
//    the gulp length; the MAD and the dropout median are exact radix
//    selections in one CTA; the boxcar ladder runs one CTA per width over a
//    bit-packed detection mask with word prefix counts; the per-sample flag
//    merges are grid-wide.
// Every arithmetic expression that decides a flag keeps the association and
// the float/double types of frost's CPU code; the file is compiled
// --fmad=false so no multiply-add is contracted.

#include "rfi_decide.hpp"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>

namespace fb::rfi {

namespace {

std::atomic<uint64_t> g_launches{0};

#define FB_DECIDE_LAUNCH()                                                                        \
    do {                                                                                          \
        FB_LAUNCH_CHECK();                                                                        \
        g_launches.fetch_add(1, std::memory_order_relaxed);                                      \
    } while (0)

constexpr int kBlock            = 1024;
constexpr size_t kSortSmemBytes = 128 * 1024;
constexpr float kMadNorm        = 0.6744897501960817F; // Phi^-1(3/4)
constexpr int kMaxVoteSlots     = 128;

unsigned grid_for(uint64_t n, unsigned block) {
    const uint64_t g = (n + block - 1) / block;
    return static_cast<unsigned>(std::max<uint64_t>(std::min<uint64_t>(g, 148ULL * 64), 1));
}

uint64_t pow2_at_least(uint64_t n) {
    uint64_t p = 1;
    while (p < n)
        p <<= 1;
    return p;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t{255}; }

// ---- block helpers (blockDim.x a multiple of 32, at most 1024) ------------

template <typename T> __device__ T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xFFFFFFFFU, v, o);
    return v;
}

/** Sum over the block; every thread gets the total. `red` holds 32 T. */
template <typename T> __device__ T block_sum(T v, T* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0)
        red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        T s = lane < nw ? red[lane] : T(0);
        s   = warp_sum(s);
        if (lane == 0)
            red[0] = s;
    }
    __syncthreads();
    const T total = red[0];
    __syncthreads();
    return total;
}

/** Exclusive scan of one value per thread (thread order); *total gets the
 * block's sum. `red` holds 32 T. */
template <typename T> __device__ T block_exclusive_scan(T v, T* red, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xFFFFFFFFU, x, o);
        if (lane >= o)
            x += y;
    }
    __syncthreads();
    if (lane == 31)
        red[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T s = lane < nw ? red[lane] : T(0);
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xFFFFFFFFU, s, o);
            if (lane >= o)
                s += y;
        }
        red[lane] = s;
    }
    __syncthreads();
    const T before = warp > 0 ? red[warp - 1] : T(0);
    *total         = red[nw - 1];
    __syncthreads();
    return before + x - v;
}

/** Ascending bitonic sort of a[0..P), P a power of two (+inf pads). */
__device__ void block_bitonic_sort(double* a, uint64_t P) {
    __syncthreads();
    for (uint64_t k = 2; k <= P; k <<= 1) {
        for (uint64_t j = k >> 1; j > 0; j >>= 1) {
            for (uint64_t i = threadIdx.x; i < P; i += blockDim.x) {
                const uint64_t l = i ^ j;
                if (l > i) {
                    const double x = a[i], y = a[l];
                    const bool up  = (i & k) == 0;
                    if (up ? (x > y) : (x < y)) {
                        a[i] = y;
                        a[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

/** numpy-style (linear interpolation) quantile of ascending s[0..m),
 * frost's quantile_sorted (lib/cpu/rfi_kernels.hpp:136-142). */
__device__ double quantile_of(const double* s, uint64_t m, double q) {
    const double h    = static_cast<double>(m - 1) * q;
    const auto lo     = static_cast<uint64_t>(h);
    const uint64_t hi = lo + 1 < m - 1 ? lo + 1 : m - 1;
    const double fr   = h - static_cast<double>(lo);
    return s[lo] + (fr * (s[hi] - s[lo]));
}

// Order-preserving 32-bit keys of non-NaN floats.
__device__ __forceinline__ uint32_t order_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000U) ? ~b : (b | 0x80000000U);
}
__device__ __forceinline__ float key_value(uint32_t k) {
    return __uint_as_float((k & 0x80000000U) ? (k & 0x7FFFFFFFU) : ~k);
}

/** The rank-th smallest (0-based) of x[0..count) (|x| when ABS) by an MSB
 * first radix selection over order keys: the element std::nth_element
 * would put at position `rank`. Whole block; `hist` holds 256 words. */
template <bool ABS>
__device__ float block_select(const float* __restrict__ x, uint64_t count, uint64_t rank, uint32_t* hist,
                              uint64_t* s_rank, uint32_t* s_bin) {
    uint32_t prefix = 0, pmask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x)
            hist[i] = 0;
        __syncthreads();
        // eight loads in flight per thread (one CTA streams the whole
        // series), then one shared-memory atomic per bin a warp's keys fall
        // in (most keys share their top bytes)
        constexpr int kU = 8;
        for (uint64_t base = 0; base < count; base += static_cast<uint64_t>(blockDim.x) * kU) {
            float v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const uint64_t i = base + static_cast<uint64_t>(u) * blockDim.x + threadIdx.x;
                v[u]             = i < count ? x[i] : 0.0F;
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const uint64_t i = base + static_cast<uint64_t>(u) * blockDim.x + threadIdx.x;
                uint32_t bin     = 256U; // none
                if (i < count) {
                    const uint32_t k = order_key(ABS ? fabsf(v[u]) : v[u]);
                    if ((k & pmask) == prefix)
                        bin = (k >> shift) & 255U;
                }
                const unsigned peers = __match_any_sync(0xFFFFFFFFU, bin);
                if (bin < 256U && static_cast<int>(threadIdx.x & 31U) == __ffs(static_cast<int>(peers)) - 1)
                    atomicAdd(&hist[bin], static_cast<uint32_t>(__popc(peers)));
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t acc = 0;
            uint32_t b   = 0;
            for (; b < 255; ++b) {
                if (acc + hist[b] > rank)
                    break;
                acc += hist[b];
            }
            *s_bin  = b;
            *s_rank = rank - acc;
        }
        __syncthreads();
        prefix |= *s_bin << shift;
        pmask |= 0xFFU << shift;
        rank = *s_rank;
        __syncthreads();
    }
    return key_value(prefix);
}

/** The element of rank `rank - 1` given the element `v` of rank `rank`
 * (|x| when ABS): v itself when fewer than `rank` elements lie below it,
 * else the largest element below it (one pass instead of a second
 * selection). */
template <bool ABS>
__device__ float block_select_prev(const float* __restrict__ x, uint64_t count, uint64_t rank, float v,
                                   unsigned long long* red, uint32_t* s_max) {
    const uint32_t K       = order_key(v);
    unsigned long long below = 0;
    uint32_t best          = 0U;
    constexpr int kU = 8; // loads in flight per thread
    for (uint64_t base = 0; base < count; base += static_cast<uint64_t>(blockDim.x) * kU) {
        float v[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t i = base + static_cast<uint64_t>(u) * blockDim.x + threadIdx.x;
            v[u]             = i < count ? x[i] : 0.0F;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t i = base + static_cast<uint64_t>(u) * blockDim.x + threadIdx.x;
            const uint32_t k = order_key(ABS ? fabsf(v[u]) : v[u]);
            if (i < count && k < K) {
                ++below;
                best = max(best, k);
            }
        }
    }
    if (threadIdx.x == 0)
        *s_max = 0U;
    below = block_sum(below, red); // its barriers also order the reset above
    atomicMax(s_max, best);
    __syncthreads();
    const uint32_t m = *s_max;
    __syncthreads();
    return below >= rank ? key_value(m) : v;
}

// ---- channel mask --------------------------------------------------------

struct SortJobs {
    uint64_t n;
    uint64_t P;  // power of two >= n
    int use_smem;
    int nstat;   // moment statistics to test
    int sid[5];  // their indices
    int niqrm;   // IQRM (lag, sign) jobs
    double k;
    float iqrm_threshold;
};

// Per channel: clipped-moment tables, the five moment statistics of the
// window-summed moments (frost's build_channel_mask arithmetic) and the
// scale-weighted std IQRM tests.
__global__ void k_channel_stats(ChannelMaskParams p, const MomentSums* __restrict__ mom,
                                const float* __restrict__ scale, const uint32_t* __restrict__ unmeasured,
                                const uint8_t* __restrict__ static_mask, float* __restrict__ clip_mean,
                                float* __restrict__ clip_inv, ChannelScratch w) {
    const uint64_t ch = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    const uint64_t n  = p.n;
    if (ch >= n)
        return;
    if (p.need_clip) {
        for (uint64_t win = 0; win < p.nwin; ++win) {
            const MomentSums& sm = mom[win * n + ch];
            float cm = 0.0F, ci = 0.0F;
            if (sm.nc > 1.0) {
                const double mean = sm.c1 / sm.nc;
                const double var  = (sm.c2 / sm.nc) - (mean * mean);
                cm                = static_cast<float>(mean);
                ci                = var > 0.0 ? static_cast<float>(1.0 / sqrt(var)) : 0.0F;
            }
            clip_mean[win * n + ch] = cm;
            clip_inv[win * n + ch]  = ci;
        }
    }
    double st[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    uint8_t good = 0;
    if (p.moments && static_mask[ch] != 0) {
        double sn = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, s4 = 0.0, lag = 0.0, lag_pairs = 0.0;
        for (uint64_t win = 0; win < p.nwin; ++win) {
            const MomentSums& sw = mom[win * n + ch];
            sn += sw.n;
            s1 += sw.s1;
            s2 += sw.s2;
            s3 += sw.s3;
            s4 += sw.s4;
            lag += sw.lag;
            const double pairs = sw.n - 1.0;
            lag_pairs += pairs < 0.0 ? 0.0 : pairs;
        }
        if (sn >= 2.0) {
            const double m1  = s1 / sn;
            const double m2  = s2 / sn;
            const double m3  = s3 / sn;
            const double m4  = s4 / sn;
            const double var = m2 - (m1 * m1);
            if (var > 0.0) {
                good            = 1;
                const double sd = sqrt(var);
                st[0]           = m1;
                st[1]           = sd;
                st[2]           = (m3 - (3.0 * m1 * m2) + (2.0 * m1 * m1 * m1)) / (var * sd);
                st[3] = ((m4 - (4.0 * m1 * m3) + (6.0 * m1 * m1 * m2) - (3.0 * m1 * m1 * m1 * m1)) / (var * var)) -
                        3.0;
                st[4] = lag_pairs > 0.0 ? ((lag / lag_pairs) - (m1 * m1)) / var : 0.0;
            }
        }
    }
    for (int s = 0; s < 5; ++s)
        w.stat[s * n + ch] = st[s];
    w.good[ch] = good;
    if (p.iqrm) {
        w.ignore[ch]  = (static_mask[ch] == 0 || unmeasured[ch] > 0) ? 1 : 0;
        double weight = 0.0, acc = 0.0;
        for (uint64_t win = 0; win < p.nwin; ++win) {
            const MomentSums& sm = mom[win * n + ch];
            if (sm.n > 1.0) {
                const double mean = sm.s1 / sm.n;
                const double var  = (sm.s2 / sm.n) - (mean * mean);
                const double sc   = scale[win * n + ch];
                acc += sm.n * (var < 0.0 ? 0.0 : var) * sc * sc;
                weight += sm.n;
            }
        }
        w.iqrm_x[ch] = weight > 0.0 ? static_cast<float>(sqrt(acc / weight)) : 0.0F;
    }
}

// One sort job per CTA: the IQR outlier test of one moment statistic over
// the good channels (lib/cpu/rfi_cpu_measure.cpp:56-84), or one (lag, sign)
// of IQRM (lib/cpu/rfi_masks_cpu.cpp:64-101): the lagged differences of
// the non-ignored pairs, their quartiles and median, and the votes of the
// channels whose difference exceeds the Tukey cut.
__global__ void __launch_bounds__(kBlock)
    k_channel_sorts(SortJobs j, ChannelScratch w, const float* __restrict__ x, const uint8_t* __restrict__ ign) {
    extern __shared__ double sm_sort[];
    __shared__ unsigned long long red[32];
    const uint64_t n = j.n, P = j.P;
    const int job    = static_cast<int>(blockIdx.x);
    double* a        = j.use_smem ? sm_sort : w.sort_buf + static_cast<uint64_t>(job) * P;
    if (job < j.nstat) {
        const int s          = j.sid[job];
        const double* stat   = w.stat + static_cast<uint64_t>(s) * n;
        unsigned long long m = 0;
        for (uint64_t i = threadIdx.x; i < P; i += blockDim.x) {
            double v = INFINITY;
            if (i < n && w.good[i] != 0) {
                v = stat[i];
                ++m;
            }
            a[i] = v;
        }
        m = block_sum(m, red);
        if (m < 4)
            return;
        block_bitonic_sort(a, P);
        const double q1  = quantile_of(a, m, 0.25);
        const double q3  = quantile_of(a, m, 0.75);
        const double iqr = q3 - q1;
        if (!(iqr > 0.0))
            return;
        const double lo = q1 - (j.k * iqr);
        const double hi = q3 + (j.k * iqr);
        uint8_t* flags  = w.flags + static_cast<uint64_t>(s) * n;
        for (uint64_t i = threadIdx.x; i < n; i += blockDim.x)
            flags[i] = (w.good[i] != 0 && (stat[i] < lo || stat[i] > hi)) ? 1 : 0;
        return;
    }
    const int q       = job - j.nstat;
    const int64_t lag = static_cast<int64_t>(w.lags[q / 2]);
    const int64_t k   = (q % 2 == 0) ? lag : -lag;
    const int64_t ni  = static_cast<int64_t>(n);
    const uint64_t S  = 2 * w.nlags;
    auto partner      = [&](uint64_t i) -> uint64_t {
        int64_t jj = static_cast<int64_t>(i) - k;
        jj         = jj < 0 ? 0 : (jj > ni - 1 ? ni - 1 : jj);
        return static_cast<uint64_t>(jj);
    };
    unsigned long long m = 0;
    for (uint64_t i = threadIdx.x; i < P; i += blockDim.x) {
        double v = INFINITY;
        if (i < n) {
            const uint64_t jj = partner(i);
            if (ign[i] == 0 && ign[jj] == 0) {
                v = static_cast<double>(x[i]) - static_cast<double>(x[jj]);
                ++m;
            }
        }
        a[i] = v;
    }
    m = block_sum(m, red);
    if (m == 0)
        return;
    block_bitonic_sort(a, P);
    const double q1  = quantile_of(a, m, 0.25);
    const double med = quantile_of(a, m, 0.5);
    const double q3  = quantile_of(a, m, 0.75);
    const double cut = static_cast<double>(j.iqrm_threshold) * (q3 - q1) / 1.349;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint64_t jj = partner(i);
        if (ign[i] == 0 && ign[jj] == 0) {
            const double diff = static_cast<double>(x[i]) - static_cast<double>(x[jj]);
            if (diff - med > cut)
                w.votes[i * S + static_cast<uint64_t>(q)] = static_cast<int32_t>(jj);
        }
    }
}

/** The channels that voted against channel i, as a set: one per lag and
 * sign, distinct except for the clamped edge channels 0 and n - 1. */
struct Voters {
    const int32_t* row;
    uint64_t S, n;
    __device__ uint32_t count() const {
        uint32_t r   = 0;
        bool first   = false, last = false;
        const auto l = static_cast<int32_t>(n - 1);
        for (uint64_t q = 0; q < S; ++q) {
            const int32_t v = row[q];
            if (v < 0)
                continue;
            if (v == 0)
                first = true;
            else if (v == l)
                last = true;
            else
                ++r;
        }
        return r + (first ? 1U : 0U) + (last ? 1U : 0U);
    }
    template <typename F> __device__ void each(F&& f) const {
        bool first   = false, last = false;
        const auto l = static_cast<int32_t>(n - 1);
        for (uint64_t q = 0; q < S; ++q) {
            const int32_t v = row[q];
            if (v < 0)
                continue;
            if (v == 0)
                first = true;
            else if (v == l)
                last = true;
            else
                f(static_cast<uint64_t>(v));
        }
        if (first)
            f(uint64_t{0});
        if (last && l != 0)
            f(static_cast<uint64_t>(l));
    }
};

// One CTA: moment flags (and the kurtosis cap) into the dynamic mask, the
// IQRM vote resolution (a channel is flagged when one of its voters cast
// fewer votes than it received), growth, then mask = static & ~dynamic and
// its exclusive prefix counts (lib/cpu/rfi_cpu_measure.cpp:140-300). With a
// null `mask` only the IQRM flags are written, to `iqrm_out`.
__global__ void __launch_bounds__(kBlock)
    k_channel_decide(ChannelMaskParams p, ChannelScratch w, const uint8_t* __restrict__ static_mask,
                     const uint8_t* __restrict__ ign, uint8_t* __restrict__ mask,
                     uint64_t* __restrict__ good_prefix, unsigned long long* __restrict__ counters,
                     uint8_t* __restrict__ iqrm_out) {
    __shared__ unsigned long long red[32];
    __shared__ uint32_t red32[32];
    const uint64_t n = p.n;
    const uint64_t S = 2 * w.nlags;
    unsigned long long cnt = 0;
    for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
        uint8_t dyn = 0;
        if (p.moments) {
            for (int s = 0; s < 5; ++s)
                if (p.stat_on[s] && w.flags[static_cast<uint64_t>(s) * n + c] != 0)
                    dyn = 1;
            if (p.kurt_max > 0.0 && w.good[c] != 0 && fabs(w.stat[3 * n + c]) > p.kurt_max)
                dyn = 1;
        }
        w.dynamic[c] = dyn;
        cnt += dyn;
    }
    cnt = block_sum(cnt, red);
    if (threadIdx.x == 0 && counters != nullptr)
        counters[kRepMoments] = p.moments ? cnt : 0;
    if (p.iqrm) {
        for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
            const Voters v{w.votes + c * S, S, n};
            v.each([&](uint64_t j) { atomicAdd(&w.cast[j], 1U); });
        }
        __syncthreads();
        unsigned long long added = 0;
        for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
            const Voters v{w.votes + c * S, S, n};
            const uint32_t received = v.count();
            bool flag               = ign[c] != 0;
            v.each([&](uint64_t j) {
                if (w.cast[j] < received)
                    flag = true;
            });
            if (iqrm_out != nullptr)
                iqrm_out[c] = flag ? 1 : 0;
            if (flag && ign[c] == 0 && w.dynamic[c] == 0) {
                w.dynamic[c] = 1;
                ++added;
            }
        }
        added = block_sum(added, red);
        if (threadIdx.x == 0 && counters != nullptr)
            counters[kRepIqrm] = added;
    }
    if (mask == nullptr)
        return;
    const uint64_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint64_t c0  = threadIdx.x * per;
    const uint64_t c1  = c0 + per < n ? c0 + per : n;
    if (p.grow > 0) {
        uint32_t local = 0, total = 0;
        for (uint64_t c = c0; c < c1; ++c)
            local += w.dynamic[c] != 0 ? 1U : 0U;
        __syncthreads();
        uint32_t run = block_exclusive_scan(local, red32, &total);
        for (uint64_t c = c0; c < c1; ++c) {
            w.prefix[c] = run;
            run += w.dynamic[c] != 0 ? 1U : 0U;
        }
        if (threadIdx.x == blockDim.x - 1)
            w.prefix[n] = total;
        __syncthreads();
        const uint64_t g         = p.grow;
        unsigned long long grown = 0;
        for (uint64_t c = threadIdx.x; c < n; c += blockDim.x) {
            const uint64_t lo = c > g ? c - g : 0;
            const uint64_t hi = (c + g < n - 1) ? c + g : n - 1;
            if (w.prefix[hi + 1] - w.prefix[lo] > 0 && w.dynamic[c] == 0) {
                if (static_mask[c] != 0)
                    ++grown;
                w.dynamic[c] = 2; // grown
            }
        }
        grown = block_sum(grown, red);
        if (threadIdx.x == 0)
            counters[kRepGrown] = grown;
    }
    __syncthreads();
    unsigned long long local = 0, total = 0;
    for (uint64_t c = c0; c < c1; ++c) {
        const uint8_t keep = (static_mask[c] != 0 && w.dynamic[c] == 0) ? 1 : 0;
        mask[c]            = keep;
        local += keep;
    }
    unsigned long long run = block_exclusive_scan(local, red, &total);
    for (uint64_t c = c0; c < c1; ++c) {
        good_prefix[c] = run;
        run += mask[c];
    }
    if (threadIdx.x == 0) {
        good_prefix[n]       = total;
        counters[kRepMasked] = n - total;
    }
}

// ---- time flags ----------------------------------------------------------

__device__ __forceinline__ bool none_good(const uint64_t* good_prefix, uint64_t n) { return good_prefix[n] == 0; }

__global__ void k_dead(uint64_t n, uint64_t nwin, const uint64_t* __restrict__ good_prefix,
                       const uint32_t* __restrict__ unmeasured, const float* __restrict__ lo,
                       const float* __restrict__ hi, uint8_t* __restrict__ mask,
                       unsigned long long* __restrict__ counters) {
    if (none_good(good_prefix, n))
        return;
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= n)
        return;
    if (mask[c] == 0 || unmeasured[c] < nwin)
        return;
    if (!(hi[c] > lo[c])) {
        mask[c] = 0;
        atomicAdd(&counters[kRepDead], 1ULL);
    }
}

__global__ void k_copy(const float* __restrict__ in, float* __restrict__ out, uint64_t count,
                       const uint64_t* __restrict__ good_prefix, uint64_t n) {
    if (none_good(good_prefix, n))
        return;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += stride)
        out[i] = in[i];
}

// Linear resampling of in[0..in_size) onto out_size points in double
// (frost's linear_stretch, lib/cpu/stats_kernels.hpp:154-181).
__device__ float stretch_at(const float* __restrict__ in, uint64_t in_size, uint64_t out_size, uint64_t i) {
    if (in_size == 0)
        return 0.0F;
    if (out_size == 1 || in_size == 1)
        return in[0];
    const double scale = static_cast<double>(in_size - 1) / static_cast<double>(out_size - 1);
    const double pos   = static_cast<double>(i) * scale;
    const auto lo      = static_cast<uint64_t>(pos);
    const double frac  = pos - static_cast<double>(lo);
    const uint64_t hi  = lo + 1 < in_size - 1 ? lo + 1 : in_size - 1;
    return static_cast<float>(static_cast<double>(in[lo]) * (1.0 - frac) + static_cast<double>(in[hi]) * frac);
}

// out[i] = the resampled value, or with `subtract` out[i] -= it.
__global__ void k_stretch(const float* __restrict__ in, uint64_t in_size, float* __restrict__ out,
                          uint64_t out_size, int subtract, const uint64_t* __restrict__ good_prefix, uint64_t n) {
    if (none_good(good_prefix, n))
        return;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < out_size; i += stride) {
        const float v = stretch_at(in, in_size, out_size, i);
        if (subtract)
            out[i] -= v;
        else
            out[i] = v;
    }
}

__device__ __forceinline__ float median3f(float a, float b, float c) {
    return a < b ? (b < c ? b : (a < c ? c : a)) : (a < c ? a : (b < c ? c : b));
}

// std::min / std::max semantics (the first argument on ties).
__device__ __forceinline__ float min_first(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float max_first(float a, float b) { return (a < b) ? b : a; }

// Median of five: the larger of the two pair minima and the smaller of the
// two pair maxima bracket the median with the fifth value
// (lib/cpu/stats_kernels.hpp:25-31).
__device__ __forceinline__ float median5f(float a, float b, float c, float d, float e) {
    const float f = max_first(min_first(a, b), min_first(c, d));
    const float g = min_first(max_first(a, b), max_first(c, d));
    return median3f(e, f, g);
}

__global__ void k_scrunch5(const float* __restrict__ in, uint64_t in_size, float* __restrict__ out,
                           const uint64_t* __restrict__ good_prefix, uint64_t n) {
    if (none_good(good_prefix, n))
        return;
    if (in_size < 5) {
        if (blockIdx.x == 0 && threadIdx.x == 0 && in_size > 0)
            out[0] = in[0];
        return;
    }
    const uint64_t out_size = in_size / 5;
    const uint64_t stride   = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < out_size; i += stride) {
        const float* q = in + 5 * i;
        out[i]         = median5f(q[0], q[1], q[2], q[3], q[4]);
    }
}

// b[0] and b[2k+1] extrapolate the stretched knots linearly.
__global__ void k_knot_edges(float* __restrict__ b, uint64_t knots, const uint64_t* __restrict__ good_prefix,
                             uint64_t n) {
    if (none_good(good_prefix, n))
        return;
    b[0]             = 2 * b[1] - b[2];
    b[knots * 2 + 1] = 2 * b[knots * 2] - b[knots * 2 - 1];
}

// MAD scale of the baseline-subtracted series (frost's compute_mad,
// lib/cpu/stats_cpu.cpp:77-93): the median of |x| by exact selection (the
// mean of the two middle values for even lengths), over 0.67449.
__global__ void __launch_bounds__(kBlock)
    k_mad(const float* __restrict__ x, uint64_t count, float* __restrict__ scalars,
          const uint64_t* __restrict__ good_prefix, uint64_t n) {
    __shared__ uint32_t hist[256];
    __shared__ uint64_t s_rank;
    __shared__ uint32_t s_bin;
    __shared__ unsigned long long red[32];
    __shared__ uint32_t s_max;
    if (none_good(good_prefix, n))
        return;
    float med = block_select<true>(x, count, count / 2, hist, &s_rank, &s_bin);
    if (count % 2 == 0) {
        const float lower = block_select_prev<true>(x, count, count / 2, med, red, &s_max);
        med               = 0.5F * lower + 0.5F * med;
    }
    if (threadIdx.x == 0)
        scalars[0] = med / kMadNorm;
}

// x /= rms and the plain |x| > threshold detections; nothing when the
// scale is not positive (frost then flags nothing).
__global__ void k_scale_threshold(float* __restrict__ x, uint64_t count, float threshold,
                                  const float* __restrict__ scalars, uint8_t* __restrict__ bb,
                                  const uint64_t* __restrict__ good_prefix, uint64_t n) {
    if (none_good(good_prefix, n))
        return;
    const float rms       = scalars[0];
    const bool ok         = rms > 0.0F;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += stride) {
        if (!ok) {
            bb[i] = 0;
            continue;
        }
        const float v = x[i] / rms;
        x[i]          = v;
        bb[i]         = fabsf(v) > threshold ? 1 : 0;
    }
}

// Inclusive prefix sum of the series in float, in sample order: the
// sequential left fold std::inclusive_scan performs, so every partial sum
// rounds exactly as frost's (lib/cpu/stats_cpu.cpp:153-170). One thread;
// loads run ahead of the add chain.
__global__ void k_scan_serial(const float* __restrict__ x, uint64_t count, float* __restrict__ scanned,
                              const float* __restrict__ scalars, const uint64_t* __restrict__ good_prefix,
                              uint64_t n) {
    if (none_good(good_prefix, n) || !(scalars[0] > 0.0F) || count == 0)
        return;
    scanned[0] = 0.0F;
    float acc  = x[0];
    scanned[1] = acc;
    uint64_t i = 1;
    for (; i + 8 <= count; i += 8) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u)
            v[u] = x[i + u];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            acc += v[u];
            scanned[i + u + 1] = acc;
        }
    }
    for (; i < count; ++i) {
        acc += x[i];
        scanned[i + 1] = acc;
    }
}

// One boxcar width per CTA (widths 1, 2, 4, ... <= bmax): the window sums
// of the scanned series centred as frost's MatchedFilterPlan centres them,
// scaled by 1/sqrt(width), thresholded into a bit mask; every detection is
// then widened by its boxcar: a sample is flagged when the width's window
// around it holds a detection (lib/cpu/device_rfi_flags_cpu.cpp:44-66).
__global__ void __launch_bounds__(kBlock)
    k_boxcar_widths(uint64_t count, uint64_t bmax, float threshold, const float* __restrict__ scanned,
                    const float* __restrict__ scalars, FlagScratch w, uint8_t* __restrict__ bb,
                    const uint64_t* __restrict__ good_prefix, uint64_t n) {
    __shared__ uint32_t red32[32];
    if (none_good(good_prefix, n) || !(scalars[0] > 0.0F))
        return;
    const uint64_t width  = uint64_t{1} << blockIdx.x;
    const uint64_t W      = (count + 31) / 32;
    uint32_t* words       = w.words + blockIdx.x * W;
    uint32_t* pre         = w.wpre + blockIdx.x * (W + 1);
    const uint64_t offset = bmax / 2;
    const uint64_t flen   = count + 1 - bmax;
    const uint64_t ahead  = ((width - 1) / 2) + 1;
    const uint64_t behind = width / 2;
    const float norm      = 1.0F / sqrtf(static_cast<float>(width));
    const int lane        = threadIdx.x & 31;
    // detection bits, one word per warp step
    for (uint64_t base = (threadIdx.x >> 5) * 32; base < W * 32; base += (blockDim.x >> 5) * 32) {
        const uint64_t p = base + lane;
        bool hit         = false;
        if (p >= offset && p < offset + flen) {
            const float f = scanned[p + ahead] - scanned[p - behind];
            hit           = fabsf(f * norm) > threshold;
        }
        const uint32_t bits = __ballot_sync(0xFFFFFFFFU, hit);
        if (lane == 0)
            words[base / 32] = bits;
    }
    __syncthreads();
    // word prefix counts
    const uint64_t per = (W + blockDim.x - 1) / blockDim.x;
    const uint64_t w0  = threadIdx.x * per;
    const uint64_t w1  = w0 + per < W ? w0 + per : W;
    uint32_t local = 0, total = 0;
    for (uint64_t k = w0; k < w1; ++k)
        local += __popc(words[k]);
    uint32_t run = block_exclusive_scan(local, red32, &total);
    for (uint64_t k = w0; k < w1; ++k) {
        pre[k] = run;
        run += __popc(words[k]);
    }
    if (threadIdx.x == 0)
        pre[W] = total;
    __syncthreads();
    if (total == 0)
        return;
    auto ones_before = [&](uint64_t q) -> uint32_t {
        const uint64_t k = q / 32, r = q % 32;
        uint32_t c       = pre[k];
        if (r != 0)
            c += __popc(words[k] & ((1U << r) - 1U));
        return c;
    };
    for (uint64_t i = threadIdx.x; i < flen; i += blockDim.x) {
        const uint64_t p = offset + i;
        if (ones_before(p + ahead) - ones_before(p - behind) > 0)
            bb[p] = 1;
    }
}

// time_flags |= src, counting the samples newly flagged.
__global__ void k_merge_flags(const uint8_t* __restrict__ src, uint64_t count, uint8_t* __restrict__ flags,
                              unsigned long long* __restrict__ counter, const uint64_t* __restrict__ good_prefix,
                              uint64_t n) {
    __shared__ unsigned long long red[32];
    if (none_good(good_prefix, n))
        return;
    unsigned long long added = 0;
    const uint64_t stride    = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count; i += stride) {
        if (src[i] != 0 && flags[i] == 0) {
            flags[i] = 1;
            ++added;
        }
    }
    added = block_sum(added, red);
    if (threadIdx.x == 0 && added)
        atomicAdd(counter, added);
}

// Dropout cut: min_std_fraction x the median row spread (the element of
// rank T/2, as std::nth_element leaves it; lib/cpu/rfi_cpu.cpp:382-387).
__global__ void __launch_bounds__(kBlock)
    k_dropout_cut(const float* __restrict__ row_std, uint64_t count, float fraction, float* __restrict__ scalars,
                  const uint64_t* __restrict__ good_prefix, uint64_t n) {
    __shared__ uint32_t hist[256];
    __shared__ uint64_t s_rank;
    __shared__ uint32_t s_bin;
    if (none_good(good_prefix, n))
        return;
    const float mid = block_select<false>(row_std, count, count / 2, hist, &s_rank, &s_bin);
    if (threadIdx.x == 0)
        scalars[1] = fraction * mid;
}

// A sample below the cut flags itself and both neighbours.
__global__ void k_dropout(const float* __restrict__ row_std, uint64_t count, const float* __restrict__ scalars,
                          uint8_t* __restrict__ flags, unsigned long long* __restrict__ counters,
                          const uint64_t* __restrict__ good_prefix, uint64_t n) {
    __shared__ unsigned long long red[32];
    if (none_good(good_prefix, n))
        return;
    const float cut          = scalars[1];
    unsigned long long added = 0;
    const uint64_t stride    = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < count; t += stride) {
        const bool drop =
            row_std[t] < cut || (t > 0 && row_std[t - 1] < cut) || (t + 1 < count && row_std[t + 1] < cut);
        if (drop && flags[t] == 0) {
            flags[t] = 1;
            ++added;
        }
    }
    added = block_sum(added, red);
    if (threadIdx.x == 0 && added)
        atomicAdd(&counters[kRepDropout], added);
}

// Zero-DM fit of each channel against the kept-sample series
// (lib/cpu/rfi_cpu.cpp:413-436): slope a and offset b in double.
__global__ void k_zdot_fit(uint64_t n, const ZdotSums* __restrict__ zsum, const uint64_t* __restrict__ good_prefix,
                           float* __restrict__ a_out, float* __restrict__ b_out) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= n)
        return;
    float fa = 0.0F, fb = 0.0F;
    const ZdotSums sm = zsum[c];
    if (!none_good(good_prefix, n) && sm.n >= 2.0) {
        const double mz    = sm.sz / sm.n;
        const double ms    = sm.ss / sm.n;
        const double var_s = (sm.sss / sm.n) - (ms * ms);
        const double cov   = (sm.szs / sm.n) - (mz * ms);
        const double a     = var_s > 0.0 ? cov / var_s : 0.0;
        fa                 = static_cast<float>(a);
        fb                 = static_cast<float>(mz - (a * ms));
    }
    a_out[c] = fa;
    b_out[c] = fb;
}

// Kadane-along-time segments of the good channels whose best run is long
// enough and whose sum / sqrt(length) clears the threshold
// (lib/cpu/rfi_cpu.cpp:437-466).
__global__ void k_kchan_accept(uint64_t n, double min_len, double threshold, const Run* __restrict__ pos,
                               const Run* __restrict__ neg, const uint8_t* __restrict__ mask,
                               const uint64_t* __restrict__ good_prefix, Segment* __restrict__ seg_pos,
                               Segment* __restrict__ seg_neg, uint8_t* __restrict__ any) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= n)
        return;
    Segment sp{0, -1}, sn{0, -1};
    if (!none_good(good_prefix, n) && mask[c] != 0) {
        auto accept = [&](const Run& r, Segment& out) {
            const auto len = static_cast<double>(r.length());
            if (len > 0.0 && len >= min_len && r.sum / sqrt(len) > threshold)
                out = {r.start, r.end};
        };
        accept(pos[c], sp);
        accept(neg[c], sn);
    }
    seg_pos[c] = sp;
    seg_neg[c] = sn;
    any[c]     = (sp.start <= sp.end || sn.start <= sn.end) ? 1 : 0;
}

// One CTA: the flagged samples in increasing order, their count and the
// masked-channel count after the dead channels.
__global__ void __launch_bounds__(kBlock)
    k_flag_list(uint64_t count, uint64_t n, const uint8_t* __restrict__ flags, const uint8_t* __restrict__ mask,
                uint64_t* __restrict__ flagged, unsigned long long* __restrict__ counters) {
    __shared__ unsigned long long red[32];
    // each warp takes one contiguous span (a multiple of 32 samples) and
    // walks it 32 samples at a time, eight ballots per step (loads in
    // flight); pass 1 counts, the warps' counts are scanned, pass 2 writes
    // each flagged sample at its rank: increasing order without a barrier
    // per step
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t below_lane = (1U << lane) - 1U;
    const uint64_t span       = ((count + nwarps - 1) / nwarps + 31) / 32 * 32;
    const uint64_t w0         = min(static_cast<uint64_t>(warp) * span, count);
    const uint64_t w1         = min(w0 + span, count);
    constexpr int kU          = 8;
    auto step = [&](uint64_t base, uint32_t (&bal)[kU]) {
        bool f[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const uint64_t t = base + 32 * u + lane;
            f[u]             = t < w1 && flags[t] != 0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u)
            bal[u] = __ballot_sync(0xFFFFFFFFU, f[u]);
    };
    unsigned long long mine = 0;
    for (uint64_t base = w0; base < w1; base += 32 * kU) {
        uint32_t bal[kU];
        step(base, bal);
#pragma unroll
        for (int u = 0; u < kU; ++u)
            mine += static_cast<unsigned long long>(__popc(bal[u]));
    }
    unsigned long long total = 0;
    unsigned long long at    = block_exclusive_scan(lane == 0 ? mine : 0ULL, red, &total);
    at                       = __shfl_sync(0xFFFFFFFFU, at, 0);
    for (uint64_t base = w0; base < w1; base += 32 * kU) {
        uint32_t bal[kU];
        step(base, bal);
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if ((bal[u] >> lane) & 1U)
                flagged[at + static_cast<uint32_t>(__popc(bal[u] & below_lane))] = base + 32 * u + lane;
            at += static_cast<unsigned long long>(__popc(bal[u]));
        }
    }
    unsigned long long kept = 0;
    for (uint64_t c = threadIdx.x; c < n; c += blockDim.x)
        kept += mask[c] != 0 ? 1 : 0;
    kept = block_sum(kept, red);
    if (threadIdx.x == 0) {
        counters[kRepFlagged] = total;
        counters[kRepMasked]  = n - kept;
    }
}

} // namespace

uint64_t decide_launch_counter() { return g_launches.load(std::memory_order_relaxed); }

std::vector<uint64_t> iqrm_lags(uint64_t n, uint64_t radius) {
    std::vector<uint64_t> lags;
    if (n == 0)
        return lags;
    for (uint64_t lag = 1; lag <= radius; lag = std::max(lag + lag / 2, lag + 1)) {
        lags.push_back(lag);
        if (lag >= n - 1)
            break;
    }
    return lags;
}

size_t ChannelScratch::size_for(uint64_t n, uint64_t nlags) {
    const uint64_t P    = pow2_at_least(std::max<uint64_t>(n, 1));
    const uint64_t jobs = 5 + 2 * nlags;
    size_t b            = 0;
    b += align_up(5 * n * sizeof(double));
    b += align_up(n) * 2;
    b += align_up(n * sizeof(float));
    b += align_up(5 * n);
    b += align_up(n * 2 * std::max<uint64_t>(nlags, 1) * sizeof(int32_t));
    b += align_up(n * sizeof(uint32_t));
    b += align_up(n);
    b += align_up((n + 1) * sizeof(uint32_t));
    b += align_up(std::max<uint64_t>(nlags, 1) * sizeof(uint64_t));
    if (P * sizeof(double) > kSortSmemBytes)
        b += align_up(jobs * P * sizeof(double));
    return b;
}

void ChannelScratch::carve(void* base, uint64_t n, uint64_t nl) {
    auto* p   = static_cast<uint8_t*>(base);
    auto take = [&](size_t bytes) {
        uint8_t* q = p;
        p += align_up(bytes);
        return q;
    };
    const uint64_t P = pow2_at_least(std::max<uint64_t>(n, 1));
    nlags            = nl;
    stat             = reinterpret_cast<double*>(take(5 * n * sizeof(double)));
    good             = take(n);
    ignore           = take(n);
    iqrm_x           = reinterpret_cast<float*>(take(n * sizeof(float)));
    flags            = take(5 * n);
    votes            = reinterpret_cast<int32_t*>(take(n * 2 * std::max<uint64_t>(nl, 1) * sizeof(int32_t)));
    cast             = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
    dynamic          = take(n);
    prefix           = reinterpret_cast<uint32_t*>(take((n + 1) * sizeof(uint32_t)));
    lags             = reinterpret_cast<uint64_t*>(take(std::max<uint64_t>(nl, 1) * sizeof(uint64_t)));
    sort_buf         = P * sizeof(double) > kSortSmemBytes
                           ? reinterpret_cast<double*>(take((5 + 2 * nl) * P * sizeof(double)))
                           : nullptr;
}

namespace {

void launch_sorts(const SortJobs& j, const ChannelScratch& w, const float* x, const uint8_t* ign, cudaStream_t s) {
    const int jobs = j.nstat + j.niqrm;
    if (jobs == 0)
        return;
    const size_t smem = j.use_smem ? j.P * sizeof(double) : 0;
    if (smem > 48 * 1024)
        allow_large_smem(reinterpret_cast<const void*>(&k_channel_sorts));
    k_channel_sorts<<<static_cast<unsigned>(jobs), kBlock, smem, s>>>(j, w, x, ign);
    FB_DECIDE_LAUNCH();
}

SortJobs sort_jobs(uint64_t n, const ChannelScratch& w) {
    SortJobs j{};
    j.n        = n;
    j.P        = pow2_at_least(std::max<uint64_t>(n, 1));
    j.use_smem = j.P * sizeof(double) <= kSortSmemBytes ? 1 : 0;
    if (!j.use_smem && w.sort_buf == nullptr)
        throw Error(FROST_ERR_INTERNAL, "RFI: channel sort scratch missing");
    return j;
}

} // namespace

void decide_channel_mask(const ChannelMaskParams& p, const ChannelScratch& w, const MomentSums* mom,
                         const float* scale, const uint32_t* unmeasured, const uint8_t* static_mask,
                         float* clip_mean, float* clip_inv, uint8_t* mask, uint64_t* good_prefix,
                         unsigned long long* counters, cudaStream_t s) {
    const uint64_t n = p.n;
    if (n == 0)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "RFI: no channels");
    if (2 * w.nlags > kMaxVoteSlots)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "RFI: too many IQRM lags");
    if (p.moments || p.iqrm || p.need_clip) {
        FB_CUDA(cudaMemsetAsync(w.flags, 0, 5 * n, s));
        if (p.iqrm) {
            FB_CUDA(cudaMemsetAsync(w.votes, 0xFF, n * 2 * w.nlags * sizeof(int32_t), s));
            FB_CUDA(cudaMemsetAsync(w.cast, 0, n * sizeof(uint32_t), s));
        }
        k_channel_stats<<<grid_for(n, 128), 128, 0, s>>>(p, mom, scale, unmeasured, static_mask, clip_mean,
                                                         clip_inv, w);
        FB_DECIDE_LAUNCH();
        SortJobs j       = sort_jobs(n, w);
        j.k              = p.k;
        j.iqrm_threshold = p.iqrm_threshold;
        if (p.moments)
            for (int k = 0; k < 5; ++k)
                if (p.stat_on[k])
                    j.sid[j.nstat++] = k;
        j.niqrm = p.iqrm ? static_cast<int>(2 * w.nlags) : 0;
        launch_sorts(j, w, w.iqrm_x, w.ignore, s);
    }
    k_channel_decide<<<1, kBlock, 0, s>>>(p, w, static_mask, w.ignore, mask, good_prefix, counters, nullptr);
    FB_DECIDE_LAUNCH();
}

void iqrm_device(uint64_t n, const float* x, const uint8_t* ignore, float threshold, const ChannelScratch& w,
                 uint8_t* out, cudaStream_t s) {
    if (n == 0)
        return;
    if (2 * w.nlags > kMaxVoteSlots)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "iqrm_mask: too many lags");
    FB_CUDA(cudaMemsetAsync(w.votes, 0xFF, n * 2 * w.nlags * sizeof(int32_t), s));
    FB_CUDA(cudaMemsetAsync(w.cast, 0, n * sizeof(uint32_t), s));
    SortJobs j       = sort_jobs(n, w);
    j.iqrm_threshold = threshold;
    j.niqrm          = static_cast<int>(2 * w.nlags);
    launch_sorts(j, w, x, ignore, s);
    ChannelMaskParams p{};
    p.n    = n;
    p.iqrm = 1;
    k_channel_decide<<<1, kBlock, 0, s>>>(p, w, nullptr, ignore, nullptr, nullptr, nullptr, out);
    FB_DECIDE_LAUNCH();
}

void iqrm_mask_host(const float* x, uint64_t n, uint64_t radius, float threshold, const uint8_t* ignore,
                    uint8_t* out) {
    if (radius == 0)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "iqrm_mask: radius must be > 0");
    if (!is_positive_finite(threshold))
        throw Error(FROST_ERR_INVALID_ARGUMENT, "iqrm_mask: threshold must be > 0");
    if (n == 0)
        return;
    const std::vector<uint64_t> lags = iqrm_lags(n, radius);
    DeviceBuffer scratch, xs, flags;
    scratch.reserve(ChannelScratch::size_for(n, lags.size()));
    xs.reserve(n * sizeof(float) + n);
    flags.reserve(n);
    ChannelScratch w{};
    w.carve(scratch.get(), n, lags.size());
    cudaStream_t s = nullptr;
    FB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
        auto* xd = xs.as<float>();
        auto* ig = reinterpret_cast<uint8_t*>(xd + n);
        FB_CUDA(cudaMemcpyAsync(w.lags, lags.data(), lags.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        FB_CUDA(cudaMemcpyAsync(xd, x, n * sizeof(float), cudaMemcpyHostToDevice, s));
        if (ignore != nullptr)
            FB_CUDA(cudaMemcpyAsync(ig, ignore, n, cudaMemcpyHostToDevice, s));
        else
            FB_CUDA(cudaMemsetAsync(ig, 0, n, s));
        iqrm_device(n, xd, ig, threshold, w, flags.as<uint8_t>(), s);
        FB_CUDA(cudaMemcpyAsync(out, flags.get(), n, cudaMemcpyDeviceToHost, s));
        FB_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    FB_CUDA(cudaStreamDestroy(s));
}

size_t FlagScratch::size_for(uint64_t T, uint64_t bmax) {
    uint32_t nw = 0;
    for (uint64_t width = 1; width <= bmax; width *= 2)
        ++nw;
    const uint64_t W = (T + 31) / 32;
    size_t b         = 0;
    b += align_up(T * sizeof(float));
    b += 2 * align_up((2 * T + 4) * sizeof(float));
    b += align_up((T + 1) * sizeof(float));
    b += align_up(std::max<uint32_t>(nw, 1) * W * sizeof(uint32_t));
    b += align_up(std::max<uint32_t>(nw, 1) * (W + 1) * sizeof(uint32_t));
    b += align_up(T);
    b += align_up(4 * sizeof(float));
    return b;
}

void FlagScratch::carve(void* base, uint64_t T, uint64_t bmax) {
    auto* p   = static_cast<uint8_t*>(base);
    auto take = [&](size_t bytes) {
        uint8_t* q = p;
        p += align_up(bytes);
        return q;
    };
    nwidths = 0;
    for (uint64_t width = 1; width <= bmax; width *= 2)
        ++nwidths;
    const uint64_t W = (T + 31) / 32;
    series           = reinterpret_cast<float*>(take(T * sizeof(float)));
    buf_a            = reinterpret_cast<float*>(take((2 * T + 4) * sizeof(float)));
    buf_b            = reinterpret_cast<float*>(take((2 * T + 4) * sizeof(float)));
    scanned          = reinterpret_cast<float*>(take((T + 1) * sizeof(float)));
    words            = reinterpret_cast<uint32_t*>(take(std::max<uint32_t>(nwidths, 1) * W * sizeof(uint32_t)));
    wpre             = reinterpret_cast<uint32_t*>(take(std::max<uint32_t>(nwidths, 1) * (W + 1) * sizeof(uint32_t)));
    bb               = take(T);
    scalars          = reinterpret_cast<float*>(take(4 * sizeof(float)));
}

namespace {

// The broad-band zero-DM detector on the detection series: baseline
// resampling and subtraction (frost's BaselineFilterPlan,
// lib/cpu/stats_cpu.cpp:210-278, sizes planned here from the length), the
// MAD scale, the plain threshold and the boxcar ladder, then the merge.
void broadband(const FlagParams& p, const FlagScratch& w, const float* s_det, const uint64_t* gp,
               uint8_t* time_flags, unsigned long long* counters, cudaStream_t s) {
    const uint64_t T = p.nsamps, n = p.nchans;
    const unsigned g = grid_for(T, 256);
    k_copy<<<g, 256, 0, s>>>(s_det, w.series, T, gp, n);
    FB_DECIDE_LAUNCH();
    const uint64_t r = p.smooth_radius;
    if (r == 0)
        throw Error(FROST_ERR_INVALID_ARGUMENT, "baseline filter: smooth_radius must be > 0");
    const uint64_t knots = T / r + ((T % r >= r / 2 + r % 2) ? 1 : 0);
    if (knots > 1) {
        uint64_t rounded = knots;
        while (rounded <= T / 5)
            rounded *= 5;
        k_stretch<<<grid_for(rounded, 256), 256, 0, s>>>(w.series, T, w.buf_a, rounded, 0, gp, n);
        FB_DECIDE_LAUNCH();
        float* cur   = w.buf_a;
        float* other = w.buf_b;
        for (uint64_t size = rounded; size > knots; size /= 5) {
            k_scrunch5<<<grid_for(std::max<uint64_t>(size / 5, 1), 256), 256, 0, s>>>(cur, size, other, gp, n);
            FB_DECIDE_LAUNCH();
            std::swap(cur, other);
        }
        k_stretch<<<grid_for(2 * knots, 256), 256, 0, s>>>(cur, knots, other + 1, 2 * knots, 0, gp, n);
        FB_DECIDE_LAUNCH();
        k_knot_edges<<<1, 1, 0, s>>>(other, knots, gp, n);
        FB_DECIDE_LAUNCH();
        k_stretch<<<g, 256, 0, s>>>(other, 2 * knots + 2, w.series, T, 1, gp, n);
        FB_DECIDE_LAUNCH();
    }
    k_mad<<<1, kBlock, 0, s>>>(w.series, T, w.scalars, gp, n);
    FB_DECIDE_LAUNCH();
    k_scale_threshold<<<g, 256, 0, s>>>(w.series, T, p.broad_threshold, w.scalars, w.bb, gp, n);
    FB_DECIDE_LAUNCH();
    if (T > p.boxcar_max && p.boxcar_max > 1) {
        k_scan_serial<<<1, 1, 0, s>>>(w.series, T, w.scanned, w.scalars, gp, n);
        FB_DECIDE_LAUNCH();
        k_boxcar_widths<<<w.nwidths, kBlock, 0, s>>>(T, p.boxcar_max, p.broad_threshold, w.scanned, w.scalars, w,
                                                     w.bb, gp, n);
        FB_DECIDE_LAUNCH();
    }
    k_merge_flags<<<g, 256, 0, s>>>(w.bb, T, time_flags, &counters[kRepBroad], gp, n);
    FB_DECIDE_LAUNCH();
}

} // namespace

void decide_flags(const FlagParams& p, const FlagScratch& w, const uint64_t* good_prefix,
                  const uint32_t* unmeasured, const float* lo, const float* hi, const float* s_det,
                  const float* row_std, const uint8_t* kspec_whole, const ZdotSums* zsum,
                  const Run* kpos_best, const Run* kneg_best, uint8_t* mask, uint8_t* time_flags,
                  float* zdot_a, float* zdot_b, Segment* kchan_pos, Segment* kchan_neg,
                  uint8_t* kchan_any, uint64_t* flagged, unsigned long long* counters, cudaStream_t s) {
    const uint64_t T = p.nsamps, n = p.nchans;
    const unsigned gt = grid_for(T, 256);
    k_dead<<<grid_for(n, 128), 128, 0, s>>>(n, p.nwin, good_prefix, unmeasured, lo, hi, mask, counters);
    FB_DECIDE_LAUNCH();
    FB_CUDA(cudaMemsetAsync(time_flags, 0, std::max<uint64_t>(T, 1), s));
    if (T > 0) {
        if (p.broad)
            broadband(p, w, s_det, good_prefix, time_flags, counters, s);
        if (p.dropout) {
            k_dropout_cut<<<1, kBlock, 0, s>>>(row_std, T, p.dropout_fraction, w.scalars, good_prefix, n);
            FB_DECIDE_LAUNCH();
            k_dropout<<<gt, 256, 0, s>>>(row_std, T, w.scalars, time_flags, counters, good_prefix, n);
            FB_DECIDE_LAUNCH();
        }
        if (p.kspec) {
            k_merge_flags<<<gt, 256, 0, s>>>(kspec_whole, T, time_flags, &counters[kRepKadane], good_prefix, n);
            FB_DECIDE_LAUNCH();
        }
    }
    if (p.zdot) {
        k_zdot_fit<<<grid_for(n, 128), 128, 0, s>>>(n, zsum, good_prefix, zdot_a, zdot_b);
        FB_DECIDE_LAUNCH();
    }
    if (p.kchan) {
        k_kchan_accept<<<grid_for(n, 128), 128, 0, s>>>(n, p.kchan_min_len, p.kchan_threshold, kpos_best, kneg_best,
                                                        mask, good_prefix, kchan_pos, kchan_neg, kchan_any);
        FB_DECIDE_LAUNCH();
    } else {
        FB_CUDA(cudaMemsetAsync(kchan_any, 0, n, s));
    }
    k_flag_list<<<1, kBlock, 0, s>>>(T, n, time_flags, mask, flagged, counters);
    FB_DECIDE_LAUNCH();
}

} // namespace fb::rfi
