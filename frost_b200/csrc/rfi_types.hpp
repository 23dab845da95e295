// Plain structs shared by the RFI kernels (device) and the RFI orchestration
// (host), plus the counter hash and the maximum-sum-run monoid. Both sides
// must produce identical bits, so every function here is written once and
// compiled for host and device.
//
// The hash (splitmix64 chained over five words), the uniform index/open
// interval maps and the Box-Muller deviate restate lib/cpu/rfi_kernels.hpp:
// 17-47; the run monoid restates KadaneState (lib/cpu/rfi_kernels.hpp:
// 65-133): its append/combine decisions must be the same ones, in the same
// order, for the flags to agree bit for bit.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define FB_HD __host__ __device__ __forceinline__
#else
#define FB_HD inline
#endif

namespace fb::rfi {

// Random-stream tags (lib/cpu/rfi_cpu_detail.hpp:45-50).
enum : uint64_t { kStreamCell = 1, kStreamTime = 2, kStreamNoise = 3, kStreamMasked = 4 };

// Cell states of the apply pass (lib/cpu/rfi_cpu_detail.hpp:52-59).
enum : uint8_t {
    kClean          = 0,
    kMasked         = 1,
    kUnmeasured     = 2,
    kNarrow         = 3,
    kKadaneSpectrum = 4,
    kKadaneChannel  = 5,
};

constexpr int kMaxBandpassRows = 3125; // 5^5 sampled spectra per window
constexpr int kMinWindow       = 5;
constexpr int kMinBlockSamps   = 64;
constexpr int kMaxDraws        = 10;
constexpr int kMaxChunks       = 64;
constexpr int kMinChunkRows    = 1024;
constexpr double kClipSigma    = 4.5;
constexpr int kClipIterations  = 2;
constexpr float kMadToStd      = 1.4826F;

struct MomentSums {
    double n, s1, s2, s3, s4, lag, nc, c1, c2;
};

struct ZdotSums {
    double n, sz, ss, sss, szs;
};

struct Span32 {
    int32_t lo, hi;
};

struct Segment {
    int64_t start, end;
};

FB_HD uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30U)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27U)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31U);
}

FB_HD uint64_t hash5(uint64_t a, uint64_t b, uint64_t c, uint64_t d, uint64_t e) {
    return splitmix64(splitmix64(splitmix64(splitmix64(splitmix64(a) ^ b) ^ c) ^ d) ^ e);
}

/** Uniform integer in [lo, hi]. */
FB_HD uint64_t uniform_index(uint64_t h, uint64_t lo, uint64_t hi) {
    return lo + h % (hi - lo + 1);
}

/** Uniform double in (0, 1). */
FB_HD double uniform_open(uint64_t h) {
    return (static_cast<double>(h >> 11U) + 0.5) * 0x1.0p-53;
}

/** Maximum-sum contiguous run [start, end]; empty when end < start. */
struct Run {
    double sum;
    int64_t start;
    int64_t end;
    FB_HD int64_t length() const { return end - start + 1; }
};

/** Associative state of the maximum-sum run over increasing positions. */
struct KadaneState {
    double total;
    int64_t first;
    int64_t last;
    int32_t empty;
    int32_t pad_;
    Run prefix;
    Run suffix;
    Run best;

    FB_HD static KadaneState make() {
        KadaneState s;
        s.total  = 0.0;
        s.first  = 0;
        s.last   = -1;
        s.empty  = 1;
        s.pad_   = 0;
        s.prefix = {0.0, 0, -1};
        s.suffix = {0.0, 0, -1};
        s.best   = {0.0, 0, -1};
        return s;
    }

    FB_HD void append(int64_t i, double u) {
        if (empty) {
            empty  = 0;
            first  = i;
            prefix = {0.0, i, i - 1};
            suffix = {0.0, i, i - 1};
            best   = suffix;
        }
        last = i;
        total += u;
        if (total > prefix.sum)
            prefix = {total, first, i};
        if (suffix.sum + u > 0.0) {
            if (suffix.length() <= 0)
                suffix.start = i;
            suffix.sum += u;
            suffix.end = i;
        } else {
            suffix = {0.0, i + 1, i};
        }
        if (suffix.sum > best.sum)
            best = suffix;
    }

    /** State of `a` followed by `b`. */
    FB_HD static KadaneState combine(const KadaneState& a, const KadaneState& b) {
        if (a.empty)
            return b;
        if (b.empty)
            return a;
        KadaneState r = make();
        r.empty       = 0;
        r.first       = a.first;
        r.last        = b.last;
        r.total       = a.total + b.total;
        r.prefix      = a.prefix;
        if (a.total + b.prefix.sum > r.prefix.sum)
            r.prefix = {a.total + b.prefix.sum, a.first, b.prefix.end};
        const int64_t join = a.suffix.length() > 0 ? a.suffix.start : b.first;
        r.suffix           = b.suffix;
        if (b.total + a.suffix.sum > r.suffix.sum)
            r.suffix = {b.total + a.suffix.sum, join, b.last};
        r.best = a.best;
        if (b.best.sum > r.best.sum)
            r.best = b.best;
        const double cross = a.suffix.sum + b.prefix.sum;
        if (cross > r.best.sum)
            r.best = {cross, join, b.prefix.end};
        return r;
    }
};

/** KadaneState::append with 32-bit positions (a block's samples and
 * channels stay below 2^31): the same sums, comparisons and runs, fewer
 * integer instructions in the per-sample scans; widened for storage. */
struct KadaneState32 {
    struct Run32 {
        double sum;
        int32_t start, end;
    };
    double total = 0.0;
    int32_t first = 0, last = -1;
    bool empty    = true;
    Run32 prefix{0.0, 0, -1}, suffix{0.0, 0, -1}, best{0.0, 0, -1};

    FB_HD void append(int32_t i, double u) {
        if (empty) {
            empty  = false;
            first  = i;
            prefix = {0.0, i, i - 1};
            suffix = {0.0, i, i - 1};
            best   = suffix;
        }
        last = i;
        total += u;
        if (total > prefix.sum) { // the prefix run always starts at `first`
            prefix.sum = total;
            prefix.end = i;
        }
        // The open (suffix) run always ends at the last position, so its end
        // is `last` (filled in by widen) and it is empty exactly when its
        // sum is zero (a kept run has a positive sum).
        const double s = suffix.sum + u;
        if (s > 0.0) {
            if (suffix.sum == 0.0)
                suffix.start = i;
            suffix.sum = s;
        } else {
            suffix.sum   = 0.0;
            suffix.start = i + 1;
        }
        if (suffix.sum > best.sum)
            best = {suffix.sum, suffix.start, i};
    }
    FB_HD static Run wide(const Run32& r) { return {r.sum, r.start, r.end}; }
    FB_HD KadaneState widen() const {
        KadaneState k = KadaneState::make();
        k.total       = total;
        k.first       = first;
        k.last        = last;
        k.empty       = empty ? 1 : 0;
        k.prefix      = wide(prefix);
        k.suffix      = {suffix.sum, suffix.start, empty ? suffix.end : last};
        k.best        = wide(best);
        return k;
    }
};

/** The two KadaneState32 of one sequence u and its negation -u, appended
 * together from a known first position (`begin`) with 32-bit positions:
 * the states of -u share the running total (negated: the sums of -u are
 * the exact negations of those of u) and compare it for their own best
 * prefix; the open runs' ends are the last position (`widen_*(last)`). The
 * same sums, comparisons and runs as two KadaneState32 appends. */
struct KadanePair32 {
    struct Side {
        double psum = 0.0, ssum = 0.0, bsum = 0.0;
        int32_t pend = -1, sstart = 0, bstart = 0, bend = -1;
    };
    double total = 0.0; // of u
    int32_t first = 0;
    bool empty    = true;
    Side pos, neg;

    FB_HD static void begin_side(Side& sd, int32_t i) {
        sd.pend   = i - 1;
        sd.sstart = i;
        sd.bstart = i;
        sd.bend   = i - 1;
    }
    FB_HD void begin(int32_t i) {
        empty = false;
        first = i;
        begin_side(pos, i);
        begin_side(neg, i);
    }
    FB_HD static void open_run(Side& sd, int32_t i, double s) {
        if (s > 0.0) {
            if (sd.ssum == 0.0)
                sd.sstart = i;
            sd.ssum = s;
        } else {
            sd.ssum   = 0.0;
            sd.sstart = i + 1;
        }
        if (sd.ssum > sd.bsum) {
            sd.bsum   = sd.ssum;
            sd.bstart = sd.sstart;
            sd.bend   = i;
        }
    }
    FB_HD void append(int32_t i, double u) {
        total += u;
        if (total > pos.psum) { // the prefix runs start at `first`
            pos.psum = total;
            pos.pend = i;
        }
        if (-total > neg.psum) {
            neg.psum = -total;
            neg.pend = i;
        }
        open_run(pos, i, pos.ssum + u);
        open_run(neg, i, neg.ssum - u);
    }
    FB_HD KadaneState widen(const Side& sd, double tot, int32_t last) const {
        KadaneState k = KadaneState::make();
        if (empty)
            return k;
        k.total  = tot;
        k.first  = first;
        k.last   = last;
        k.empty  = 0;
        k.prefix = {sd.psum, first, sd.pend};
        k.suffix = {sd.ssum, sd.sstart, last};
        k.best   = {sd.bsum, sd.bstart, sd.bend};
        return k;
    }
    /** The state of u after appends up to position `last`. */
    FB_HD KadaneState widen_pos(int32_t last) const { return widen(pos, total, last); }
    /** The state of -u (its total is 0 - total: +0 rather than -0 for a
     * zero total, as the sum of -u would be). */
    FB_HD KadaneState widen_neg(int32_t last) const { return widen(neg, 0.0 - total, last); }
};

/** The best run of KadaneState::append over a sequence that is never
 * combined with another: only the open (suffix) run and the best one are
 * kept, with 32-bit positions. The open run always ends at the position
 * just appended and is empty exactly when its sum is zero. When no run
 * ever has a positive sum the best run is empty (length 0) and reported at
 * position 0 rather than at the first position appended; callers use only
 * a best run's length when it is empty. */
struct KadaneBest {
    double ssum = 0.0, bsum = 0.0;
    int32_t sstart = 0, bstart = 0, bend = -1;

    FB_HD void append(int32_t i, double u) {
        const double s = ssum + u;
        if (s > 0.0) {
            if (ssum == 0.0)
                sstart = i;
            ssum = s;
        } else {
            ssum   = 0.0;
            sstart = i + 1;
        }
        if (ssum > bsum) {
            bsum   = ssum;
            bstart = sstart;
            bend   = i;
        }
    }
    FB_HD Run best() const { return {bsum, bstart, bend}; }
};

/** Largest power of five not above `count` (0 for 0). */
FB_HD uint64_t largest_power_of_five_leq(uint64_t count) {
    if (count == 0)
        return 0;
    uint64_t p = 1;
    while (p <= count / 5)
        p *= 5;
    return p;
}

} // namespace fb::rfi
