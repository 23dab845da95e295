// Host statistics on per-gulp series. The arithmetic follows the reference
// step for step (same float/double types, same order) because the flags it
// produces must match frost's CPU cleaner exactly; the code is this
// project's own.

#include "host_stats.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace fb::stats {

namespace {

inline float median3(float a, float b, float c) {
    return a < b ? (b < c ? b : (a < c ? c : a)) : (a < c ? a : (b < c ? c : b));
}

inline float median5(float a, float b, float c, float d, float e) {
    const float f = std::max(std::min(a, b), std::min(c, d));
    const float g = std::min(std::max(a, b), std::max(c, d));
    return median3(e, f, g);
}

// Resamples `in` onto `out_size` points by linear interpolation in double
// (lib/cpu/stats_kernels.hpp:154-181).
void stretch(const float* in, SizeType in_size, float* out, SizeType out_size) {
    if (out_size == 0)
        return;
    if (in_size == 0) {
        std::fill(out, out + out_size, 0.0F);
        return;
    }
    if (out_size == 1) {
        out[0] = in[0];
        return;
    }
    if (in_size == 1) {
        std::fill(out, out + out_size, in[0]);
        return;
    }
    const double scale = static_cast<double>(in_size - 1) / static_cast<double>(out_size - 1);
    for (SizeType i = 0; i < out_size; ++i) {
        const double pos  = static_cast<double>(i) * scale;
        const auto lo     = static_cast<SizeType>(pos);
        const double frac = pos - static_cast<double>(lo);
        const SizeType hi = std::min(lo + 1, in_size - 1);
        out[i] = static_cast<float>(static_cast<double>(in[lo]) * (1.0 - frac) +
                                    static_cast<double>(in[hi]) * frac);
    }
}

void scrunch5(const float* in, SizeType in_size, float* out) {
    if (in_size == 0)
        return;
    if (in_size < 5) {
        out[0] = in[0];
        return;
    }
    for (SizeType i = 0; i < in_size / 5; ++i) {
        const float* p = in + 5 * i;
        out[i]         = median5(p[0], p[1], p[2], p[3], p[4]);
    }
}

// Inclusive prefix sum with a leading zero, then trailing-window sums of
// `width` centred as the reference's MatchedFilterPlan does
// (lib/cpu/stats_cpu.cpp:153-208).
struct PrefixFilter {
    std::vector<float> scanned;
    SizeType max_width = 0;

    void prepare(const float* in, SizeType count, SizeType mw) {
        scanned.resize(count + 1);
        scanned[0] = 0.0F;
        float acc  = 0.0F;
        for (SizeType i = 0; i < count; ++i) {
            acc += in[i];
            scanned[i + 1] = acc;
        }
        max_width = mw;
    }
    void execute(float* out, SizeType width) const {
        const SizeType out_count = scanned.size() - max_width;
        const SizeType offset    = max_width / 2;
        const SizeType ahead     = ((width - 1) / 2) + 1;
        const SizeType behind    = width / 2;
        for (SizeType i = 0; i < out_count; ++i) {
            const SizeType idx = offset + i;
            out[i]             = scanned[idx + ahead] - scanned[idx - behind];
        }
    }
};

} // namespace

double quantile_sorted(std::span<const double> sorted, double q) {
    const double h  = static_cast<double>(sorted.size() - 1) * q;
    const auto lo   = static_cast<SizeType>(h);
    const auto hi   = std::min(lo + 1, sorted.size() - 1);
    const double fr = h - static_cast<double>(lo);
    return sorted[lo] + (fr * (sorted[hi] - sorted[lo]));
}

float mad_scale(std::span<const float> data) {
    constexpr float kMadNorm = 0.6744897501960817F;
    const SizeType count     = data.size();
    std::vector<float> a(count);
    for (SizeType i = 0; i < count; ++i)
        a[i] = std::abs(data[i]);
    auto middle = a.begin() + static_cast<IndexType>(count / 2);
    std::nth_element(a.begin(), middle, a.end());
    float med = *middle;
    if (count % 2 == 0) {
        const float lower = *std::max_element(a.begin(), middle);
        med               = 0.5F * lower + 0.5F * med;
    }
    return med / kMadNorm;
}

void baseline_subtract(std::vector<float>& data, SizeType r) {
    const SizeType count = data.size();
    if (r == 0)
        invalid("baseline filter: smooth_radius must be > 0");
    if (count == 0)
        return;
    // Knot count: count / r rounded to nearest, in integers.
    const SizeType knots = count / r + (count % r >= r / 2 + r % 2 ? 1 : 0);
    if (knots <= 1)
        return;
    SizeType rounded = knots;
    while (rounded <= count / 5)
        rounded *= 5;
    std::vector<float> a(rounded), b(rounded / 5);
    stretch(data.data(), count, a.data(), rounded);
    for (SizeType size = rounded; size > knots; size /= 5) {
        scrunch5(a.data(), size, b.data());
        std::swap(a, b);
    }
    b.resize(knots * 2 + 2);
    stretch(a.data(), knots, b.data() + 1, knots * 2);
    b[0]             = 2 * b[1] - b[2];
    b[knots * 2 + 1] = 2 * b[knots * 2] - b[knots * 2 - 1];
    std::vector<float> base(count);
    stretch(b.data(), knots * 2 + 2, base.data(), count);
    for (SizeType i = 0; i < count; ++i)
        data[i] -= base[i];
}

SizeType broadband_time_flags(std::vector<float> series, SizeType smooth_radius, float threshold,
                              SizeType boxcar_max, std::span<uint8_t> flags) {
    const SizeType n = series.size();
    if (flags.size() < n)
        invalid("broadband flags are shorter than the series");
    baseline_subtract(series, smooth_radius);
    if (n == 0)
        return 0;
    const float rms = mad_scale(series);
    if (!(rms > 0.0F))
        return 0;
    for (auto& v : series)
        v /= rms;
    std::vector<uint8_t> mask(n, 0);
    for (SizeType t = 0; t < n; ++t)
        mask[t] = std::abs(series[t]) > threshold ? 1 : 0;
    if (n > boxcar_max && boxcar_max > 1) {
        PrefixFilter sf;
        sf.prepare(series.data(), n, boxcar_max);
        const SizeType flen   = n + 1 - boxcar_max;
        const SizeType offset = boxcar_max / 2;
        std::vector<float> filtered(flen), fmask(n, 0.0F), widened(flen);
        for (SizeType width = 1; width <= boxcar_max; width *= 2) {
            sf.execute(filtered.data(), width);
            const float norm = 1.0F / std::sqrt(static_cast<float>(width));
            std::fill(fmask.begin(), fmask.end(), 0.0F);
            for (SizeType i = 0; i < flen; ++i)
                fmask[offset + i] = std::abs(filtered[i] * norm) > threshold ? 1.0F : 0.0F;
            PrefixFilter mf;
            mf.prepare(fmask.data(), n, boxcar_max);
            mf.execute(widened.data(), width);
            for (SizeType i = 0; i < flen; ++i)
                if (widened[i] > 0.5F)
                    mask[offset + i] = 1;
        }
    }
    SizeType count = 0;
    for (SizeType t = 0; t < n; ++t) {
        if (mask[t] != 0 && flags[t] == 0) {
            flags[t] = 1;
            ++count;
        }
    }
    return count;
}

std::vector<uint8_t> iqrm_mask(std::span<const float> x, SizeType radius, float threshold,
                               std::span<const uint8_t> ignore) {
    const SizeType n = x.size();
    if (radius == 0)
        invalid("iqrm_mask: radius must be > 0");
    if (!is_positive_finite(threshold))
        invalid("iqrm_mask: threshold must be > 0");
    if (!ignore.empty() && ignore.size() != n)
        invalid("iqrm_mask: ignore size must match x");
    std::vector<uint8_t> mask(n, 0);
    if (n == 0)
        return mask;
    auto ignored = [&](SizeType i) { return !ignore.empty() && ignore[i] != 0; };
    const auto ni = static_cast<IndexType>(n);
    auto clampi   = [&](IndexType i) { return static_cast<SizeType>(std::clamp<IndexType>(i, 0, ni - 1)); };

    // Votes are kept as bitsets-by-list: cast[j] = channels j voted against,
    // received[i] = channels that voted against i; duplicates are removed.
    std::vector<std::vector<SizeType>> cast(n), received(n);
    std::vector<double> diff(n);
    std::vector<uint8_t> valid(n);
    std::vector<double> sorted;
    for (SizeType lag = 1; lag <= radius; lag = std::max(lag + lag / 2, lag + 1)) {
        for (const IndexType k : {static_cast<IndexType>(lag), -static_cast<IndexType>(lag)}) {
            sorted.clear();
            for (IndexType i = 0; i < ni; ++i) {
                const SizeType j  = clampi(i - k);
                const auto ui     = static_cast<SizeType>(i);
                valid[ui]         = (!ignored(ui) && !ignored(j)) ? 1 : 0;
                diff[ui]          = static_cast<double>(x[ui]) - static_cast<double>(x[j]);
                if (valid[ui])
                    sorted.push_back(diff[ui]);
            }
            if (sorted.empty())
                continue;
            std::sort(sorted.begin(), sorted.end());
            const double q1  = quantile_sorted(sorted, 0.25);
            const double med = quantile_sorted(sorted, 0.5);
            const double q3  = quantile_sorted(sorted, 0.75);
            const double cut = static_cast<double>(threshold) * (q3 - q1) / 1.349;
            for (IndexType i = 0; i < ni; ++i) {
                const auto ui = static_cast<SizeType>(i);
                if (valid[ui] && diff[ui] - med > cut) {
                    const SizeType j = clampi(i - k);
                    cast[j].push_back(ui);
                    received[ui].push_back(j);
                }
            }
        }
        // Lags beyond n-1 repeat the edge-clamped comparisons.
        if (lag >= n - 1)
            break;
    }
    for (auto& v : cast) {
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
    }
    for (SizeType i = 0; i < n; ++i) {
        auto& from = received[i];
        std::sort(from.begin(), from.end());
        from.erase(std::unique(from.begin(), from.end()), from.end());
        for (const SizeType j : from) {
            if (cast[j].size() < from.size()) {
                mask[i] = 1;
                break;
            }
        }
        if (ignored(i))
            mask[i] = 1;
    }
    return mask;
}

void flag_iqr_outliers(std::span<const double> stat, std::span<const uint8_t> good, double k,
                       std::span<uint8_t> flags) {
    std::vector<double> vals;
    vals.reserve(stat.size());
    for (SizeType c = 0; c < stat.size(); ++c)
        if (good[c])
            vals.push_back(stat[c]);
    if (vals.size() < 4)
        return;
    std::sort(vals.begin(), vals.end());
    const double q1  = quantile_sorted(vals, 0.25);
    const double q3  = quantile_sorted(vals, 0.75);
    const double iqr = q3 - q1;
    if (!(iqr > 0.0))
        return;
    const double lo = q1 - (k * iqr);
    const double hi = q3 + (k * iqr);
    for (SizeType c = 0; c < stat.size(); ++c)
        if (good[c] && (stat[c] < lo || stat[c] > hi))
            flags[c] = 1;
}

} // namespace fb::stats
