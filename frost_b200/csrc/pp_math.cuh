// Coincidence and dispersion-curve predicates of frost's candidate
// post-processing, shared by the device kernels (postprocess_kernels.cu) and
// the host entry points (postprocess.cpp).
//
//   time_reach, are_coincident (both overloads)   lib/search/clustering.cpp:18-67
//   subband_time_shift_samples, subband_dm_step,
//   dm_within_smear, on_same_curve                 lib/search/subband_dedup.cpp:70-192
//
// Every floating-point expression keeps the reference's operation order in
// double precision; both compilation units are built without FMA
// contraction (nvcc --fmad=false, g++ -ffp-contract=off), and CUDA's double
// division and square root are correctly rounded, so host and device give
// the bits the reference's strict-IEEE build gives.
#pragma once

#include <cmath>
#include <cstdint>

#include "frost_b200.h"

#ifdef __CUDACC__
#define PP_HD __host__ __device__ __forceinline__
#else
#define PP_HD inline
#endif

namespace fb::pp {

using u64 = std::uint64_t;

/** dmt::kDispConst, s MHz^2 cm^3 / pc (the value the FDMT plan uses). */
constexpr double kDispConst = 4.148808e3;

/** The fields the predicates read, gathered from a frost_giant or from the
 * kernels' time-ordered columns. `width` is giant_boxcar_width. */
struct Pt {
    u64 samp, filter, width, dm_idx, cb, ce, plane;
    float dm, snr, flo, fhi;
};

PP_HD u64 absdiff(u64 a, u64 b) { return a > b ? a - b : b - a; }
PP_HD u64 max_u(u64 a, u64 b) { return (a < b) ? b : a; }
PP_HD double max_d(double a, double b) { return (a < b) ? b : a; }
PP_HD float max_f(float a, float b) { return (a < b) ? b : a; }

PP_HD double abs_d(double x) { return x < 0.0 ? -x : x; }

PP_HD bool finite_f(float x) {
    union {
        float f;
        std::uint32_t u;
    } v{x};
    return (v.u & 0x7F800000U) != 0x7F800000U;
}
PP_HD bool finite_d(double x) {
    union {
        double f;
        u64 u;
    } v{x};
    return (v.u & 0x7FF0000000000000ULL) != 0x7FF0000000000000ULL;
}
PP_HD bool posfin_f(float x) { return finite_f(x) && x > 0.0F; }
PP_HD bool posfin_d(double x) { return finite_d(x) && x > 0.0; }

/** giant_boxcar_width (include/frost/search/candidate.hpp:75-81). */
PP_HD u64 box_width(u64 filter_width, u64 filter_idx) {
    if (filter_width > 0)
        return filter_width;
    return u64{1} << (filter_idx < 63 ? filter_idx : 63);
}

/** width * tol, saturating at the largest sample distance. */
PP_HD u64 time_reach(u64 width, u64 tol) {
    return (tol != 0 && width > ~u64{0} / tol) ? ~u64{0} : width * tol;
}

PP_HD Pt pt_of(const frost_giant& g) {
    return Pt{g.samp_idx, g.filter_idx, box_width(g.filter_width, g.filter_idx), g.dm_idx, g.chan_begin,
              g.chan_end,  g.plane,      g.dm,  g.snr,  g.f_low,  g.f_high};
}

PP_HD double dm_step(float f_low, float f_high, float tsamp) {
    if (!posfin_f(tsamp) || !posfin_f(f_low) || !finite_f(f_high) || !(f_high > f_low))
        return 0.0;
    const double lo    = static_cast<double>(f_low);
    const double hi    = static_cast<double>(f_high);
    const double denom = (1.0 / (lo * lo)) - (1.0 / (hi * hi));
    if (!posfin_d(denom))
        return 0.0;
    return static_cast<double>(tsamp) / (kDispConst * denom);
}

PP_HD double time_shift(float dm, float f_wide, float f_narrow, float tsamp) {
    if (!posfin_f(tsamp) || !posfin_f(f_wide) || !posfin_f(f_narrow))
        return 0.0;
    const double w   = static_cast<double>(f_wide);
    const double n   = static_cast<double>(f_narrow);
    const double inv = (1.0 / (w * w)) - (1.0 / (n * n));
    return (static_cast<double>(dm) * kDispConst * inv) / static_cast<double>(tsamp);
}

/** are_coincident(a, b, time_tol, filter_tol, dm_tol). */
PP_HD bool coincident_basic(const Pt& a, const Pt& b, u64 time_tol, u64 filter_tol, u64 dm_tol) {
    if (a.plane != b.plane || a.cb != b.cb || a.ce != b.ce)
        return false;
    const u64 widest = max_u(a.width, b.width);
    return absdiff(a.samp, b.samp) <= time_reach(widest, time_tol) &&
           absdiff(a.filter, b.filter) <= filter_tol && absdiff(a.dm_idx, b.dm_idx) <= dm_tol;
}

/** The physical DM gate of are_coincident(a, b, ClusterTolerances), for a
 * pair that already passed coincident_basic. */
PP_HD bool dm_gate(const Pt& a, const Pt& b, const frost_cluster_tolerances& t) {
    if (!(t.dm_smear > 0.0) || !(t.tsamp > 0.0) || absdiff(a.dm_idx, b.dm_idx) <= 1)
        return true;
    const double step = dm_step(a.flo, a.fhi, static_cast<float>(t.tsamp));
    if (!(step > 0.0))
        return true;
    const double widest = static_cast<double>(max_u(a.width, b.width));
    const double ddm    = abs_d(static_cast<double>(a.dm) - static_cast<double>(b.dm));
    double growth       = 1.0;
    if (t.snr_floor > 0.0) {
        const double ratio = static_cast<double>(max_f(a.snr, b.snr)) / t.snr_floor;
        growth             = max_d(1.0, sqrt(max_d(0.0, (ratio * ratio) - 1.0)));
    }
    return ddm <= t.dm_smear * widest * step * growth;
}

PP_HD bool coincident(const Pt& a, const Pt& b, const frost_cluster_tolerances& t) {
    return coincident_basic(a, b, t.time_tol, t.filter_tol, t.dm_tol) && dm_gate(a, b, t);
}

PP_HD u64 span_of(u64 cb, u64 ce) { return ce < cb ? 0 : (ce - cb) + 1; }

PP_HD bool dm_within_smear(const Pt& a, const Pt& b, const frost_cluster_tolerances& t, double widest,
                           double step) {
    const double smear = t.dm_smear > 0.0 ? t.dm_smear : 1.0;
    const double delay = max_d(2.0, widest);
    const double delta = abs_d(static_cast<double>(a.dm) - static_cast<double>(b.dm));
    return delta <= (smear * delay * step);
}

/** on_same_curve(a, b, tol, tsamp) (subband_dedup.cpp:85-150). */
PP_HD bool on_same_curve(const Pt& a, const Pt& b, const frost_cluster_tolerances& t, float tsamp) {
    const u64 sa = span_of(a.cb, a.ce), sb = span_of(b.cb, b.ce);
    if (sa == 0 || sb == 0)
        return false;
    if (sa == sb) {
        if (a.plane == b.plane || a.cb != b.cb || a.ce != b.ce || absdiff(a.filter, b.filter) > t.filter_tol)
            return false;
        const double step   = dm_step(a.flo, a.fhi, tsamp);
        const double widest = static_cast<double>(max_u(a.width, b.width));
        return posfin_d(step) && dm_within_smear(a, b, t, widest, step) &&
               static_cast<double>(absdiff(a.samp, b.samp)) <= static_cast<double>(t.time_tol) * widest;
    }
    const bool a_holds_b = a.cb <= b.cb && a.ce >= b.ce;
    const bool b_holds_a = b.cb <= a.cb && b.ce >= a.ce;
    if (!a_holds_b && !b_holds_a)
        return false;
    const Pt& wide   = sa > sb ? a : b;
    const Pt& narrow = sa > sb ? b : a;
    if (absdiff(wide.filter, narrow.filter) > t.filter_tol)
        return false;
    const double step = dm_step(narrow.flo, narrow.fhi, tsamp);
    if (!posfin_d(step))
        return false;
    if (!dm_within_smear(wide, narrow, t, static_cast<double>(max_u(wide.width, narrow.width)), step))
        return false;
    const double wide_step = dm_step(wide.flo, wide.fhi, tsamp);
    if (posfin_d(wide_step) && step > 4.0 * wide_step) {
        const double expected = static_cast<double>(wide.snr) *
                                sqrt(static_cast<double>(sa < sb ? sa : sb) / static_cast<double>(max_u(sa, sb)));
        if (static_cast<double>(narrow.snr) > (2.0 * expected) + 3.0)
            return false;
    }
    const double shift   = time_shift(wide.dm, wide.flo, narrow.flo, tsamp);
    const double aligned = static_cast<double>(narrow.samp) + shift;
    const double delta   = abs_d(aligned - static_cast<double>(wide.samp));
    const double widest  = static_cast<double>(max_u(wide.width, narrow.width));
    return delta <= static_cast<double>(t.time_tol) * widest;
}

} // namespace fb::pp
