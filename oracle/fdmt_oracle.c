/*
 * TEST INFRASTRUCTURE ONLY — the FP64 CPU oracle of the dedispersion search.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it, as the checker; the product (frost_b200) never links or calls it.
 *
 * frost delegates FDMT + boxcar + noise + peaks to dmt v0.8.0
 * (github.com/pravirkr/dmt, tag v0.8.0, fetched by CPM in
 * cmake/frostDependencies.cmake:65-102). dmt is not vendored with the
 * reference and there is no network, so dmt itself cannot run here: PARITY
 * WITH dmt IS UNPINNED. This file restates the published algorithm
 * (Zackay & Ofek 2017, cited by frost's README.md:86) under frost's own
 * contracts, and the tests pin it to those contracts (unit noise of every
 * plane, S/N = window sum / sqrt(variance grid), peak at the end of the
 * trailing window, times referenced to the bottom of the band, cold prefix,
 * plane geometry; tests/cpp/api/calibration_test.cpp,
 * gpu_parity_test.cpp:83-150, pipeline_end_to_end_test.cpp:116-196,
 * dedisp_test.cpp:30-54).
 *
 * The oracle computes each dedispersed row directly — not level by level —
 * as sum over channels of a window of L_c samples ending s_c samples before
 * t, with (s_c, L_c) found by descending the sub-band split rule:
 *   K(a,b) = a^-2 - b^-2; band [f_a, f_b] split at f_m; a row of delay d
 *   takes d_hi = round(d K(f_m,f_b)/K(f_a,f_b)) from the upper part (shifted
 *   by d_lo = d - d_hi) and d_lo from the lower part; one channel with delay
 *   d is a window of d + 1 samples.
 * Every sum is FP64.
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KDISP 4.148808e3

static double kfac(double a, double b) { return 1.0 / (a * a) - 1.0 / (b * b); }

static double edge(int64_t c, int64_t C, double f_min, double f_max) {
    const double bw = (f_max - f_min) / (double)C;
    return f_min + (double)c * bw;
}

/* Delay (samples) across [f_lo, f_hi] at dm. */
int64_t oracle_band_delay(double dm, double f_lo, double f_hi, double tsamp) {
    return llround(KDISP * dm * kfac(f_lo, f_hi) / tsamp);
}

/* Regular split point of channel range [a, b). */
static int64_t mid_of(int64_t a, int64_t b) { return a + (b - a) / 2; }

static void descend(int64_t C, double f_min, double f_max, int64_t a, int64_t m, int64_t b,
                    int64_t d, int64_t shift, int64_t base, int64_t* shifts, int64_t* lens) {
    if (b - a == 1) {
        shifts[a - base] = shift;
        lens[a - base]   = d + 1;
        return;
    }
    const double fa = edge(a, C, f_min, f_max);
    const double fm = edge(m, C, f_min, f_max);
    const double fb = edge(b, C, f_min, f_max);
    const int64_t d_hi = llround((double)d * (kfac(fm, fb) / kfac(fa, fb)));
    const int64_t d_lo = d - d_hi;
    descend(C, f_min, f_max, a, mid_of(a, m), m, d_lo, shift, base, shifts, lens);
    descend(C, f_min, f_max, m, mid_of(m, b), b, d_hi, shift + d_lo, base, shifts, lens);
}

/* For each of nrows delays of the band [a, b) split first at m: per channel
 * the shift s_c and window length L_c ([row][b - a] each). */
int oracle_row_geometry(int64_t C, double f_min, double f_max, int64_t a, int64_t m, int64_t b,
                        const int64_t* delays, int64_t nrows, int64_t* shifts, int64_t* lens) {
    if (!(a < m && m < b) || b > C)
        return -1;
    for (int64_t r = 0; r < nrows; ++r)
        descend(C, f_min, f_max, a, m, b, delays[r], 0, a, shifts + r * (b - a), lens + r * (b - a));
    return 0;
}

/* out[r][t] = sum_c sum_{j<L} in[c][t - s - j] over channels [a, b) of the
 * [C][T] input (samples before 0 are zero), FP64. */
int oracle_dedisperse(const double* in, int64_t C, int64_t T, int64_t a, int64_t b,
                      const int64_t* shifts, const int64_t* lens, int64_t nrows, double* out) {
    const int64_t n = b - a;
    double* pre     = (double*)malloc(sizeof(double) * (size_t)(n * (T + 1)));
    if (pre == NULL)
        return -1;
    for (int64_t c = 0; c < n; ++c) {
        double acc = 0.0;
        pre[c * (T + 1)] = 0.0;
        for (int64_t t = 0; t < T; ++t) {
            acc += in[(a + c) * T + t];
            pre[c * (T + 1) + t + 1] = acc;
        }
    }
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < nrows; ++r) {
        double* o = out + r * T;
        for (int64_t t = 0; t < T; ++t)
            o[t] = 0.0;
        for (int64_t c = 0; c < n; ++c) {
            const int64_t s = shifts[r * n + c], L = lens[r * n + c];
            const double* p = pre + c * (T + 1);
            for (int64_t t = 0; t < T; ++t) {
                int64_t hi = t - s + 1;       /* window [t - s - L + 1, t - s] */
                int64_t lo = t - s - L + 1;
                if (hi <= 0)
                    continue;
                if (lo < 0)
                    lo = 0;
                o[t] += p[hi] - p[lo];
            }
        }
    }
    free(pre);
    return 0;
}

/* Window weights: boxcar, or trapezoid with half-weight edges of (W+1)/4. */
static void weights(int64_t W, int trap, double* w) {
    for (int64_t i = 0; i < W; ++i)
        w[i] = 1.0;
    if (trap && W >= 3) {
        const int64_t e = (W + 1) / 4;
        for (int64_t i = 0; i < e; ++i) {
            w[i]         = 0.5;
            w[W - 1 - i] = 0.5;
        }
    }
}

/* Sum over k of m(k)^2, m = the width-W weights convolved with an L-sample
 * box: m(k) = sum of w[i] over max(0, k-L+1) <= i <= min(W-1, k), for
 * k = 0 .. W+L-2. For L >= W the middle L-W+1 values all equal sum(w), so
 * only the two ramps are summed term by term. Every term is a multiple of
 * 1/4 and every partial sum stays far below 2^51, so the result is exact and
 * independent of the summation order. */
static double box_sq(int64_t L, int64_t W, const double* wpre) {
    double v = 0.0;
#define MULT(k) (wpre[((k) < W - 1 ? (k) : W - 1) + 1] - wpre[((k) - L + 1 > 0 ? (k) - L + 1 : 0)])
    if (L >= W) {
        const double s = wpre[W];
        for (int64_t k = 0; k < W - 1; ++k) {
            const double m = MULT(k);
            v += m * m;
        }
        v += (double)(L - W + 1) * s * s;
        for (int64_t k = L; k < W + L - 1; ++k) {
            const double m = MULT(k);
            v += m * m;
        }
    } else {
        for (int64_t k = 0; k < W + L - 1; ++k) {
            const double m = MULT(k);
            v += m * m;
        }
    }
#undef MULT
    return v;
}

/* Noise variance of the width-W window for unit-variance input: per active
 * channel, the sum of squared multiplicities of the window convolved with
 * the channel's L-sample box (box_sq, memoised per distinct L). */
int oracle_variance(const int64_t* lens, int64_t nrows, int64_t n, const uint8_t* mask,
                    int64_t W, int trap, double* out) {
    double* w    = (double*)malloc(sizeof(double) * (size_t)W);
    double* wpre = (double*)malloc(sizeof(double) * (size_t)(W + 1));
    int64_t lmax = 1;
    for (int64_t i = 0; i < nrows * n; ++i)
        if (lens[i] > lmax)
            lmax = lens[i];
    double* memo = (double*)malloc(sizeof(double) * (size_t)(lmax + 1));
    if (w == NULL || wpre == NULL || memo == NULL) {
        free(w);
        free(wpre);
        free(memo);
        return -1;
    }
    weights(W, trap, w);
    wpre[0] = 0.0;
    for (int64_t i = 0; i < W; ++i)
        wpre[i + 1] = wpre[i] + w[i];
    for (int64_t l = 0; l <= lmax; ++l)
        memo[l] = -1.0;
    for (int64_t r = 0; r < nrows; ++r) {
        double v = 0.0;
        for (int64_t c = 0; c < n; ++c) {
            if (!mask[c])
                continue;
            const int64_t L = lens[r * n + c];
            if (memo[L] < 0.0)
                memo[L] = box_sq(L, W, wpre);
            v += memo[L];
        }
        out[r] = v;
    }
    free(w);
    free(wpre);
    free(memo);
    return 0;
}

/* Selected rows of one band straight from a float32 [C][T] input:
 * out[i][t] = sum over channels [a, b) of the FP64 window sum
 * in[c][t - s - L + 1 .. t - s] (samples before 0 are zero), with (s, L)
 * the row's per-channel shift and length ([nrows][b - a] each). The window
 * slides along t in FP64 (one add and one subtract per sample), so no
 * prefix array of the whole input is held. */
int oracle_dedisperse_rows(const float* in, int64_t C, int64_t T, int64_t a, int64_t b,
                           const int64_t* shifts, const int64_t* lens, int64_t nrows, double* out) {
    const int64_t n = b - a;
    if (a < 0 || b > C || n <= 0)
        return -1;
#pragma omp parallel for schedule(dynamic)
    for (int64_t r = 0; r < nrows; ++r) {
        double* o = out + r * T;
        for (int64_t t = 0; t < T; ++t)
            o[t] = 0.0;
        for (int64_t c = 0; c < n; ++c) {
            const int64_t s = shifts[r * n + c], L = lens[r * n + c];
            const float* x  = in + (a + c) * T;
            double acc      = 0.0;
            /* window of output t covers input [t - s - L + 1, t - s] */
            for (int64_t t = 0; t < T; ++t) {
                const int64_t hi = t - s;
                const int64_t lo = t - s - L;
                if (hi >= 0)
                    acc += (double)x[hi];
                if (lo >= 0)
                    acc -= (double)x[lo];
                o[t] += acc;
            }
        }
    }
    return 0;
}

typedef struct {
    int64_t row;
    int64_t width_idx;
    int64_t peak;
    int64_t begin;
    int64_t end;
    double snr;
} oracle_cand;

/* Matched-filter search of FP64 rows [nrows][T]: S/N(t, w) = window sum /
 * sqrt(var[row][w]), or var_or[row][w] when t - gulp_start(t) <
 * delay + W - 1 and the gulp's mask changed (or_gulp[g] != 0). Samples with
 * t < delay + W - 1 are skipped when skip_cold. Peaks: mode 0 one per run
 * per width, 1 one per run over all widths (ties: earliest sample, then the
 * smaller width), 2 every sample. Open runs at T are emitted. Returns the
 * number of candidates written (at most cap), or -1. */
int64_t oracle_search(const double* rows, int64_t nrows, int64_t T, const int64_t* delays,
                      const int64_t* widths, int64_t nw, const double* var, const double* var_or,
                      int64_t gulp, const uint8_t* or_gulp, double thresh, int mode, int trap,
                      int skip_cold, oracle_cand* out, int64_t cap) {
    int64_t n        = 0;
    double* pre      = (double*)malloc(sizeof(double) * (size_t)(T + 1));
    double* wts      = (double*)malloc(sizeof(double) * 4096 * 2);
    double* snr      = (double*)malloc(sizeof(double) * (size_t)(T * nw));
    if (pre == NULL || wts == NULL || snr == NULL)
        return -1;
    for (int64_t r = 0; r < nrows; ++r) {
        const double* x = rows + r * T;
        pre[0]          = 0.0;
        for (int64_t t = 0; t < T; ++t)
            pre[t + 1] = pre[t] + x[t];
        for (int64_t wi = 0; wi < nw; ++wi) {
            const int64_t W = widths[wi];
            const int64_t e = (trap && W >= 3) ? (W + 1) / 4 : 0;
            for (int64_t t = 0; t < T; ++t) {
                double v = -INFINITY;
                const int cold = skip_cold && t < delays[r] + W - 1;
                if (!cold) {
                    /* samples before the stream start are zero */
#define PRE(i) ((i) <= 0 ? 0.0 : pre[(i)])
                    double s = PRE(t + 1) - PRE(t + 1 - W);
                    if (e > 0)
                        s -= 0.5 * ((PRE(t + 1) - PRE(t + 1 - e)) + (PRE(t + 1 - W + e) - PRE(t + 1 - W)));
#undef PRE
                    const int64_t g = t / gulp;
                    const int use_or = or_gulp[g] && (t - g * gulp) < delays[r] + W - 1;
                    const double vv  = use_or ? var_or[r * nw + wi] : var[r * nw + wi];
                    if (vv > 0.0)
                        v = s / sqrt(vv);
                }
                snr[wi * T + t] = v;
            }
        }
        if (mode == 2) {
            for (int64_t t = 0; t < T; ++t)
                for (int64_t wi = 0; wi < nw; ++wi)
                    if (snr[wi * T + t] > thresh) {
                        if (n < cap)
                            out[n] = (oracle_cand){r, wi, t, t, t, snr[wi * T + t]};
                        ++n;
                    }
            continue;
        }
        const int64_t passes = mode == 0 ? nw : 1;
        for (int64_t pw = 0; pw < passes; ++pw) {
            int open = 0;
            oracle_cand cur;
            for (int64_t t = 0; t <= T; ++t) {
                double best = -INFINITY;
                int64_t bw  = 0;
                if (t < T) {
                    if (mode == 0) {
                        best = snr[pw * T + t];
                        bw   = pw;
                    } else {
                        for (int64_t wi = 0; wi < nw; ++wi)
                            if (snr[wi * T + t] > best) {
                                best = snr[wi * T + t];
                                bw   = wi;
                            }
                    }
                }
                const int up = t < T && best > thresh;
                if (up && open) {
                    if (best > cur.snr) {
                        cur.snr       = best;
                        cur.peak      = t;
                        cur.width_idx = bw;
                    }
                    cur.end = t;
                } else if (up) {
                    open = 1;
                    cur  = (oracle_cand){r, bw, t, t, t, best};
                } else if (open) {
                    if (n < cap)
                        out[n] = cur;
                    ++n;
                    open = 0;
                }
            }
        }
    }
    free(pre);
    free(wts);
    free(snr);
    return n;
}
