// Correctly rounded a / n (n a positive integer count) from a precomputed
// two-term reciprocal y_hi = RN(1/n), y_lo = RN((1 - n y_hi) / n):
// q = RN(a y_hi + RN(a y_lo)), the division the Welford kernel uses
// (frost_b200/csrc/rfi_kernels.cu: WelfordAcc::step_recip), checked bit for
// bit against IEEE division on random operands. A zero numerator may give
// a zero of the other sign; the kernel adds q to a mean that is never -0,
// so only the value of a zero quotient matters there.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static uint64_t state = 88172645463325252ULL;
static uint64_t next(void) {
    state ^= state << 13;
    state ^= state >> 7;
    state ^= state << 17;
    return state;
}

static double div_by_count(double a, double n, double yh, double yl) {
    double q = fma(a, yh, a * yl);
    if (!(fabs(a) > 0x1p-900) && a != 0.0)
        q = a / n;
    return q;
}

int main(void) {
    long bad = 0, tested = 0;
    for (long i = 0; i < 30000000L; ++i) {
        const uint64_t n = 1 + ((i % 11 == 0) ? next() % 4294967296ULL : next() % 262144);
        double a;
        if (i % 3 == 0) {
            a = ((double)(int64_t)next() / 9.2e18) * 100.0; // typical deviations
        } else if (i % 3 == 1) {
            const uint64_t bits = next(); // any finite double
            memcpy(&a, &bits, 8);
            if (!isfinite(a) || fabs(a) > 1e300)
                continue;
        } else {
            a = ((double)(next() % 1000000) - 500000.0) * 0.125; // dyadic values, zeros included
            if (i % 7 == 0)
                a = (i % 2) ? 0.0 : -0.0;
        }
        const double dn = (double)n;
        const double yh = 1.0 / dn;
        const double yl = fma(-dn, yh, 1.0) / dn;
        const double q = div_by_count(a, dn, yh, yl), t = a / dn;
        ++tested;
        const int same = (a == 0.0) ? (q == 0.0) : (memcmp(&q, &t, sizeof q) == 0);
        if (!same) {
            if (bad < 10)
                printf("a=%a n=%lu got %a want %a\n", a, (unsigned long)n, q, t);
            ++bad;
        }
    }
    printf("tested %ld bad %ld\n", tested, bad);
    return bad != 0;
}
