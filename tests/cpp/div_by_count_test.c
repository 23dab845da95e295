// Correctly rounded a / n (n a positive integer count) from a precomputed
// y = RN(1/n) with one fused multiply-add correction, the division the
// Welford kernel uses (frost_b200/csrc/rfi_kernels.cu: div_by_count),
// checked bit for bit against IEEE division on random operands.
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

static double div_by_count(double a, double n, double y) {
    if (a == 0.0)
        return a;
    if (!(fabs(a) > 0x1p-900))
        return a / n;
    const double q0 = a * y;
    const double r  = fma(-q0, n, a);
    return fma(r, y, q0);
}

int main(void) {
    long bad = 0, tested = 0;
    for (long i = 0; i < 30000000L; ++i) {
        const uint64_t n = 1 + next() % 262144;
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
        const double y = 1.0 / (double)n;
        const double q = div_by_count(a, (double)n, y), t = a / (double)n;
        ++tested;
        if (memcmp(&q, &t, sizeof q) != 0) {
            if (bad < 10)
                printf("a=%a n=%lu got %a want %a\n", a, (unsigned long)n, q, t);
            ++bad;
        }
    }
    printf("tested %ld bad %ld\n", tested, bad);
    return bad != 0;
}
