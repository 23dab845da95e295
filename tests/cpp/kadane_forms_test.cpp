// The reduced Kadane forms of the RFI scans (KadaneState32: 32-bit
// positions, the open run's end implied; KadaneBest: open and best runs
// only; KadanePair32: the states of u and -u together) against the full
// KadaneState on random sequences: integer values
// (exact zero sums and ties), small and large floats, runs of equal values,
// gaps in the positions. Prints "bad N" with N the mismatches.

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "rfi_types.hpp"

using namespace fb::rfi;

namespace {

bool same(const Run& a, const Run& b) { return a.sum == b.sum && a.start == b.start && a.end == b.end; }

bool same_state(const KadaneState& a, const KadaneState& b) {
    return a.total == b.total && a.first == b.first && a.last == b.last && a.empty == b.empty &&
           same(a.prefix, b.prefix) && same(a.suffix, b.suffix) && same(a.best, b.best);
}

} // namespace

int main() {
    std::mt19937_64 rng(20241204);
    long bad = 0, cases = 0;
    for (int trial = 0; trial < 200000; ++trial) {
        const int n    = static_cast<int>(rng() % 40);
        const int kind = static_cast<int>(rng() % 4);
        KadaneState full = KadaneState::make(), fneg = KadaneState::make();
        KadaneState32 k32;
        KadaneBest kb;
        KadanePair32 pair;
        int32_t last = -1;
        int32_t pos = static_cast<int32_t>(rng() % 5);
        for (int i = 0; i < n; ++i) {
            double u = 0.0;
            switch (kind) {
            case 0: u = static_cast<double>(static_cast<int>(rng() % 7) - 3); break;
            case 1: u = std::ldexp(static_cast<double>(static_cast<int64_t>(rng() % 2001) - 1000), -7); break;
            case 2: u = std::normal_distribution<double>(-0.1, 1.0)(rng); break;
            default: u = (rng() % 3 == 0) ? 0.0 : std::ldexp(static_cast<double>(static_cast<int>(rng() % 5) - 2), static_cast<int>(rng() % 60) - 30); break;
            }
            full.append(pos, u);
            fneg.append(pos, -u);
            k32.append(pos, u);
            kb.append(pos, u);
            if (i == 0)
                pair.begin(pos);
            pair.append(pos, u);
            last = pos;
            pos += 1 + static_cast<int32_t>(rng() % 3 == 0 ? rng() % 4 : 0);
        }
        ++cases;
        const KadaneState w = k32.widen();
        if (!same_state(w, full))
            ++bad;
        // bit-level equality of the totals (the sign of a zero included)
        const KadaneState pp = pair.widen_pos(last), pn = pair.widen_neg(last);
        if (!same_state(pp, full) || !same_state(pn, fneg) ||
            std::signbit(pp.total) != std::signbit(full.total) || std::signbit(pn.total) != std::signbit(fneg.total))
            ++bad;
        const Run b = kb.best();
        if (full.best.length() > 0 ? !same(b, full.best) : (b.length() > 0 || b.sum != full.best.sum))
            ++bad;
    }
    std::printf("cases %ld bad %ld\n", cases, bad);
    return bad == 0 ? 0 : 1;
}
