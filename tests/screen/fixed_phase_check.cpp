// Host check of the mixed sweeps' fixed-point eclipse test
// (lcurve_re_b200/csrc/fixed_phase.cuh, compiled here for the host) against
// the reference's double test, ecl_range (comp_light_flat.cpp:171-173):
//   eclipsed = (phin >= in && phin <= out) || phin <= out - 1.
// Triples (phin, in, out) come at random and adversarially: phin on a
// boundary and one or two ulps either side of it, ranges that wrap past
// phase 1, out exactly 1, in exactly 0, phin exactly 1, empty ranges. Every
// decision must agree where the phase and the boundary it is compared with
// are >= 2^-12; below that they may differ only within 2^-64 of each other.
// Prints "cases mismatches tiny_mismatches" and exits 1 on a mismatch.
#include <cmath>
#include <cstdio>
#include <random>

struct ulonglong2 {
    unsigned long long x, y;
};
static inline ulonglong2 make_ulonglong2(unsigned long long x, unsigned long long y) {
    return ulonglong2{x, y};
}
#define LCG_FX_FN static inline
#include "../../lcurve_re_b200/csrc/fixed_phase.cuh"

using lcg::ecl_fx64;
using lcg::phase_fx64;

static long long cases = 0, bad = 0, tiny = 0;

static void check(double phin, double in, double out) {
    if (!(in >= 0.0 && in < 1.0 && out >= in && out <= in + 1.0 && out <= 2.0)) return;
    if (!(phin >= 0.0 && phin <= 1.0)) return;
    const bool ref = (phin >= in && phin <= out) || phin <= out - 1.0;
    const ulonglong2 E = ecl_fx64(in, out);
    const bool fx = !((phase_fx64(phin) - E.x) >= E.y);
    cases++;
    if (ref == fx) return;
    const double b = out >= 1.0 ? out - 1.0 : out;
    const double lim = std::ldexp(1.0, -12), eps = std::ldexp(1.0, -64);
    const bool small = (phin < lim) && (in < lim || b < lim) &&
                       (std::fabs(phin - in) <= eps || std::fabs(phin - b) <= eps);
    if (small) {
        tiny++;
        return;
    }
    if (bad < 10)
        std::printf("mismatch phin=%.17g in=%.17g out=%.17g ref=%d fx=%d\n", phin, in, out, ref,
                    fx);
    bad++;
}

static void around(double x, double in, double out) {
    double lo = x, hi = x;
    check(x, in, out);
    for (int k = 0; k < 3; k++) {
        lo = std::nextafter(lo, -1.0);
        hi = std::nextafter(hi, 2.0);
        check(lo, in, out);
        check(hi, in, out);
    }
}

int main() {
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    for (int r = 0; r < 400000; r++) {
        const double in = r % 97 == 0 ? 0.0 : u(rng);
        double w = u(rng) * (r % 3 == 0 ? 1e-6 : 0.6);
        if (r % 89 == 0) w = 0.0;
        double out = in + w;
        if (r % 101 == 0) out = 1.0;
        if (out < in) continue;
        check(u(rng), in, out);
        around(in, in, out);
        around(out, in, out);
        if (out >= 1.0) around(out - 1.0, in, out);
        check(1.0, in, out);
        check(0.0, in, out);
    }
    // small phases and boundaries (below 2^-12)
    for (int r = 0; r < 200000; r++) {
        const double in = u(rng) * 1e-4, out = in + u(rng) * 1e-4;
        around(in, in, out);
        around(out, in, out);
        check(u(rng) * 2e-4, in, out);
    }
    std::printf("%lld %lld %lld\n", cases, bad, tiny);
    return bad ? 1 : 0;
}
