// Host check of the FP32 eclipse screen (lcurve_re_b200/csrc/ecl_screen.cuh)
// against the FP64 line-of-sight test it screens.
//
// The device restatement of Roche::ingress_egress (eclipse.cuh) is compiled
// here for the host, with the CUDA qualifiers defined away. For every face
// of the grid given on stdin (header: q, cos i, sin i, delta_phase, spin of
// the eclipser, radius of the eclipser, unused, eclipser index; then the
// face count and the positions) it runs the sphere test and pot_min, then
// both bisections twice: with Roche::fblink alone, and with the screen
// deciding first and fblink only where the screen is unsure. Prints one
// line "faces hits tests fp64_tests screened_true screened_false
// mismatches" and exits 1 if any ingress or egress differs.
#include <cstdio>
#include <cstdlib>
#include <vector>
#define __device__
#define __noinline__
#define __forceinline__ inline
static struct { unsigned x; } threadIdx;
#define __shfl_sync(m, v, l) (v)
#define __shfl_xor_sync(m, v, l) (v)
#define __any_sync(m, p) (p)
#define __ballot_sync(m, p) ((p) ? 1u : 0u)
#define __clz(x) __builtin_clz(x)
#include "../../lcurve_re_b200/csrc/eclipse.cuh"
#include "../../lcurve_re_b200/csrc/ecl_screen.cuh"
using namespace lcg;

int main() {
    double h[8];
    long long n = 0;
    if (fread(h, 8, 8, stdin) != 8 || fread(&n, 8, 1, stdin) != 1) return 2;
    std::vector<double> pos(3 * (size_t)n);
    if (fread(pos.data(), 8, pos.size(), stdin) != pos.size()) return 2;
    const double q = h[0], cosi = h[1], sini = h[2], delta = h[3], spin = h[4], rad = h[5];
    const int star = (int)h[7];
    const double rl = star == kStar1 ? xl11(q, spin) : 1. - xl12(q, spin);
    double rref, pref;
    ref_sphere(star, q, spin, rad / rl, rref, pref);
    EclScreen S = make_ecl_screen(star, q, spin, rref, pref);
    const V3 cofm = star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    long long hits = 0, tests = 0, t64 = 0, st_true = 0, st_false = 0, bad = 0;
    for (long long i = 0; i < n; i++) {
        const V3 r = v3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        double phi1, phi2, lam1, lam2, phi, lam;
        if (!sphere_eclipse_ph(cosi, sini, r, cofm, rref, phi1, phi2, lam1, lam2)) continue;
        const double acc = 2. * sqrt(2. * kTwoPi * (lam2 - lam1) * delta);
        int st = 0;
        if (!pot_min(star, q, spin, cosi, sini, r, phi1, phi2, lam1, lam2, rref, pref, acc, phi,
                     lam, st))
            continue;
        hits++;
        const float u0x = (float)(r.x - cofm.x), u0y = (float)r.y, u0z = (float)r.z;
        for (int side = 0; side < 2; side++) {
            double res[2];
            for (int screened = 0; screened < 2; screened++) {
                double pin = phi, pout = side ? phi2 : phi1, pmid;
                while (fabs(pin - pout) > delta) {
                    pmid = (pin + pout) / 2.;
                    int d = kScreenUnsure;
                    if (screened) {
                        tests++;
                        const double ph = pmid - rint(pmid);
                        const float ang = (float)(kTwoPi * ph);
                        const float si = (float)sini;
                        d = fblink_screen(S, u0x, u0y, u0z, si * cosf(ang), -si * sinf(ang),
                                          (float)cosi, (float)acc);
                        if (d == kScreenTrue) st_true++;
                        if (d == kScreenFalse) st_false++;
                        if (d == kScreenUnsure) t64++;
                    }
                    const bool in = d == kScreenUnsure
                                        ? fblink(star, q, spin, acc, set_earth(cosi, sini, pmid),
                                                 r, rref, pref, st)
                                        : d == kScreenTrue;
                    if (in) pin = pmid; else pout = pmid;
                }
                res[screened] = (pin + pout) / 2.;
            }
            if (res[0] != res[1]) bad++;
        }
    }
    printf("%lld %lld %lld %lld %lld %lld %lld\n", n, hits, tests, t64, st_true, st_false, bad);
    return bad ? 1 : 0;
}
