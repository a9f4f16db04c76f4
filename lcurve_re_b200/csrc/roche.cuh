// roche.cuh — Roche geometry shared by the host engine and the kernels.
//
// Every function keeps the floating-point operation order of the reference
// routine it restates (cited per function, lcurve_re source tree) so that,
// compiled without FMA contraction (nvcc --fmad=false, g++
// -ffp-contract=off), FP64 results equal the reference's up to the libm
// differences of sin/cos/acos/atan2/exp/pow (sqrt and division are IEEE on
// both sides).
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define LCG_HD __host__ __device__ __forceinline__
#else
#define LCG_HD inline
#endif

namespace lcg {

constexpr double kPi = 3.14159265358979323846264;  // constants.h:89
constexpr double kTwoPi = 2. * kPi;                 // constants.h:92
constexpr double kC = 2.99792458e8;                 // constants.h:15
constexpr double kH = 6.6262e-34;                   // constants.h:21
constexpr double kK = 1.3806e-23;                   // constants.h:24
constexpr double kDay = 86400.;                     // constants.h:73 (float 86400)
constexpr double kM_PI = 3.14159265358979323846;    // <math.h> M_PI

struct V3 {
    double x, y, z;
};

LCG_HD V3 v3(double x, double y, double z) { return V3{x, y, z}; }
LCG_HD double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
LCG_HD double norm2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
LCG_HD double len(V3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
LCG_HD V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
LCG_HD V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
LCG_HD V3 scale(double c, V3 a) { return V3{c * a.x, c * a.y, c * a.z}; }
LCG_HD double sq(double a) { return a * a; }
LCG_HD double deg2rad(double d) { return kM_PI * d / 180.; }  // new_subs.h:187
LCG_HD double rad2deg(double r) { return 180. * r / kM_PI; }  // new_subs.h:192
// std::min / std::max argument conventions
LCG_HD double dmin(double a, double b) { return (b < a) ? b : a; }
LCG_HD double dmax(double a, double b) { return (a < b) ? b : a; }
LCG_HD double dsign(double a, double b) { return b >= 0. ? fabs(a) : -fabs(a); }

enum { kStar1 = 0, kStar2 = 1 };

// Roche::rpot1 (rpot.cpp:37-51)
LCG_HD double rpot1(double q, double spin, V3 p) {
    double mu = q / (1 + q), comp = 1. - mu;
    double x2y2 = sq(p.x) + sq(p.y), z2 = sq(p.z);
    double r1sq = x2y2 + z2, r1 = sqrt(r1sq);
    double r2 = sqrt(r1sq + 1. - 2. * p.x);
    return (-comp / r1 - mu / r2 - sq(spin) * x2y2 / 2. + mu * p.x);
}

// Roche::rpot2 (rpot.cpp:61-86)
LCG_HD double rpot2(double q, double spin, V3 p) {
    const double mu = q / (1 + q), comp = 1. - mu;
    const double x2y2 = p.x * p.x + p.y * p.y;
    const double r1sq = x2y2 + p.z * p.z;
    const double r1 = sqrt(r1sq);
    const double r2 = sqrt(r1sq + 1.0 - 2.0 * p.x);
    const double ss = spin * spin;
    return -comp / r1 - mu / r2 - ss * (0.5 + 0.5 * x2y2 - p.x) - comp * p.x;
}

LCG_HD double rpot(int star, double q, double spin, V3 p) {
    return star == kStar1 ? rpot1(q, spin, p) : rpot2(q, spin, p);
}

// Roche::drpot1 / drpot2 (drpot.cpp:40-85)
LCG_HD V3 drpot(int star, double q, double spin, V3 p) {
    double r1sq = norm2(p), r1 = sqrt(r1sq);
    double r2sq = r1sq + 1. - 2. * p.x, r2 = sqrt(r2sq);
    double mu = q / (1 + q);
    double mu1 = mu / r2 / r2sq;
    double comp = (1. - mu) / r1 / r1sq;
    double ssq = sq(spin);
    if (star == kStar1)
        return V3{comp * p.x + mu1 * (p.x - 1.) - ssq * p.x + mu,
                  comp * p.y + mu1 * p.y - ssq * p.y, comp * p.z + mu1 * p.z};
    return V3{comp * p.x + mu1 * (p.x - 1.) - ssq * (p.x - 1.) + mu - 1.,
              comp * p.y + mu1 * p.y - ssq * p.y, comp * p.z + mu1 * p.z};
}

// Newton iteration on the L1 quintic (roche.cpp:8-80, xl1.cpp:47-76).
// Returns a negative value when the iteration cap is reached.
LCG_HD double xl_quintic(double a1, double a2, double a3, double a4, double a5,
                         double a6, double q) {
    double d1 = 1. * a2, d2 = 2. * a3, d3 = 3. * a4, d4 = 4. * a5, d5 = 5. * a6;
    int n = 0;
    double xold = 0., x = 1. / (1. + q), f, df;
    while (n < 1000 && fabs(x - xold) > 1.e-12 * fabs(x)) {
        xold = x;
        f = x * (x * (x * (x * (x * a6 + a5) + a4) + a3) + a2) + a1;
        df = x * (x * (x * (x * d5 + d4) + d3) + d2) + d1;
        x -= f / df;
        n++;
    }
    return n == 1000 ? -1. : x;
}

LCG_HD double xl11(double q, double spin) {
    double ssq = spin * spin, mu = q / (1. + q);
    return xl_quintic(-1. + mu, 2. - 2. * mu, -1. + mu, ssq + 2. * mu, -2. * ssq - mu, ssq, q);
}

LCG_HD double xl12(double q, double spin) {
    double ssq = spin * spin, mu = q / (1. + q);
    return xl_quintic(-1. + mu, 2. - 2. * mu, -ssq + mu, 3. * ssq + 2. * mu - 2.,
                      1. - mu - 3. * ssq, ssq, q);
}

LCG_HD double xl1(double q) {
    double mu = q / (1. + q);
    return xl_quintic(-1. + mu, 2. - 2. * mu, -1. + mu, 1. + 2. * mu, -2. - mu, 1., q);
}

// Roche::ref_sphere (ref_sphere.cpp:30-40)
LCG_HD void ref_sphere(int star, double q, double spin, double ffac, double &rref,
                       double &pref) {
    if (star == kStar1) {
        double tref = xl11(q, spin);
        rref = dmin(1.001 * ffac, 1.0) * tref;
        pref = rpot1(q, spin, v3(ffac * tref, 0., 0.));
    } else {
        double tref = 1. - xl12(q, spin);
        rref = dmin(1.001 * ffac, 1.0) * tref;
        pref = rpot2(q, spin, v3(1. - ffac * tref, 0., 0.));
    }
}

// Roche::set_earth (set_earth.cpp:39-46)
LCG_HD V3 set_earth(double cosi, double sini, double phase) {
    double rp = kTwoPi * phase;
    double cosp = cos(rp), sinp = sin(rp);
    return V3{sini * cosp, -sini * sinp, cosi};
}

// Potential along a face ray, as in Roche::face_chop_batch (face.cpp:85-102):
// the distance to the star's own centre is the ray parameter itself.
LCG_HD double chop_pot(int star, double q, double spin, double dx, double dy, double r) {
    const double mu = q / (1 + q), comp = 1. - mu, ss = spin * spin;
    const bool primary = (star == kStar1);
    double rdx = r * dx;
    double px = (primary ? 0. : 1.) + rdx;
    double py = r * dy;
    double x2y2 = px * px + py * py;
    double rr = r * r;
    double dcomp = sqrt(rr + 1. + (primary ? -2. : 2.) * rdx);
    if (primary) return -comp / r - mu / dcomp - ss * x2y2 / 2. + mu * px;
    return -comp / dcomp - mu / r - ss * (0.5 + 0.5 * x2y2 - px) - comp * px;
}

// Potential along a face ray as in RayPot (face.cpp:34-62).
LCG_HD double ray_pot(int star, double q, double spin, V3 d, double rad) {
    const double mu = q / (1 + q), comp = 1. - mu, ss = spin * spin;
    double px = (star == kStar1 ? 0. : 1.) + rad * d.x, py = rad * d.y, pz = rad * d.z;
    double x2y2 = px * px + py * py;
    double r1sq = x2y2 + pz * pz;
    double r1 = sqrt(r1sq);
    double r2 = sqrt(r1sq + 1. - 2. * px);
    if (star == kStar1) return -comp / r1 - mu / r2 - ss * x2y2 / 2. + mu * px;
    return -comp / r1 - mu / r2 - ss * (0.5 + 0.5 * x2y2 - px) - comp * px;
}

// One lane of Roche::face_chop_batch (face.cpp:71-161): 0 ok, 1 reference
// radius below pref, 2 search failed, 3 chop cap.
LCG_HD int face_chop(int star, double q, double spin, double dx, double dy, double rref,
                     double pref, double acc, double &rad) {
    int fail = chop_pot(star, q, spin, dx, dy, rref) < pref ? 1 : 0;
    double r1 = rref / 2, r2 = rref, tref = pref + 1.;
    if (!fail) {
        for (int it = 0; it < 30 && tref > pref; it++) {
            r1 = r2 / 2;
            double t = chop_pot(star, q, spin, dx, dy, r1);
            tref = t;
            if (t > pref) r2 = r1;
        }
        if (tref > pref) fail = 2;
    }
    if (!fail) {
        for (int nchop = 0; nchop < 100 && r2 - r1 > acc; nchop++) {
            double r = (r1 + r2) / 2.;
            if (chop_pot(star, q, spin, dx, dy, r) < pref) r1 = r;
            else r2 = r;
        }
        if (r2 - r1 > acc) fail = 3;
    }
    rad = (r1 + r2) / 2.;
    return fail;
}

// Roche::face (face.cpp:163-220) without the exception: returns 0 on
// success, 1/2/3 for the three failure modes.
LCG_HD int face_scalar(int star, double q, double spin, V3 dirn, double rref, double pref,
                       double acc, V3 &pvec, V3 &dvec, double &r, double &g) {
    double tref = ray_pot(star, q, spin, dirn, rref);
    if (tref < pref) return 1;
    double r1 = rref / 2, r2 = rref;
    tref = pref + 1;
    for (int i = 0; i < 30 && tref > pref; i++) {
        r1 = r2 / 2;
        tref = ray_pot(star, q, spin, dirn, r1);
        if (tref > pref) r2 = r1;
    }
    if (tref > pref) return 2;
    int nchop = 0;
    while (r2 - r1 > acc && nchop < 100) {
        double rr = (r1 + r2) / 2.;
        if (ray_pot(star, q, spin, dirn, rr) < pref) r1 = rr;
        else r2 = rr;
        nchop++;
    }
    if (nchop == 100) return 3;
    r = (r1 + r2) / 2.;
    const V3 cofm = star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    pvec = add(cofm, scale(r, dirn));
    dvec = drpot(star, q, spin, pvec);
    g = len(dvec);
    dvec.x /= g;
    dvec.y /= g;
    dvec.z /= g;
    return 0;
}

// Roche::sphere_eclipse, phase form (sphere_eclipse.cpp:33-79)
LCG_HD bool sphere_eclipse_ph(double cosi, double sini, V3 r, V3 c, double rs, double &phi1,
                              double &phi2, double &lam1, double &lam2) {
    const V3 d = sub(r, c);
    const double PDIST = sqrt(sq(d.x) + sq(d.y));
    const double BQUAD = d.z * cosi - PDIST * sini;
    if (BQUAD >= 0.) return false;
    const double CQUAD = norm2(d) - sq(rs);
    double fac = sq(BQUAD) - CQUAD;
    if (fac <= 0.) return false;
    fac = sqrt(fac);
    lam2 = -BQUAD + fac;
    lam1 = dmax(0., CQUAD / lam2);
    if (CQUAD < 0.) {
        phi1 = 0.;
        phi2 = 1.;
    } else {
        double delta = acos((cosi * d.z + sqrt(CQUAD)) / (sini * PDIST));
        double phi = atan2(d.y, -d.x);
        phi1 = (phi - delta) / kTwoPi;
        phi1 -= floor(phi1);
        phi2 = phi1 + 2. * delta / kTwoPi;
    }
    return true;
}

// Roche::sphere_eclipse, line-of-sight form (sphere_eclipse.cpp:94-115)
LCG_HD bool sphere_eclipse_los(V3 earth, V3 r, V3 c, double rs, double &lam1, double &lam2) {
    const V3 d = sub(r, c);
    const double BQUAD = dot(earth, d);
    if (BQUAD >= 0.) return false;
    const double CQUAD = norm2(d) - sq(rs);
    double fac = sq(BQUAD) - CQUAD;
    if (fac <= 0.) return false;
    fac = sqrt(fac);
    lam2 = -BQUAD + fac;
    lam1 = dmax(0., CQUAD / lam2);
    return true;
}

// Subs::planck / Subs::dlpdlt (new_subs.cpp:125-164)
LCG_HD double planck(double wave, double temp) {
    const double FAC1 = 2.e27 * kH * kC;
    const double FAC2 = 1.e9 * kH * kC / kK;
    double efac = FAC2 / (wave * temp);
    if (efac > 40.) return FAC1 * exp(-efac) / (wave * sq(wave));
    return FAC1 / (exp(efac) - 1.) / (wave * sq(wave));
}

LCG_HD double dlpdlt(double wave, double temp) {
    const double FAC2 = 1.e9 * kH * kC / kK;
    double efac = FAC2 / (wave * temp);
    return efac / (1. - exp(-efac));
}

// Lcurve::Ginterp (lcurve.h:92-148)
struct Ginterp {
    double phase1, phase2, scale11, scale12, scale21, scale22;
};

LCG_HD double gi_scale1(const Ginterp &g, double phase) {
    double pnorm = phase - floor(phase);
    if (pnorm <= g.phase1 || pnorm >= 1. - g.phase1) return 1.;
    return (g.scale11 * (1. - g.phase1 - pnorm) + g.scale12 * (pnorm - g.phase1)) /
           (1 - 2. * g.phase1);
}

LCG_HD double gi_scale2(const Ginterp &g, double phase) {
    double pnorm = phase - floor(phase);
    if (pnorm >= g.phase2 && pnorm <= 1. - g.phase2) return 1.;
    if (pnorm < 0.5)
        return (g.scale22 * (g.phase2 - pnorm) + g.scale21 * (pnorm + g.phase2)) /
               (2. * g.phase2);
    return (g.scale21 * (1. + g.phase2 - pnorm) + g.scale22 * (pnorm - 1. + g.phase2)) /
           (2. * g.phase2);
}

LCG_HD int gi_type(const Ginterp &g, double phase) {
    double pnorm = phase - floor(phase);
    if (pnorm <= g.phase1 || pnorm >= 1. - g.phase1) return 1;
    if ((pnorm > g.phase1 && pnorm < g.phase2) || (pnorm > 1. - g.phase2 && pnorm < 1. - g.phase1))
        return 2;
    return 3;
}

}  // namespace lcg
