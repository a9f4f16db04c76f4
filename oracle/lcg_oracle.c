/*
 * lcg_oracle.c — CPU restatement of lcurve_re's model-evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine, never part of
 * the product. Each routine restates one reference routine (cited by
 * file:line of the lcurve_re source tree) in the same floating-point
 * operation order, so that with -ffp-contract=off and the same libm it
 * reproduces the reference bit for bit. tests/test_oracle_pin.py checks that
 * against the reference compiled from its own sources (oracle/_ref).
 *
 * C++ exceptions of the reference become integer statuses (lcg_status) with
 * the reference's message text.
 */
#define _DEFAULT_SOURCE
#include "lcg_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- constants (src/lcurve_base/constants.h:15-95) --------------------- */
static const double C_LIGHT = 2.99792458e8;
static const double H_PLANCK = 6.6262e-34;
static const double K_BOLTZ = 1.3806e-23;
static const double PI_ = 3.14159265358979323846264;
#define TWOPI_ (2. * PI_)
static const float DAY_F = 86400.f;

typedef struct { double x, y, z; } v3;

static inline v3 mk3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline double dot3(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline double len3(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline double sqr3(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline v3 add3(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub3(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 scl3(double c, v3 a) { return mk3(c * a.x, c * a.y, c * a.z); }
static inline double sqr(double a) { return a * a; }
/* new_subs.h:187-195 */
static inline double deg2rad(double d) { return M_PI * d / 180.; }
static inline double rad2deg(double r) { return 180. * r / M_PI; }
/* std::min / std::max argument conventions */
static inline double dmin(double a, double b) { return (b < a) ? b : a; }
static inline double dmax(double a, double b) { return (a < b) ? b : a; }
/* new_subs.h:95-99 */
static inline double dsign(double a, double b) { return b >= 0. ? fabs(a) : -fabs(a); }

typedef struct { int st; char msg[256]; } oerr;

static int seterr(oerr *e, int st, const char *fmt, ...) {
    if (e && e->st == LCG_OK) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(e->msg, sizeof(e->msg), fmt, ap);
        va_end(ap);
        e->st = st;
    }
    return st;
}

static void copyerr(const oerr *e, char *err, int errlen) {
    if (err && errlen > 0) {
        strncpy(err, e->msg, (size_t)errlen - 1);
        err[errlen - 1] = 0;
    }
}

/* ---- black body (src/new_subs.cpp:125-164) ----------------------------- */
static double planck(double wave, double temp) {
    const double FAC1 = 2.e27 * H_PLANCK * C_LIGHT;
    const double FAC2 = 1.e9 * H_PLANCK * C_LIGHT / K_BOLTZ;
    double efac = FAC2 / (wave * temp);
    if (efac > 40.)
        return FAC1 * exp(-efac) / (wave * sqr(wave));
    return FAC1 / (exp(efac) - 1.) / (wave * sqr(wave));
}

static double dlpdlt(double wave, double temp) {
    const double FAC2 = 1.e9 * H_PLANCK * C_LIGHT / K_BOLTZ;
    double efac = FAC2 / (wave * temp);
    return efac / (1. - exp(-efac));
}

/* ---- L1 point (src/lroche_base/roche.cpp:8-80, xl1.cpp:47-76) ----------- */
static double xl_newton(double a1, double a2, double a3, double a4, double a5,
                        double a6, double q, oerr *e, const char *who) {
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
    if (n == 1000)
        seterr(e, LCG_E_NOCONVERGE, "Roche::%s: exceeded maximum iterations", who);
    return x;
}

static double xl11(double q, double spin, oerr *e) {
    if (q <= 0.) {
        seterr(e, LCG_E_INVALID, "Roche::xl11(double, double): q = %f <= 0.", q);
        return 0.;
    }
    double ssq = spin * spin, mu = q / (1. + q);
    return xl_newton(-1. + mu, 2. - 2. * mu, -1. + mu, ssq + 2. * mu,
                     -2. * ssq - mu, ssq, q, e, "xl11(double, double)");
}

static double xl12(double q, double spin, oerr *e) {
    if (q <= 0.) {
        seterr(e, LCG_E_INVALID, "Roche::xl12(double, double): q = %f <= 0.", q);
        return 0.;
    }
    double ssq = spin * spin, mu = q / (1. + q);
    return xl_newton(-1. + mu, 2. - 2. * mu, -ssq + mu, 3. * ssq + 2. * mu - 2.,
                     1. - mu - 3. * ssq, ssq, q, e, "xl12(double,double)");
}

static double xl1(double q, oerr *e) {
    if (q <= 0.) {
        seterr(e, LCG_E_INVALID, "Roche::xl1(double): q = %f <= 0.", q);
        return 0.;
    }
    double mu = q / (1. + q);
    return xl_newton(-1. + mu, 2. - 2. * mu, -1. + mu, 1. + 2. * mu, -2. - mu,
                     1., q, e, "xl1(double)");
}

/* ---- Roche potential and gradient (rpot.cpp:37-86, drpot.cpp:40-85) ---- */
static double rpot1(double q, double spin, v3 p) {
    double mu = q / (1 + q), comp = 1. - mu;
    double x2y2 = sqr(p.x) + sqr(p.y), z2 = sqr(p.z);
    double r1sq = x2y2 + z2, r1 = sqrt(r1sq);
    double r2 = sqrt(r1sq + 1. - 2. * p.x);
    return (-comp / r1 - mu / r2 - sqr(spin) * x2y2 / 2. + mu * p.x);
}

static double rpot2(double q, double spin, v3 p) {
    const double mu = q / (1 + q), comp = 1. - mu;
    const double px = p.x, py = p.y, pz = p.z;
    const double x2y2 = px * px + py * py;
    const double r1sq = x2y2 + pz * pz;
    const double r1 = sqrt(r1sq);
    const double r2 = sqrt(r1sq + 1.0 - 2.0 * px);
    const double spin_sq = spin * spin;
    return -comp / r1 - mu / r2 - spin_sq * (0.5 + 0.5 * x2y2 - px) - comp * px;
}

static v3 drpot1(double q, double spin, v3 p) {
    double r1sq = sqr3(p), r1 = sqrt(r1sq);
    double r2sq = r1sq + 1. - 2. * p.x, r2 = sqrt(r2sq);
    double mu = q / (1 + q);
    double mu1 = mu / r2 / r2sq;
    double comp = (1. - mu) / r1 / r1sq;
    double ssq = sqr(spin);
    return mk3(comp * p.x + mu1 * (p.x - 1.) - ssq * p.x + mu,
               comp * p.y + mu1 * p.y - ssq * p.y,
               comp * p.z + mu1 * p.z);
}

static v3 drpot2(double q, double spin, v3 p) {
    double r1sq = sqr3(p), r1 = sqrt(r1sq);
    double r2sq = r1sq + 1. - 2. * p.x, r2 = sqrt(r2sq);
    double mu = q / (1 + q);
    double mu1 = mu / r2 / r2sq;
    double comp = (1. - mu) / r1 / r1sq;
    double ssq = sqr(spin);
    return mk3(comp * p.x + mu1 * (p.x - 1.) - ssq * (p.x - 1.) + mu - 1.,
               comp * p.y + mu1 * p.y - ssq * p.y,
               comp * p.z + mu1 * p.z);
}

/* ref_sphere.cpp:30-40 */
static void ref_sphere(double q, int star, double spin, double ffac,
                       double *rref, double *pref, oerr *e) {
    double tref;
    if (star == LCG_STAR1) {
        tref = xl11(q, spin, e);
        *rref = dmin(1.001 * ffac, 1.0) * tref;
        *pref = rpot1(q, spin, mk3(ffac * tref, 0., 0.));
    } else {
        tref = 1. - xl12(q, spin, e);
        *rref = dmin(1.001 * ffac, 1.0) * tref;
        *pref = rpot2(q, spin, mk3(1. - ffac * tref, 0., 0.));
    }
}

/* set_earth.cpp:39-46 */
static inline v3 set_earth(double cosi, double sini, double phase) {
    double rp = TWOPI_ * phase;
    double cosp = cos(rp), sinp = sin(rp);
    return mk3(sini * cosp, -sini * sinp, cosi);
}

/* ---- face radius solve ------------------------------------------------- */

/* Potential along a ray as in Roche::face_chop_batch (face.cpp:85-102). */
static inline double chop_pot(double q, int star, double spin, double dx,
                              double dy, double r) {
    const double mu = q / (1 + q), comp = 1. - mu, spin_sq = spin * spin;
    const int primary = (star == LCG_STAR1);
    const double cx = primary ? 0. : 1.;
    double rdx = r * dx;
    double px = cx + rdx;
    double py = r * dy;
    double x2y2 = px * px + py * py;
    double rr = r * r;
    double down = r;
    double dcomp = sqrt(rr + 1. + (primary ? -2. : 2.) * rdx);
    if (primary)
        return -comp / down - mu / dcomp - spin_sq * x2y2 / 2. + mu * px;
    return -comp / dcomp - mu / down - spin_sq * (0.5 + 0.5 * x2y2 - px) - comp * px;
}

/* One lane of Roche::face_chop_batch (face.cpp:71-161). Returns the fail
 * code: 0 ok, 1 reference radius below pref, 2 search failed, 3 chop cap. */
static int face_chop(double q, int star, double spin, double dx, double dy,
                     double rref, double pref, double acc, double *rad) {
    int fail = chop_pot(q, star, spin, dx, dy, rref) < pref ? 1 : 0;
    double r1 = rref / 2, r2 = rref, tref = pref + 1.;
    if (!fail) {
        for (int it = 0; it < 30 && tref > pref; it++) {
            r1 = r2 / 2;
            double t = chop_pot(q, star, spin, dx, dy, r1);
            tref = t;
            if (t > pref) r2 = r1;
        }
        if (tref > pref) fail = 2;
    }
    if (!fail) {
        for (int nchop = 0; nchop < 100 && r2 - r1 > acc; nchop++) {
            double r = (r1 + r2) / 2.;
            if (chop_pot(q, star, spin, dx, dy, r) < pref) r1 = r;
            else r2 = r;
        }
        if (r2 - r1 > acc) fail = 3;
    }
    *rad = (r1 + r2) / 2.;
    return fail;
}

/* Potential along a ray as in RayPot (face.cpp:34-62). */
static inline double ray_pot(double q, int star, double spin, v3 d, double rad) {
    const double mu = q / (1 + q), comp = 1. - mu, spin_sq = spin * spin;
    const double cx = (star == LCG_STAR1) ? 0. : 1.;
    double px = cx + rad * d.x, py = rad * d.y, pz = rad * d.z;
    double x2y2 = px * px + py * py;
    double r1sq = x2y2 + pz * pz;
    double r1 = sqrt(r1sq);
    double r2 = sqrt(r1sq + 1. - 2. * px);
    if (star == LCG_STAR1)
        return -comp / r1 - mu / r2 - spin_sq * x2y2 / 2. + mu * px;
    return -comp / r1 - mu / r2 - spin_sq * (0.5 + 0.5 * x2y2 - px) - comp * px;
}

/* Roche::face (face.cpp:163-220). */
static int face_scalar(double q, int star, double spin, v3 dirn, double rref,
                       double pref, double acc, v3 *pvec, v3 *dvec, double *r,
                       double *g, oerr *e) {
    const v3 cofm = (star == LCG_STAR1) ? mk3(0., 0., 0.) : mk3(1., 0., 0.);
    double tref = ray_pot(q, star, spin, dirn, rref);
    if (tref < pref)
        return seterr(e, LCG_E_ROCHE,
                      "Roche::face error: point at reference radius = %f appears "
                      "to have a lower potential = %f than the reference = %f",
                      rref, tref, pref);
    double r1 = rref / 2, r2 = rref;
    tref = pref + 1;
    for (int i = 0; i < 30 && tref > pref; i++) {
        r1 = r2 / 2;
        tref = ray_pot(q, star, spin, dirn, r1);
        if (tref > pref) r2 = r1;
    }
    if (tref > pref)
        return seterr(e, LCG_E_ROCHE,
                      "Roche::face error: could not find a radius with a potential "
                      "below the reference potential; probably bad inputs.");
    int nchop = 0;
    while (r2 - r1 > acc && nchop < 100) {
        double rr = (r1 + r2) / 2.;
        if (ray_pot(q, star, spin, dirn, rr) < pref) r1 = rr;
        else r2 = rr;
        nchop++;
    }
    if (nchop == 100)
        return seterr(e, LCG_E_ROCHE,
                      "Roche::face error: reached maximum number of binary chops = 100");
    *r = (r1 + r2) / 2.;
    *pvec = add3(cofm, scl3(*r, dirn));
    *dvec = (star == LCG_STAR1) ? drpot1(q, spin, *pvec) : drpot2(q, spin, *pvec);
    *g = len3(*dvec);
    dvec->x /= *g; dvec->y /= *g; dvec->z /= *g;
    return LCG_OK;
}

/* ---- eclipse by a sphere (sphere_eclipse.cpp:33-79, 94-115) ------------- */
static int sphere_eclipse_ph(double cosi, double sini, v3 r, v3 c, double rs,
                             double *phi1, double *phi2, double *lam1,
                             double *lam2) {
    const v3 d = sub3(r, c);
    const double PDIST = sqrt(sqr(d.x) + sqr(d.y));
    const double BQUAD = d.z * cosi - PDIST * sini;
    if (BQUAD >= 0.) return 0;
    const double CQUAD = sqr3(d) - sqr(rs);
    double fac = sqr(BQUAD) - CQUAD;
    if (fac <= 0.) return 0;
    fac = sqrt(fac);
    *lam2 = -BQUAD + fac;
    *lam1 = dmax(0., CQUAD / *lam2);
    if (CQUAD < 0.) {
        *phi1 = 0.;
        *phi2 = 1.;
    } else {
        double delta = acos((cosi * d.z + sqrt(CQUAD)) / (sini * PDIST));
        double phi = atan2(d.y, -d.x);
        *phi1 = (phi - delta) / TWOPI_;
        *phi1 -= floor(*phi1);
        *phi2 = *phi1 + 2. * delta / TWOPI_;
    }
    return 1;
}

static int sphere_eclipse_los(v3 earth, v3 r, v3 c, double rs, double *lam1,
                              double *lam2) {
    const v3 d = sub3(r, c);
    const double BQUAD = dot3(earth, d);
    if (BQUAD >= 0.) return 0;
    const double CQUAD = sqr3(d) - sqr(rs);
    double fac = sqr(BQUAD) - CQUAD;
    if (fac <= 0.) return 0;
    fac = sqrt(fac);
    *lam2 = -BQUAD + fac;
    *lam1 = dmax(0., CQUAD / *lam2);
    return 1;
}

/* ---- potential along lines of sight (rpot_val.cpp, rpot_grad.cpp,
 *      rpot_val_grad.cpp) -------------------------------------------------- */
typedef struct {
    double q, spin, cosi, sini;
    int star;
    v3 p;
    /* line in (phi, lambda): phi + dphi*x, lam + dlam*x (roche.h:258-324) */
    double phi, dphi, lam, dlam;
    /* fixed earth for the lambda-only functions (roche.h:328-365) */
    v3 earth;
    int mode; /* 0: (phi, lam) line, 1: lambda with fixed earth */
} linefn;

static inline double rpot_at(double q, int star, double spin, v3 r) {
    return star == LCG_STAR1 ? rpot1(q, spin, r) : rpot2(q, spin, r);
}

static inline void rpot_grad(double q, int star, double spin, v3 earth, v3 p,
                             double lam, double *dphi, double *dlam) {
    v3 r = add3(p, scl3(lam, earth));
    v3 d = star == LCG_STAR1 ? drpot1(q, spin, r) : drpot2(q, spin, r);
    v3 ed = mk3(earth.y, -earth.x, 0.);
    *dphi = TWOPI_ * lam * dot3(d, ed);
    *dlam = dot3(d, earth);
}

static double lf_val(const linefn *f, double x) {
    if (f->mode == 1)
        return rpot_at(f->q, f->star, f->spin, add3(f->p, scl3(x, f->earth)));
    v3 earth = set_earth(f->cosi, f->sini, f->phi + f->dphi * x);
    return rpot_at(f->q, f->star, f->spin,
                   add3(f->p, scl3(f->lam + f->dlam * x, earth)));
}

static double lf_der(const linefn *f, double x) {
    double dp, dl;
    if (f->mode == 1) {
        rpot_grad(f->q, f->star, f->spin, f->earth, f->p, x, &dp, &dl);
        return dl;
    }
    rpot_grad(f->q, f->star, f->spin,
              set_earth(f->cosi, f->sini, f->phi + f->dphi * x), f->p,
              f->lam + f->dlam * x, &dp, &dl);
    return (dp * f->dphi + dl * f->dlam);
}

/* Subs::dbrent with early exit (src/dbrent.cpp:21-126). */
static double dbrent(double ax, double bx, double cx, const linefn *f,
                     double acc, int stopfast, double fref, double *xmin,
                     oerr *e) {
    double a = (ax < cx ? ax : cx);
    double b = (ax > cx ? ax : cx);
    double x, w, v;
    x = w = v = bx;
    double fw, fv, fx;
    fw = fv = fx = lf_val(f, x);
    if (stopfast && fx < fref) { *xmin = x; return fx; }
    double dw, dv, dx;
    dw = dv = dx = lf_der(f, x);
    double xm, tol1, tol2, e_ = 0., d1, d2, u1, u2, olde, d = 0, u, fu, du;
    int ok1, ok2;
    for (int iter = 0; iter < 100; iter++) {
        xm = 0.5 * (a + b);
        tol1 = acc;
        tol2 = 2. * tol1;
        if (fabs(x - xm) <= (tol2 - 0.5 * (b - a))) { *xmin = x; return fx; }
        if (fabs(e_) > tol1) {
            d2 = d1 = 2. * (b - a);
            if (dw != dx) d1 = (w - x) * dx / (dx - dw);
            if (dv != dx) d2 = (v - x) * dx / (dx - dv);
            u1 = x + d1;
            u2 = x + d2;
            ok1 = (a - u1) * (u1 - b) > 0. && dx * d1 <= 0.;
            ok2 = (a - u2) * (u2 - b) > 0. && dx * d2 <= 0.;
            olde = e_;
            e_ = d;
            if (ok1 || ok2) {
                if (ok1 && ok2) d = (fabs(d1) < fabs(d2) ? d1 : d2);
                else if (ok1) d = d1;
                else d = d2;
                if (fabs(d) <= fabs(0.5 * olde)) {
                    u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = dsign(tol1, xm - x);
                } else {
                    d = 0.5 * (e_ = (dx >= 0. ? a - x : b - x));
                }
            } else {
                d = 0.5 * (e_ = (dx >= 0. ? a - x : b - x));
            }
        } else {
            d = 0.5 * (e_ = (dx >= 0. ? a - x : b - x));
        }
        if (fabs(d) >= tol1) {
            u = x + d;
            fu = lf_val(f, u);
            if (stopfast && fu < fref) { *xmin = u; return fu; }
        } else {
            u = x + dsign(tol1, d);
            fu = lf_val(f, u);
            if (stopfast && fu < fref) { *xmin = u; return fu; }
            if (fu > fx) { *xmin = x; return fx; }
        }
        du = lf_der(f, u);
        if (fu <= fx) {
            if (u >= x) a = x; else b = x;
            v = w; fv = fw; dv = dw;
            w = x; fw = fx; dw = dx;
            x = u; fx = fu; dx = du;
        } else {
            if (u < x) a = u; else b = u;
            if (fu <= fw || w == x) {
                v = w; fv = fw; dv = dw;
                w = u; fw = fu; dw = du;
            } else if (fu < fv || v == x || v == w) {
                v = u; fv = fu; dv = du;
            }
        }
    }
    (void)fv;
    seterr(e, LCG_E_NOCONVERGE, "Subs::dbrent: too many iterations");
    *xmin = x;
    return fx;
}

/* Roche::linmin (pot_min.cpp:127-420). The reference leaves `jammed` unset
 * on its early returns; every such return reaches pot_min's
 * |pmin - pot| < DELPHI test with pmin == pot, so initialising it to false
 * gives the same result. */
static void linmin(double q, int star, double spin, double cosi, double sini,
                   v3 p, double *phi, double *lam, double dphi, double dlam,
                   double phi1, double phi2, double lam1, double lam2,
                   double pref, double acc, double *pmin, int *jammed,
                   oerr *e) {
    linefn f = {q, spin, cosi, sini, star, p, *phi, dphi, *lam, dlam, {0, 0, 0}, 0};
    *jammed = 0;
    double xmax = 1.e30, xend;
    int nbound = 0;
    if (dphi != 0.) {
        xend = (phi1 - *phi) / dphi;
        if (xend > 0. && xend < xmax) { nbound = 1; xmax = xend; }
        xend = (phi2 - *phi) / dphi;
        if (xend > 0. && xend < xmax) { nbound = 2; xmax = xend; }
    }
    if (dlam != 0.) {
        xend = (lam1 - *lam) / dlam;
        if (xend > 0. && xend < xmax) { nbound = 3; xmax = xend; }
        xend = (lam2 - *lam) / dlam;
        if (xend > 0. && xend < xmax) { nbound = 4; xmax = xend; }
    }
    double xa = 0., fa = lf_val(&f, xa);
    double xb = 1.e-8 * xmax, fb = lf_val(&f, xb);
    int nten = 0;
    const int NTEN = 7;
    while ((fb >= fa || xa == xb) && nten < NTEN) {
        nten++;
        xb *= 10.;
        fb = lf_val(&f, xb);
    }
    if (fb <= pref) { *phi += dphi * xb; *lam += dlam * xb; *pmin = fb; return; }
    if (fb >= fa) { *pmin = fa; return; }

    int bracketted = 0;
    double xc = 0., fc = 0., dc, xbold = xb, fbold = fb;
    const int NTRY = 5;
    xmax -= xb;
    for (int n = 1; n <= NTRY; n++) {
        xc = xbold + xmax * n / NTRY;
        fc = lf_val(&f, xc);
        if (fc <= pref) { *phi += dphi * xc; *lam += dlam * xc; *pmin = fc; return; }
        if (fc < fb) { xb = xc; fb = fc; }
        else { bracketted = 1; break; }
    }
    *jammed = 0;
    if (!bracketted) {
        dc = lf_der(&f, xc);
        if (dc > 0.) {
            xb = xbold;
            double db = lf_der(&f, xb);
            if (db < 0.) {
                double xm = (xb + xc) / 2.;
                while ((xc - xb) > 1.e-8 * xc) {
                    xm = (xb + xc) / 2.;
                    if (lf_der(&f, xm) > 0.) xc = xm;
                    else xb = xm;
                }
                double fm = lf_val(&f, xm);
                if (fm <= pref) { *phi += dphi * xm; *lam += dlam * xm; *pmin = fm; return; }
                if (fm < fc && fm < fbold) {
                    xb = xm;
                    bracketted = 1;
                } else {
                    seterr(e, LCG_E_ROCHE, "Roche::linmin: failed to bracket minimum, error 3");
                    *pmin = fa;
                    return;
                }
            } else {
                seterr(e, LCG_E_ROCHE, "Roche::linmin: failed to bracket minimum, error 1");
                *pmin = fa;
                return;
            }
        } else {
            *jammed = 1;
            *phi += dphi * xmax;
            *lam += dlam * xmax;
            xmax = 1.;
            rpot_grad(q, star, spin, set_earth(cosi, sini, *phi), p, *lam, &dphi, &dlam);
            switch (nbound) {
            case 1:
                *phi = phi1; dphi = 0.;
                dlam = (dlam > 0.) ? lam1 - *lam : lam2 - *lam;
                break;
            case 2:
                *phi = phi2; dphi = 0.;
                dlam = (dlam > 0.) ? lam1 - *lam : lam2 - *lam;
                break;
            case 3:
                *lam = lam1; dlam = 0.;
                dphi = (dphi > 0.) ? phi1 - *phi : phi2 - *phi;
                break;
            case 4:
                *lam = lam2; dlam = 0.;
                dphi = (dphi > 0.) ? phi1 - *phi : phi2 - *phi;
                break;
            }
            f.phi = *phi; f.dphi = dphi; f.lam = *lam; f.dlam = dlam;
            nten = 0;
            xb = 1.e-6;
            fb = lf_val(&f, xb);
            while (fb >= fa && nten < NTEN) {
                xb *= 10.;
                nten++;
                fb = lf_val(&f, xb);
            }
            if (fb <= pref) { *phi += dphi * xb; *lam += dlam * xb; *pmin = fb; return; }
            if (fb >= fa) { *pmin = fa; return; }
            bracketted = 0;
            for (int n = 1; n <= NTRY; n++) {
                xc = xmax * n / NTRY;
                fc = lf_val(&f, xc);
                if (fc <= pref) { *phi += dphi * xc; *lam += dlam * xc; *pmin = fc; return; }
                if (fc < fb) { xb = xc; fb = fc; }
                else { bracketted = 1; break; }
            }
            if (!bracketted) {
                if (lf_der(&f, xc) > 0.) {
                    seterr(e, LCG_E_ROCHE, "Roche::linmin failed to bracket minimum, error 2");
                    *pmin = fa;
                    return;
                }
                *phi += dphi * xmax;
                *lam += dlam * xmax;
                *pmin = fc;
                return;
            }
        }
    }
    double xmin;
    double xacc = acc / sqrt(sqr(TWOPI_ * dphi) + sqr(dlam));
    *pmin = dbrent(xa, xb, xc, &f, xacc, 1, pref, &xmin, e);
    *phi += dphi * xmin;
    *lam += dlam * xmin;
}

/* Roche::pot_min (pot_min.cpp:38-100). */
static int pot_min(double q, double cosi, double sini, int star, double spin,
                   v3 p, double phi1, double phi2, double lam1, double lam2,
                   double rref, double pref, double acc, double *phi,
                   double *lam, oerr *e) {
    double dphi, dlam, gdphi, gdlam, hdphi, hdlam;
    *phi = (phi1 + phi2) / 2.;
    *lam = (lam1 + lam2) / 2.;
    double rp = TWOPI_ * *phi;
    double cosp = cos(rp), sinp = sin(rp);
    v3 earth = mk3(sini * cosp, -sini * sinp, cosi);
    double pot;
    {
        v3 r = add3(p, scl3(*lam, earth));
        v3 d = star == LCG_STAR1 ? drpot1(q, spin, r) : drpot2(q, spin, r);
        pot = rpot_at(q, star, spin, r);
        v3 ed = mk3(earth.y, -earth.x, 0.);
        dphi = TWOPI_ * *lam * dot3(d, ed);
        dlam = dot3(d, earth);
    }
    if (pot <= pref) return 1;
    gdphi = -dphi;
    gdlam = -dlam;
    dphi = hdphi = gdphi;
    dlam = hdlam = gdlam;
    const double DELPHI = q / (1. + q) * sqr(acc / rref) / 2.;
    double pmin, gam, dgg, gg;
    int jammed;
    for (int its = 0; its < 200; its++) {
        linmin(q, star, spin, cosi, sini, p, phi, lam, dphi, dlam, phi1, phi2,
               lam1, lam2, pref, acc, &pmin, &jammed, e);
        if (e->st) return 0;
        if (pmin <= pref) return 1;
        if (jammed || fabs(pmin - pot) < DELPHI) return 0;
        pot = pmin;
        rp = TWOPI_ * *phi;
        cosp = cos(rp);
        sinp = sin(rp);
        earth = mk3(sini * cosp, -sini * sinp, cosi);
        rpot_grad(q, star, spin, earth, p, *lam, &dphi, &dlam);
        gg = gdphi * gdphi + gdlam * gdlam;
        if (gg == 0.) return 0;
        dgg = (dphi + gdphi) * dphi + (dlam + gdlam) * dlam;
        gam = dgg / gg;
        gdphi = -dphi;
        gdlam = -dlam;
        dphi = hdphi = gdphi + gam * hdphi;
        dlam = hdlam = gdlam + gam * hdlam;
    }
    seterr(e, LCG_E_ROCHE, "Roche::pot_min: too many iterations.");
    return 0;
}

/* Roche::fblink (fblink.cpp:34-104). */
static int fblink(double q, int star, double spin, double acc, v3 earth, v3 p,
                  double rref, double pref, oerr *e) {
    v3 cofm = (star == LCG_STAR1) ? mk3(0., 0., 0.) : mk3(1., 0., 0.);
    double lam1, lam2;
    if (!sphere_eclipse_los(earth, p, cofm, rref, &lam1, &lam2)) return 0;
    if (lam1 == 0.) return 1;
    linefn f = {q, spin, 0., 0., star, p, 0., 0., 0., 0., earth, 1};
    int nstep = 1;
    double step = (lam2 - lam1);
    double f1 = 0., f2 = 0., flam = 1., lam = lam1;
    while (step > acc) {
        lam = lam1 + step / 2.;
        for (int n = 0; n < nstep; n++) {
            flam = lf_val(&f, lam);
            if (flam <= pref) return 1;
            if (nstep == 1) {
                f1 = lf_val(&f, lam1);
                f2 = lf_val(&f, lam2);
            }
            if (flam < f1 && flam < f2) break;
            lam += step;
        }
        if (flam < f1 && flam < f2) break;
        step /= 2.;
        nstep *= 2;
    }
    if (flam < f1 && flam < f2) {
        double xmin;
        oerr sub = {0, ""};
        flam = dbrent(lam1, lam, lam2, &f, acc, 1, pref, &xmin, &sub);
        if (sub.st) {
            seterr(e, LCG_E_ROCHE, "fblink died");
            return 0;
        }
        return (flam < pref);
    }
    return 0;
}

/* Roche::ingress_egress (ingress_egress.cpp:35-97). */
static int ingress_egress(double q, int star, double spin, double iangle,
                          double delta, v3 r, double *ingress, double *egress,
                          double rref, double pref, oerr *e) {
    double ri = deg2rad(iangle);
    double cosi = cos(ri), sini = sin(ri);
    v3 cofm = (star == LCG_STAR1) ? mk3(0., 0., 0.) : mk3(1., 0., 0.);
    double phi1, phi2, lam1, lam2, phi, lam;
    if (!sphere_eclipse_ph(cosi, sini, r, cofm, rref, &phi1, &phi2, &lam1, &lam2))
        return 0;
    const double ACC = 2. * sqrt(2. * TWOPI_ * (lam2 - lam1) * delta);
    if (!pot_min(q, cosi, sini, star, spin, r, phi1, phi2, lam1, lam2, rref,
                 pref, ACC, &phi, &lam, e))
        return 0;
    double pin = phi, pout = phi1, pmid;
    while (fabs(pin - pout) > delta) {
        pmid = (pin + pout) / 2.;
        if (fblink(q, star, spin, ACC, set_earth(cosi, sini, pmid), r, rref, pref, e))
            pin = pmid;
        else
            pout = pmid;
        if (e->st) return 0;
    }
    *ingress = (pin + pout) / 2.;
    *ingress = *ingress - floor(*ingress);
    pin = phi;
    pout = phi2;
    while (fabs(pin - pout) > delta) {
        pmid = (pin + pout) / 2.;
        if (fblink(q, star, spin, ACC, set_earth(cosi, sini, pmid), r, rref, pref, e))
            pin = pmid;
        else
            pout = pmid;
        if (e->st) return 0;
    }
    *egress = (pin + pout) / 2.;
    *egress = *egress - floor(*egress);
    if (*egress < *ingress) *egress += 1;
    return 1;
}

/* ---- model scalars ----------------------------------------------------- */

/* Model::get_r1r2 (lcurve.h:399-410). */
static void get_r1r2(const lcg_model *m, double *rr1, double *rr2) {
    if (m->use_radii) {
        *rr1 = m->r1;
        *rr2 = m->r2;
    } else {
        double sini = sin(deg2rad(m->iangle));
        double r2pr1 = sqrt(1.0 - pow(sini * cos(2.0 * M_PI * m->cphi4), 2));
        double r2mr1 = sqrt(1.0 - pow(sini * cos(2.0 * M_PI * m->cphi3), 2));
        *rr1 = (r2pr1 - r2mr1) / 2.0;
        *rr2 = (r2pr1 + r2mr1) / 2.0;
    }
}

/* Everything set_star_grid derives before tiling (set_star_grid.cpp:52-197). */
typedef struct {
    double r1, r2, rl1, rl2;
    double rref1, pref1, rref2, pref2, ffac1, ffac2;
    double gref;
    int infill;
    double thelo, thehi;
    int nlat, nlatfill, nlngfill, eclipse;
} grid_setup;

/* set_star_grid.cpp:528-538 */
static void envelope(double rangle, double lambda, double r1, double *x, double *y) {
    double sini = sin(rangle), cosi = cos(rangle);
    double sinl = sin(lambda), cosl = cos(lambda);
    double norm = sqrt(cosi * cosi + sini * sini * cosl * cosl);
    *x = sinl + r1 * cosi * sinl / norm;
    *y = -cosi * cosl - r1 * cosl / norm;
}

static int grid_prepare(const lcg_model *m, int star, int fine, grid_setup *s,
                        oerr *e) {
    double r1, r2;
    get_r1r2(m, &r1, &r2);
    s->eclipse = star == LCG_STAR1 ? m->eclipse1 : m->eclipse2;
    s->nlat = star == LCG_STAR1 ? (fine ? m->nlat1f : m->nlat1c)
                                : (fine ? m->nlat2f : m->nlat2c);
    s->nlatfill = star == LCG_STAR1 ? 0 : (fine ? m->nlatfill : 0);
    s->nlngfill = star == LCG_STAR1 ? 0 : (fine ? m->nlngfill : 0);
    double latlo = star == LCG_STAR1 ? 0 : m->llo;
    double lathi = star == LCG_STAR1 ? 0 : m->lhi;
    if (s->nlat <= 0)
        return seterr(e, LCG_E_INVALID, "set_star_grid: nlat = %d must be positive", s->nlat);
    if (m->q <= 0.)
        return seterr(e, LCG_E_INVALID, "Roche::xl11(double, double): q = %f <= 0.", m->q);

    double rl1 = xl11(m->q, m->spin1, e);
    if (e->st) return e->st;
    if (r1 < 0) r1 = rl1;
    else if (r1 > rl1)
        return seterr(e, LCG_E_LOBE, "set_star_grid: the primary star is larger than its Roche lobe!");
    double rl2 = 1. - xl12(m->q, m->spin2, e);
    if (e->st) return e->st;
    if (r2 < 0) r2 = rl2;
    else if (r2 > rl2)
        return seterr(e, LCG_E_LOBE, "set_star_grid: the secondary star is larger than its Roche lobe!");
    if (m->glens1 && star == LCG_STAR2 && m->roche1 && m->eclipse2)
        return seterr(e, LCG_E_INVALID,
                      "set_star_grid: cannot have gravitational lensing, eclipse and Roche lobe geometry at the same time");
    if (m->glens1 && star == LCG_STAR2) {
        double gm = pow(1000. * m->velocity_scale, 3) * m->tperiod * DAY_F / TWOPI_;
        double a = pow(gm / sqr(TWOPI_ / DAY_F / m->tperiod), 1. / 3.);
        double rlens1 = 4. * gm / (1. + m->q) / a / sqr(C_LIGHT);
        r1 -= rlens1 / (r1 / (1. - r2 / 2.));
        if (r1 < 0)
            return seterr(e, LCG_E_INVALID,
                          "set_star_grid: gravitational lensing correction more than the current program can cope with.");
    }
    s->r1 = r1; s->r2 = r2; s->rl1 = rl1; s->rl2 = rl2;
    s->ffac1 = r1 / rl1;
    ref_sphere(m->q, LCG_STAR1, m->spin1, s->ffac1, &s->rref1, &s->pref1, e);
    s->ffac2 = r2 / rl2;
    ref_sphere(m->q, LCG_STAR2, m->spin2, s->ffac2, &s->rref2, &s->pref2, e);
    if (e->st) return e->st;

    int infill = m->npole && (star == LCG_STAR2) && (s->nlatfill > 0 || s->nlngfill > 0) && r2 > r1;
    double thelo = 0, thehi = 0;
    if (infill) {
        double rangle = deg2rad(m->iangle);
        double cosi = cos(rangle);
        double ratio = (cosi + r1) / r2;
        if (ratio >= 1.) {
            thehi = PI_ / 2. + rangle;
        } else {
            double llo = 0., lhi = PI_ / 2., x = 0., y = 0.;
            while (lhi > llo + 1.e-7) {
                double lmid = (llo + lhi) / 2.;
                envelope(rangle, lmid, r1, &x, &y);
                if (x * x + y * y < r2 * r2) llo = lmid;
                else lhi = lmid;
            }
            double sini = sin(rangle);
            thehi = dmax(PI_ / 2. - deg2rad(latlo),
                         dmin(PI_ / 2. + rangle, acos(y * sini / r2) + deg2rad(m->lfudge)));
        }
        ratio = (cosi - r1) / r2;
        if (ratio >= 1.) {
            infill = 0;
        } else if (ratio <= -1.) {
            thelo = 0.;
        } else {
            thelo = dmin(PI_ / 2. - deg2rad(lathi),
                         dmax(0., PI_ / 2. - acos(ratio) + rangle - deg2rad(m->lfudge)));
        }
    }
    s->infill = infill;
    s->thelo = thelo;
    s->thehi = thehi;

    const double ACC = m->delta_phase / 10.;
    v3 posn, dvec;
    double rad, gref;
    if (star == LCG_STAR1 && m->roche1) {
        if (face_scalar(m->q, LCG_STAR1, m->spin1, mk3(-1., 0., 0.), s->rref1,
                        s->pref1, ACC, &posn, &dvec, &rad, &gref, e))
            return e->st;
    } else if (star == LCG_STAR2 && m->roche2) {
        if (face_scalar(m->q, LCG_STAR2, m->spin2, mk3(1., 0., 0.), s->rref2,
                        s->pref2, ACC, &posn, &dvec, &rad, &gref, e))
            return e->st;
    } else {
        gref = 1.;
    }
    s->gref = gref;
    return LCG_OK;
}

/* Lcurve::numface (numface.cpp:14-52). */
static int numface(int nlat, int infill, double thelo, double thehi,
                   int nlatfill, int nlngfill) {
    int nface = 0;
    double theta, dphi, dtheta = PI_ / nlat;
    if (infill) {
        int nl1 = (int)ceil(thelo / dtheta);
        for (int i = 0; i < nl1; i++) {
            theta = thelo * (i + 0.5) / nl1;
            dphi = dtheta / sin(theta);
            int k = (int)(2 * PI_ / dphi);
            nface += k > 16 ? k : 16;
        }
        int nl2 = (int)ceil((1 + nlatfill) * (thehi - thelo) / dtheta);
        for (int i = 0; i < nl2; i++) {
            theta = thelo + (thehi - thelo) * (i + 0.5) / nl2;
            dphi = dtheta / sin(theta) / (1 + nlngfill);
            int k = (int)(PI_ / dphi);
            nface += k > 8 ? k : 8;
        }
        int nl3 = (int)ceil((thehi - thelo) / dtheta);
        for (int i = 0; i < nl3; i++) {
            theta = thelo + (thehi - thelo) * (i + 0.5) / nl3;
            dphi = dtheta / sin(theta);
            int k = (int)(PI_ / dphi);
            nface += k > 8 ? k : 8;
        }
        int nl4 = (int)ceil((PI_ - thehi) / dtheta);
        for (int i = 0; i < nl4; i++) {
            theta = thehi + (PI_ - thehi) * (i + 0.5) / nl4;
            dphi = dtheta / sin(theta);
            int k = (int)(2 * PI_ / dphi);
            nface += k > 16 ? k : 16;
        }
    } else {
        nlat = (int)ceil(PI_ / dtheta);
        for (int i = 0; i < nlat; i++) {
            theta = PI_ * (i + 0.5) / nlat;
            dphi = dtheta / sin(theta);
            int k = (int)(2 * PI_ / dphi);
            nface += k > 16 ? k : 16;
        }
    }
    return nface;
}

static int grid_nface(const grid_setup *s) {
    return numface(s->nlat, s->infill, s->thelo, s->thehi, s->nlatfill, s->nlngfill);
}

/* Output arrays of one star grid. */
typedef struct {
    double *posn, *dirn;
    float *area, *gravity, *flux;
    int32_t *necl;
    double *ein, *eout;
} gridout;

/* One latitude ring (set_star_grid.cpp:280-320). */
typedef struct {
    double theta, sint, cost, phi1, phi2;
    int nphi, nl;
} ring;

static void ring_geometry(int star, int infill, int nlat, int nlat1, int nlat2,
                          int nlngfill, double tlo, double thi, double dtheta,
                          int nt, ring *g) {
    if (infill) {
        if (nt < nlat1) {
            g->theta = tlo + (thi - tlo) * (nt + 0.5) / nlat1;
            g->sint = sin(g->theta);
            g->cost = cos(g->theta);
            int k = (int)(PI_ * g->sint * (1 + nlngfill) / dtheta);
            g->nphi = k > 8 ? k : 8;
            g->nl = nlat1;
            if (star == LCG_STAR1) { g->phi1 = -PI_ / 2.; g->phi2 = +PI_ / 2.; }
            else { g->phi1 = +PI_ / 2.; g->phi2 = +3. * PI_ / 2.; }
        } else {
            g->theta = tlo + (thi - tlo) * (nt - nlat1 + 0.5) / nlat2;
            g->sint = sin(g->theta);
            g->cost = cos(g->theta);
            int k = (int)(PI_ * g->sint / dtheta);
            g->nphi = k > 8 ? k : 8;
            g->nl = nlat2;
            if (star == LCG_STAR1) { g->phi1 = +PI_ / 2.; g->phi2 = +3. * PI_ / 2.; }
            else { g->phi1 = -PI_ / 2.; g->phi2 = +PI_ / 2.; }
        }
    } else {
        g->theta = tlo + (thi - tlo) * (nt + 0.5) / nlat;
        g->sint = sin(g->theta);
        g->cost = cos(g->theta);
        int k = (int)(2 * PI_ * g->sint / dtheta);
        g->nphi = k > 16 ? k : 16;
        g->nl = nlat;
        g->phi1 = 0.;
        g->phi2 = TWOPI_;
    }
}

/* Eclipse of one face by the other star (set_star_grid.cpp:372-386). */
static int face_eclipse(const lcg_model *m, const grid_setup *s, int star,
                        v3 pos, double *ein, double *eout, oerr *e) {
    if (!s->eclipse) return 0;
    double ri = deg2rad(m->iangle), cosi = cos(ri), sini = sin(ri);
    double ingress = 0., egress = 0., lam1, lam2;
    int ecl;
    if (star == LCG_STAR1) {
        if (m->roche2)
            ecl = ingress_egress(m->q, LCG_STAR2, m->spin2, m->iangle, m->delta_phase,
                                 pos, &ingress, &egress, s->rref2, s->pref2, e);
        else
            ecl = sphere_eclipse_ph(cosi, sini, pos, mk3(1., 0., 0.), s->r2,
                                    &ingress, &egress, &lam1, &lam2);
    } else {
        if (m->roche1)
            ecl = ingress_egress(m->q, LCG_STAR1, m->spin1, m->iangle, m->delta_phase,
                                 pos, &ingress, &egress, s->rref1, s->pref1, e);
        else
            ecl = sphere_eclipse_ph(cosi, sini, pos, mk3(0., 0., 0.), s->r1,
                                    &ingress, &egress, &lam1, &lam2);
    }
    if (ecl) { *ein = ingress; *eout = egress; }
    return ecl;
}

/* Lcurve::add_faces (set_star_grid.cpp:226-523). */
static int add_faces(const lcg_model *m, const grid_setup *s, int star,
                     gridout *o, int *nface, int cap, double tlo, double thi,
                     double dtheta, int nlatfill, int nlngfill, oerr *e) {
    const int infill = (nlatfill > 0) || (nlngfill > 0);
    int nlat, nlat1 = 0, nlat2 = 0;
    if (infill) {
        nlat1 = (int)ceil((1 + nlatfill) * (thi - tlo) / dtheta);
        nlat2 = (int)ceil((thi - tlo) / dtheta);
        nlat = nlat1 + nlat2;
    } else {
        nlat = (int)ceil((thi - tlo) / dtheta);
    }
    if (nlat <= 0) return LCG_OK;
    int *off = (int *)malloc(sizeof(int) * (size_t)nlat);
    for (int nt = 0; nt < nlat; nt++) {
        off[nt] = *nface;
        ring g;
        ring_geometry(star, infill, nlat, nlat1, nlat2, nlngfill, tlo, thi, dtheta, nt, &g);
        *nface += g.nphi;
    }
    /* The reference sizes its vector by numface (set_star_grid.cpp:162-166)
     * and writes each face at off[nt] + np (:490, :508). For a few nlat
     * (153, 297, 315, 333, 339, ...) the ring tiling has one or two faces
     * more than numface; those writes land past the vector's end and are not
     * part of the grid it goes on to use. Only faces below cap are kept. */
    const double ACC = m->delta_phase / 10.;
    const double q = m->q;
    const int roche_solve = (star == LCG_STAR1 && m->roche1) || (star == LCG_STAR2 && m->roche2);
    const double spin = star == LCG_STAR1 ? m->spin1 : m->spin2;
    const double rref = star == LCG_STAR1 ? s->rref1 : s->rref2;
    const double pref = star == LCG_STAR1 ? s->pref1 : s->pref2;
    const v3 cofm = star == LCG_STAR1 ? mk3(0., 0., 0.) : mk3(1., 0., 0.);
    int first_bad = nlat;
    oerr bad = {0, ""};

#pragma omp parallel for schedule(dynamic)
    for (int nt = 0; nt < nlat; nt++) {
        ring g;
        ring_geometry(star, infill, nlat, nlat1, nlat2, nlngfill, tlo, thi, dtheta, nt, &g);
        const int nhalf = (g.nphi + 1) / 2;
        oerr le = {0, ""};
        for (int np = 0; np < nhalf && !le.st; np++) {
            double phi = g.phi1 + (g.phi2 - g.phi1) * (np + 0.5) / g.nphi;
            double sinp = sin(phi), cosp = cos(phi);
            v3 dirn = m->npole ? mk3(g.sint * cosp, g.sint * sinp, g.cost)
                               : mk3(g.cost, g.sint * cosp, g.sint * sinp);
            v3 posn, dvec;
            double rad, gravity, area;
            if (roche_solve) {
                int fail = face_chop(q, star, spin, dirn.x, dirn.y, rref, pref, ACC, &rad);
                if (fail) {
                    if (face_scalar(q, star, spin, dirn, rref, pref, ACC, &posn, &dvec,
                                    &rad, &gravity, &le))
                        break;
                } else {
                    posn = add3(cofm, scl3(rad, dirn));
                    dvec = star == LCG_STAR1 ? drpot1(q, spin, posn) : drpot2(q, spin, posn);
                    gravity = len3(dvec);
                    dvec.x /= gravity; dvec.y /= gravity; dvec.z /= gravity;
                }
            } else {
                rad = star == LCG_STAR1 ? s->r1 : s->r2;
                posn = add3(cofm, scl3(rad, dirn));
                dvec = dirn;
                gravity = 1.;
            }
            area = ((g.phi2 - g.phi1) / g.nphi * rad * g.sint) *
                   ((thi - tlo) / g.nl * rad) / dot3(dirn, dvec);
            const int i1 = off[nt] + np;
            double ein = 0., eout = 0.;
            int ecl = face_eclipse(m, s, star, posn, &ein, &eout, &le);
            if (i1 < cap) {
                o->posn[3 * i1] = posn.x; o->posn[3 * i1 + 1] = posn.y; o->posn[3 * i1 + 2] = posn.z;
                o->dirn[3 * i1] = dvec.x; o->dirn[3 * i1 + 1] = dvec.y; o->dirn[3 * i1 + 2] = dvec.z;
                o->area[i1] = (float)area;
                o->gravity[i1] = (float)(gravity / s->gref);
                o->necl[i1] = ecl;
                o->ein[i1] = ecl ? ein : 0.;
                o->eout[i1] = ecl ? eout : 0.;
            }
            const int np2 = g.nphi - 1 - np;
            if (np2 != np) {
                v3 dirn2 = dirn, posn2 = posn, dvec2 = dvec;
                if (m->npole) { dirn2.y = -dirn.y; posn2.y = -posn.y; dvec2.y = -dvec.y; }
                else { dirn2.z = -dirn.z; posn2.z = -posn.z; dvec2.z = -dvec.z; }
                (void)dirn2;
                const int i2 = off[nt] + np2;
                ein = eout = 0.;
                ecl = face_eclipse(m, s, star, posn2, &ein, &eout, &le);
                if (i2 >= cap) continue;
                o->posn[3 * i2] = posn2.x; o->posn[3 * i2 + 1] = posn2.y; o->posn[3 * i2 + 2] = posn2.z;
                o->dirn[3 * i2] = dvec2.x; o->dirn[3 * i2 + 1] = dvec2.y; o->dirn[3 * i2 + 2] = dvec2.z;
                o->area[i2] = (float)area;
                o->gravity[i2] = (float)(gravity / s->gref);
                o->necl[i2] = ecl;
                o->ein[i2] = ecl ? ein : 0.;
                o->eout[i2] = ecl ? eout : 0.;
            }
        }
        if (le.st) {
#pragma omp critical(lco_grid_err)
            {
                if (nt < first_bad) { first_bad = nt; bad = le; }
            }
        }
    }
    free(off);
    if (bad.st) {
        if (e->st == LCG_OK) *e = bad;
        return bad.st;
    }
    return LCG_OK;
}

/* set_star_grid.cpp:206-223 */
static int build_grid(const lcg_model *m, const grid_setup *s, int star,
                      gridout *o, int nface_expected, oerr *e) {
    int nface = 0;
    double dtheta = PI_ / s->nlat;
    const int cap = nface_expected;
    int st;
    if (s->infill) {
        st = add_faces(m, s, star, o, &nface, cap, 0., s->thelo, dtheta, 0, 0, e);
        if (!st) st = add_faces(m, s, star, o, &nface, cap, s->thelo, s->thehi, dtheta,
                                s->nlatfill, s->nlngfill, e);
        if (!st) st = add_faces(m, s, star, o, &nface, cap, s->thehi, PI_, dtheta, 0, 0, e);
    } else {
        st = add_faces(m, s, star, o, &nface, cap, 0., PI_, dtheta, 0, 0, e);
    }
    if (st) return st;
    /* fewer tiled faces than numface (nlat 813, 879, ...): the rest of the
     * reference's vector holds default Points (lcurve.h:53-54) */
    for (int i = nface; i < nface_expected; i++) {
        for (int k = 0; k < 3; k++) o->posn[3 * i + k] = o->dirn[3 * i + k] = 0.;
        o->area[i] = 0.f;
        o->gravity[i] = 1.f;
        o->necl[i] = 0;
        o->ein[i] = o->eout[i] = 0.;
    }
    return LCG_OK;
}

/* ---- continuum (set_star_continuum.cpp:26-297) -------------------------- */
static void continuum(const lcg_model *m, int star, int nface,
                      const double *posn, const double *dirn,
                      const float *area, const float *gravity, float *flux) {
    double r1, r2;
    get_r1r2(m, &r1, &r2);
    oerr dummy = {0, ""};
    double rl1 = xl1(m->q, &dummy);
    if (r1 < 0) r1 = rl1;
    double rl2 = 1. - rl1;
    if (r2 < 0) r2 = rl2;
    const double EFAC = sqrt(8. * log(2.));

    if (star == LCG_STAR1) {
        const v3 cofm2 = mk3(1., 0., 0.);
        const double GDCBOL1 = m->gdark_bolom1 ? m->gravity_dark1
                                               : m->gravity_dark1 / dlpdlt(m->wavelength, m->t1);
        v3 spot[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, uespot = {0, 0, 0};
        int is_spot[3];
        for (int k = 0; k < 3; k++) {
            is_spot[k] = m->stsp_defined[k];
            if (is_spot[k]) {
                double clong = cos(deg2rad(m->stsp[k][0]));
                double slong = sin(deg2rad(m->stsp[k][0]));
                double clat = cos(deg2rad(m->stsp[k][1]));
                double slat = sin(deg2rad(m->stsp[k][1]));
                spot[k] = mk3(clat * clong, clat * slong, slat);
            }
        }
        int is_uespot = m->uesp_defined;
        double longhw = 0.;
        if (is_uespot) {
            longhw = (m->uesp[1] - m->uesp[0]) / 2.;
            double lcen = deg2rad((m->uesp[0] + m->uesp[1]) / 2.);
            uespot = mk3(cos(lcen), sin(lcen), 0.);
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nface; i++) {
            v3 p = mk3(posn[3 * i], posn[3 * i + 1], posn[3 * i + 2]);
            v3 d = mk3(dirn[3 * i], dirn[3 * i + 1], dirn[3 * i + 2]);
            v3 vec = sub3(cofm2, p);
            double r = len3(vec);
            double mu = dot3(d, vec) / r;
            double t1 = m->t1;
            for (int k = 0; k < 3; k++) {
                if (is_spot[k]) {
                    double dist = rad2deg(acos(dot3(p, spot[k]) / len3(p)));
                    t1 += (m->stsp[k][3] - m->t1) *
                          exp(-sqr(dist / (m->stsp[k][2] / EFAC)) / 2.);
                }
            }
            if (is_uespot) {
                v3 evec = mk3(p.x, p.y, 0);
                double evecl = len3(evec);
                if (evecl > 0.) {
                    double rd = len3(p);
                    double clat = dot3(p, evec) / evecl / rd;
                    clat = dmin(1.0, dmax(-1., clat));
                    double dlat = rad2deg(acos(clat));
                    double clong = dot3(uespot, evec) / evecl;
                    clong = dmin(1.0, dmax(-1., clong));
                    double dlong = rad2deg(acos(clong));
                    const double lathw = m->uesp[2], taper = m->uesp[3], temp = m->uesp[4];
                    if (dlat <= lathw && dlong <= longhw) {
                        t1 = temp;
                    } else if (dlat <= lathw) {
                        t1 += (temp - m->t1) * exp(-(dlong - longhw) / taper);
                    } else if (dlong <= longhw) {
                        t1 += (temp - m->t1) * exp(-(dlat - lathw) / taper);
                    } else {
                        t1 += (temp - m->t1) * exp(-(dlat - lathw) / taper) *
                              exp(-(dlong - longhw) / taper);
                    }
                }
            }
            double temp, geom;
            if (mu >= r2) {
                geom = sqr(r2 / r) * mu;
                temp = pow(pow(t1 * pow((double)gravity[i], GDCBOL1), 4) +
                               m->absorb * pow(m->t2, 4) * geom, 0.25);
            } else if (mu > -r2) {
                double x0 = -mu / r2;
                geom = sqr(r2 / r) * r2 *
                       (sqrt(1. - x0 * x0) * (2 + x0 * x0) / 3 - x0 * (PI_ / 2 - asin(x0))) / PI_;
                temp = pow(pow(t1 * pow((double)gravity[i], GDCBOL1), 4) +
                               m->absorb * pow(m->t2, 4) * geom, 0.25);
            } else {
                geom = 0.;
                temp = t1 * pow((double)gravity[i], GDCBOL1);
            }
            flux[i] = (float)(area[i] * planck(m->wavelength, temp));
            if (m->mirror)
                flux[i] = (float)(flux[i] + area[i] * geom * planck(m->wavelength, fabs(m->t2)));
        }
    } else {
        const v3 cofm1 = mk3(0., 0., 0.), cofm2 = mk3(1., 0., 0.);
        const double GDCBOL2 = m->gdark_bolom2 ? m->gravity_dark2
                                               : m->gravity_dark2 / dlpdlt(m->wavelength, fabs(m->t2));
        v3 spot[2] = {{0, 0, 0}, {0, 0, 0}};
        int is_spot[2];
        for (int k = 0; k < 2; k++) {
            is_spot[k] = m->stsp_defined[3 + k];
            if (is_spot[k]) {
                double clong = cos(deg2rad(m->stsp[3 + k][0]));
                double slong = sin(deg2rad(m->stsp[3 + k][0]));
                double clat = cos(deg2rad(m->stsp[3 + k][1]));
                double slat = sin(deg2rad(m->stsp[3 + k][1]));
                spot[k] = mk3(clat * clong, clat * slong, slat);
            }
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nface; i++) {
            v3 p = mk3(posn[3 * i], posn[3 * i + 1], posn[3 * i + 2]);
            v3 d = mk3(dirn[3 * i], dirn[3 * i + 1], dirn[3 * i + 2]);
            v3 vec = sub3(cofm1, p);
            double r = len3(vec);
            double mu = dot3(d, vec) / r;
            double t2 = fabs(m->t2);
            for (int k = 0; k < 2; k++) {
                if (is_spot[k]) {
                    v3 off = sub3(p, cofm2);
                    double dist = rad2deg(acos(dot3(off, spot[k]) / len3(off)));
                    t2 += (m->stsp[3 + k][3] - t2) *
                          exp(-sqr(dist / (m->stsp[3 + k][2] / EFAC)) / 2.);
                }
            }
            double temp, geom;
            if (mu >= r1) {
                geom = sqr(r1 / r) * mu;
                temp = pow(pow(t2 * pow((double)gravity[i], GDCBOL2), 4) +
                               m->absorb * pow(m->t1, 4.) * geom, 0.25);
            } else if (mu > -r1) {
                double x0 = -mu / r1;
                geom = sqr(r1 / r) * r1 *
                       (sqrt(1. - x0 * x0) * (2 + x0 * x0) / 3 - x0 * (PI_ / 2 - asin(x0))) / PI_;
                temp = pow(pow(t2 * pow((double)gravity[i], GDCBOL2), 4) +
                               m->absorb * pow(m->t1, 4.) * geom, 0.25);
            } else {
                geom = 0.;
                temp = t2 * pow((double)gravity[i], GDCBOL2);
            }
            flux[i] = (float)(area[i] * planck(m->wavelength, temp));
            if (m->mirror)
                flux[i] = (float)(flux[i] + area[i] * geom * planck(m->wavelength, m->t1));
        }
    }
}

/* ---- public: grids ------------------------------------------------------ */
int lco_face_count(const lcg_model *m, int star, int fine, int32_t *nface,
                   char *err, int errlen) {
    oerr e = {0, ""};
    grid_setup s;
    if (grid_prepare(m, star, fine, &s, &e)) {
        copyerr(&e, err, errlen);
        return e.st;
    }
    *nface = grid_nface(&s);
    return LCG_OK;
}

int lco_star_grid(const lcg_model *m, int star, int fine, int32_t nface,
                  double *posn, double *dirn, float *area, float *gravity,
                  float *flux, int32_t *neclipse, double *ecl_in,
                  double *ecl_out, char *err, int errlen) {
    oerr e = {0, ""};
    grid_setup s;
    if (grid_prepare(m, star, fine, &s, &e)) {
        copyerr(&e, err, errlen);
        return e.st;
    }
    if (grid_nface(&s) != nface) {
        seterr(&e, LCG_E_INVALID, "nface mismatch");
        copyerr(&e, err, errlen);
        return e.st;
    }
    gridout o = {posn, dirn, area, gravity, flux, neclipse, ecl_in, ecl_out};
    if (build_grid(m, &s, star, &o, nface, &e)) {
        copyerr(&e, err, errlen);
        return e.st;
    }
    continuum(m, star, nface, posn, dirn, area, gravity, flux);
    return LCG_OK;
}

int lco_model_scalars(const lcg_model *m, double *o, char *err, int errlen) {
    oerr e = {0, ""};
    grid_setup s1, s2;
    if (grid_prepare(m, LCG_STAR1, 1, &s1, &e) || grid_prepare(m, LCG_STAR2, 1, &s2, &e)) {
        copyerr(&e, err, errlen);
        return e.st;
    }
    o[0] = s1.r1; o[1] = s1.r2; o[2] = s1.rl1; o[3] = s1.rl2;
    o[4] = s1.rref1; o[5] = s1.pref1; o[6] = s1.rref2; o[7] = s1.pref2;
    o[8] = s1.ffac1; o[9] = s1.ffac2; o[10] = s1.gref; o[11] = s2.gref;
    return LCG_OK;
}

/* ---- FlatGrid (comp_light_flat.cpp:26-65) ------------------------------- */
int lco_flatten(int32_t nface, const double *posn, const double *dirn,
                const float *flux, const int32_t *neclipse,
                const double *ecl_in, const double *ecl_out, double *dx,
                double *dy, double *dz, double *px, double *py, double *pz,
                double *fflux, double *in1, double *out1, int64_t *n0_out,
                int64_t *n1_out) {
    int64_t c0 = 0, c1 = 0;
    for (int i = 0; i < nface; i++) {
        c0 += (neclipse[i] == 0);
        c1 += (neclipse[i] == 1);
    }
    if (c0 + c1 != nface) return LCG_E_UNSUPPORTED;
    int64_t n0 = c0, n1 = c0 + c1, i0 = 0, i1 = n0;
    for (int j = 0; j < nface; j++) {
        int k = neclipse[j];
        int64_t i = (k == 0) ? i0++ : i1++;
        dx[i] = dirn[3 * j]; dy[i] = dirn[3 * j + 1]; dz[i] = dirn[3 * j + 2];
        px[i] = posn[3 * j]; py[i] = posn[3 * j + 1]; pz[i] = posn[3 * j + 2];
        fflux[i] = flux[j];
        if (k == 1) {
            in1[i - n0] = ecl_in[j];
            out1[i - n0] = ecl_out[j];
        }
    }
    *n0_out = n0;
    *n1_out = n1;
    return LCG_OK;
}

/* ---- flux sweep (comp_light_flat.cpp:80-168, 241-372) ------------------- */
typedef struct { double c1, c2, c3, c4, base, mucrit; } ldcc;

static inline double imu_bl(int ltype, double mu, const ldcc *L) {
    double mm = dmin(mu, 1.0);
    double im;
    if (ltype == LCG_LIMB_POLY) {
        double om = 1.0 - mm;
        im = 1.0 - om * (L->c1 + om * (L->c2 + om * (L->c3 + om * L->c4)));
    } else {
        double msq = sqrt(dmax(mm, 0.0));
        im = L->base + msq * (L->c1 + msq * (L->c2 + msq * (L->c3 + msq * L->c4)));
    }
    return (double)(mu > 0.0) * im;
}

typedef struct {
    const double *dx, *dy, *dz, *px, *py, *pz, *flux;
    int ltype, star, glens, beam_on;
    ldcc L;
    double beam, spin, vfac, xcofm, rlens1;
} sweep;

static inline double elem(const sweep *g, int64_t i, double ex, double ey, double ez) {
    double mu = ex * g->dx[i] + ey * g->dy[i] + ez * g->dz[i];
    if (g->star == LCG_STAR1) {
        double val;
        if (!g->beam_on) {
            val = mu * g->flux[i] * imu_bl(g->ltype, mu, &g->L);
        } else {
            double vx = -g->vfac * g->spin * g->py[i];
            double vy = g->vfac * (g->spin * g->px[i] - g->xcofm);
            double vr = -(ex * vx + ey * vy);
            double vn = g->dx[i] * vx + g->dy[i] * vy;
            double mud = mu - mu * vr - vn;
            val = mu * g->flux[i] * (1.0 - g->beam * vr) * imu_bl(g->ltype, mud, &g->L);
        }
        return (double)(mu > g->L.mucrit) * val;
    }
    double magn = 1.0;
    if (g->glens) {
        double sx = g->px[i], sy = g->py[i], sz = g->pz[i];
        double d = -(sx * ex + sy * ey + sz * ez);
        double qx = sx + d * ex, qy = sy + d * ey, qz = sz + d * ez;
        double p = sqrt(qx * qx + qy * qy + qz * qz);
        double ph = 0.5 * p;
        double rd = g->rlens1 * d;
        double pd = (ph * ph > 25.0 * rd) ? p + rd / p : ph + sqrt(ph * ph + rd);
        double mg = pd * pd / (pd - ph) / ph / 4.0;
        magn = d > 0.0 ? mg : 1.0;
    }
    double val;
    if (!g->beam_on) {
        val = mu * magn * g->flux[i] * imu_bl(g->ltype, mu, &g->L);
    } else {
        double vx = -g->vfac * g->spin * g->py[i];
        double vy = g->vfac * (g->spin * (g->px[i] - 1.0) + 1.0 - g->xcofm);
        double vr = -(ex * vx + ey * vy);
        double vn = g->dx[i] * vx + g->dy[i] * vy;
        double mud = mu - mu * vr - vn;
        val = mu * magn * g->flux[i] * (1.0 - g->beam * vr) * imu_bl(g->ltype, mud, &g->L);
    }
    if (g->glens) return mu > g->L.mucrit ? val : 0.0;
    return (double)(mu > g->L.mucrit) * val;
}

static inline int ecl_range(double phin, double in, double out) {
    return (phin >= in && phin <= out) || phin <= out - 1.0;
}

/* The blocked sweep over [never | one range | ragged] faces: faces [n1, n)
 * have ranges moff[i - n1] .. moff[i - n1 + 1] of rmin / rmout. */
static int sum_multi_r(int star, int64_t n, int64_t n0, int64_t n1, const double *dx,
                       const double *dy, const double *dz, const double *px,
                       const double *py, const double *pz, const double *flux,
                       const double *in1, const double *out1, const int64_t *moff,
                       const double *rmin, const double *rmout, int32_t nent,
                       const double *ex, const double *ey, const double *ez,
                       const double *phin, const double *ldc, int32_t ltype,
                       double mucrit, double beam, double spin, double vfac,
                       double xcofm, int32_t glens1, double rlens1, double *out) {
    sweep g;
    g.dx = dx; g.dy = dy; g.dz = dz; g.px = px; g.py = py; g.pz = pz; g.flux = flux;
    g.ltype = ltype; g.star = star; g.glens = (star == LCG_STAR2) && glens1;
    g.beam_on = (beam != 0.0);
    g.L.c1 = ldc[0]; g.L.c2 = ldc[1]; g.L.c3 = ldc[2]; g.L.c4 = ldc[3];
    g.L.base = 1.0 - (ldc[0] + ldc[1] + ldc[2] + ldc[3]);
    g.L.mucrit = mucrit;
    g.beam = beam; g.spin = spin; g.vfac = vfac; g.xcofm = xcofm; g.rlens1 = rlens1;
    const int64_t FACE_BLOCK = 1024;
    const int64_t nblk = (n + FACE_BLOCK - 1) / FACE_BLOCK;
    for (int k = 0; k < nent; k++) out[k] = 0.0;
    if (nblk == 0 || nent == 0) return LCG_OK;
    double *blk = (double *)malloc(sizeof(double) * (size_t)nblk * (size_t)nent);
    if (!blk) return LCG_E_NOMEM;
#pragma omp parallel for schedule(dynamic)
    for (int64_t b = 0; b < nblk; b++) {
        double *brow = blk + b * nent;
        const int64_t lo = b * FACE_BLOCK;
        const int64_t hi = (n < lo + FACE_BLOCK) ? n : lo + FACE_BLOCK;
        const int64_t a1 = hi < n0 ? hi : n0;
        const int64_t b0 = lo > n0 ? lo : n0;
        const int64_t b1 = hi < n1 ? hi : n1;
        const int64_t c0 = lo > n1 ? lo : n1;
        for (int k = 0; k < nent; k++) brow[k] = 0.0;
        for (int64_t i = lo; i < a1; i++)
            for (int k = 0; k < nent; k++)
                brow[k] += elem(&g, i, ex[k], ey[k], ez[k]);
        for (int64_t i = b0; i < b1; i++) {
            const double ein = in1[i - n0], eout = out1[i - n0];
            for (int k = 0; k < nent; k++) {
                double v = elem(&g, i, ex[k], ey[k], ez[k]);
                brow[k] += ecl_range(phin[k], ein, eout) ? 0.0 : v;
            }
        }
        for (int64_t i = c0; i < hi; i++) {
            for (int k = 0; k < nent; k++) {
                int ecl = 0;
                for (int64_t j = moff[i - n1]; j < moff[i - n1 + 1]; j++)
                    if (ecl_range(phin[k], rmin[j], rmout[j])) { ecl = 1; break; }
                if (!ecl) brow[k] += elem(&g, i, ex[k], ey[k], ez[k]);
            }
        }
    }
    for (int64_t b = 0; b < nblk; b++) {
        const double *brow = blk + b * nent;
        for (int k = 0; k < nent; k++) out[k] += brow[k];
    }
    free(blk);
    return LCG_OK;
}

int lco_sum_star_multi(int star, int64_t n, int64_t n0, const double *dx,
                       const double *dy, const double *dz, const double *px,
                       const double *py, const double *pz, const double *flux,
                       const double *in1, const double *out1, int32_t nent,
                       const double *ex, const double *ey, const double *ez,
                       const double *phin, const double *ldc, int32_t ltype,
                       double mucrit, double beam, double spin, double vfac,
                       double xcofm, int32_t glens1, double rlens1,
                       double *out) {
    const int64_t moff0 = 0;
    return sum_multi_r(star, n, n0, n, dx, dy, dz, px, py, pz, flux, in1, out1, &moff0, NULL,
                       NULL, nent, ex, ey, ez, phin, ldc, ltype, mucrit, beam, spin, vfac,
                       xcofm, glens1, rlens1, out);
}

/* ---- Ginterp (lcurve.h:92-148) ------------------------------------------ */
typedef struct { double phase1, phase2, scale11, scale12, scale21, scale22; } ginterp;

static double gi_scale1(const ginterp *g, double phase) {
    double pnorm = phase - floor(phase);
    if (pnorm <= g->phase1 || pnorm >= 1. - g->phase1) return 1.;
    return (g->scale11 * (1. - g->phase1 - pnorm) + g->scale12 * (pnorm - g->phase1)) /
           (1 - 2. * g->phase1);
}

static double gi_scale2(const ginterp *g, double phase) {
    double pnorm = phase - floor(phase);
    if (pnorm >= g->phase2 && pnorm <= 1. - g->phase2) return 1.;
    if (pnorm < 0.5)
        return (g->scale22 * (g->phase2 - pnorm) + g->scale21 * (pnorm + g->phase2)) /
               (2. * g->phase2);
    return (g->scale21 * (1. + g->phase2 - pnorm) + g->scale22 * (pnorm - 1. + g->phase2)) /
           (2. * g->phase2);
}

static int gi_type(const ginterp *g, double phase) {
    double pnorm = phase - floor(phase);
    if (pnorm <= g->phase1 || pnorm >= 1. - g->phase1) return 1;
    if ((pnorm > g->phase1 && pnorm < g->phase2) ||
        (pnorm > 1. - g->phase2 && pnorm < 1. - g->phase1))
        return 2;
    return 3;
}

/* A star grid held in Point order plus its flattened form. */
typedef struct {
    int n;
    double *posn, *dirn, *ein, *eout;
    float *area, *gravity, *flux;
    int32_t *necl;
    /* ranges appended by an opaque disc (light_curve_comp.cpp:288-323) */
    int32_t *ndx;
    double *xin, *xout;  /* LCO_DISC_R per face */
    /* FlatGrid */
    double *dx, *dy, *dz, *px, *py, *pz, *ff, *in1, *out1;
    int64_t n0, n1;
    int64_t *moff;       /* ragged faces [n1, n): ranges moff[k] .. moff[k + 1] */
    double *rmin, *rmout;
} sgrid;
#define LCO_DISC_R 2

static void sgrid_free(sgrid *g) {
    free(g->posn); free(g->dirn); free(g->ein); free(g->eout);
    free(g->area); free(g->gravity); free(g->flux); free(g->necl);
    free(g->dx); free(g->dy); free(g->dz); free(g->px); free(g->py); free(g->pz);
    free(g->ff); free(g->in1); free(g->out1);
    free(g->ndx); free(g->xin); free(g->xout); free(g->moff); free(g->rmin); free(g->rmout);
    memset(g, 0, sizeof(*g));
}

static int sgrid_build(const lcg_model *m, int star, int fine, sgrid *g, oerr *e) {
    memset(g, 0, sizeof(*g));
    grid_setup s;
    if (grid_prepare(m, star, fine, &s, e)) return e->st;
    int n = grid_nface(&s);
    g->n = n;
    size_t N = (size_t)(n > 0 ? n : 1);
    g->posn = (double *)calloc(3 * N, sizeof(double));
    g->dirn = (double *)calloc(3 * N, sizeof(double));
    g->ein = (double *)calloc(N, sizeof(double));
    g->eout = (double *)calloc(N, sizeof(double));
    g->area = (float *)calloc(N, sizeof(float));
    g->gravity = (float *)calloc(N, sizeof(float));
    g->flux = (float *)calloc(N, sizeof(float));
    g->necl = (int32_t *)calloc(N, sizeof(int32_t));
    gridout o = {g->posn, g->dirn, g->area, g->gravity, g->flux, g->necl, g->ein, g->eout};
    if (build_grid(m, &s, star, &o, n, e)) return e->st;
    return LCG_OK;
}

static void sgrid_flatten(sgrid *g) {
    size_t N = (size_t)(g->n > 0 ? g->n : 1);
    g->dx = (double *)malloc(N * sizeof(double));
    g->dy = (double *)malloc(N * sizeof(double));
    g->dz = (double *)malloc(N * sizeof(double));
    g->px = (double *)malloc(N * sizeof(double));
    g->py = (double *)malloc(N * sizeof(double));
    g->pz = (double *)malloc(N * sizeof(double));
    g->ff = (double *)malloc(N * sizeof(double));
    g->in1 = (double *)malloc(N * sizeof(double));
    g->out1 = (double *)malloc(N * sizeof(double));
    g->moff = (int64_t *)calloc(N + 1, sizeof(int64_t));
    g->rmin = (double *)malloc((1 + LCO_DISC_R) * N * sizeof(double));
    g->rmout = (double *)malloc((1 + LCO_DISC_R) * N * sizeof(double));
    /* FlatGrid::build (comp_light_flat.cpp:26-65): a face's ranges are its
       Roche eclipse, if any, then the disc's */
    int64_t c0 = 0, c1 = 0;
    for (int j = 0; j < g->n; j++) {
        int k = g->necl[j] + (g->ndx ? g->ndx[j] : 0);
        c0 += (k == 0);
        c1 += (k == 1);
    }
    g->n0 = c0;
    g->n1 = c0 + c1;
    int64_t i0 = 0, i1 = g->n0, i2 = g->n1, nr = 0;
    g->moff[0] = 0;
    for (int j = 0; j < g->n; j++) {
        const int nd = g->ndx ? g->ndx[j] : 0, k = g->necl[j] + nd;
        int64_t i = (k == 0) ? i0++ : (k == 1 ? i1++ : i2++);
        g->dx[i] = g->dirn[3 * j]; g->dy[i] = g->dirn[3 * j + 1]; g->dz[i] = g->dirn[3 * j + 2];
        g->px[i] = g->posn[3 * j]; g->py[i] = g->posn[3 * j + 1]; g->pz[i] = g->posn[3 * j + 2];
        g->ff[i] = g->flux[j];
        double rin[1 + LCO_DISC_R], rout[1 + LCO_DISC_R];
        int q = 0;
        if (g->necl[j]) { rin[q] = g->ein[j]; rout[q++] = g->eout[j]; }
        for (int r = 0; r < nd; r++) {
            rin[q] = g->xin[LCO_DISC_R * j + r];
            rout[q++] = g->xout[LCO_DISC_R * j + r];
        }
        if (k == 1) {
            g->in1[i - g->n0] = rin[0];
            g->out1[i - g->n0] = rout[0];
        } else if (k >= 2) {
            for (int r = 0; r < q; r++) { g->rmin[nr] = rin[r]; g->rmout[nr++] = rout[r]; }
            g->moff[i - g->n1 + 1] = nr;
        }
    }
}

/* LDC::imu (lcurve.h:216-231) */
static double ldc_imu(const double *c, int ltype, double mu) {
    if (mu <= 0) return 0.;
    mu = dmin(mu, 1.);
    double ommu = 1. - mu, im = 1.;
    if (ltype == LCG_LIMB_POLY) {
        im -= ommu * (c[0] + ommu * (c[1] + ommu * (c[2] + ommu * c[3])));
    } else {
        im -= c[0] + c[1] + c[2] + c[3];
        double msq = sqrt(mu);
        im += msq * (c[0] + msq * (c[1] + msq * (c[2] + msq * c[3])));
    }
    return im;
}

/* Point-path single-phase star sums comp_star1 / comp_star2 with ndiv = 1
 * (comp_light.cpp:20-92, 225-315); used only for the Ginterp scales. */
static double comp_star_point(const lcg_model *m, int star, double phase,
                              const ginterp *gi, const sgrid *gf,
                              const sgrid *gc, double rlens1) {
    const double XCOFM = m->q / (1.0 + m->q);
    const double VFAC = (double)(float)m->velocity_scale / (C_LIGHT / 1.e3);
    double ri = deg2rad(m->iangle);
    double cosi = cos(ri), sini = sin(ri);
    double phi = phase, wgt = 1.0;
    v3 earth = set_earth(cosi, sini, phi);
    const double *c = star == LCG_STAR1 ? m->ldc1 : m->ldc2;
    const int ltype = star == LCG_STAR1 ? m->limb1 : m->limb2;
    const double mucrit = star == LCG_STAR1 ? m->mucrit1 : m->mucrit2;
    const double beam = star == LCG_STAR1 ? m->beam_factor1 : m->beam_factor2;
    const sgrid *g = star == LCG_STAR1 ? ((gi_type(gi, phi) == 1) ? gf : gc)
                                       : ((gi_type(gi, phi) == 3) ? gf : gc);
    double s = 0.0, pn = phi - floor(phi);
    for (int i = 0; i < g->n; i++) {
        if (g->necl[i] && ecl_range(pn, g->ein[i], g->eout[i])) continue;
        v3 d = mk3(g->dirn[3 * i], g->dirn[3 * i + 1], g->dirn[3 * i + 2]);
        v3 p = mk3(g->posn[3 * i], g->posn[3 * i + 1], g->posn[3 * i + 2]);
        double mu = dot3(earth, d);
        if (!(mu > mucrit)) continue;
        double magn = 1.0;
        if (star == LCG_STAR2 && m->glens1) {
            double dd = -dot3(p, earth);
            if (dd > 0.0) {
                double pp = len3(add3(p, scl3(dd, earth)));
                double ph = 0.5 * pp, rd = rlens1 * dd;
                double pd = (ph * ph > 25.0 * rd) ? pp + rd / pp : ph + sqrt(ph * ph + rd);
                magn = pd * pd / (pd - ph) / ph / 4.0;
            }
        }
        if (beam == 0.0) {
            s += (star == LCG_STAR1) ? mu * g->flux[i] * ldc_imu(c, ltype, mu)
                                     : mu * magn * g->flux[i] * ldc_imu(c, ltype, mu);
            continue;
        }
        double vx = -VFAC * 1.0 * p.y;
        double vy = (star == LCG_STAR1) ? VFAC * (1.0 * p.x - XCOFM)
                                        : VFAC * (1.0 * (p.x - 1.0) + 1.0 - XCOFM);
        double vr = -(earth.x * vx + earth.y * vy);
        double vn = d.x * vx + d.y * vy;
        double mud = mu - mu * vr - vn;
        s += (star == LCG_STAR1)
                 ? mu * g->flux[i] * (1.0 - beam * vr) * ldc_imu(c, ltype, mud)
                 : mu * magn * g->flux[i] * (1.0 - beam * vr) * ldc_imu(c, ltype, mud);
    }
    double part = wgt * (star == LCG_STAR1 ? gi_scale1(gi, phi) : gi_scale2(gi, phi)) * s;
    return part / 1;
}

/* ---- phase batch (light_curve_comp.cpp:350-455) -------------------------- */
typedef struct {
    int64_t n, cap;
    double *ex, *ey, *ez, *phin, *w;
    int32_t *idx;
} pbatch;

static void pb_push(pbatch *b, double ex, double ey, double ez, double phin,
                    double w, int32_t idx) {
    if (b->n == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 1024;
        b->ex = (double *)realloc(b->ex, (size_t)b->cap * sizeof(double));
        b->ey = (double *)realloc(b->ey, (size_t)b->cap * sizeof(double));
        b->ez = (double *)realloc(b->ez, (size_t)b->cap * sizeof(double));
        b->phin = (double *)realloc(b->phin, (size_t)b->cap * sizeof(double));
        b->w = (double *)realloc(b->w, (size_t)b->cap * sizeof(double));
        b->idx = (int32_t *)realloc(b->idx, (size_t)b->cap * sizeof(int32_t));
    }
    b->ex[b->n] = ex; b->ey[b->n] = ey; b->ez[b->n] = ez;
    b->phin[b->n] = phin; b->w[b->n] = w; b->idx[b->n] = idx;
    b->n++;
}

static void pb_free(pbatch *b) {
    free(b->ex); free(b->ey); free(b->ez); free(b->phin); free(b->w); free(b->idx);
    memset(b, 0, sizeof(*b));
}

/* Per-point phase and polynomial factor (light_curve_comp.cpp:350-376). */
static void point_phases(const lcg_model *m, const lcg_datum *data, int32_t n,
                         double *phases, double *slfacs) {
    double xmin = data[0].time, xmax = data[0].time;
    for (int np = 1; np < n; np++) {
        xmin = data[np].time > xmin ? xmin : data[np].time;
        xmax = data[np].time < xmax ? xmax : data[np].time;
    }
    double middle = (xmin + xmax) / 2., range = (xmax - xmin) / 2.;
    for (int np = 0; np < n; np++) {
        double phase = (data[np].time - m->t0) / m->period;
        for (int it = 0; it < 4; it++)
            phase -= (m->t0 + phase * (m->period + m->pdot * phase) - data[np].time) /
                     (m->period + 2. * m->pdot * phase);
        phase += m->deltat / m->period / 2. * (cos(2. * PI_ * phase) - 1.);
        phases[np] = phase;
        double frac = (data[np].time - middle) / range;
        slfacs[np] = 1. + frac * (m->slope + frac * (m->quad + frac * m->cube));
    }
}

int64_t lco_phase_batch(const lcg_model *m, const lcg_datum *data, int32_t n,
                        double *ex, double *ey, double *ez, double *phin,
                        double *w1, double *w2, int32_t *idx) {
    if (n < 1) return 0;
    double *phases = (double *)malloc(sizeof(double) * (size_t)n);
    double *slfacs = (double *)malloc(sizeof(double) * (size_t)n);
    point_phases(m, data, n, phases, slfacs);
    const double ri = deg2rad(m->iangle);
    const double cosi = cos(ri), sini = sin(ri);
    ginterp gi = {m->phase1, m->phase2, 1., 1., 1., 1.};
    int64_t k = 0;
    for (int np = 0; np < n; np++) {
        double phase = phases[np], slfac = slfacs[np];
        double expose = data[np].expose / m->period;
        int ndiv = data[np].ndiv;
        double norm = (ndiv - 1 > 1) ? ndiv - 1 : 1;
        for (int nd = 0; nd < ndiv; ++nd) {
            double phi, wgt;
            if (ndiv == 1) { phi = phase; wgt = 1.0; }
            else {
                phi = phase + expose * (nd - (ndiv - 1) / 2.0) / (ndiv - 1);
                wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
            }
            v3 earth = set_earth(cosi, sini, phi);
            ex[k] = earth.x; ey[k] = earth.y; ez[k] = earth.z;
            phin[k] = phi - floor(phi);
            w1[k] = slfac * wgt * gi_scale1(&gi, phi) / norm;
            w2[k] = slfac * wgt * gi_scale2(&gi, phi) / norm;
            idx[k] = np;
            k++;
        }
    }
    free(phases);
    free(slfacs);
    return k;
}

static double sweep_flat(const lcg_model *m, int star, const sgrid *g,
                         const pbatch *pb, double *out, double spin, double vfac,
                         double xcofm, double rlens1) {
    return (double)sum_multi_r(
        star, g->n, g->n0, g->n1, g->dx, g->dy, g->dz, g->px, g->py, g->pz, g->ff, g->in1,
        g->out1, g->moff, g->rmin, g->rmout, (int32_t)pb->n, pb->ex, pb->ey, pb->ez, pb->phin,
        star == LCG_STAR1 ? m->ldc1 : m->ldc2, star == LCG_STAR1 ? m->limb1 : m->limb2,
        star == LCG_STAR1 ? m->mucrit1 : m->mucrit2,
        star == LCG_STAR1 ? m->beam_factor1 : m->beam_factor2, spin, vfac, xcofm,
        star == LCG_STAR2 ? m->glens1 : 0, rlens1, out);
}

/* Single-phase flat sum in face order: the scalar sum_star{1,2}_t. The
 * reference vectorises this reduction (omp simd), so its summation order is
 * compiler-dependent; agreement is to rounding. */
static double flat_sum_one(const lcg_model *m, int star, const sgrid *g, v3 earth,
                           double phin, double vfac, double xcofm, double rlens1) {
    pbatch pb = {0, 0, 0, 0, 0, 0, 0, 0};
    pb_push(&pb, earth.x, earth.y, earth.z, phin, 1.0, 0);
    double out = 0.;
    sweep_flat(m, star, g, &pb, &out, 1.0, vfac, xcofm, rlens1);
    pb_free(&pb);
    return out;
}

/* comp_star1_flat / comp_star2_flat (comp_light_flat.cpp:538-602): the
 * sub-exposure sums of one star, Ginterp-scaled, spin 1 in the beaming. */
static double comp_star_flat(const lcg_model *m, int star, double phase, double expose,
                             int ndiv, const ginterp *gi, const sgrid *gf, const sgrid *gc,
                             double vfac, double xcofm, double rlens1) {
    const double ri = deg2rad(m->iangle);
    const double cosi = cos(ri), sini = sin(ri);
    double sum = 0.0;
    for (int nd = 0; nd < ndiv; ++nd) {
        double phi, wgt;
        if (ndiv == 1) { phi = phase; wgt = 1.0; }
        else {
            phi = phase + expose * (nd - (ndiv - 1) / 2.0) / (ndiv - 1);
            wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
        }
        v3 earth = set_earth(cosi, sini, phi);
        double phin = phi - floor(phi);
        const sgrid *g = star == LCG_STAR1 ? ((gi_type(gi, phi) == 1) ? gf : gc)
                                           : ((gi_type(gi, phi) == 3) ? gf : gc);
        sum += wgt * (star == LCG_STAR1 ? gi_scale1(gi, phi) : gi_scale2(gi, phi)) *
               flat_sum_one(m, star, g, earth, phin, vfac, xcofm, rlens1);
    }
    return sum / ((ndiv - 1 > 1) ? ndiv - 1 : 1);
}

/* The iscale fit from the components (light_curve_comp.cpp:532-556). */
static void iscale_calc(const lcg_model *m, int32_t n, const double *fcomp,
                        const double *sfac, double *calc) {
    for (int np = 0; np < n; np++) {
        const double *f = fcomp + 5 * np;
        calc[np] = sfac[0] * f[0] + sfac[1] * f[1] + sfac[2] * f[2] + sfac[3] * f[3];
        if (m->t2 > 0.) calc[np] += sfac[4] * f[4];
    }
}

/* comp_gravity1/2 (comp_gravity.cpp:20-155) and comp_radius1/2
 * (comp_radius.cpp:16-86). */
static double comp_gravity(const lcg_model *m, int star, const sgrid *g, oerr *e) {
    double gm = pow(1000. * m->velocity_scale, 3) * m->tperiod * DAY_F / TWOPI_;
    double a = pow(gm / sqr(TWOPI_ / DAY_F / m->tperiod), 1. / 3.);
    double gscale = 100 * gm / sqr(a), gref;
    double r1, r2;
    get_r1r2(m, &r1, &r2);
    double rl1 = xl12(m->q, m->spin1, e);
    double rl2 = 1. - xl12(m->q, m->spin2, e);
    if (m->r2 < 0) r2 = rl2;
    const double ACC = m->delta_phase / 10.;
    v3 posn, dvec;
    double rad;
    if (star == LCG_STAR1) {
        if (m->roche1) {
            double rref1, pref1, ffac1 = r1 / rl1;
            ref_sphere(m->q, LCG_STAR1, m->spin1, ffac1, &rref1, &pref1, e);
            face_scalar(m->q, LCG_STAR1, m->spin1, mk3(-1., 0., 0.), rref1, pref1, ACC,
                        &posn, &dvec, &rad, &gref, e);
            gref *= gscale;
        } else {
            gref = gscale / (1 + m->q) / sqr(r1);
        }
    } else {
        if (m->roche2) {
            double rref2, pref2, ffac2 = r2 / rl2;
            ref_sphere(m->q, LCG_STAR2, m->spin2, ffac2, &rref2, &pref2, e);
            face_scalar(m->q, LCG_STAR2, m->spin2, mk3(1., 0., 0.), rref2, pref2, ACC,
                        &posn, &dvec, &rad, &gref, e);
            gref *= gscale;
        } else {
            gref = gscale * m->q / (1 + m->q) / sqr(r2);
        }
    }
    const int BLK = 8192, nn = g->n, nblk = (nn + BLK - 1) / BLK;
    double sumfg = 0., sumf = 0;
    for (int b = 0; b < nblk; b++) {
        double bfg = 0., bf = 0.;
        int end = (nn < b * BLK + BLK) ? nn : b * BLK + BLK;
        for (int i = b * BLK; i < end; i++) {
            float fg = g->flux[i] * g->gravity[i];
            bfg += fg;
            bf += g->flux[i];
        }
        sumfg += bfg;
        sumf += bf;
    }
    if ((gref > 0) & (sumfg > 0) & (sumf > 0)) return log10(gref * sumfg / sumf);
    return 0.;
}

static double comp_radius(int star, const sgrid *g) {
    const v3 cofm = star == LCG_STAR1 ? mk3(0., 0., 0.) : mk3(1., 0., 0.);
    const int BLK = 8192, nn = g->n, nblk = (nn + BLK - 1) / BLK;
    double sumsa = 0., sumvol = 0.;
    for (int b = 0; b < nblk; b++) {
        double bsa = 0., bvol = 0.;
        int end = (nn < b * BLK + BLK) ? nn : b * BLK + BLK;
        for (int i = b * BLK; i < end; i++) {
            v3 p = mk3(g->posn[3 * i], g->posn[3 * i + 1], g->posn[3 * i + 2]);
            v3 d = mk3(g->dirn[3 * i], g->dirn[3 * i + 1], g->dirn[3 * i + 2]);
            v3 vec = sub3(p, cofm);
            double r = len3(vec);
            double rcosa = dot3(d, vec);
            bsa += g->area[i] * rcosa / pow(r, 3);
            bvol += g->area[i] * rcosa;
        }
        sumsa += bsa;
        sumvol += bvol;
    }
    return pow(sumvol / sumsa, 1. / 3.);
}

/* ---- the whole path (light_curve_comp.cpp:119-599) ---------------------- */
/* ---- accretion disc, disc edge and bright spot --------------------------
 * set_disc_grid.cpp:27-127 (disc), :144-264 (edge), set_bright_spot_grid.cpp
 * :27-100 (spot), set_disc_continuum.cpp:19-88, disc_eclipse.cpp:38-366,
 * star_eclipse.cpp:15-26. Elements are kept in the reference's vector order;
 * each carries up to LCO_MAXR eclipse ranges in the order they were pushed. */
#define LCO_MAXR 4

typedef struct {
    int n;
    double *posn, *dirn;  /* 3 per element */
    float *area, *flux;
    int32_t *nr;          /* eclipse ranges per element */
    double *rin, *rout;   /* LCO_MAXR per element */
} elist;

static void el_free(elist *d) {
    free(d->posn); free(d->dirn); free(d->area); free(d->flux);
    free(d->nr); free(d->rin); free(d->rout);
    memset(d, 0, sizeof(*d));
}

static void el_alloc(elist *d, int n) {
    memset(d, 0, sizeof(*d));
    size_t N = (size_t)(n > 0 ? n : 1);
    d->n = n;
    d->posn = (double *)calloc(3 * N, sizeof(double));
    d->dirn = (double *)calloc(3 * N, sizeof(double));
    d->area = (float *)calloc(N, sizeof(float));
    d->flux = (float *)calloc(N, sizeof(float));
    d->nr = (int32_t *)calloc(N, sizeof(int32_t));
    d->rin = (double *)calloc(LCO_MAXR * N, sizeof(double));
    d->rout = (double *)calloc(LCO_MAXR * N, sizeof(double));
}

/* Appends one range to a list of at most LCO_MAXR. */
static void push_range(int32_t *nr, double *rin, double *rout, double in, double out) {
    if (*nr < LCO_MAXR) {
        rin[*nr] = in;
        rout[*nr] = out;
    }
    (*nr)++;
}

enum { CIRC_ABOVE, CIRC_INSIDE, CIRC_OUTSIDE, CIRC_SEPARATE, CIRC_CROSSING };

/* cut_phase (disc_eclipse.cpp:349-366) */
static double cut_phase(double rxy, double rcone, double radius, oerr *e) {
    if (rxy + rcone <= radius) { seterr(e, LCG_E_ROCHE, "rxy + rcone <= radius"); return 0.; }
    if (rxy >= radius + rcone) { seterr(e, LCG_E_ROCHE, "rxy >= radius + rcone"); return 0.; }
    if (rcone >= radius + rxy) { seterr(e, LCG_E_ROCHE, "rcone >= radius + rxy"); return 0.; }
    return acos((sqr(rxy) + sqr(rcone) - sqr(radius)) / (2. * rcone * rxy)) / TWOPI_;
}

/* circle_eclipse (disc_eclipse.cpp:316-340) */
static int circle_eclipse(double rxy, double z, double zcirc, double radius, double tani,
                          double *phase, oerr *e) {
    if (z >= zcirc) return CIRC_ABOVE;
    const double RCONE = tani * (zcirc - z);
    if (RCONE >= rxy + radius) return CIRC_OUTSIDE;
    if (rxy >= RCONE + radius) return CIRC_SEPARATE;
    if (rxy + RCONE <= radius) return CIRC_INSIDE;
    *phase = cut_phase(rxy, RCONE, radius, e);
    return CIRC_CROSSING;
}

/* Roche::disc_eclipse (disc_eclipse.cpp:38-301): the phase ranges over which
 * the flared disc hides point r; 0, 1 or 2 ranges appended. */
static void disc_eclipse(double iangle, double rdisc1, double rdisc2, double beta,
                         double height, v3 r, int32_t *nr, double *rin, double *rout,
                         oerr *e) {
    if (beta < 1) { seterr(e, LCG_E_ROCHE, "Roche::disc_eclipse: beta must be >= 1"); return; }
    const double sini = sin(PI_ / 180. * iangle);
    const double cosi = cos(PI_ / 180. * iangle);
    const double HOUT = height * pow(rdisc2, beta);
    if (r.z >= HOUT) return;
    if (cosi == 0.) {
        if (fabs(r.z) < HOUT) {
            double rxy = sqrt(sqr(r.x) + sqr(r.y));
            if (rxy <= rdisc2) {
                push_range(nr, rin, rout, 0., 1.);
            } else {
                double subtend = asin(rdisc2 / rxy) / TWOPI_;
                double pcen = atan2(r.y, -r.x) / TWOPI_;
                double ingress = pcen - subtend;
                ingress = ingress - floor(ingress);
                double egress = ingress + 2. * subtend;
                push_range(nr, rin, rout, ingress, egress);
            }
        }
        return;
    }
    const double RXY = sqrt(sqr(r.x) + sqr(r.y));
    if (rdisc1 < RXY && RXY < rdisc2 && fabs(r.z) < height * pow(RXY, beta)) {
        push_range(nr, rin, rout, 0., 1.1);
        return;
    }
    const double TANI = sini / cosi;
    int result;
    double phase = 0., ingress, egress;
    if (RXY < rdisc2 && r.z >= height * pow(dmax(rdisc1, RXY), beta)) {
        result = circle_eclipse(RXY, r.z, HOUT, rdisc2, TANI, &phase, e);
        if (e->st) return;
        if (result == CIRC_OUTSIDE) {
            push_range(nr, rin, rout, 0., 1.1);
        } else if (result == CIRC_CROSSING) {
            double phi0 = atan2(r.y, -r.x) / TWOPI_;
            ingress = phi0 + phase;
            ingress -= floor(ingress);
            egress = ingress + 1 - 2. * phase;
            push_range(nr, rin, rout, ingress, egress);
        }
        return;
    }
    const double RCONE_LO = dmax(0., TANI * (-HOUT - r.z));
    if (RCONE_LO >= RXY + rdisc2) return;
    const double RCONE_HI = TANI * (HOUT - r.z);
    if (RXY >= RCONE_HI + rdisc2) return;
    double eclipse_phase = 0;
    if (RXY + RCONE_LO <= rdisc2) {
        eclipse_phase = 0.5;
    } else if (RXY <= rdisc2) {
        eclipse_phase = cut_phase(RXY, RCONE_LO, rdisc2, e);
    } else {
        if (sqr(RCONE_HI) + sqr(rdisc2) >= sqr(RXY) && sqr(RCONE_LO) + sqr(rdisc2) <= sqr(RXY)) {
            eclipse_phase = asin(rdisc2 / RXY) / TWOPI_;
        } else if (sqr(RCONE_HI) + sqr(rdisc2) < sqr(RXY)) {
            eclipse_phase = cut_phase(RXY, RCONE_HI, rdisc2, e);
        } else {
            eclipse_phase = cut_phase(RXY, RCONE_LO, rdisc2, e);
        }
    }
    if (e->st) return;
    const double HIN = height * pow(rdisc1, beta);
    double appear_phase = -1;
    /* the LOSC passes the rims in turn; the first sets appear_phase, the
       rest can only lower it or rule out a view through the hole */
    double zc[4], rc[4];
    int nc = 0;
    if (r.z < -HOUT) {
        zc[0] = -HOUT; rc[0] = rdisc2; zc[1] = -HIN; rc[1] = rdisc1;
        zc[2] = HIN; rc[2] = rdisc1; zc[3] = HOUT; rc[3] = rdisc2; nc = 4;
    } else if (RXY < rdisc1) {
        if (r.z < -HIN) {
            zc[0] = -HIN; rc[0] = rdisc1; zc[1] = HIN; rc[1] = rdisc1;
            zc[2] = HOUT; rc[2] = rdisc2; nc = 3;
        } else if (r.z < HIN) {
            zc[0] = HIN; rc[0] = rdisc1; zc[1] = HOUT; rc[1] = rdisc2; nc = 2;
        }
    }
    for (int k = 0; k < nc; k++) {
        if (k > 0 && !(appear_phase > 0)) break;
        result = circle_eclipse(RXY, r.z, zc[k], rc[k], TANI, &phase, e);
        if (e->st) return;
        if (k == 0) {
            if (result == CIRC_INSIDE) appear_phase = 0.5;
            else if (result == CIRC_CROSSING) appear_phase = phase;
        } else if (result == CIRC_CROSSING) {
            appear_phase = dmin(appear_phase, phase);
        } else if (result != CIRC_INSIDE) {
            appear_phase = -1.;
        }
    }
    double phi0 = atan2(r.y, -r.x) / TWOPI_;
    if (appear_phase <= 0) {
        ingress = phi0 - eclipse_phase;
        ingress -= floor(ingress);
        egress = ingress + 2. * eclipse_phase;
        push_range(nr, rin, rout, ingress, egress);
    } else if (appear_phase < eclipse_phase) {
        ingress = phi0 - eclipse_phase;
        ingress -= floor(ingress);
        egress = ingress + (eclipse_phase - appear_phase);
        push_range(nr, rin, rout, ingress, egress);
        ingress = phi0 + appear_phase;
        ingress -= floor(ingress);
        egress = ingress + (eclipse_phase - appear_phase);
        push_range(nr, rin, rout, ingress, egress);
    }
}

/* Lcurve::star_eclipse (star_eclipse.cpp:15-26): eclipse of point posn by
 * star `star` (Roche-distorted with reference sphere rref/pref, or a sphere
 * of radius r); one range appended when eclipsed. */
static void star_eclipse(double q, double r, double spin, double iangle, v3 posn,
                         double delta, int roche, int star, double rref, double pref,
                         int32_t *nr, double *rin, double *rout, oerr *e) {
    double ri = deg2rad(iangle);
    const double cosi = cos(ri), sini = sin(ri);
    double ingress = 0., egress = 0., lam1, lam2;
    v3 cofm = (star == LCG_STAR1) ? mk3(0., 0., 0.) : mk3(1., 0., 0.);
    int ecl = roche ? ingress_egress(q, star, spin, iangle, delta, posn, &ingress, &egress,
                                     rref, pref, e)
                    : sphere_eclipse_ph(cosi, sini, posn, cofm, r, &ingress, &egress, &lam1,
                                        &lam2);
    if (e->st) return;
    if (ecl) push_range(nr, rin, rout, ingress, egress);
}

/* What set_disc_grid / set_disc_edge / set_bright_spot_grid derive from the
 * model before making elements (set_disc_grid.cpp:31-66). */
typedef struct {
    double r1, r2, rl1, rl2, rdisc1, rdisc2;
    double rref1, pref1, rref2, pref2, ffac1, ffac2;
} comp_setup;

static int comp_prepare(const lcg_model *m, const char *who, comp_setup *s, oerr *e) {
    get_r1r2(m, &s->r1, &s->r2);
    s->rl1 = xl11(m->q, m->spin1, e);
    if (e->st) return e->st;
    if (s->r1 < 0) s->r1 = s->rl1;
    else if (s->r1 > s->rl1)
        return seterr(e, LCG_E_LOBE, "%s: the primary star is larger than its Roche lobe!", who);
    s->rl2 = 1. - xl12(m->q, m->spin2, e);
    if (e->st) return e->st;
    if (s->r2 < 0) s->r2 = s->rl2;
    else if (s->r2 > s->rl2)
        return seterr(e, LCG_E_LOBE, "%s: the secondary star is larger than its Roche lobe!", who);
    s->rdisc1 = m->rdisc1 > 0. ? m->rdisc1 : s->r1;
    s->rdisc2 = m->rdisc2 > 0. ? m->rdisc2 : m->radius_spot;
    s->ffac1 = s->r1 / s->rl1;
    ref_sphere(m->q, LCG_STAR1, m->spin1, s->ffac1, &s->rref1, &s->pref1, e);
    s->ffac2 = s->r2 / s->rl2;
    ref_sphere(m->q, LCG_STAR2, m->spin2, s->ffac2, &s->rref2, &s->pref2, e);
    return e->st;
}

/* The eclipses every component element gets: the opaque disc, then star 1,
 * then star 2. trap1: a Roche_Error from star 1's eclipse becomes a range
 * (0, 1) (the edge's upper rim, set_disc_grid.cpp:222-231). */
static void element_eclipses(const lcg_model *m, const comp_setup *s, v3 posn, int opaque,
                             int trap1, int32_t *nr, double *rin, double *rout, oerr *e) {
    *nr = 0;
    if (opaque)
        disc_eclipse(m->iangle, s->rdisc1, s->rdisc2, m->beta_disc, m->height_disc, posn, nr,
                     rin, rout, e);
    if (e->st) return;
    if (m->eclipse1) {
        star_eclipse(m->q, s->r1, m->spin1, m->iangle, posn, m->delta_phase, m->roche1,
                     LCG_STAR1, s->rref1, s->pref1, nr, rin, rout, e);
        if (e->st && trap1 && e->st == LCG_E_ROCHE) {
            e->st = 0;
            e->msg[0] = 0;
            push_range(nr, rin, rout, 0., 1.);
        }
        if (e->st) return;
    }
    if (m->eclipse2)
        star_eclipse(m->q, s->r2, m->spin2, m->iangle, posn, m->delta_phase, m->roche2,
                     LCG_STAR2, s->rref2, s->pref2, nr, rin, rout, e);
}

static void el_set(elist *d, int i, v3 posn, v3 dirn, double area) {
    d->posn[3 * i] = posn.x; d->posn[3 * i + 1] = posn.y; d->posn[3 * i + 2] = posn.z;
    d->dirn[3 * i] = dirn.x; d->dirn[3 * i + 1] = dirn.y; d->dirn[3 * i + 2] = dirn.z;
    d->area[i] = (float)area;
}

/* Lcurve::set_disc_grid (set_disc_grid.cpp:27-127) */
static int disc_grid(const lcg_model *m, elist *d, oerr *e) {
    const double EFAC = 1.0000001;
    comp_setup s;
    if (comp_prepare(m, "set_disc_grid", &s, e)) return e->st;
    int nface = 0, ntheta = 0;
    double drad = (s.rdisc2 - s.rdisc1) / m->nrad, drrad = s.rdisc2 / m->nrad;
    for (int i = 0; i < m->nrad; i++) {
        ntheta = (int)ceil(TWOPI_ * (s.rdisc1 + (s.rdisc2 - s.rdisc1) * (i + 0.5) / m->nrad) / drrad);
        ntheta = ntheta > 8 ? ntheta : 8;
        nface += ntheta;
    }
    el_alloc(d, nface);
    nface = 0;
    for (int i = 0; i < m->nrad; i++) {
        double rad = s.rdisc1 + (s.rdisc2 - s.rdisc1) * (i + 0.5) / m->nrad;
        ntheta = (int)ceil(TWOPI_ * rad / drrad);
        ntheta = ntheta > 8 ? ntheta : 8;
        double h = EFAC * m->height_disc * pow(rad, m->beta_disc);
        double tanp = m->beta_disc * h / rad;
        double cosp = 1. / sqrt(1 + sqr(tanp));
        double sinp = tanp * cosp;
        double area = TWOPI_ / ntheta * rad * drad;
        for (int j = 0; j < ntheta; j++, nface++) {
            double theta = TWOPI_ * j / ntheta;
            double sint = sin(theta), cost = cos(theta);
            v3 posn = mk3(rad * cost, rad * sint, h);
            v3 dirn = mk3(-cost * sinp, -sint * sinp, cosp);
            element_eclipses(m, &s, posn, m->opaque, 0, d->nr + nface, d->rin + LCO_MAXR * nface,
                             d->rout + LCO_MAXR * nface, e);
            if (e->st) return e->st;
            el_set(d, nface, posn, dirn, area);
        }
    }
    return LCG_OK;
}

/* Lcurve::set_disc_edge with outer = true, visual = false
 * (set_disc_grid.cpp:144-264) */
static int disc_edge(const lcg_model *m, elist *d, oerr *e) {
    const double EFAC = 1.0000001;
    comp_setup s;
    if (comp_prepare(m, "set_disc_grid", &s, e)) return e->st;
    const double size = s.rdisc2 / m->nrad;
    const double RAD = s.rdisc2;
    const double H = m->height_disc * pow(RAD, m->beta_disc);
    const int NOUT = (int)(2 * H / size) + 2;
    const int NTHETA = (int)ceil(TWOPI_ * RAD / size) > 8 ? (int)ceil(TWOPI_ * RAD / size) : 8;
    el_alloc(d, NTHETA * NOUT);
    double area = TWOPI_ / NTHETA * RAD * 2 * H / (NOUT - 1);
    int nface = 0;
    for (int i = 0; i < NTHETA; i++) {
        double theta = TWOPI_ * i / NTHETA;
        double sint = sin(theta), cost = cos(theta);
        v3 posn = mk3(EFAC * RAD * cost, EFAC * RAD * sint, EFAC * H);
        v3 dirn = mk3(cost, sint, 0);
        element_eclipses(m, &s, posn, m->opaque, 1, d->nr + nface, d->rin + LCO_MAXR * nface,
                         d->rout + LCO_MAXR * nface, e);
        if (e->st) return e->st;
        el_set(d, nface++, posn, dirn, area / 2.);
        for (int j = 0; j < NOUT - 1; j++) {
            posn = mk3(EFAC * RAD * cost, EFAC * RAD * sint, -H + 2 * H * j / (NOUT - 1));
            dirn = mk3(cost, sint, 0);
            element_eclipses(m, &s, posn, m->opaque, 0, d->nr + nface,
                             d->rin + LCO_MAXR * nface, d->rout + LCO_MAXR * nface, e);
            if (e->st) return e->st;
            el_set(d, nface++, posn, dirn, area);
        }
    }
    return LCG_OK;
}

/* set_disc_continuum (set_disc_continuum.cpp:19-31) */
static void disc_continuum(double rdisc, double tdisc, double texp, double wave, elist *d) {
    const double BRIGHT = planck(wave, tdisc);
    for (int i = 0; i < d->n; i++) {
        double r = len3(mk3(d->posn[3 * i], d->posn[3 * i + 1], d->posn[3 * i + 2]));
        d->flux[i] = (float)(BRIGHT * pow(r / rdisc, texp) * d->area[i]);
    }
}

/* set_edge_continuum (set_disc_continuum.cpp:48-88) */
static void edge_continuum(double tedge, double r2, double t2, double absorb, double wave,
                           elist *d) {
    const v3 cofm2 = mk3(1., 0., 0.);
    for (int i = 0; i < d->n; i++) {
        v3 p = mk3(d->posn[3 * i], d->posn[3 * i + 1], d->posn[3 * i + 2]);
        v3 n = mk3(d->dirn[3 * i], d->dirn[3 * i + 1], d->dirn[3 * i + 2]);
        v3 vec = sub3(cofm2, p);
        double r = len3(vec);
        double mu = dot3(n, vec) / r, geom, temp;
        if (mu >= r2) {
            geom = sqr(r2 / r) * mu;
            temp = pow(pow(tedge, 4) + absorb * pow(t2, 4) * geom, 0.25);
        } else if (mu > -r2) {
            double x0 = -mu / r2;
            geom = sqr(r2 / r) * r2 *
                   (sqrt(1. - x0 * x0) * (2 + x0 * x0) / 3 - x0 * (PI_ / 2 - asin(x0))) / PI_;
            temp = pow(pow(tedge, 4) + absorb * pow(t2, 4) * geom, 0.25);
        } else {
            temp = tedge;
        }
        d->flux[i] = (float)(d->area[i] * planck(wave, temp));
    }
}

/* ---- gas stream to the bright spot --------------------------------------
 * Roche::strinit (strining.cpp:14-33) starts a particle just inside L1 with
 * the Lubow & Shu velocity; the reference then integrates the restricted
 * three-body motion (rocacc.cpp) with a Bulirsch-Stoer stepper until the
 * stream reaches radius_spot (stradv.cpp:27-80, accuracy 1e-10 in radius).
 * Here the same motion is integrated with the Dormand-Prince 5(4) pair
 * (Dormand & Prince 1980, J. Comp. Appl. Math. 6, 19) under a much tighter
 * tolerance, and the crossing is bisected in time to the same radius
 * accuracy, so the spot lands on the stream within the reference's own
 * integration error (the reference's stepper keeps its step size in a
 * static between calls, so its result depends on call history). */
static void rocacc(double q, const double *y, double *dy) {
    double f1 = 1.0 / (1.0 + q), f2 = f1 * q;
    double yzsq = sqr(y[1]) + sqr(y[2]);
    double r1sq = sqr(y[0]) + yzsq, r2sq = sqr(y[0] - 1.0) + yzsq;
    double fm1 = f1 / (r1sq * sqrt(r1sq)), fm2 = f2 / (r2sq * sqrt(r2sq)), fm3 = fm1 + fm2;
    dy[0] = y[3]; dy[1] = y[4]; dy[2] = y[5];
    dy[3] = -fm3 * y[0] + fm2 + 2.0 * y[4] + y[0] - f2;
    dy[4] = -fm3 * y[1] - 2.0 * y[3] + y[1];
    dy[5] = -fm3 * y[2];
}

/* One Dormand-Prince step of size h from y; returns the error norm. */
static double dp_step(double q, const double *y, double h, double *yo) {
    static const double a21 = 1. / 5, a31 = 3. / 40, a32 = 9. / 40, a41 = 44. / 45,
                        a42 = -56. / 15, a43 = 32. / 9, a51 = 19372. / 6561,
                        a52 = -25360. / 2187, a53 = 64448. / 6561, a54 = -212. / 729,
                        a61 = 9017. / 3168, a62 = -355. / 33, a63 = 46732. / 5247,
                        a64 = 49. / 176, a65 = -5103. / 18656, b1 = 35. / 384,
                        b3 = 500. / 1113, b4 = 125. / 192, b5 = -2187. / 6784, b6 = 11. / 84,
                        e1 = 71. / 57600, e3 = -71. / 16695, e4 = 71. / 1920,
                        e5 = -17253. / 339200, e6 = 22. / 525, e7 = -1. / 40;
    double k1[6], k2[6], k3[6], k4[6], k5[6], k6[6], k7[6], t[6];
    int i;
    rocacc(q, y, k1);
    for (i = 0; i < 6; i++) t[i] = y[i] + h * (a21 * k1[i]);
    rocacc(q, t, k2);
    for (i = 0; i < 6; i++) t[i] = y[i] + h * (a31 * k1[i] + a32 * k2[i]);
    rocacc(q, t, k3);
    for (i = 0; i < 6; i++) t[i] = y[i] + h * (a41 * k1[i] + a42 * k2[i] + a43 * k3[i]);
    rocacc(q, t, k4);
    for (i = 0; i < 6; i++)
        t[i] = y[i] + h * (a51 * k1[i] + a52 * k2[i] + a53 * k3[i] + a54 * k4[i]);
    rocacc(q, t, k5);
    for (i = 0; i < 6; i++)
        t[i] = y[i] + h * (a61 * k1[i] + a62 * k2[i] + a63 * k3[i] + a64 * k4[i] + a65 * k5[i]);
    rocacc(q, t, k6);
    for (i = 0; i < 6; i++)
        yo[i] = y[i] + h * (b1 * k1[i] + b3 * k3[i] + b4 * k4[i] + b5 * k5[i] + b6 * k6[i]);
    rocacc(q, yo, k7);
    double err = 0.;
    for (i = 0; i < 6; i++) {
        double ei = h * (e1 * k1[i] + e3 * k3[i] + e4 * k4[i] + e5 * k5[i] + e6 * k6[i] +
                         e7 * k7[i]);
        double sc = 1e-14 + 1e-13 * fmax(fabs(y[i]), fabs(yo[i]));
        err = fmax(err, fabs(ei) / sc);
    }
    return err;
}

/* The stream position where it first reaches radius rad from star 1. */
static int stream_to_radius(double q, double rad, v3 *pos, oerr *e) {
    const double SMALL = 1.e-5, ACC = 1.e-10, SMAX = 1.e-3, TMAX = 10.;
    double rl1 = xl1(q, e);
    if (e->st) return e->st;
    double mu = q / (1.0 + q);
    double a = (1.0 - mu) / pow(rl1, 3) + mu / pow((1. - rl1), 3);
    double lambda1 = sqrt(((a - 2.0) + sqrt(a * (9.0 * a - 8.0))) / 2.0);
    double m1 = (lambda1 * lambda1 - 2.0 * a - 1.0) / 2.0 / lambda1;
    double y[6] = {rl1 - SMALL, -m1 * SMALL, 0., -lambda1 * SMALL, -lambda1 * m1 * SMALL, 0.};
    double yo[6], ylo[6], h = 1e-4, t = 0.;
    const double rinit = sqrt(sqr(y[0]) + sqr(y[1]) + sqr(y[2]));
    double rnow = rinit;
    int guard = 0;
    while ((rinit > rad && rnow > rad) || (rinit < rad && rnow < rad)) {
        if (++guard > 1000000 || t > TMAX)
            return seterr(e, LCG_E_ROCHE, "Roche::stradv: taken too long without crossing radius");
        h = fmin(h, SMAX);
        double err = dp_step(q, y, h, yo);
        if (err > 1.) {
            h *= fmax(0.2, 0.9 * pow(err, -0.2));
            continue;
        }
        memcpy(ylo, y, sizeof y);
        memcpy(y, yo, sizeof y);
        t += h;
        rnow = sqrt(sqr(y[0]) + sqr(y[1]) + sqr(y[2]));
        double hstep = h;
        h *= err > 0. ? fmin(5., 0.9 * pow(err, -0.2)) : 5.;
        if (!((rinit > rad && rnow > rad) || (rinit < rad && rnow < rad))) {
            /* bisect the last step in time until the radius is pinned */
            double lo = 0., hi = hstep;
            double rlo = sqrt(sqr(ylo[0]) + sqr(ylo[1]) + sqr(ylo[2])), rhi = rnow;
            int g2 = 0;
            while (fabs(rhi - rlo) > ACC && ++g2 < 200) {
                double tt = (lo + hi) / 2.;
                dp_step(q, ylo, tt, y);
                rnow = sqrt(sqr(y[0]) + sqr(y[1]) + sqr(y[2]));
                if ((rhi > rad && rnow > rad) || (rhi < rad && rnow < rad)) {
                    rhi = rnow;
                    hi = tt;
                } else {
                    rlo = rnow;
                    lo = tt;
                }
            }
            break;
        }
    }
    *pos = mk3(y[0], y[1], y[2]);
    return LCG_OK;
}

/* Lcurve::set_bright_spot_grid (set_bright_spot_grid.cpp:27-100) */
static int spot_grid(const lcg_model *m, elist *d, oerr *e) {
    comp_setup s;
    if (comp_prepare(m, "set_bright_spot_grid", &s, e)) return e->st;
    v3 bspot = {0., 0., 0.};
    if (stream_to_radius(m->q, m->radius_spot, &bspot, e)) return e->st;
    double theta = atan2(bspot.y, bspot.x) + TWOPI_ / 4. + deg2rad(m->angle_spot);
    double alpha = deg2rad(m->yaw_spot);
    double tilt = deg2rad(m->tilt_spot);
    v3 bvec = mk3(cos(theta), sin(theta), 0);
    v3 pvec = mk3(0, 0, 1);
    v3 tvec = mk3(sin(tilt) * sin(theta + alpha), -sin(tilt) * cos(theta + alpha), cos(tilt));
    const double BMAX = pow(m->expon_spot / m->epow_spot, 1. / m->epow_spot);
    const double SFAC = 20. + BMAX;
    const int ns = m->nspot;
    el_alloc(d, 2 * ns);
    const double AREA = SFAC * m->length_spot * m->height_spot / (ns - 1);
    const double BRIGHT = planck(m->wavelength, m->temp_spot);
    for (int i = 0; i < ns; i++) {
        double dist = SFAC * i / (ns - 1);
        v3 posn = add3(bspot, scl3(m->length_spot * (dist - BMAX), bvec));
        int32_t nr = 0;
        double rin[LCO_MAXR], rout[LCO_MAXR];
        element_eclipses(m, &s, posn, 0, 0, &nr, rin, rout, e);
        if (e->st) return e->st;
        double bright = BRIGHT * pow(dist / BMAX, m->expon_spot) *
                        exp(m->expon_spot / m->epow_spot - pow(dist, m->epow_spot));
        el_set(d, i, posn, tvec, AREA);
        el_set(d, ns + i, posn, pvec, AREA);
        d->flux[i] = (float)(bright * (1 - m->cfrac_spot) * d->area[i]);
        d->flux[ns + i] = (float)(bright * m->cfrac_spot * d->area[i]);
        for (int k = 0; k < 2; k++) {
            int j = k ? ns + i : i;
            d->nr[j] = nr;
            memcpy(d->rin + LCO_MAXR * j, rin, sizeof rin);
            memcpy(d->rout + LCO_MAXR * j, rout, sizeof rout);
        }
    }
    return LCG_OK;
}

/* Point::visible (lcurve.h:81-89) over an element's ranges. */
static inline int el_visible(const elist *d, int i, double phase) {
    double phi = phase - floor(phase);
    for (int k = 0; k < d->nr[i]; k++) {
        double in = d->rin[LCO_MAXR * i + k], out = d->rout[LCO_MAXR * i + k];
        if ((phi >= in && phi <= out) || phi <= out - 1.0) return 0;
    }
    return 1;
}

/* comp_disc / comp_edge / comp_spot (comp_light.cpp:323-408): per
 * sub-exposure a serial sum over the elements in vector order, weighted and
 * merged in order. spot selects spot_elem (mu flux) over disc_elem (linear +
 * quadratic limb darkening). */
static double comp_elements(const lcg_model *m, const elist *d, int spot, double phase,
                            double expose, int ndiv) {
    double sum = 0.0;
    for (int nd = 0; nd < ndiv; ++nd) {
        double phi, wgt;
        if (ndiv == 1) { phi = phase; wgt = 1.0; }
        else {
            phi = phase + expose * (nd - (ndiv - 1) / 2.0) / (ndiv - 1);
            wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
        }
        double ri = deg2rad(m->iangle);
        double cosi = cos(ri), sini = sin(ri);
        v3 earth = set_earth(cosi, sini, phi);
        double s = 0.0;
        for (int i = 0; i < d->n; i++) {
            double v = 0.0;
            if (el_visible(d, i, phi)) {
                double mu = dot3(earth, mk3(d->dirn[3 * i], d->dirn[3 * i + 1], d->dirn[3 * i + 2]));
                if (spot) {
                    v = (mu > 0.0) ? mu * d->flux[i] : 0.0;
                } else if (mu > 0.0) {
                    double om = 1.0 - mu;
                    v = mu * d->flux[i] * (1.0 - om * (m->lin_limb_disc + m->quad_limb_disc * om));
                }
            }
            s += v;
        }
        sum += wgt * s;
    }
    return sum / ((ndiv - 1 > 1) ? ndiv - 1 : 1);
}

/* ---- iscale: Subs::svdfit (svdfit.cpp:22-80) ----------------------------
 * Least squares for the component scale factors: rows with sigma z > 0,
 * weighted by 1/z; singular values below 1e-5 of the largest are dropped.
 * The decomposition is a one-sided Jacobi SVD (Hestenes 1958) of the
 * weighted design matrix: the reference's svdcmp is a different SVD
 * algorithm, so the factors agree to rounding, not bit for bit. */
static void svd_solve(int nrow, int nc, double *A, const double *b, double *x) {
    double V[25], w[5];
    for (int i = 0; i < nc * nc; i++) V[i] = 0.;
    for (int i = 0; i < nc; i++) V[i * nc + i] = 1.;
    for (int sweep = 0; sweep < 60; sweep++) {
        int rotated = 0;
        for (int p = 0; p < nc - 1; p++)
            for (int q = p + 1; q < nc; q++) {
                double al = 0., be = 0., ga = 0.;
                for (int i = 0; i < nrow; i++) {
                    al += A[i * nc + p] * A[i * nc + p];
                    be += A[i * nc + q] * A[i * nc + q];
                    ga += A[i * nc + p] * A[i * nc + q];
                }
                if (ga == 0. || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
                rotated = 1;
                double zeta = (be - al) / (2. * ga);
                double t = (zeta >= 0. ? 1. : -1.) / (fabs(zeta) + sqrt(1. + zeta * zeta));
                double c = 1. / sqrt(1. + t * t), sn = c * t;
                for (int i = 0; i < nrow; i++) {
                    double ap = A[i * nc + p], aq = A[i * nc + q];
                    A[i * nc + p] = c * ap - sn * aq;
                    A[i * nc + q] = sn * ap + c * aq;
                }
                for (int i = 0; i < nc; i++) {
                    double vp = V[i * nc + p], vq = V[i * nc + q];
                    V[i * nc + p] = c * vp - sn * vq;
                    V[i * nc + q] = sn * vp + c * vq;
                }
            }
        if (!rotated) break;
    }
    double wmax = 0.;
    for (int j = 0; j < nc; j++) {
        double s = 0.;
        for (int i = 0; i < nrow; i++) s += A[i * nc + j] * A[i * nc + j];
        w[j] = sqrt(s);
        wmax = fmax(wmax, w[j]);
    }
    for (int j = 0; j < nc; j++) x[j] = 0.;
    for (int j = 0; j < nc; j++) {
        if (!(w[j] >= 1e-5 * wmax) || w[j] == 0.) continue;
        double ub = 0.;
        for (int i = 0; i < nrow; i++) ub += A[i * nc + j] * b[i];
        ub /= w[j] * w[j];  /* (u_j . b) / w_j with u_j = column j / w_j */
        for (int k = 0; k < nc; k++) x[k] += V[k * nc + j] * ub;
    }
}

/* sfac[0..nc-1] from the per-point components fcomp[n][5] (svdfit.cpp:22-80,
 * light_curve_comp.cpp:511-530). */
static void iscale_fit(const lcg_datum *data, int32_t n, const double *fcomp, int nc,
                       double *sfac) {
    int nrow = 0;
    for (int i = 0; i < n; i++) {
        double z = data[i].weight <= 0. ? -1. : data[i].ferr / sqrt(data[i].weight);
        if (z > 0) nrow++;
    }
    double *A = (double *)malloc(sizeof(double) * (size_t)(nrow > 0 ? nrow : 1) * nc);
    double *b = (double *)malloc(sizeof(double) * (size_t)(nrow > 0 ? nrow : 1));
    int k = 0;
    for (int i = 0; i < n; i++) {
        double z = data[i].weight <= 0. ? -1. : data[i].ferr / sqrt(data[i].weight);
        if (!(z > 0)) continue;
        double invsig = 1. / z;
        for (int j = 0; j < nc; j++) A[k * nc + j] = invsig * fcomp[5 * i + j];
        b[k++] = invsig * data[i].flux;
    }
    svd_solve(nrow, nc, A, b, sfac);
    free(A);
    free(b);
}

int lco_components(const lcg_model *m, int32_t which, int32_t cap, int32_t maxr,
                   int32_t *nout, double *posn, double *dirn, float *area, float *flux,
                   int32_t *nr, double *rin, double *rout, char *err, int errlen) {
    oerr e = {0, ""};
    elist d;
    memset(&d, 0, sizeof(d));
    double r1, r2;
    get_r1r2(m, &r1, &r2);
    const double rl2 = 1. - xl12(m->q, m->spin2, &e);
    if (r2 < 0) r2 = rl2;
    const double rdisc2 = m->rdisc2 > 0. ? m->rdisc2 : m->radius_spot;
    if (!e.st) {
        if (which == 0 && !disc_grid(m, &d, &e))
            disc_continuum(rdisc2, m->temp_disc, m->texp_disc, m->wavelength, &d);
        else if (which == 1 && !disc_edge(m, &d, &e))
            edge_continuum(m->temp_edge, r2, fabs(m->t2), m->absorb_edge, m->wavelength, &d);
        else if (which == 2)
            spot_grid(m, &d, &e);
    }
    if (!e.st) {
        *nout = d.n;
        if (d.n <= cap && posn) {
            memcpy(posn, d.posn, 3 * sizeof(double) * (size_t)d.n);
            memcpy(dirn, d.dirn, 3 * sizeof(double) * (size_t)d.n);
            memcpy(area, d.area, sizeof(float) * (size_t)d.n);
            memcpy(flux, d.flux, sizeof(float) * (size_t)d.n);
            for (int i = 0; i < d.n; i++) {
                nr[i] = d.nr[i];
                for (int k = 0; k < maxr && k < d.nr[i] && k < LCO_MAXR; k++) {
                    rin[maxr * i + k] = d.rin[LCO_MAXR * i + k];
                    rout[maxr * i + k] = d.rout[LCO_MAXR * i + k];
                }
            }
        }
    }
    el_free(&d);
    copyerr(&e, err, errlen);
    return e.st;
}

int lco_light_curve(const lcg_model *m, const lcg_datum *data, int32_t n,
                    int32_t flags, double *sfac, double *calc, double *scalars,
                    char *err, int errlen) {
    oerr e = {0, ""};
    sgrid s1f, s2f, s1c, s2c;
    memset(&s1f, 0, sizeof(s1f)); memset(&s2f, 0, sizeof(s2f));
    memset(&s1c, 0, sizeof(s1c)); memset(&s2c, 0, sizeof(s2c));
    pbatch pb1f = {0}, pb1c = {0}, pb2f = {0}, pb2c = {0};
    double *phases = NULL, *slfacs = NULL, *fcomp = NULL;
    double *o1f = NULL, *o1c = NULL, *o2f = NULL, *o2c = NULL;
    elist disc, edge, spot;
    memset(&disc, 0, sizeof(disc)); memset(&edge, 0, sizeof(edge)); memset(&spot, 0, sizeof(spot));

    if (n < 1) { seterr(&e, LCG_E_INVALID, "light_curve_comp: no data points"); goto done; }
    if (m->q <= 0.) { seterr(&e, LCG_E_INVALID, "Roche::xl12(double, double): q = %f <= 0.", m->q); goto done; }

    double r1, r2;
    get_r1r2(m, &r1, &r2);
    double rl2 = 1. - xl12(m->q, m->spin2, &e);
    if (e.st) goto done;
    if (r2 < 0) r2 = rl2;
    else if (r2 > rl2) {
        seterr(&e, LCG_E_LOBE, "light_curve_comp: the secondary star is larger than its Roche lobe!");
        goto done;
    }
    double rlens1 = 0.;
    if (m->glens1) {
        double gm = pow(1000. * m->velocity_scale, 3) * m->tperiod * DAY_F / TWOPI_;
        double a = pow(gm / (TWOPI_ / DAY_F / m->tperiod * TWOPI_ / DAY_F / m->tperiod), 1. / 3.);
        rlens1 = 4. * gm / (1. + m->q) / a / (C_LIGHT * C_LIGHT);
    }

    if (sgrid_build(m, LCG_STAR1, 1, &s1f, &e)) goto done;
    if (sgrid_build(m, LCG_STAR2, 1, &s2f, &e)) goto done;
    const int copy1 = (m->nlat1f == m->nlat1c);
    const int copy2 = (m->nlat2f == m->nlat2c) &&
                      (!m->npole || r1 >= r2 || (m->nlatfill == 0 && m->nlngfill == 0));
    if (!copy1 && sgrid_build(m, LCG_STAR1, 0, &s1c, &e)) goto done;
    if (!copy2 && sgrid_build(m, LCG_STAR2, 0, &s2c, &e)) goto done;
    sgrid *g1c = copy1 ? &s1f : &s1c;
    sgrid *g2c = copy2 ? &s2f : &s2c;

    if (flags & LCG_FLAG_INFO) {
        fprintf(stderr, "Number of points for star 1 (fine) = %d\n", s1f.n);
        fprintf(stderr, "Number of points for star 2 (fine) = %d\n", s2f.n);
        fprintf(stderr, "Number of points for star 1 (coarse) = %d\n", g1c->n);
        fprintf(stderr, "Number of points for star 2 (coarse) = %d\n", g2c->n);
    }

    continuum(m, LCG_STAR1, s1f.n, s1f.posn, s1f.dirn, s1f.area, s1f.gravity, s1f.flux);
    continuum(m, LCG_STAR2, s2f.n, s2f.posn, s2f.dirn, s2f.area, s2f.gravity, s2f.flux);
    if (!copy1) continuum(m, LCG_STAR1, s1c.n, s1c.posn, s1c.dirn, s1c.area, s1c.gravity, s1c.flux);
    if (!copy2) continuum(m, LCG_STAR2, s2c.n, s2c.posn, s2c.dirn, s2c.area, s2c.gravity, s2c.flux);

    ginterp gi = {m->phase1, m->phase2, 1., 1., 1., 1.};
    if (m->nlat1c != m->nlat1f) {
        double ff = comp_star_point(m, LCG_STAR1, 0.9999999999 * m->phase1, &gi, &s1f, g1c, rlens1);
        double fc = comp_star_point(m, LCG_STAR1, 1.0000000001 * m->phase1, &gi, &s1f, g1c, rlens1);
        gi.scale11 = ff / fc;
        ff = comp_star_point(m, LCG_STAR1, 1. - 0.9999999999 * m->phase1, &gi, &s1f, g1c, rlens1);
        fc = comp_star_point(m, LCG_STAR1, 1. - 1.0000000001 * m->phase1, &gi, &s1f, g1c, rlens1);
        gi.scale12 = ff / fc;
    }
    if (!copy2) {
        double ff = comp_star_point(m, LCG_STAR2, 1 - 1.0000000001 * m->phase2, &gi, &s2f, g2c, rlens1);
        double fc = comp_star_point(m, LCG_STAR2, 1 - 0.9999999999 * m->phase2, &gi, &s2f, g2c, rlens1);
        gi.scale21 = ff / fc;
        ff = comp_star_point(m, LCG_STAR2, 1.0000000001 * m->phase2, &gi, &s2f, g2c, rlens1);
        fc = comp_star_point(m, LCG_STAR2, 0.9999999999 * m->phase2, &gi, &s2f, g2c, rlens1);
        gi.scale22 = ff / fc;
    }
    /* disc, edge, opaque-disc eclipses of the stars, bright spot
       (light_curve_comp.cpp:272-333) */
    if (m->add_disc) {
        if (disc_grid(m, &disc, &e)) goto done;
        if (disc_edge(m, &edge, &e)) goto done;
        double rdisc1 = m->rdisc1 > 0. ? m->rdisc1 : r1;
        double rdisc2 = m->rdisc2 > 0. ? m->rdisc2 : m->radius_spot;
        if (m->opaque) {
            sgrid *gs[4] = {&s1f, copy1 ? NULL : &s1c, &s2f, copy2 ? NULL : &s2c};
            for (int k = 0; k < 4; k++) {
                sgrid *g = gs[k];
                if (!g) continue;
                size_t N = (size_t)(g->n > 0 ? g->n : 1);
                g->ndx = (int32_t *)calloc(N, sizeof(int32_t));
                g->xin = (double *)calloc(LCO_DISC_R * N, sizeof(double));
                g->xout = (double *)calloc(LCO_DISC_R * N, sizeof(double));
                for (int i = 0; i < g->n; i++) {
                    disc_eclipse(m->iangle, rdisc1, rdisc2, m->beta_disc, m->height_disc,
                                 mk3(g->posn[3 * i], g->posn[3 * i + 1], g->posn[3 * i + 2]),
                                 g->ndx + i, g->xin + LCO_DISC_R * i, g->xout + LCO_DISC_R * i,
                                 &e);
                    if (e.st) goto done;
                }
            }
        }
        disc_continuum(rdisc2, m->temp_disc, m->texp_disc, m->wavelength, &disc);
        edge_continuum(m->temp_edge, r2, fabs(m->t2), m->absorb_edge, m->wavelength, &edge);
    }
    if (m->add_spot && spot_grid(m, &spot, &e)) goto done;
    sgrid_flatten(&s1f);
    sgrid_flatten(&s2f);
    if (!copy1) sgrid_flatten(&s1c);
    if (!copy2) sgrid_flatten(&s2c);

    phases = (double *)malloc(sizeof(double) * (size_t)n);
    slfacs = (double *)malloc(sizeof(double) * (size_t)n);
    point_phases(m, data, n, phases, slfacs);
    {
        const double ri = deg2rad(m->iangle);
        const double cosi = cos(ri), sini = sin(ri);
        float vs = (float)m->velocity_scale;
        const double XCOFM = m->q / (1.0 + m->q);
        const double VFAC = vs / (C_LIGHT / 1.e3);
        if (m->iscale) {
            /* per-point components (light_curve_comp.cpp:378-414) */
            fcomp = (double *)calloc(5 * (size_t)n, sizeof(double));
            for (int np = 0; np < n; np++) {
                double phase = phases[np], slfac = slfacs[np];
                double expose = data[np].expose / m->period;
                const int ndiv = data[np].ndiv;
                double *f = fcomp + 5 * np;
                f[0] = slfac * comp_star_flat(m, LCG_STAR1, phase, expose, ndiv, &gi, &s1f, g1c,
                                              VFAC, XCOFM, rlens1);
                f[1] = slfac * comp_elements(m, &disc, 0, phase, expose, ndiv);
                f[2] = slfac * comp_elements(m, &edge, 0, phase, expose, ndiv);
                f[3] = slfac * comp_elements(m, &spot, 1, phase, expose, ndiv);
                if (m->t2 > 0)
                    f[4] = slfac * comp_star_flat(m, LCG_STAR2, phase, expose, ndiv, &gi, &s2f,
                                                  g2c, VFAC, XCOFM, rlens1);
            }
        }
        for (int np = 0; !m->iscale && np < n; np++) {
            double phase = phases[np], slfac = slfacs[np];
            double expose = data[np].expose / m->period;
            int ndiv = data[np].ndiv;
            double norm = (ndiv - 1 > 1) ? ndiv - 1 : 1;
            for (int nd = 0; nd < ndiv; ++nd) {
                double phi, wgt;
                if (ndiv == 1) { phi = phase; wgt = 1.0; }
                else {
                    phi = phase + expose * (nd - (ndiv - 1) / 2.0) / (ndiv - 1);
                    wgt = (nd == 0 || nd == ndiv - 1) ? 0.5 : 1.0;
                }
                v3 earth = set_earth(cosi, sini, phi);
                double phin = phi - floor(phi);
                double w1 = slfac * wgt * gi_scale1(&gi, phi) / norm;
                double w2 = slfac * wgt * gi_scale2(&gi, phi) / norm;
                pbatch *b1 = copy1 ? &pb1f : ((gi_type(&gi, phi) == 1) ? &pb1f : &pb1c);
                pbatch *b2 = copy2 ? &pb2f : ((gi_type(&gi, phi) == 3) ? &pb2f : &pb2c);
                pb_push(b1, earth.x, earth.y, earth.z, phin, w1, np);
                pb_push(b2, earth.x, earth.y, earth.z, phin, w2, np);
            }
        }
        for (int np = 0; np < n; np++) calc[np] = 0.;
        o1f = (double *)calloc((size_t)pb1f.n + 1, sizeof(double));
        o1c = (double *)calloc((size_t)pb1c.n + 1, sizeof(double));
        o2f = (double *)calloc((size_t)pb2f.n + 1, sizeof(double));
        o2c = (double *)calloc((size_t)pb2c.n + 1, sizeof(double));
        if (pb1f.n) sweep_flat(m, LCG_STAR1, &s1f, &pb1f, o1f, m->spin1, VFAC, XCOFM, rlens1);
        if (pb1c.n) sweep_flat(m, LCG_STAR1, g1c, &pb1c, o1c, m->spin1, VFAC, XCOFM, rlens1);
        if (pb2f.n) sweep_flat(m, LCG_STAR2, &s2f, &pb2f, o2f, m->spin2, VFAC, XCOFM, rlens1);
        if (pb2c.n) sweep_flat(m, LCG_STAR2, g2c, &pb2c, o2c, m->spin2, VFAC, XCOFM, rlens1);
        for (int64_t k = 0; k < pb1f.n; k++) calc[pb1f.idx[k]] += pb1f.w[k] * o1f[k];
        for (int64_t k = 0; k < pb1c.n; k++) calc[pb1c.idx[k]] += pb1c.w[k] * o1c[k];
        for (int64_t k = 0; k < pb2f.n; k++) calc[pb2f.idx[k]] += pb2f.w[k] * o2f[k];
        for (int64_t k = 0; k < pb2c.n; k++) calc[pb2c.idx[k]] += pb2c.w[k] * o2c[k];
        if (!m->iscale && (disc.n || edge.n || spot.n)) {
            for (int np = 0; np < n; np++) {
                double expose = data[np].expose / m->period;
                const int ndiv = data[np].ndiv;
                calc[np] += slfacs[np] * (comp_elements(m, &disc, 0, phases[np], expose, ndiv) +
                                          comp_elements(m, &edge, 0, phases[np], expose, ndiv) +
                                          comp_elements(m, &spot, 1, phases[np], expose, ndiv));
            }
        }
        if (!m->iscale)
            for (int np = 0; np < n; np++) calc[np] += m->third;

        const int diagnostics = (flags & LCG_FLAG_DIAGNOSTICS) != 0;
        double wdwarf = 0.0;
        if (diagnostics) {
            double phi = 0.5;
            v3 earth = set_earth(cosi, sini, phi);
            const sgrid *g = (gi_type(&gi, phi) == 1) ? &s1f : g1c;
            wdwarf = 1.0 * gi_scale1(&gi, phi) *
                     flat_sum_one(m, LCG_STAR1, g, earth, phi - floor(phi), VFAC, XCOFM, rlens1);
            wdwarf = wdwarf / 1;
        }
        const int nc = m->t2 > 0 ? 5 : 4;
        if ((flags & LCG_FLAG_SCALE) && m->iscale) {
            iscale_fit(data, n, fcomp, nc, sfac);
            wdwarf *= sfac[0];
            if (m->t2 <= 0.) sfac[4] = 0.;
            iscale_calc(m, n, fcomp, sfac, calc);
            double wnok = 0., chisq = 0.;
            for (int i = 0; i < n; i++) {
                if (data[i].weight > 0.) {
                    wnok += data[i].weight;
                    chisq += data[i].weight * sqr((data[i].flux - calc[i]) / data[i].ferr);
                }
            }
            scalars[LCG_OUT_CHISQ] = chisq;
            scalars[LCG_OUT_WNOK] = wnok;
        } else if (flags & LCG_FLAG_SCALE) {
            /* re_scale (re_scale.cpp:16-42) */
            double wgt, sdy = 0., syy = 0., wnok = 0., chisq = 0.;
            for (int i = 0; i < n; i++) {
                if (data[i].weight > 0.) {
                    wgt = data[i].weight / sqr(data[i].ferr);
                    sdy += wgt * data[i].flux * calc[i];
                    syy += wgt * calc[i] * calc[i];
                    wnok += data[i].weight;
                }
            }
            double ssfac;
            if (wnok > 0.0) {
                ssfac = sdy / syy;
                for (int i = 0; i < n; i++) calc[i] = calc[i] * ssfac;
                chisq = 0.;
                for (int i = 0; i < n; i++)
                    if (data[i].weight > 0.0)
                        chisq += data[i].weight * sqr((data[i].flux - calc[i]) / data[i].ferr);
            } else {
                ssfac = 1.;
                chisq = 0.;
            }
            wdwarf *= ssfac;
            for (int k = 0; k < 5; k++) sfac[k] = ssfac;
            scalars[LCG_OUT_CHISQ] = chisq;
            scalars[LCG_OUT_WNOK] = wnok;
        } else {
            wdwarf *= sfac[0];
            if (m->iscale) iscale_calc(m, n, fcomp, sfac, calc);
            else
                for (int np = 0; np < n; np++) calc[np] *= sfac[0];
            if (flags & LCG_FLAG_RDATA) {
                double wnok = 0., chisq = 0.;
                for (int i = 0; i < n; i++) {
                    if (data[i].weight > 0.) {
                        wnok += data[i].weight;
                        chisq += data[i].weight * sqr((data[i].flux - calc[i]) / data[i].ferr);
                    }
                }
                scalars[LCG_OUT_CHISQ] = chisq;
                scalars[LCG_OUT_WNOK] = wnok;
            }
        }
        scalars[LCG_OUT_WDWARF] = wdwarf;
        if (diagnostics) {
            scalars[LCG_OUT_LOGG1] = comp_gravity(m, LCG_STAR1, &s1f, &e);
            scalars[LCG_OUT_LOGG2] = comp_gravity(m, LCG_STAR2, &s2f, &e);
            scalars[LCG_OUT_RV1] = comp_radius(LCG_STAR1, &s1f);
            scalars[LCG_OUT_RV2] = comp_radius(LCG_STAR2, &s2f);
        } else {
            scalars[LCG_OUT_LOGG1] = scalars[LCG_OUT_LOGG2] = 0.0;
            scalars[LCG_OUT_RV1] = scalars[LCG_OUT_RV2] = 0.0;
        }
    }

done:
    sgrid_free(&s1f); sgrid_free(&s2f); sgrid_free(&s1c); sgrid_free(&s2c);
    pb_free(&pb1f); pb_free(&pb1c); pb_free(&pb2f); pb_free(&pb2c);
    free(phases); free(slfacs); free(fcomp);
    free(o1f); free(o1c); free(o2f); free(o2c);
    el_free(&disc); el_free(&edge); el_free(&spot);
    copyerr(&e, err, errlen);
    return e.st;
}

/* ---- light_curve_comp_fast (light_curve_comp_fast.cpp:6-84) ---------------
 * Above max_pts points, the curve is computed on max_pts points picked
 * uniformly by index (both ends included), interpolated linearly in time to
 * every point, and chi**2 / wnok are recomputed over all points (serial sums
 * in point order) when rdata is set. */
int lco_light_curve_fast(const lcg_model *m, const lcg_datum *data, int32_t n,
                         int32_t flags, int32_t max_pts, double *sfac, double *calc,
                         double *scalars, char *err, int errlen) {
    if (n <= max_pts)
        return lco_light_curve(m, data, n, flags, sfac, calc, scalars, err, errlen);
    if (max_pts < 2) {
        if (err && errlen > 0) snprintf(err, (size_t)errlen, "light_curve_comp_fast: max_model_points < 2");
        return LCG_E_INVALID;
    }
    size_t *idx = (size_t *)malloc(sizeof(size_t) * (size_t)max_pts);
    lcg_datum *sub = (lcg_datum *)malloc(sizeof(lcg_datum) * (size_t)max_pts);
    double *mc = (double *)malloc(sizeof(double) * (size_t)max_pts);
    for (int i = 0; i < max_pts; i++) {
        idx[i] = (size_t)i * (size_t)(n - 1) / (size_t)(max_pts - 1);
        sub[i] = data[idx[i]];
    }
    int st = lco_light_curve(m, sub, max_pts, flags, sfac, mc, scalars, err, errlen);
    if (st == 0) {
        for (int32_t i = 0; i < n; i++) {
            /* first sample index >= i */
            int lo = 0, hi = max_pts;
            while (lo < hi) {
                int mid = (lo + hi) / 2;
                if (idx[mid] < (size_t)i) lo = mid + 1;
                else hi = mid;
            }
            if (lo == 0) {
                calc[i] = mc[0];
            } else if (lo == max_pts) {
                calc[i] = mc[max_pts - 1];
            } else {
                const size_t i1 = idx[lo - 1], i2 = idx[lo];
                const double t = (data[i].time - data[i1].time) / (data[i2].time - data[i1].time);
                calc[i] = mc[lo - 1] * (1.0 - t) + mc[lo] * t;
            }
        }
        if (flags & LCG_FLAG_RDATA) {
            double wnok = 0., chisq = 0.;
            for (int32_t i = 0; i < n; i++) {
                if (data[i].weight > 0.) {
                    wnok += data[i].weight;
                    const double d = (data[i].flux - calc[i]) / data[i].ferr;
                    chisq += data[i].weight * (d * d);
                }
            }
            scalars[LCG_OUT_WNOK] = wnok;
            scalars[LCG_OUT_CHISQ] = chisq;
        }
    }
    free(idx);
    free(sub);
    free(mc);
    return st;
}
