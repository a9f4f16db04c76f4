// eclipse.cuh — per-face eclipse ingress/egress by a Roche-distorted star.
//
// Device restatement of Roche::ingress_egress (ingress_egress.cpp:35-97)
// with its helpers pot_min / linmin (pot_min.cpp:38-420), fblink
// (fblink.cpp:34-104) and Subs::dbrent (dbrent.cpp:21-126), one thread per
// surface element. FP64 throughout, same operation order (the file that
// includes this is compiled with --fmad=false), so the eclipse flags and
// phases follow the reference decision for decision. Every loop that the
// reference leaves unbounded carries an iteration cap; hitting one returns
// kEclNoConverge instead of spinning. linmin, pot_min and fblink are
// out-of-line functions: inlined into every caller they overflow the
// instruction cache and the warps stall on instruction fetch (dbrent stays
// inline in its two callers).
#pragma once

#include "roche.cuh"

namespace lcg {
// internal linkage: every translation unit that includes this header gets
// its own copy of these device functions
namespace {

enum {
    kEclOk = 0,
    kEclRoche = 3,       // LCG_E_ROCHE: linmin / pot_min failure (Roche_Error)
    kEclNoConverge = 4,  // LCG_E_NOCONVERGE: dbrent or a cap
};

// Potential along a line in (phase, lambda) space (roche.h:258-324) or
// along lambda with a fixed earth vector (roche.h:328-365).
struct LineFn {
    double q, spin, cosi, sini;
    int star;
    V3 p;
    double phi, dphi, lam, dlam;
    V3 earth;
    bool fixed_earth;

    __device__ __forceinline__ double val(double x) const {
        if (fixed_earth) return rpot(star, q, spin, add(p, scale(x, earth)));
        V3 e = set_earth(cosi, sini, phi + dphi * x);
        return rpot(star, q, spin, add(p, scale(lam + dlam * x, e)));
    }
    // Roche::rpot_grad (rpot_grad.cpp:25-39) projected on the line
    __device__ __forceinline__ double der(double x) const {
        V3 e = fixed_earth ? earth : set_earth(cosi, sini, phi + dphi * x);
        double l = fixed_earth ? x : lam + dlam * x;
        V3 d = drpot(star, q, spin, add(p, scale(l, e)));
        V3 ed = v3(e.y, -e.x, 0.);
        double dp = kTwoPi * l * dot(d, ed);
        double dl = dot(d, e);
        if (fixed_earth) return dl;
        return (dp * dphi + dl * dlam);
    }
};

__device__ __forceinline__ void rpot_grad_pl(int star, double q, double spin, V3 earth, V3 p,
                                             double lam, double &dphi, double &dlam) {
    V3 d = drpot(star, q, spin, add(p, scale(lam, earth)));
    V3 ed = v3(earth.y, -earth.x, 0.);
    dphi = kTwoPi * lam * dot(d, ed);
    dlam = dot(d, earth);
}

// Subs::dbrent with early exit below fref (dbrent.cpp:21-126).
__device__ double dbrent(double ax, double bx, double cx, const LineFn &f, double acc,
                         bool stopfast, double fref, double &xmin, int &st) {
    double a = (ax < cx ? ax : cx);
    double b = (ax > cx ? ax : cx);
    double x, w, v;
    x = w = v = bx;
    double fw, fv, fx;
    fw = fv = fx = f.val(x);
    if (stopfast && fx < fref) { xmin = x; return fx; }
    double dw, dv, dx;
    dw = dv = dx = f.der(x);
    double xm, tol1, tol2, e = 0., d1, d2, u1, u2, olde, d = 0, u, fu, du;
    for (int iter = 0; iter < 100; iter++) {
        xm = 0.5 * (a + b);
        tol1 = acc;
        tol2 = 2. * tol1;
        if (fabs(x - xm) <= (tol2 - 0.5 * (b - a))) { xmin = x; return fx; }
        if (fabs(e) > tol1) {
            d2 = d1 = 2. * (b - a);
            if (dw != dx) d1 = (w - x) * dx / (dx - dw);
            if (dv != dx) d2 = (v - x) * dx / (dx - dv);
            u1 = x + d1;
            u2 = x + d2;
            bool ok1 = (a - u1) * (u1 - b) > 0. && dx * d1 <= 0.;
            bool ok2 = (a - u2) * (u2 - b) > 0. && dx * d2 <= 0.;
            olde = e;
            e = d;
            if (ok1 || ok2) {
                if (ok1 && ok2) d = (fabs(d1) < fabs(d2) ? d1 : d2);
                else if (ok1) d = d1;
                else d = d2;
                if (fabs(d) <= fabs(0.5 * olde)) {
                    u = x + d;
                    if (u - a < tol2 || b - u < tol2) d = dsign(tol1, xm - x);
                } else {
                    d = 0.5 * (e = (dx >= 0. ? a - x : b - x));
                }
            } else {
                d = 0.5 * (e = (dx >= 0. ? a - x : b - x));
            }
        } else {
            d = 0.5 * (e = (dx >= 0. ? a - x : b - x));
        }
        if (fabs(d) >= tol1) {
            u = x + d;
            fu = f.val(u);
            if (stopfast && fu < fref) { xmin = u; return fu; }
        } else {
            u = x + dsign(tol1, d);
            fu = f.val(u);
            if (stopfast && fu < fref) { xmin = u; return fu; }
            if (fu > fx) { xmin = x; return fx; }
        }
        du = f.der(u);
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
    st = kEclNoConverge;
    xmin = x;
    return fx;
}

// Roche::linmin (pot_min.cpp:127-420). jammed starts false: the reference
// leaves it unset on early returns whose pmin equals the starting potential,
// where pot_min stops regardless of it.
__device__ __noinline__ void linmin(int star, double q, double spin, double cosi, double sini, V3 p,
                       double &phi, double &lam, double dphi, double dlam, double phi1,
                       double phi2, double lam1, double lam2, double pref, double acc,
                       double &pmin, bool &jammed, int &st) {
    LineFn f{q, spin, cosi, sini, star, p, phi, dphi, lam, dlam, v3(0., 0., 0.), false};
    jammed = false;
    double xmax = 1.e30, xend;
    int nbound = 0;
    if (dphi != 0.) {
        xend = (phi1 - phi) / dphi;
        if (xend > 0. && xend < xmax) { nbound = 1; xmax = xend; }
        xend = (phi2 - phi) / dphi;
        if (xend > 0. && xend < xmax) { nbound = 2; xmax = xend; }
    }
    if (dlam != 0.) {
        xend = (lam1 - lam) / dlam;
        if (xend > 0. && xend < xmax) { nbound = 3; xmax = xend; }
        xend = (lam2 - lam) / dlam;
        if (xend > 0. && xend < xmax) { nbound = 4; xmax = xend; }
    }
    double xa = 0., fa = f.val(xa);
    double xb = 1.e-8 * xmax, fb = f.val(xb);
    int nten = 0;
    const int NTEN = 7, NTRY = 5;
    while ((fb >= fa || xa == xb) && nten < NTEN) {
        nten++;
        xb *= 10.;
        fb = f.val(xb);
    }
    if (fb <= pref) { phi += dphi * xb; lam += dlam * xb; pmin = fb; return; }
    if (fb >= fa) { pmin = fa; return; }

    bool bracketted = false;
    double xc = 0., fc = 0., xbold = xb, fbold = fb;
    xmax -= xb;
    for (int n = 1; n <= NTRY; n++) {
        xc = xbold + xmax * n / NTRY;
        fc = f.val(xc);
        if (fc <= pref) { phi += dphi * xc; lam += dlam * xc; pmin = fc; return; }
        if (fc < fb) { xb = xc; fb = fc; }
        else { bracketted = true; break; }
    }
    if (!bracketted) {
        double dc = f.der(xc);
        if (dc > 0.) {
            xb = xbold;
            double db = f.der(xb);
            if (!(db < 0.)) { st = kEclRoche; pmin = fa; return; }  // "error 1"
            double xm = (xb + xc) / 2.;
            int guard = 0;
            while ((xc - xb) > 1.e-8 * xc) {
                if (++guard > 400) { st = kEclNoConverge; pmin = fa; return; }
                xm = (xb + xc) / 2.;
                if (f.der(xm) > 0.) xc = xm;
                else xb = xm;
            }
            double fm = f.val(xm);
            if (fm <= pref) { phi += dphi * xm; lam += dlam * xm; pmin = fm; return; }
            if (!(fm < fc && fm < fbold)) { st = kEclRoche; pmin = fa; return; }  // "error 3"
            xb = xm;
        } else {
            jammed = true;
            phi += dphi * xmax;
            lam += dlam * xmax;
            xmax = 1.;
            rpot_grad_pl(star, q, spin, set_earth(cosi, sini, phi), p, lam, dphi, dlam);
            switch (nbound) {
            case 1:
                phi = phi1; dphi = 0.;
                dlam = (dlam > 0.) ? lam1 - lam : lam2 - lam;
                break;
            case 2:
                phi = phi2; dphi = 0.;
                dlam = (dlam > 0.) ? lam1 - lam : lam2 - lam;
                break;
            case 3:
                lam = lam1; dlam = 0.;
                dphi = (dphi > 0.) ? phi1 - phi : phi2 - phi;
                break;
            case 4:
                lam = lam2; dlam = 0.;
                dphi = (dphi > 0.) ? phi1 - phi : phi2 - phi;
                break;
            }
            f.phi = phi; f.dphi = dphi; f.lam = lam; f.dlam = dlam;
            nten = 0;
            xb = 1.e-6;
            fb = f.val(xb);
            while (fb >= fa && nten < NTEN) {
                xb *= 10.;
                nten++;
                fb = f.val(xb);
            }
            if (fb <= pref) { phi += dphi * xb; lam += dlam * xb; pmin = fb; return; }
            if (fb >= fa) { pmin = fa; return; }
            bracketted = false;
            for (int n = 1; n <= NTRY; n++) {
                xc = xmax * n / NTRY;
                fc = f.val(xc);
                if (fc <= pref) { phi += dphi * xc; lam += dlam * xc; pmin = fc; return; }
                if (fc < fb) { xb = xc; fb = fc; }
                else { bracketted = true; break; }
            }
            if (!bracketted) {
                if (f.der(xc) > 0.) { st = kEclRoche; pmin = fa; return; }  // "error 2"
                phi += dphi * xmax;
                lam += dlam * xmax;
                pmin = fc;
                return;
            }
        }
    }
    double xmin;
    double xacc = acc / sqrt(sq(kTwoPi * dphi) + sq(dlam));
    pmin = dbrent(xa, xb, xc, f, xacc, true, pref, xmin, st);
    phi += dphi * xmin;
    lam += dlam * xmin;
}

// Roche::pot_min (pot_min.cpp:38-100): conjugate gradients in (phase,
// lambda) for the lowest potential on the line-of-sight cone.
__device__ __noinline__ bool pot_min(int star, double q, double spin, double cosi, double sini, V3 p,
                        double phi1, double phi2, double lam1, double lam2, double rref,
                        double pref, double acc, double &phi, double &lam, int &st) {
    double dphi, dlam, gdphi, gdlam, hdphi, hdlam;
    phi = (phi1 + phi2) / 2.;
    lam = (lam1 + lam2) / 2.;
    double rp = kTwoPi * phi;
    double cosp = cos(rp), sinp = sin(rp);
    V3 earth = v3(sini * cosp, -sini * sinp, cosi);
    double pot;
    {
        V3 r = add(p, scale(lam, earth));
        V3 d = drpot(star, q, spin, r);
        pot = rpot(star, q, spin, r);
        V3 ed = v3(earth.y, -earth.x, 0.);
        dphi = kTwoPi * lam * dot(d, ed);
        dlam = dot(d, earth);
    }
    if (pot <= pref) return true;
    gdphi = -dphi;
    gdlam = -dlam;
    dphi = hdphi = gdphi;
    dlam = hdlam = gdlam;
    const double DELPHI = q / (1. + q) * sq(acc / rref) / 2.;
    for (int its = 0; its < 200; its++) {
        double pmin;
        bool jammed;
        linmin(star, q, spin, cosi, sini, p, phi, lam, dphi, dlam, phi1, phi2, lam1, lam2,
               pref, acc, pmin, jammed, st);
        if (st) return false;
        if (pmin <= pref) return true;
        if (jammed || fabs(pmin - pot) < DELPHI) return false;
        pot = pmin;
        rp = kTwoPi * phi;
        cosp = cos(rp);
        sinp = sin(rp);
        earth = v3(sini * cosp, -sini * sinp, cosi);
        rpot_grad_pl(star, q, spin, earth, p, lam, dphi, dlam);
        double gg = gdphi * gdphi + gdlam * gdlam;
        if (gg == 0.) return false;
        double dgg = (dphi + gdphi) * dphi + (dlam + gdlam) * dlam;
        double gam = dgg / gg;
        gdphi = -dphi;
        gdlam = -dlam;
        dphi = hdphi = gdphi + gam * hdphi;
        dlam = hdlam = gdlam + gam * hdlam;
    }
    st = kEclRoche;  // "Roche::pot_min: too many iterations."
    return false;
}

// Roche::fblink (fblink.cpp:34-104): is p hidden along earth by the star?
__device__ __noinline__ bool fblink(int star, double q, double spin, double acc, V3 earth, V3 p,
                       double rref, double pref, int &st) {
    const V3 cofm = star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    double lam1, lam2;
    if (!sphere_eclipse_los(earth, p, cofm, rref, lam1, lam2)) return false;
    if (lam1 == 0.) return true;
    LineFn f{q, spin, 0., 0., star, p, 0., 0., 0., 0., earth, true};
    int nstep = 1;
    double step = (lam2 - lam1);
    double f1 = 0., f2 = 0., flam = 1., lam = lam1;
    long long evals = 0;
    while (step > acc) {
        lam = lam1 + step / 2.;
        for (int n = 0; n < nstep; n++) {
            flam = f.val(lam);
            if (flam <= pref) return true;
            if (nstep == 1) {
                f1 = f.val(lam1);
                f2 = f.val(lam2);
            }
            if (flam < f1 && flam < f2) break;
            lam += step;
        }
        if (flam < f1 && flam < f2) break;
        evals += nstep;
        if (evals > (1LL << 22)) { st = kEclNoConverge; return false; }
        step /= 2.;
        nstep *= 2;
    }
    if (flam < f1 && flam < f2) {
        double xmin;
        int sub = 0;
        flam = dbrent(lam1, lam, lam2, f, acc, true, pref, xmin, sub);
        if (sub) { st = kEclRoche; return false; }  // "fblink died"
        return (flam < pref);
    }
    return false;
}

// Roche::ingress_egress (ingress_egress.cpp:35-97) with the reference
// sphere (rref, pref) precomputed. Returns true when eclipsed.
__device__ bool ingress_egress(int star, double q, double spin, double cosi, double sini,
                               double delta, V3 r, double rref, double pref, double &ingress,
                               double &egress, int &st) {
    const V3 cofm = star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    double phi1, phi2, lam1, lam2, phi, lam;
    if (!sphere_eclipse_ph(cosi, sini, r, cofm, rref, phi1, phi2, lam1, lam2)) return false;
    const double ACC = 2. * sqrt(2. * kTwoPi * (lam2 - lam1) * delta);
    if (!pot_min(star, q, spin, cosi, sini, r, phi1, phi2, lam1, lam2, rref, pref, ACC, phi,
                 lam, st))
        return false;
    double pin = phi, pout = phi1, pmid;
    int guard = 0;
    while (fabs(pin - pout) > delta) {
        if (++guard > 400) { st = kEclNoConverge; return false; }
        pmid = (pin + pout) / 2.;
        if (fblink(star, q, spin, ACC, set_earth(cosi, sini, pmid), r, rref, pref, st))
            pin = pmid;
        else
            pout = pmid;
        if (st) return false;
    }
    ingress = (pin + pout) / 2.;
    ingress = ingress - floor(ingress);
    pin = phi;
    pout = phi2;
    guard = 0;
    while (fabs(pin - pout) > delta) {
        if (++guard > 400) { st = kEclNoConverge; return false; }
        pmid = (pin + pout) / 2.;
        if (fblink(star, q, spin, ACC, set_earth(cosi, sini, pmid), r, rref, pref, st))
            pin = pmid;
        else
            pout = pmid;
        if (st) return false;
    }
    egress = (pin + pout) / 2.;
    egress = egress - floor(egress);
    if (egress < ingress) egress++;
    return true;
}

}  // namespace
}  // namespace lcg

namespace lcg {
namespace {

// Warp-cooperative Roche::ingress_egress, for grids with few eclipse
// candidates, where one thread per face leaves the GPU idle. Lane 0 runs the
// sphere test and pot_min; then lanes 0-15 bisect the ingress and lanes 16-31
// the egress. Each half evaluates at once the 15 midpoints of the next four
// bisection steps (a complete binary tree of brackets in heap order: child 2n
// is "not hidden", pout = mid; child 2n+1 is "hidden", pin = mid) and then
// follows the path the results select. Each midpoint is computed from the
// same bracket by the same arithmetic as the sequential loop
// (ingress_egress.cpp:61-86), and fblink has no state, so the phases are
// identical to the sequential ones; only failures on the taken path count.
// All 32 lanes must call this with the same face.
__device__ bool ingress_egress_warp(int star, double q, double spin, double cosi, double sini,
                                    double delta, V3 r, double rref, double pref,
                                    double &ingress, double &egress, int &st) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int half = lane >> 4;
    const int node = (lane & 15) + 1;  // 1..16; node 16 has nothing to evaluate
    const V3 cofm = star == kStar1 ? v3(0., 0., 0.) : v3(1., 0., 0.);
    double phi1 = 0., phi2 = 0., lam1 = 0., lam2 = 0., phi = 0., lam = 0., ACC = 0.;
    int ok = 0, s0 = 0;
    if (lane == 0) {
        if (sphere_eclipse_ph(cosi, sini, r, cofm, rref, phi1, phi2, lam1, lam2)) {
            ACC = 2. * sqrt(2. * kTwoPi * (lam2 - lam1) * delta);
            ok = pot_min(star, q, spin, cosi, sini, r, phi1, phi2, lam1, lam2, rref, pref, ACC, phi,
                         lam, s0) ? 1 : 0;
        }
    }
    ok = __shfl_sync(full, ok, 0);
    s0 = __shfl_sync(full, s0, 0);
    if (s0) {
        st = s0;
        return false;
    }
    if (!ok) return false;
    phi = __shfl_sync(full, phi, 0);
    phi1 = __shfl_sync(full, phi1, 0);
    phi2 = __shfl_sync(full, phi2, 0);
    ACC = __shfl_sync(full, ACC, 0);
    double pin = phi, pout = half ? phi2 : phi1;
    const int depth = 31 - __clz(node);
    int fail = 0;  // uniform within a half: the status of a failed node on its path
    for (int round = 0;; round++) {
        const bool live = fabs(pin - pout) > delta && fail == 0;
        if (!__any_sync(full, live)) break;
        if (round >= 100) {  // uniform: every lane counts the same rounds
            st = kEclNoConverge;
            return false;
        }
        // this lane's bracket: replay the path below the root
        double a = pin, b = pout;
        bool valid = node < 16 && live;
        for (int lev = depth - 1; lev >= 0 && valid; lev--) {
            if (!(fabs(a - b) > delta)) {
                valid = false;
                break;
            }
            const double mid = (a + b) / 2.;
            if ((node >> lev) & 1) a = mid;
            else b = mid;
        }
        if (valid && !(fabs(a - b) > delta)) valid = false;
        int ls = 0;
        bool hidden = false;
        if (valid)
            hidden = fblink(star, q, spin, ACC, set_earth(cosi, sini, (a + b) / 2.), r, rref, pref,
                            ls);
        const unsigned res = __ballot_sync(full, hidden);
        const unsigned bad = __ballot_sync(full, ls != 0);
        // follow the taken path (the same in every lane of a half)
        int bad_src = -1;
        if (live) {
            int n = 1;
            for (int lev = 0; lev < 4; lev++) {
                if (!(fabs(pin - pout) > delta)) break;
                const int src = half * 16 + n - 1;
                if ((bad >> src) & 1u) {
                    bad_src = src;
                    break;
                }
                const double mid = (pin + pout) / 2.;
                const int h = (res >> src) & 1u;
                if (h) pin = mid;
                else pout = mid;
                n = 2 * n + h;
            }
        }
        const int code = __shfl_sync(full, ls, bad_src >= 0 ? bad_src : lane);
        if (bad_src >= 0) fail = code;
    }
    // the sequential routine bisects the ingress first: its failure wins
    const int fail_i = __shfl_sync(full, fail, 0), fail_e = __shfl_sync(full, fail, 16);
    if (fail_i || fail_e) {
        st = fail_i ? fail_i : fail_e;
        return false;
    }
    const double other_pin = __shfl_xor_sync(full, pin, 16);
    const double other_pout = __shfl_xor_sync(full, pout, 16);
    const double pin_i = half ? other_pin : pin, pout_i = half ? other_pout : pout;
    const double pin_e = half ? pin : other_pin, pout_e = half ? pout : other_pout;
    ingress = (pin_i + pout_i) / 2.;
    ingress = ingress - floor(ingress);
    egress = (pin_e + pout_e) / 2.;
    egress = egress - floor(egress);
    if (egress < ingress) egress++;
    return true;
}

}  // namespace
}  // namespace lcg
