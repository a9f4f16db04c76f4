// ecl_screen.cuh — an FP32 screen of the eclipse line-of-sight test.
//
// Roche::fblink (fblink.cpp:34-104) decides whether the line of sight from a
// point towards the earth passes inside the companion's Roche lobe: it cuts
// the line with the reference sphere, evaluates the potential at the chord
// midpoint (true at once if that is at or below the lobe potential pref),
// brackets a minimum and runs dbrent down to it. In the ingress/egress
// bisections most of these tests are far from the lobe's edge, where the
// answer does not depend on rounding or on the search path:
//
//   * the line misses the reference sphere by a margin: FP64 returns false;
//   * the potential at the chord midpoint is below pref by a margin: the
//     FP64 test takes the same first evaluation and returns true;
//   * the minimum of the potential along the chord is above pref by a
//     margin: nothing the FP64 search evaluates can reach pref, false.
//
// fblink_screen decides those cases in FP32 from one evaluation of the
// potential and its first two derivatives along the line at the chord
// midpoint (rsqrt on the MUFU unit), and answers kScreenUnsure for
// everything else, which the caller hands to the FP64 fblink. On B200 the
// FP64 pipe runs at half the FP32 rate, so the screen must stay a small
// fraction of an FP64 test: no iterations. The chord midpoint is the
// closest approach to the eclipser's centre (distance b); the minimum lies
// a step delta = |f'| / f'' away, and over |t| <= tau = 2 delta (at most b / 10)
// the second derivative stays above h_min = f'' - 0.05 m_e / b^3 - c3 tau (the
// eclipser's term -m_e / r loses at most 4.4% of its curvature there; c3
// bounds the change of the other star's), so f + f' t + h_min t^2 / 2 is a
// lower bound whose minimum f - f'^2 / (2 h_min) lies inside |t| < tau:
// the potential's minimum along the chord is at least that (it is unimodal
// along a chord of the reference sphere, where the eclipser's well
// dominates the centrifugal and tidal terms). The margin covers the FP32
// evaluation error (positions to ~4e-7, the potential to a few ulps of its
// largest terms); the decisions the screen takes are those of the FP64
// test, so the bisections follow the same midpoints to the same ingress and
// egress.
//
// The potential is evaluated about the eclipser's centre u = P - c with the
// constant terms dropped (pref shifted to match):
//   phi(u) = -m_e/|u| - m_o/|u - d| - ss/2 (ux^2 + uy^2) + k ux
// star 1 eclipses (c = 0):        m_e = 1-mu, m_o = mu, d = (+1,0,0), k = mu
// star 2 eclipses (c = (1,0,0)):  m_e = mu, m_o = 1-mu, d = (-1,0,0), k = -(1-mu),
//                                 constant -(1-mu) moved into pref
// which is Roche::rpot1 / rpot2 (rpot.cpp:37-86) rewritten about c.
#pragma once

#include "roche.cuh"

namespace lcg {

enum { kScreenFalse = 0, kScreenTrue = 1, kScreenUnsure = 2 };

struct EclScreen {
    float me, mo, dx, ss, k;  // potential about the eclipser's centre
    float rref2;              // reference sphere radius squared
    float pref;               // lobe potential, shifted
    float margin;             // decision margin on the potential
    float c3;                 // bound on |d/dlam| of the other star's curvature
    int32_t on;               // 0: every test goes to FP64
};

// Host: the screen constants for eclipser `star` (kStar1 / kStar2) of a
// binary with mass ratio q, spin of the eclipser, reference sphere (rref,
// pref) as ref_sphere gives them.
inline EclScreen make_ecl_screen(int star, double q, double spin, double rref, double pref) {
    EclScreen s;
    const double mu = q / (1 + q), comp = 1. - mu;
    if (star == kStar1) {
        s.me = (float)comp; s.mo = (float)mu; s.dx = 1.f; s.k = (float)mu;
        s.pref = (float)pref;
    } else {
        s.me = (float)mu; s.mo = (float)comp; s.dx = -1.f; s.k = (float)-comp;
        s.pref = (float)(pref + comp);
    }
    s.ss = (float)(spin * spin);
    s.rref2 = (float)(rref * rref);
    // FP32 error of the potential: a few ulps of its largest terms (the
    // eclipser's well at its reference sphere, the other star's well at
    // least 1 - rref away), plus its gradient there times 4e-7 of position
    // error (the point, the earth vector and the line parameter in FP32)
    const double dob = (1. - rref > 0.1) ? 1. - rref : 0.1;
    const double pot = s.me / rref + s.mo / dob + 1.;
    const double grad = s.me / (rref * rref) + s.mo / (dob * dob) + 1.;
    s.margin = (float)(4e-6 * pot + 4e-7 * grad + 1e-6);
    // |third derivative| of -m_o / r along a line is at most 6 m_o / r^4
    s.c3 = (float)(6. * s.mo / (dob * dob * dob * dob));
    s.on = 1;
    return s;
}

namespace {

LCG_HD float scr_rsqrt(float x) {
#ifdef __CUDA_ARCH__
    return rsqrtf(x);
#else
    return 1.f / sqrtf(x);
#endif
}

// potential, first and second derivatives along e at u (explicit fmaf: the
// files that include this are compiled without FMA contraction)
LCG_HD void scr_phi(const EclScreen &S, float ux, float uy, float uz, float ex, float ey,
                    float ez, float &f, float &g, float &h) {
    const float vx = ux - S.dx;
    const float ryz = fmaf(uy, uy, uz * uz);
    const float ie = scr_rsqrt(fmaf(ux, ux, ryz)), io = scr_rsqrt(fmaf(vx, vx, ryz));
    const float ie2 = ie * ie, io2 = io * io;
    const float ae = S.me * ie * ie2, ao = S.mo * io * io2;  // m / r^3
    const float eyz = fmaf(ey, uy, ez * uz);
    const float eu = fmaf(ex, ux, eyz), ev = fmaf(ex, vx, eyz);
    const float rxy = fmaf(ux, ux, uy * uy);
    f = fmaf(S.k, ux, fmaf(-0.5f * S.ss, rxy, -fmaf(S.me, ie, S.mo * io)));
    g = fmaf(ae, eu, fmaf(ao, ev, fmaf(-S.ss, fmaf(ex, ux, ey * uy), S.k * ex)));
    // d/dlam of m e.u / |u|^3 = m (1 / |u|^3 - 3 (e.u)^2 / |u|^5)
    h = fmaf(ae, fmaf(-3.f * eu * eu, ie2, 1.f),
             fmaf(ao, fmaf(-3.f * ev * ev, io2, 1.f), -S.ss * fmaf(ex, ex, ey * ey)));
}

}  // namespace

// u0: the point relative to the eclipser's centre; e: the earth vector;
// acc: fblink's accuracy on the line parameter.
LCG_HD int fblink_screen(const EclScreen &S, float u0x, float u0y, float u0z, float ex, float ey,
                         float ez, float acc) {
    const float B = ex * u0x + ey * u0y + ez * u0z;
    const float C = u0x * u0x + u0y * u0y + u0z * u0z - S.rref2;
    const float tiny = 4e-6f * (1.f + S.rref2 + u0x * u0x + u0y * u0y + u0z * u0z);
    if (B >= tiny) return kScreenFalse;  // pointing away from the eclipser
    if (B > -tiny || C <= tiny) return kScreenUnsure;
    const float fac = B * B - C;
    if (fac <= -tiny) return kScreenFalse;  // misses the reference sphere
    if (fac < tiny) return kScreenUnsure;
    const float hc = sqrtf(fac);  // half chord: lam2 - lam1 = 2 hc
    // FP64 runs its search only while the chord exceeds acc; 2 hc carries an
    // error up to about tiny / hc from fac
    const float slack = 2.f * tiny / hc + 1e-6f * acc;
    if (2.f * hc < acc - slack) return kScreenFalse;
    if (2.f * hc <= acc + slack) return kScreenUnsure;
    const float M = S.margin;
    // the chord midpoint -B: fblink's first evaluation, and the closest
    // approach to the eclipser's centre
    const float x = -B;
    float f, g, h;
    scr_phi(S, u0x + x * ex, u0y + x * ey, u0z + x * ez, ex, ey, ez, f, g, h);
    if (f <= S.pref - M) return kScreenTrue;
    if (f <= S.pref + M) return kScreenUnsure;
    // lower bound on the minimum along the chord: a quadratic about x with
    // the least curvature over |t| <= tau
    const float b2 = S.rref2 - fac;  // |u0|^2 - B^2
    if (!(b2 > 0.f) || !(h > 0.f)) return kScreenUnsure;
    const float b = sqrtf(b2);
    const float tau = 2.f * fabsf(g) / h + 1e-6f * b;
    if (tau > 0.1f * b || tau > hc) return kScreenUnsure;
    const float hmin = h - 0.05f * S.me / (b2 * b) - S.c3 * tau;
    if (!(hmin > 0.f)) return kScreenUnsure;
    const float fmin = f - g * g / (2.f * hmin);
    return fmin > S.pref + M ? kScreenFalse : kScreenUnsure;
}

}  // namespace lcg
