// engine.cu — host side of the light-curve engine and the C ABI (include/lcg.h).
//
// Restates the orchestration of Lcurve::light_curve_comp
// (light_curve_comp.cpp:119-599) over device-resident stages:
//   per model (host, FP64, the reference's libm): radii and Roche-lobe
//   checks, reference spheres, gref, the latitude-ring table
//   (set_star_grid.cpp:49-320, numface.cpp);
//   per face (device): grid -> eclipse -> continuum -> FlatGrid partition;
//   per sub-exposure (device): phases -> flux sweeps -> scatter -> scale/chi**2.
// Grids and continuum are rebuilt only when the parameters they depend on
// change (the exact-reuse cache, light_curve_comp.cpp:28-117).
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <string>
#include <vector>

#include "context.h"

using namespace lcg;
using namespace lcg::eng;

namespace {

thread_local std::string g_create_error;
std::atomic<long long> g_launches{0};

}  // namespace

namespace lcg {
namespace eng {

// ---- per-model host setup ---------------------------------------------------

// Model::get_r1r2 (lcurve.h:399-410)
void get_r1r2(const lcg_model &m, double &rr1, double &rr2) {
    if (m.use_radii) {
        rr1 = m.r1;
        rr2 = m.r2;
    } else {
        double sini = sin(deg2rad(m.iangle));
        double r2pr1 = sqrt(1.0 - pow(sini * cos(2.0 * kM_PI * m.cphi4), 2));
        double r2mr1 = sqrt(1.0 - pow(sini * cos(2.0 * kM_PI * m.cphi3), 2));
        rr1 = (r2pr1 - r2mr1) / 2.0;
        rr2 = (r2pr1 + r2mr1) / 2.0;
    }
}

// set_star_grid.cpp:528-538
void envelope(double rangle, double lambda, double r1, double &x, double &y) {
    double sini = sin(rangle), cosi = cos(rangle);
    double sinl = sin(lambda), cosl = cos(lambda);
    double norm = sqrt(cosi * cosi + sini * sini * cosl * cosl);
    x = sinl + r1 * cosi * sinl / norm;
    y = -cosi * cosl - r1 * cosl / norm;
}

// Lcurve::numface (numface.cpp:14-52)
int numface(int nlat, bool infill, double thelo, double thehi, int nlatfill, int nlngfill) {
    int nface = 0;
    double theta, dphi, dtheta = kPi / nlat;
    if (infill) {
        int nl1 = (int)ceil(thelo / dtheta);
        for (int i = 0; i < nl1; i++) {
            theta = thelo * (i + 0.5) / nl1;
            dphi = dtheta / sin(theta);
            nface += std::max(16, (int)(2 * kPi / dphi));
        }
        int nl2 = (int)ceil((1 + nlatfill) * (thehi - thelo) / dtheta);
        for (int i = 0; i < nl2; i++) {
            theta = thelo + (thehi - thelo) * (i + 0.5) / nl2;
            dphi = dtheta / sin(theta) / (1 + nlngfill);
            nface += std::max(8, (int)(kPi / dphi));
        }
        int nl3 = (int)ceil((thehi - thelo) / dtheta);
        for (int i = 0; i < nl3; i++) {
            theta = thelo + (thehi - thelo) * (i + 0.5) / nl3;
            dphi = dtheta / sin(theta);
            nface += std::max(8, (int)(kPi / dphi));
        }
        int nl4 = (int)ceil((kPi - thehi) / dtheta);
        for (int i = 0; i < nl4; i++) {
            theta = thehi + (kPi - thehi) * (i + 0.5) / nl4;
            dphi = dtheta / sin(theta);
            nface += std::max(16, (int)(2 * kPi / dphi));
        }
    } else {
        nlat = (int)ceil(kPi / dtheta);
        for (int i = 0; i < nlat; i++) {
            theta = kPi * (i + 0.5) / nlat;
            dphi = dtheta / sin(theta);
            nface += std::max(16, (int)(2 * kPi / dphi));
        }
    }
    return nface;
}


// Appends the rings of one add_faces call (set_star_grid.cpp:241-320).
bool add_rings(int star, StarSetup &s, int &nface, double tlo, double thi, double dtheta,
               int nlatfill, int nlngfill) {
    const bool infill = (nlatfill > 0) || (nlngfill > 0);
    int nlat, nlat1 = 0, nlat2 = 0;
    if (infill) {
        nlat1 = (int)ceil((1 + nlatfill) * (thi - tlo) / dtheta);
        nlat2 = (int)ceil((thi - tlo) / dtheta);
        nlat = nlat1 + nlat2;
    } else {
        nlat = (int)ceil((thi - tlo) / dtheta);
    }
    for (int nt = 0; nt < nlat; nt++) {
        RingRec R;
        double theta, phi1, phi2;
        int nl, nphi;
        if (infill) {
            if (nt < nlat1) {
                theta = tlo + (thi - tlo) * (nt + 0.5) / nlat1;
                R.sint = sin(theta);
                R.cost = cos(theta);
                nphi = std::max(8, (int)(kPi * R.sint * (1 + nlngfill) / dtheta));
                nl = nlat1;
                if (star == kStar1) { phi1 = -kPi / 2.; phi2 = +kPi / 2.; }
                else { phi1 = +kPi / 2.; phi2 = +3. * kPi / 2.; }
            } else {
                theta = tlo + (thi - tlo) * (nt - nlat1 + 0.5) / nlat2;
                R.sint = sin(theta);
                R.cost = cos(theta);
                nphi = std::max(8, (int)(kPi * R.sint / dtheta));
                nl = nlat2;
                if (star == kStar1) { phi1 = +kPi / 2.; phi2 = +3. * kPi / 2.; }
                else { phi1 = -kPi / 2.; phi2 = +kPi / 2.; }
            }
        } else {
            theta = tlo + (thi - tlo) * (nt + 0.5) / nlat;
            R.sint = sin(theta);
            R.cost = cos(theta);
            nphi = std::max(16, (int)(2 * kPi * R.sint / dtheta));
            nl = nlat;
            phi1 = 0.;
            phi2 = kTwoPi;
        }
        R.phi1 = phi1;
        R.span = phi2 - phi1;
        R.latspan = thi - tlo;
        R.nphi = nphi;
        R.nl = nl;
        R.off = nface;
        R.hoff = (int32_t)s.nhalf;
        nface += nphi;
        s.nhalf += (nphi + 1) / 2;
        s.rings.push_back(R);
    }
    return true;
}

// set_star_grid.cpp:49-223 up to the tiling.
bool prepare_star(const lcg_model &m, int star, int fine, StarSetup &s, Fail &f, bool tiling) {
    double r1, r2;
    get_r1r2(m, r1, r2);
    s.eclipse = star == kStar1 ? m.eclipse1 : m.eclipse2;
    s.nlat = star == kStar1 ? (fine ? m.nlat1f : m.nlat1c) : (fine ? m.nlat2f : m.nlat2c);
    s.nlatfill = star == kStar1 ? 0 : (fine ? m.nlatfill : 0);
    s.nlngfill = star == kStar1 ? 0 : (fine ? m.nlngfill : 0);
    const double latlo = star == kStar1 ? 0 : m.llo, lathi = star == kStar1 ? 0 : m.lhi;
    if (s.nlat <= 0) {
        f = {LCG_E_INVALID, "set_star_grid: the number of latitude strips must be positive"};
        return false;
    }
    const double rl1 = xl11(m.q, m.spin1);
    if (rl1 < 0) {
        f = {LCG_E_NOCONVERGE, "Roche::xl11(double, double): exceeded maximum iterations"};
        return false;
    }
    if (r1 < 0) r1 = rl1;
    else if (r1 > rl1) {
        f = {LCG_E_LOBE, "set_star_grid: the primary star is larger than its Roche lobe!"};
        return false;
    }
    const double xl2 = xl12(m.q, m.spin2);
    if (xl2 < 0) {
        f = {LCG_E_NOCONVERGE, "Roche::xl12(double,double): exceeded maximum iterations"};
        return false;
    }
    const double rl2 = 1. - xl2;
    if (r2 < 0) r2 = rl2;
    else if (r2 > rl2) {
        f = {LCG_E_LOBE, "set_star_grid: the secondary star is larger than its Roche lobe!"};
        return false;
    }
    if (m.glens1 && star == kStar2 && m.roche1 && m.eclipse2) {
        f = {LCG_E_INVALID, "set_star_grid: cannot have gravitational lensing, eclipse and "
                            "Roche lobe geometry at the same time"};
        return false;
    }
    if (m.glens1 && star == kStar2) {
        double gm = pow(1000. * m.velocity_scale, 3) * m.tperiod * kDay / kTwoPi;
        double a = pow(gm / sq(kTwoPi / kDay / m.tperiod), 1. / 3.);
        double rlens1 = 4. * gm / (1. + m.q) / a / sq(kC);
        r1 -= rlens1 / (r1 / (1. - r2 / 2.));
        if (r1 < 0) {
            f = {LCG_E_INVALID, "set_star_grid: gravitational lensing correction more than the "
                                "current program can cope with."};
            return false;
        }
    }
    s.r1 = r1; s.r2 = r2; s.rl1 = rl1; s.rl2 = rl2;
    s.ffac1 = r1 / rl1;
    ref_sphere(kStar1, m.q, m.spin1, s.ffac1, s.rref1, s.pref1);
    s.ffac2 = r2 / rl2;
    ref_sphere(kStar2, m.q, m.spin2, s.ffac2, s.rref2, s.pref2);

    bool infill = m.npole && (star == kStar2) && (s.nlatfill > 0 || s.nlngfill > 0) && r2 > r1;
    double thelo = 0, thehi = 0;
    if (infill) {
        double rangle = deg2rad(m.iangle);
        double cosi = cos(rangle);
        double ratio = (cosi + r1) / r2;
        if (ratio >= 1.) {
            thehi = kPi / 2. + rangle;
        } else {
            double llo = 0., lhi = kPi / 2., x = 0., y = 0.;
            while (lhi > llo + 1.e-7) {
                double lmid = (llo + lhi) / 2.;
                envelope(rangle, lmid, r1, x, y);
                if (x * x + y * y < r2 * r2) llo = lmid;
                else lhi = lmid;
            }
            double sini = sin(rangle);
            thehi = dmax(kPi / 2. - deg2rad(latlo),
                         dmin(kPi / 2. + rangle, acos(y * sini / r2) + deg2rad(m.lfudge)));
        }
        ratio = (cosi - r1) / r2;
        if (ratio >= 1.) infill = false;
        else if (ratio <= -1.) thelo = 0.;
        else
            thelo = dmin(kPi / 2. - deg2rad(lathi),
                         dmax(0., kPi / 2. - acos(ratio) + rangle - deg2rad(m.lfudge)));
    }
    s.infill = infill;
    s.thelo = thelo;
    s.thehi = thehi;
    s.nface = tiling ? numface(s.nlat, infill, thelo, thehi, s.nlatfill, s.nlngfill) : 0;

    const double ACC = m.delta_phase / 10.;
    V3 posn, dvec;
    double rad, gref = 1.;
    int bad = 0;
    if (star == kStar1 && m.roche1)
        bad = face_scalar(kStar1, m.q, m.spin1, v3(-1., 0., 0.), s.rref1, s.pref1, ACC, posn, dvec,
                          rad, gref);
    else if (star == kStar2 && m.roche2)
        bad = face_scalar(kStar2, m.q, m.spin2, v3(1., 0., 0.), s.rref2, s.pref2, ACC, posn, dvec,
                          rad, gref);
    if (bad) {
        f = {LCG_E_ROCHE, "Roche::face error: could not solve the reference gravity point"};
        return false;
    }
    s.gref = gref;
    if (!tiling) return true;

    s.rings.clear();
    s.nhalf = 0;
    int nface = 0;
    const double dtheta = kPi / s.nlat;
    if (infill) {
        add_rings(star, s, nface, 0., thelo, dtheta, 0, 0);
        add_rings(star, s, nface, thelo, thehi, dtheta, s.nlatfill, s.nlngfill);
        add_rings(star, s, nface, thehi, kPi, dtheta, 0, 0);
    } else {
        add_rings(star, s, nface, 0., kPi, dtheta, 0, 0);
    }
    // the ring tiling can differ from numface by a face or two (nlat 153, 297,
    // 315, 333, 339, 813, ...); the grid keeps numface faces (GridDev)
    s.ntiled = nface;
    return true;
}

const char *status_text(int code) {
    switch (code) {
    case 3: return "set_star_grid: Roche face or eclipse computation failed";
    case 4: return "set_star_grid: an iteration cap was reached in the eclipse computation";
    case 6: return "flux sweep: shared-memory staging timed out";
    default: return "device failure";
    }
}

bool same_geometry(const lcg_model &a, const lcg_model &b) {
    // GeomKey (light_curve_comp.cpp:34-86)
    const bool g = a.glens1 != 0;
    return a.q == b.q && a.iangle == b.iangle && a.r1 == b.r1 && a.r2 == b.r2 &&
           a.cphi3 == b.cphi3 && a.cphi4 == b.cphi4 && a.spin1 == b.spin1 &&
           a.spin2 == b.spin2 &&
           (g ? a.velocity_scale : 0.) == (b.glens1 ? b.velocity_scale : 0.) &&
           (g ? a.tperiod : 0.) == (b.glens1 ? b.tperiod : 0.) && a.llo == b.llo &&
           a.lhi == b.lhi && a.lfudge == b.lfudge && a.delta_phase == b.delta_phase &&
           a.phase1 == b.phase1 && a.phase2 == b.phase2 && a.nlat1f == b.nlat1f &&
           a.nlat2f == b.nlat2f && a.nlat1c == b.nlat1c && a.nlat2c == b.nlat2c &&
           a.nlatfill == b.nlatfill && a.nlngfill == b.nlngfill && a.use_radii == b.use_radii &&
           a.roche1 == b.roche1 && a.roche2 == b.roche2 && a.eclipse1 == b.eclipse1 &&
           a.eclipse2 == b.eclipse2 && a.glens1 == b.glens1 && a.npole == b.npole;
}

bool same_continuum(const lcg_model &a, const lcg_model &b) {
    // ContKey (light_curve_comp.cpp:43-52,88-115)
    if (!(a.t1 == b.t1 && a.t2 == b.t2 && a.gravity_dark1 == b.gravity_dark1 &&
          a.gravity_dark2 == b.gravity_dark2 && a.wavelength == b.wavelength &&
          a.absorb == b.absorb && a.mucrit1 == b.mucrit1 && a.mucrit2 == b.mucrit2 &&
          a.beam_factor1 == b.beam_factor1 && a.beam_factor2 == b.beam_factor2 &&
          a.limb1 == b.limb1 && a.limb2 == b.limb2 && a.gdark_bolom1 == b.gdark_bolom1 &&
          a.gdark_bolom2 == b.gdark_bolom2 && a.mirror == b.mirror))
        return false;
    for (int k = 0; k < 4; k++)
        if (!(a.ldc1[k] == b.ldc1[k] && a.ldc2[k] == b.ldc2[k])) return false;
    for (int s = 0; s < 5; s++) {
        if (a.stsp_defined[s] != b.stsp_defined[s]) return false;
        for (int k = 0; k < 4; k++)
            if (!(a.stsp[s][k] == b.stsp[s][k])) return false;
    }
    if (a.uesp_defined != b.uesp_defined) return false;
    for (int k = 0; k < 5; k++)
        if (!(a.uesp[k] == b.uesp[k])) return false;
    return true;
}

ContParams continuum_params(const lcg_model &m, int star) {
    // set_star_continuum.cpp:30-101, 205-237
    double r1, r2;
    get_r1r2(m, r1, r2);
    double rl1 = xl1(m.q);
    if (r1 < 0) r1 = rl1;
    double rl2 = 1. - rl1;
    if (r2 < 0) r2 = rl2;
    ContParams p{};
    p.star = star;
    p.mirror = m.mirror;
    p.absorb = m.absorb;
    p.wavelength = m.wavelength;
    p.efac = sqrt(8. * log(2.));
    p.fp32 = 0;  // the callers that run mixed turn it on
    p.irr32 = (float)(m.absorb * pow(star == kStar1 ? m.t2 : m.t1, 4.));
    p.planck_c1 = (float)(2.e27 * kH * kC / (m.wavelength * m.wavelength * m.wavelength));
    p.planck_c2 = (float)(1.e9 * kH * kC / kK / m.wavelength);
    if (star == kStar1) {
        p.t_own = m.t1;
        p.t_other = m.t2;
        p.rcomp = r2;
        p.gdcbol = m.gdark_bolom1 ? m.gravity_dark1 : m.gravity_dark1 / dlpdlt(m.wavelength, m.t1);
        for (int s = 0; s < 3; s++) {
            if (!m.stsp_defined[s]) continue;
            const int k = p.nspot++;
            double clong = cos(deg2rad(m.stsp[s][0])), slong = sin(deg2rad(m.stsp[s][0]));
            double clat = cos(deg2rad(m.stsp[s][1])), slat = sin(deg2rad(m.stsp[s][1]));
            p.spot_dir[k][0] = clat * clong;
            p.spot_dir[k][1] = clat * slong;
            p.spot_dir[k][2] = slat;
            p.spot_fwhm[k] = m.stsp[s][2];
            p.spot_tcen[k] = m.stsp[s][3];
        }
        p.uesp_on = m.uesp_defined;
        if (p.uesp_on) {
            p.uesp_longhw = (m.uesp[1] - m.uesp[0]) / 2.;
            double lcen = deg2rad((m.uesp[0] + m.uesp[1]) / 2.);
            p.uesp_dir[0] = cos(lcen);
            p.uesp_dir[1] = sin(lcen);
            p.uesp_dir[2] = 0.;
            p.uesp_lathw = m.uesp[2];
            p.uesp_taper = m.uesp[3];
            p.uesp_temp = m.uesp[4];
        }
    } else {
        p.t_own = m.t2;
        p.t_other = m.t1;
        p.rcomp = r1;
        p.gdcbol = m.gdark_bolom2 ? m.gravity_dark2
                                  : m.gravity_dark2 / dlpdlt(m.wavelength, fabs(m.t2));
        for (int s = 3; s < 5; s++) {
            if (!m.stsp_defined[s]) continue;
            const int k = p.nspot++;
            double clong = cos(deg2rad(m.stsp[s][0])), slong = sin(deg2rad(m.stsp[s][0]));
            double clat = cos(deg2rad(m.stsp[s][1])), slat = sin(deg2rad(m.stsp[s][1]));
            p.spot_dir[k][0] = clat * clong;
            p.spot_dir[k][1] = clat * slong;
            p.spot_dir[k][2] = slat;
            p.spot_fwhm[k] = m.stsp[s][2];
            p.spot_tcen[k] = m.stsp[s][3];
        }
    }
    return p;
}

FluxConsts flux_consts(const lcg_model &m, int star, double spin, double rlens1) {
    FluxConsts k{};
    const double *c = star == kStar1 ? m.ldc1 : m.ldc2;
    for (int i = 0; i < 4; i++) k.c[i] = c[i];
    k.base = 1.0 - (c[0] + c[1] + c[2] + c[3]);
    k.mucrit = star == kStar1 ? m.mucrit1 : m.mucrit2;
    k.ltype = star == kStar1 ? m.limb1 : m.limb2;
    k.beam = star == kStar1 ? m.beam_factor1 : m.beam_factor2;
    k.beam_on = k.beam != 0.0;
    k.glens = star == kStar2 ? m.glens1 : 0;
    k.spin = spin;
    const float vs = (float)m.velocity_scale;
    k.vfac = vs / (kC / 1.e3);
    k.xcofm = m.q / (1.0 + m.q);
    k.rlens1 = rlens1;
    return k;
}

// Grid + eclipse (+ nothing else): the geometry stage of one star grid, on
// stream st (the grid's own candidate queue, so two grids can build at once).
lcg_status build_geometry(lcg_ctx *c, const lcg_model &m, int star, int fine, Grid &g,
                          cudaStream_t st) {
    Fail f{0, ""};
    if (!prepare_star(m, star, fine, g.setup, f)) return c->fail(f.code, "%s", f.msg.c_str());
    const StarSetup &s = g.setup;
    cudaError_t e;
    if ((e = g.alloc_points(s.nface)) != cudaSuccess) return c->cuda_fail(e, "grid allocation");
    g.ntiled = s.ntiled;
    if ((e = g.rings.ensure(s.rings.size())) != cudaSuccess) return c->cuda_fail(e, "rings");
    cudaMemcpyAsync(g.rings.p, s.rings.data(), s.rings.size() * sizeof(RingRec),
                    cudaMemcpyHostToDevice, st);
    GridParams gp{};
    gp.star = star;
    gp.roche = star == kStar1 ? m.roche1 : m.roche2;
    gp.npole = m.npole;
    gp.nrings = (int32_t)s.rings.size();
    gp.nhalf = s.nhalf;
    gp.q = m.q;
    gp.spin = star == kStar1 ? m.spin1 : m.spin2;
    gp.rref = star == kStar1 ? s.rref1 : s.rref2;
    gp.pref = star == kStar1 ? s.pref1 : s.pref2;
    gp.acc = m.delta_phase / 10.;
    gp.gref = s.gref;
    gp.rad_sphere = star == kStar1 ? s.r1 : s.r2;
    {
        StageScope t(c, LCG_STAGE_GRID);
        launch_grid(gp, g.rings.p, g.dev(), c->status.p, st);
    }
    if ((e = g.queue.ensure(s.nface)) || (e = g.counters.ensure(8)) ||
        (e = g.es.ensure(s.nface)) || (e = g.hits.ensure(s.nface)))
        return c->cuda_fail(e, "queue");
    EclParams ep{};
    ep.comp_star = star == kStar1 ? kStar2 : kStar1;
    ep.comp_roche = star == kStar1 ? m.roche2 : m.roche1;
    ep.q = m.q;
    ep.comp_spin = star == kStar1 ? m.spin2 : m.spin1;
    ep.comp_rref = star == kStar1 ? s.rref2 : s.rref1;
    ep.comp_pref = star == kStar1 ? s.pref2 : s.pref1;
    ep.comp_r = star == kStar1 ? s.r2 : s.r1;
    const double ri = deg2rad(m.iangle);
    ep.cosi = cos(ri);
    ep.sini = sin(ri);
    ep.delta = m.delta_phase;
    set_ecl_screen(ep, c->precision == LCG_PREC_MIXED, star == kStar1 ? s.r1 : s.r2);
    {
        StageScope t(c, LCG_STAGE_ECLIPSE);
        launch_eclipse(ep, s.eclipse, g.dev(), g.queue.p, g.counters.p, g.es.p, g.hits.p,
                       c->status.p, c->nsm, c->eclipse_warp, st);
    }
    return LCG_OK;
}

// Fast mixed-sweep records apply without beaming or lensing and with
// mucrit <= 0, where the reference's masks reduce to mu > 0.
FastCoef fast_coef(const lcg_model &m, int star, int mixed) {
    FastCoef f{};
    const double beam = star == kStar1 ? m.beam_factor1 : m.beam_factor2;
    const double mucrit = star == kStar1 ? m.mucrit1 : m.mucrit2;
    const bool glens = star == kStar2 && m.glens1;
    f.on = mixed && beam == 0.0 && !glens && mucrit <= 0.0;
    f.ltype = star == kStar1 ? m.limb1 : m.limb2;
    f.cosi = cos(deg2rad(m.iangle));
    const double *c = star == kStar1 ? m.ldc1 : m.ldc2;
    f.p[0] = 1.0 - (c[0] + c[1] + c[2] + c[3]);
    if (f.ltype == LCG_LIMB_CLARET) {
        for (int k = 0; k < 4; k++) f.p[k + 1] = c[k];
    } else {  // 1 - sum_k c_k (1 - mu)^k in powers of mu
        f.p[1] = c[0] + 2. * c[1] + 3. * c[2] + 4. * c[3];
        f.p[2] = -(c[1] + 3. * c[2] + 6. * c[3]);
        f.p[3] = c[2] + 4. * c[3];
        f.p[4] = -c[3];
    }
    return f;
}

// side: run on side[0] with its own partition scratch (star 2, concurrent
// order); otherwise on the context's stream.
lcg_status flatten(lcg_ctx *c, Grid &g, int need_pos, const FastCoef &fc, bool side = false) {
    const int mixed = c->precision == LCG_PREC_MIXED;
    cudaError_t e;
    if ((e = g.alloc_flat(mixed, need_pos, fc.on)) != cudaSuccess)
        return c->cuda_fail(e, "flat grid");
    g.fast = fc.on;
    DBuf<int32_t> &bc = side ? c->blockcnt2 : c->blockcnt;
    if ((e = bc.ensure(2 * ((g.n + 1023) / 1024) + 1)) != cudaSuccess)
        return c->cuda_fail(e, "partition");
    StageScope t(c, LCG_STAGE_FLATTEN);
    launch_flatten(g.dev(), g.flat(), bc.p, mixed, need_pos, fc, c->status.p,
                   side ? c->side[0] : c->stream);
    return LCG_OK;
}

// Unweighted single-phase flux sum of one flattened grid, spin = 1 as in
// comp_star1 / comp_star2 (comp_light.cpp:225-315).
lcg_status sweep_one(lcg_ctx *c, const lcg_model &m, Grid &g, int star, double phase,
                     double cosi, double sini, double rlens1, double &sum) {
    const V3 e = set_earth(cosi, sini, phase);
    double v[4] = {e.x, e.y, e.z, phase - floor(phase)};
    cudaError_t err;
    if ((err = c->pex.ensure(1)) || (err = c->pey.ensure(1)) || (err = c->pez.ensure(1)) ||
        (err = c->pphin.ensure(1)) || (err = c->pef.ensure(1)) || (err = c->ppfx.ensure(1)))
        return c->cuda_fail(err, "phases");
    cudaMemcpyAsync(c->pex.p, &v[0], 8, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->pey.p, &v[1], 8, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->pez.p, &v[2], 8, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->pphin.p, &v[3], 8, cudaMemcpyHostToDevice, c->stream);
    PhaseDev ph{c->pex.p, c->pey.p, c->pez.p, c->pphin.p, nullptr, nullptr, c->pef.p, nullptr, 1,
                c->ppfx.p};
    const int mixed = c->precision == LCG_PREC_MIXED;
    if (mixed) launch_pack_phases(ph, c->stream);
    FluxPlan plan = plan_flux(mixed, g.fast, g.n, 1, c->nsm);
    if ((err = c->part1f.ensure((size_t)std::max<int64_t>(plan.nchunk, 1) * 4)))
        return c->cuda_fail(err, "partials");
    FluxConsts k = flux_consts(m, star, 1.0, rlens1);
    launch_flux(mixed, star, k, g.flat(), ph, plan, c->part1f.p, 4, c->status.p, c->stream);
    if (g.disc)
        launch_flux_ragged(star, k, g.flat(), g.dev(), ph, plan.chunk, plan.nchunk,
                           c->part1f.p, 4, c->stream);
    std::vector<double> col((size_t)std::max<int64_t>(plan.nchunk, 1));
    if (plan.nchunk)
        cudaMemcpy2DAsync(col.data(), 8, c->part1f.p, 4 * 8, 8, (size_t)plan.nchunk,
                          cudaMemcpyDeviceToHost, c->stream);
    if ((err = cudaStreamSynchronize(c->stream))) return c->cuda_fail(err, "sweep");
    sum = 0.0;
    for (int64_t b = 0; b < plan.nchunk; b++) sum += col[(size_t)b];
    return LCG_OK;
}

// Grid-switching scale factors (light_curve_comp.cpp:214-254).
lcg_status ginterp_scales(lcg_ctx *c, const lcg_model &m, double rlens1) {
    Ginterp &gi = c->gi;
    gi = Ginterp{m.phase1, m.phase2, 1., 1., 1., 1.};
    const double ri = deg2rad(m.iangle), cosi = cos(ri), sini = sin(ri);
    auto comp = [&](int star, double phase, double &out) -> lcg_status {
        const int t = gi_type(gi, phase);
        Grid &g = star == kStar1 ? (t == 1 ? c->g1f : (c->copy1 ? c->g1f : c->g1c))
                                 : (t == 3 ? c->g2f : (c->copy2 ? c->g2f : c->g2c));
        double s = 0.;
        lcg_status rc = sweep_one(c, m, g, star, phase, cosi, sini, rlens1, s);
        const double sc = star == kStar1 ? gi_scale1(gi, phase) : gi_scale2(gi, phase);
        out = 1.0 * sc * s / 1;
        return rc;
    };
    lcg_status rc;
    double ff, fc;
    if (m.nlat1c != m.nlat1f) {
        if ((rc = comp(kStar1, 0.9999999999 * m.phase1, ff)) ||
            (rc = comp(kStar1, 1.0000000001 * m.phase1, fc)))
            return rc;
        gi.scale11 = ff / fc;
        if ((rc = comp(kStar1, 1. - 0.9999999999 * m.phase1, ff)) ||
            (rc = comp(kStar1, 1. - 1.0000000001 * m.phase1, fc)))
            return rc;
        gi.scale12 = ff / fc;
    }
    if (!c->copy2) {
        if ((rc = comp(kStar2, 1 - 1.0000000001 * m.phase2, ff)) ||
            (rc = comp(kStar2, 1 - 0.9999999999 * m.phase2, fc)))
            return rc;
        gi.scale21 = ff / fc;
        if ((rc = comp(kStar2, 1.0000000001 * m.phase2, ff)) ||
            (rc = comp(kStar2, 0.9999999999 * m.phase2, fc)))
            return rc;
        gi.scale22 = ff / fc;
    }
    return LCG_OK;
}

lcg_status check_model(lcg_ctx *c, const lcg_model *m) {
    if (!m) return c->fail(LCG_E_INVALID, "null model");
    if (m->add_disc && m->nrad < 1)
        return c->fail(LCG_E_INVALID, "nrad = %d: the disc needs at least one radius", m->nrad);
    if (!(m->q > 0.))
        return c->fail(LCG_E_INVALID, "Roche::xl12(double, double): q = %f <= 0.", m->q);
    if (!(m->delta_phase > 0.))
        return c->fail(LCG_E_INVALID, "delta_phase = %g must be positive", m->delta_phase);
    if (m->nlat1f <= 0 || m->nlat2f <= 0 || m->nlat1c <= 0 || m->nlat2c <= 0)
        return c->fail(LCG_E_INVALID, "the numbers of latitude strips must be positive");
    return LCG_OK;
}

lcg_status finish_status(lcg_ctx *c) {
    cudaError_t le = cudaGetLastError();
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (le != cudaSuccess) {
        c->collect_timers();
        c->has_geom = c->has_cont = false;
        return c->cuda_fail(le, "kernel launch");
    }
    c->collect_timers();
    if (e != cudaSuccess) return c->cuda_fail(e, "stream");
    DevStatus st{};
    e = cudaMemcpy(&st, c->status.p, sizeof st, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return c->cuda_fail(e, "status");
    if (st.code) {
        c->has_geom = c->has_cont = false;
        if (st.face < 0)  // a disc, rim or spot element (components.cu)
            return c->fail(st.code, "%s (disc, rim or spot element %d)",
                           st.code == 3 ? "disc or star eclipse of a component failed"
                                        : status_text(st.code),
                           -st.face - 1);
        return c->fail(st.code, "%s (face %d)", status_text(st.code), st.face);
    }
    return LCG_OK;
}

}  // namespace eng
}  // namespace lcg

void lcg::count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void lcg::count_launches(int64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// ---- C ABI --------------------------------------------------------------------

// Best of five timed launches of an FMA-chain probe on the context's stream,
// after one warm-up: TFLOP/s (2 FLOP per FMA).
template <class Launch>
lcg_status measure_peak(lcg_ctx *c, double *tflops, Launch launch) {
    if (!c || !tflops) return LCG_E_INVALID;
    cudaSetDevice(c->device);
    void *sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, 16);
    if (e) return c->cuda_fail(e, "probe");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = c->nsm * 8, iters = 4096;
    double gflop = 0.;
    launch(sink, blocks, iters, &gflop, c->stream);  // warm-up
    double best = 0.;
    for (int r = 0; r < 5; r++) {
        cudaEventRecord(a, c->stream);
        launch(sink, blocks, iters, &gflop, c->stream);
        cudaEventRecord(b, c->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        const double t = gflop / (ms * 1e-3) * 1e-3;
        if (t > best) best = t;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    e = cudaGetLastError();
    if (e) return c->cuda_fail(e, "probe");
    *tflops = best;
    return LCG_OK;
}

extern "C" {

void lcg_default_options(lcg_options *opt) {
    if (!opt) return;
    memset(opt, 0, sizeof *opt);
    opt->device = 0;
    opt->precision = LCG_PREC_MIXED;
}

int32_t lcg_abi_version(void) { return LCG_ABI_VERSION; }

lcg_status lcg_create(lcg_ctx **out, const lcg_options *opt) {
    if (!out) return LCG_E_INVALID;
    *out = nullptr;
    lcg_options o;
    lcg_default_options(&o);
    if (opt) o = *opt;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
        return LCG_E_CUDA;
    }
    if (o.device < 0 || o.device >= ndev) {
        g_create_error = "device ordinal out of range";
        return LCG_E_INVALID;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, o.device);
    if (prop.major < 10) {
        g_create_error = std::string("device ") + prop.name + " is not sm_100 class";
        return LCG_E_CUDA;
    }
    if ((e = cudaSetDevice(o.device)) != cudaSuccess) {
        g_create_error = cudaGetErrorString(e);
        return LCG_E_CUDA;
    }
    lcg_ctx *c = new lcg_ctx();
    c->device = o.device;
    c->precision = o.precision == LCG_PREC_FP64 ? LCG_PREC_FP64 : LCG_PREC_MIXED;
    c->verbose = o.verbose;
    c->eclipse_warp = o.eclipse_warp;
    c->nsm = prop.multiProcessorCount;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->side[0], cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&c->side[1], cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_join[0], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_join[1], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&c->ev_phases, cudaEventDisableTiming)) != cudaSuccess ||
        (e = c->status.ensure(1)) != cudaSuccess || (e = c->counters.ensure(2)) != cudaSuccess ||
        (e = c->sfac.ensure(8)) != cudaSuccess || (e = c->out.ensure(4)) != cudaSuccess) {
        g_create_error = cudaGetErrorString(e);
        delete c;
        return LCG_E_CUDA;
    }
    *out = c;
    return LCG_OK;
}

void lcg_destroy(lcg_ctx *c) {
    if (!c) return;
    for (lcg_ctx *w : c->workers) lcg_destroy(w);
    c->workers.clear();
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->collect_timers();
    if (c->verbose > 0) {
        const char *names[LCG_NSTAGE] = {"grid", "eclipse", "continuum", "flatten",
                                         "phases", "flux", "reduce"};
        for (int s = 0; s < LCG_NSTAGE; s++)
            fprintf(stderr, "lcg stage %-9s %10.3f ms over %lld launches\n", names[s],
                    c->stage_ms[s], (long long)c->stage_n[s]);
    }
    Grid *gs[] = {&c->g1f, &c->g2f, &c->g1c, &c->g2c};
    for (Grid *g : gs) g->release();
    DBuf<double> *d[] = {&c->pex, &c->pey, &c->pez, &c->pphin, &c->pw1, &c->pw2, &c->part1f,
                         &c->part1c, &c->part2f, &c->part2c, &c->calc, &c->scratch, &c->sfac,
                         &c->out, &c->diag, &c->osum};
    for (auto *b : d) b->release();
    c->status.release(); c->queue.release(); c->counters.release(); c->blockcnt.release();
    c->blockcnt2.release();
    c->data.release(); c->off.release(); c->pef.release(); c->ppfx.release(); c->ptype.release();
    c->fdata.release(); c->fidx.release(); c->fcalc.release(); c->fout.release();
    c->elem.release(); c->epos.release(); c->drings.release(); c->csum.release();
    c->fcomp.release(); c->iwork.release();
    batch_release(c->batch);
    c->batch = nullptr;
    for (int k = 0; k < 2; k++)
        if (c->side[k]) {
            cudaStreamSynchronize(c->side[k]);
            cudaStreamDestroy(c->side[k]);
            cudaEventDestroy(c->ev_join[k]);
        }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_phases) cudaEventDestroy(c->ev_phases);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *lcg_last_error(const lcg_ctx *c) {
    return c ? c->err.c_str() : g_create_error.c_str();
}

void *lcg_stream(lcg_ctx *c) { return c ? (void *)c->stream : nullptr; }

void lcg_set_profiling(lcg_ctx *c, int32_t on) {
    if (c) c->profiling = on != 0;
}

void lcg_stage_times(lcg_ctx *c, double *ms, int64_t *launches, int32_t reset) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    c->collect_timers();
    for (int s = 0; s < LCG_NSTAGE; s++) {
        if (ms) ms[s] = c->stage_ms[s];
        if (launches) launches[s] = c->stage_n[s];
        if (reset) {
            c->stage_ms[s] = 0.;
            c->stage_n[s] = 0;
        }
    }
}

int64_t lcg_flux_elements(lcg_ctx *c, int32_t reset) {
    if (!c) return 0;
    int64_t v = c->flux_elements;
    if (reset) c->flux_elements = 0;
    return v;
}

lcg_status lcg_set_data(lcg_ctx *c, const lcg_datum *data, int32_t n) {
    if (!c) return LCG_E_INVALID;
    c->err.clear();
    if (!data) return c->fail(LCG_E_INVALID, "null argument");
    if (n < 1) return c->fail(LCG_E_INVALID, "light_curve_comp: no data points");
    cudaSetDevice(c->device);
    // per-point offsets of the sub-exposure entries and the time range used
    // by the polynomial factor (light_curve_comp.cpp:351-356)
    std::vector<int64_t> &off = c->h_off;
    off.resize((size_t)n + 1);
    off[0] = 0;
    double xmin = data[0].time, xmax = data[0].time;
    for (int i = 0; i < n; i++) {
        off[i + 1] = off[i] + (data[i].ndiv > 0 ? data[i].ndiv : 0);
        if (i > 0) {
            xmin = data[i].time > xmin ? xmin : data[i].time;
            xmax = data[i].time < xmax ? xmax : data[i].time;
        }
    }
    cudaError_t e;
    if ((e = c->data.ensure(n)) || (e = c->off.ensure(n + 1)))
        return c->cuda_fail(e, "data buffers");
    cudaMemcpyAsync(c->data.p, data, (size_t)n * sizeof(DatumRec), cudaMemcpyHostToDevice,
                    c->stream);
    c->h_data.assign(reinterpret_cast<const DatumRec *>(data),
                     reinterpret_cast<const DatumRec *>(data) + n);
    cudaMemcpyAsync(c->off.p, off.data(), (size_t)(n + 1) * sizeof(int64_t),
                    cudaMemcpyHostToDevice, c->stream);
    c->data_n = n;
    c->data_version++;
    c->data_nent = off[n];
    c->data_xmin = xmin;
    c->data_xmax = xmax;
    return LCG_OK;
}

lcg_status lcg_light_curve(lcg_ctx *c, const lcg_model *mp, const lcg_datum *data, int32_t n,
                           int32_t flags, double *sfac, double *calc, double *scalars) {
    if (!c) return LCG_E_INVALID;
    c->err.clear();
    lcg_status rc = check_model(c, mp);
    if (rc) return rc;
    if (!data || !calc || !sfac || !scalars) return c->fail(LCG_E_INVALID, "null argument");
    if ((rc = lcg_set_data(c, data, n))) return rc;
    return lcg_light_curve_resident(c, mp, flags, sfac, calc, scalars);
}

const double *lcg_device_calc(lcg_ctx *c) { return c ? c->calc.p : nullptr; }

lcg_status lcg_light_curve_fast(lcg_ctx *c, const lcg_model *mp, const lcg_datum *data,
                                int32_t n, int32_t flags, int32_t max_model_points, double *sfac,
                                double *calc, double *scalars) {
    if (!c) return LCG_E_INVALID;
    c->err.clear();
    if (n <= max_model_points)
        return lcg_light_curve(c, mp, data, n, flags, sfac, calc, scalars);
    if (!data || !calc || !sfac || !scalars) return c->fail(LCG_E_INVALID, "null argument");
    if (max_model_points < 2)
        return c->fail(LCG_E_INVALID, "light_curve_comp_fast: max_model_points must be >= 2");
    // points uniform in index, both ends included (light_curve_comp_fast.cpp:32-37)
    const int32_t m = max_model_points;
    std::vector<int64_t> idx((size_t)m);
    std::vector<lcg_datum> sub((size_t)m);
    for (int32_t i = 0; i < m; i++) {
        idx[(size_t)i] = (int64_t)((size_t)i * (size_t)(n - 1) / (size_t)(m - 1));
        sub[(size_t)i] = data[idx[(size_t)i]];
    }
    lcg_status rc;
    if ((rc = lcg_set_data(c, sub.data(), m))) return rc;
    if ((rc = lcg_light_curve_resident(c, mp, flags, sfac, nullptr, scalars))) return rc;
    cudaError_t e;
    if ((e = c->fdata.ensure(n)) || (e = c->fidx.ensure(m)) || (e = c->fcalc.ensure(n)) ||
        (e = c->fout.ensure(2)))
        return c->cuda_fail(e, "interpolation buffers");
    cudaMemcpyAsync(c->fdata.p, data, (size_t)n * sizeof(DatumRec), cudaMemcpyHostToDevice,
                    c->stream);
    cudaMemcpyAsync(c->fidx.p, idx.data(), (size_t)m * sizeof(int64_t), cudaMemcpyHostToDevice,
                    c->stream);
    const int32_t rdata = (flags & LCG_FLAG_RDATA) != 0;
    launch_interp(c->fdata.p, n, c->fidx.p, m, c->calc.p, c->fcalc.p, rdata, c->fout.p,
                  c->stream);
    double out[2] = {0., 0.};
    cudaMemcpyAsync(calc, c->fcalc.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                    c->stream);
    if (rdata)
        cudaMemcpyAsync(out, c->fout.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    if ((rc = finish_status(c))) return rc;
    if (rdata) {
        scalars[LCG_OUT_CHISQ] = out[0];
        scalars[LCG_OUT_WNOK] = out[1];
    }
    return LCG_OK;
}

lcg_status lcg_light_curve_resident(lcg_ctx *c, const lcg_model *mp, int32_t flags, double *sfac,
                                    double *calc, double *scalars) {
    if (!c) return LCG_E_INVALID;
    c->err.clear();
    lcg_status rc = check_model(c, mp);
    if (rc) return rc;
    if (!sfac || !scalars) return c->fail(LCG_E_INVALID, "null argument");
    if (c->data_n < 1) return c->fail(LCG_E_INVALID, "no data: call lcg_set_data first");
    cudaSetDevice(c->device);
    const int32_t n = c->data_n;
    const lcg_model &m = *mp;
    const int mixed = c->precision == LCG_PREC_MIXED;
    cudaError_t e;

    // light_curve_comp.cpp:130-154
    double r1, r2;
    get_r1r2(m, r1, r2);
    const double xl2 = xl12(m.q, m.spin2);
    if (xl2 < 0)
        return c->fail(LCG_E_NOCONVERGE, "Roche::xl12(double,double): exceeded maximum iterations");
    const double rl2 = 1. - xl2;
    if (r2 < 0) r2 = rl2;
    else if (r2 > rl2)
        return c->fail(LCG_E_LOBE,
                       "light_curve_comp: the secondary star is larger than its Roche lobe!");
    double rlens1 = 0.;
    if (m.glens1) {
        double gm = pow(1000. * m.velocity_scale, 3) * m.tperiod * kDay / kTwoPi;
        double a = pow(gm / (kTwoPi / kDay / m.tperiod * kTwoPi / kDay / m.tperiod), 1. / 3.);
        rlens1 = 4. * gm / (1. + m.q) / a / (kC * kC);
    }
    const bool need_pos = m.beam_factor1 != 0. || m.beam_factor2 != 0. || m.glens1;
    // disc / rim / bright spot; an opaque disc also eclipses the stars;
    // iscale fits one scale factor per component (light_curve_comp.cpp:272-414)
    const bool comps = m.add_disc || m.add_spot;
    const bool opaque = m.add_disc && m.opaque;
    const bool iscale = m.iscale != 0;
    cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream);
    cudaEventRecord(c->ev_fork, c->stream);  // side-stream work starts here

    // geometry (GeomKey)
    const bool geom_hit = c->has_geom && !(flags & LCG_FLAG_NO_CACHE) && same_geometry(c->key, m);
    if (!geom_hit) {
        c->has_geom = c->has_cont = false;
        // star 2's grids on side[0], beside star 1's (joined before the continuum)
        cudaStreamWaitEvent(c->side[0], c->ev_fork, 0);
        if ((rc = build_geometry(c, m, kStar1, 1, c->g1f, c->stream))) return rc;
        if ((rc = build_geometry(c, m, kStar2, 1, c->g2f, c->side[0]))) return rc;
        c->copy1 = (m.nlat1f == m.nlat1c);
        c->copy2 = (m.nlat2f == m.nlat2c) &&
                   (!m.npole || r1 >= r2 || (m.nlatfill == 0 && m.nlngfill == 0));
        if (!c->copy1 && (rc = build_geometry(c, m, kStar1, 0, c->g1c, c->stream))) return rc;
        if (!c->copy2 && (rc = build_geometry(c, m, kStar2, 0, c->g2c, c->side[0]))) return rc;
    }
    // concurrent order (see lcg_ctx::side): star 2 stays on side[0] up to its
    // sweep; otherwise the streams join here
    const bool conc = c->copy1 && c->copy2 && !opaque && !c->profiling;
    if (conc) {
        cudaStreamWaitEvent(c->side[0], c->ev_fork, 0);  // also when the grids were reused
    } else if (!geom_hit) {
        cudaEventRecord(c->ev_join[0], c->side[0]);
        cudaStreamWaitEvent(c->stream, c->ev_join[0], 0);
    }
    Grid &g1f = c->g1f, &g2f = c->g2f;
    Grid &g1c = c->copy1 ? c->g1f : c->g1c;
    Grid &g2c = c->copy2 ? c->g2f : c->g2c;
    if (flags & LCG_FLAG_INFO) {
        fprintf(stderr, "Number of points for star 1 (fine) = %lld\n", (long long)g1f.n);
        fprintf(stderr, "Number of points for star 2 (fine) = %lld\n", (long long)g2f.n);
        fprintf(stderr, "Number of points for star 1 (coarse) = %lld\n", (long long)g1c.n);
        fprintf(stderr, "Number of points for star 2 (coarse) = %lld\n", (long long)g2c.n);
    }

    // disc, rim and bright-spot elements (set_disc_grid, set_disc_edge,
    // set_bright_spot_grid with their continua), rebuilt every call on the
    // side stream, beside the star grids; joined before the component sums
    int32_t ncomp = 0;
    if (comps) {

        std::vector<DiscRing> rings;
        Fail f{0, ""};
        if (!comp_setup(m, c->comp, rings, f)) return c->fail(f.code, "%s", f.msg.c_str());
        ncomp = c->comp.nd + c->comp.ne + c->comp.ns;
        if ((e = c->elem.ensure(ncomp)) || (e = c->epos.ensure(ncomp)) ||
            (e = c->drings.ensure(rings.size())))
            return c->cuda_fail(e, "component elements");
        cudaStreamWaitEvent(c->side[1], c->ev_fork, 0);
        if (!rings.empty())
            cudaMemcpyAsync(c->drings.p, rings.data(), rings.size() * sizeof(DiscRing),
                            cudaMemcpyHostToDevice, c->side[1]);
        c->comp.rings = c->drings.p;
        launch_components(c->comp, c->elem.p, c->epos.p, c->status.p, c->side[1]);
        cudaEventRecord(c->ev_join[1], c->side[1]);
        if ((flags & LCG_FLAG_INFO) && m.add_disc)
            fprintf(stderr, "Number of points for the disc = %d\n", c->comp.nd);
    }

    // continuum (ContKey) + FlatGrid
    // (opaque discs bypass the reuse, light_curve_comp.cpp:163)
    const bool cont_hit = c->has_cont && geom_hit && same_continuum(c->key, m) &&
                          c->cached_mixed_pos == (int)need_pos && !opaque && !c->g1f.disc &&
                          !c->g2f.disc && !c->g1c.disc && !c->g2c.disc;
    if (!cont_hit) {
        Grid *gl[] = {&c->g1f, &c->g2f, &c->g1c, &c->g2c};
        const int stars[] = {kStar1, kStar2, kStar1, kStar2};
        const bool use[] = {true, true, !c->copy1, !c->copy2};
        for (int k = 0; k < 4; k++) {
            gl[k]->disc = false;
            if (!use[k]) continue;
            ContParams cp = continuum_params(m, stars[k]);
            cp.fp32 = c->precision == LCG_PREC_MIXED;
            const bool on_side = conc && k == 1;  // star 2's fine grid
            {
                StageScope t(c, LCG_STAGE_CONTINUUM);
                launch_continuum(cp, gl[k]->dev(), on_side ? c->side[0] : c->stream);
            }
            // (with an opaque disc the grids are flattened below, after the
            // disc's ranges; first without them when the Ginterp scales need it)
            if (!opaque || !c->copy1 || !c->copy2)
                if ((rc = flatten(c, *gl[k], need_pos,
                                  fast_coef(m, stars[k], c->precision == LCG_PREC_MIXED),
                                  on_side)))
                    return rc;
        }
        c->gi = Ginterp{m.phase1, m.phase2, 1., 1., 1., 1.};
        if (!c->copy1 || !c->copy2) {
            if ((rc = ginterp_scales(c, m, rlens1))) return rc;
        }
        if (opaque) {
            // the disc's ranges join the stars' after the Ginterp scales were
            // taken (light_curve_comp.cpp:279-323, 327-333); rdisc1 defaults
            // to r1 as given, before any lobe filling
            double r1g, r2g;
            get_r1r2(m, r1g, r2g);
            const DiscGeom dg{sin(kPi / 180. * m.iangle), cos(kPi / 180. * m.iangle),
                              m.rdisc1 > 0. ? m.rdisc1 : r1g,
                              m.rdisc2 > 0. ? m.rdisc2 : m.radius_spot, m.beta_disc,
                              m.height_disc};
            for (int k = 0; k < 4; k++) {
                if (!use[k]) continue;
                Grid &g = *gl[k];
                if ((e = g.ndx.ensure(g.n)) || (e = g.xr.ensure(kDiscRanges * g.n)))
                    return c->cuda_fail(e, "disc eclipses");
                {
                    StageScope t(c, LCG_STAGE_ECLIPSE);
                    launch_disc_faces(dg, g.dev(), g.ndx.p, g.xr.p, c->status.p, c->stream);
                }
                g.disc = true;
                if ((rc = flatten(c, g, need_pos,
                                  fast_coef(m, stars[k], c->precision == LCG_PREC_MIXED))))
                    return rc;
            }
        }
        c->cached_mixed_pos = (int)need_pos;
    }

    // phase entries (light_curve_comp.cpp:358-455) over the resident points
    const int64_t nent = c->data_nent;
    const double xmin = c->data_xmin, xmax = c->data_xmax;
    const bool diag = (flags & LCG_FLAG_DIAGNOSTICS) != 0;
    const int64_t nall = nent + (diag ? 1 : 0);  // + the phase-0.5 entry of wdwarf
    const int64_t ldp = ((nall + 3) / 4) * 4;
    if ((e = c->pex.ensure(nall)) || (e = c->pey.ensure(nall)) || (e = c->pez.ensure(nall)) ||
        (e = c->pphin.ensure(nall)) || (e = c->pw1.ensure(nall)) || (e = c->pw2.ensure(nall)) ||
        (e = c->pef.ensure(nall)) || (e = c->ppfx.ensure(nall)) || (e = c->ptype.ensure(nall)) || (e = c->calc.ensure(n)) ||
        (e = c->scratch.ensure(3 * (size_t)n)))
        return c->cuda_fail(e, "phase buffers");
    PhaseDev ph{c->pex.p, c->pey.p, c->pez.p, c->pphin.p, c->pw1.p, c->pw2.p,
                c->pef.p, c->ptype.p, nall, c->ppfx.p};
    const double ri = deg2rad(m.iangle);
    const double cosi = cos(ri), sini = sin(ri);
    PhaseParams pp{};
    pp.t0 = m.t0; pp.period = m.period; pp.pdot = m.pdot; pp.deltat = m.deltat;
    pp.slope = m.slope; pp.quad = m.quad; pp.cube = m.cube;
    pp.middle = (xmin + xmax) / 2.;
    pp.range = (xmax - xmin) / 2.;
    pp.cosi = cosi; pp.sini = sini;
    pp.gi = c->gi;
    {
        StageScope t(c, LCG_STAGE_PHASES);
        launch_phases(pp, c->data.p, c->off.p, n, ph, c->stream);
        if (diag) {
            // comp_star1_flat at phase 0.5 (light_curve_comp.cpp:504-508)
            const V3 ew = set_earth(cosi, sini, 0.5);
            double v[4] = {ew.x, ew.y, ew.z, 0.5};
            cudaMemcpyAsync(c->pex.p + nent, &v[0], 8, cudaMemcpyHostToDevice, c->stream);
            cudaMemcpyAsync(c->pey.p + nent, &v[1], 8, cudaMemcpyHostToDevice, c->stream);
            cudaMemcpyAsync(c->pez.p + nent, &v[2], 8, cudaMemcpyHostToDevice, c->stream);
            cudaMemcpyAsync(c->pphin.p + nent, &v[3], 8, cudaMemcpyHostToDevice, c->stream);
            PhaseDev one = ph;
            one.ex += nent; one.ey += nent; one.ez += nent; one.phin += nent; one.ef += nent;
            one.pfx += nent;
            one.nent = 1;
            launch_pack_phases(one, c->stream);
        }
    }
    if (conc) {
        cudaEventRecord(c->ev_phases, c->stream);
        cudaStreamWaitEvent(c->side[0], c->ev_phases, 0);
    }

    // flux sweeps (light_curve_comp.cpp:457-473)
    struct Sweep {
        Grid *g;
        int star;
        double spin;
        DBuf<double> *part;
        int64_t nent;
        FluxPlan plan;
    };
    // iscale's components are comp_star1_flat / comp_star2_flat sums, which
    // take spin 1 in the beaming (comp_light_flat.cpp:538-602)
    const double spin1 = iscale ? 1.0 : m.spin1, spin2 = iscale ? 1.0 : m.spin2;
    Sweep sw[4] = {{&g1f, kStar1, spin1, &c->part1f, nall, {}},
                   {&g1c, kStar1, spin1, &c->part1c, nall, {}},
                   {&g2f, kStar2, spin2, &c->part2f, nent, {}},
                   {&g2c, kStar2, spin2, &c->part2c, nent, {}}};
    const bool use_sw[4] = {true, !c->copy1, true, !c->copy2};
    for (int k = 0; k < 4; k++) {
        if (!use_sw[k]) continue;
        Sweep &s = sw[k];
        s.plan = plan_flux(mixed, s.g->fast, s.g->n, s.nent, c->nsm);
        if ((e = s.part->ensure((size_t)std::max<int64_t>(s.plan.nchunk, 1) * ldp)))
            return c->cuda_fail(e, "flux partials");
        PhaseDev phk = ph;
        phk.nent = s.nent;
        FluxConsts kc = flux_consts(m, s.star, s.spin, rlens1);
        StageScope t(c, LCG_STAGE_FLUX);
        cudaStream_t fs = (conc && k == 2) ? c->side[0] : c->stream;  // star 2's fine sweep
        launch_flux(mixed, s.star, kc, s.g->flat(), phk, s.plan, s.part->p, ldp, c->status.p,
                    fs);
        if (s.g->disc)
            launch_flux_ragged(s.star, kc, s.g->flat(), s.g->dev(), phk, s.plan.chunk,
                               s.plan.nchunk, s.part->p, ldp, fs);
        c->flux_elements += s.g->n * s.nent;
    }
    if (conc) {
        cudaEventRecord(c->ev_join[0], c->side[0]);
        cudaStreamWaitEvent(c->stream, c->ev_join[0], 0);
    }
    if (comps) {
        if ((e = c->csum.ensure(3 * (size_t)ldp + (size_t)comp_sums_scratch(ncomp, ldp))))
            return c->cuda_fail(e, "component sums");
        PhaseDev phc = ph;
        phc.nent = nent;
        cudaStreamWaitEvent(c->stream, c->ev_join[1], 0);
        StageScope t(c, LCG_STAGE_FLUX);
        launch_comp_sums(c->elem.p, c->comp.nd, c->comp.ne, ncomp, m.lin_limb_disc,
                         m.quad_limb_disc, phc, c->csum.p + 3 * ldp, c->csum.p, ldp, c->stream);
    }

    // scatter, third light, scale, chi**2
    {
        ScatterParams sp{};
        sp.copy1 = c->copy1;
        sp.copy2 = c->copy2;
        sp.third = m.third;
        sp.csum = comps ? c->csum.p : nullptr;
        sp.ldc = ldp;
        sp.pp = pp;
        if (iscale) {
            if ((e = c->fcomp.ensure(5 * (size_t)n)) || (e = c->iwork.ensure(6 * (size_t)n)))
                return c->cuda_fail(e, "iscale components");
            sp.fcomp = c->fcomp.p;
        }
        if ((e = c->osum.ensure(4 * (size_t)ldp))) return c->cuda_fail(e, "entry sums");
        ReduceParams rp{};
        rp.ldp = ldp;
        for (int k = 0; k < 4; k++) {
            rp.part[k] = use_sw[k] ? sw[k].part->p : nullptr;
            rp.nchunk[k] = use_sw[k] ? sw[k].plan.nchunk : 0;
            rp.nent[k] = use_sw[k] ? sw[k].nent : 0;
            rp.osum[k] = c->osum.p + k * ldp;
        }
        StageScope t(c, LCG_STAGE_REDUCE);
        launch_scatter(sp, rp, ph, c->data.p, c->off.p, n, c->calc.p, c->stream);
        cudaMemcpyAsync(c->sfac.p, sfac, 5 * sizeof(double), cudaMemcpyHostToDevice, c->stream);
        if (iscale)
            launch_iscale(flags & 3, m.t2 > 0 ? 5 : 4, c->data.p, n, c->fcomp.p, c->iwork.p,
                          c->calc.p, c->sfac.p, c->out.p, c->stream);
        else
            launch_finalize(flags & 3, c->data.p, n, c->calc.p, c->sfac.p, c->out.p, c->stream);
    }
    double hout[4] = {0, 0, 0, 0};
    if (calc)
        cudaMemcpyAsync(calc, c->calc.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost,
                        c->stream);
    cudaMemcpyAsync(sfac, c->sfac.p, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(hout, c->out.p, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream);

    // diagnostics: wdwarf's phase-0.5 sum, logg / rv block sums
    double wsum = 0.;
    if (diag) {
        // star1c aliases star1f when copy1 (light_curve_comp.cpp:192-195)
        const bool fine = c->copy1 || gi_type(c->gi, 0.5) == 1;
        cudaMemcpyAsync(&wsum, c->osum.p + (fine ? 0 : 1) * ldp + nent, sizeof(double),
                        cudaMemcpyDeviceToHost, c->stream);
        const int64_t nb1 = (g1f.n + 8191) / 8192, nb2 = (g2f.n + 8191) / 8192;
        if ((e = c->diag.ensure(4 * (size_t)(nb1 + nb2))))
            return c->cuda_fail(e, "diagnostics");
        launch_diagnostics(kStar1, g1f.dev(), c->diag.p, c->stream);
        launch_diagnostics(kStar2, g2f.dev(), c->diag.p + 4 * nb1, c->stream);
        c->h_diag.resize(4 * (size_t)(nb1 + nb2));
        cudaMemcpyAsync(c->h_diag.data(), c->diag.p, c->h_diag.size() * sizeof(double),
                        cudaMemcpyDeviceToHost, c->stream);
    }
    if ((rc = finish_status(c))) return rc;
    c->key = m;
    c->has_geom = c->has_cont = true;
    if (diag && m.beam_factor1 != 0. && m.spin1 != 1.0 && !iscale) {
        // wdwarf is comp_star1_flat at phase 0.5, which beams with spin 1
        // (light_curve_comp.cpp:504-508); the sweeps above used spin1
        const bool fine = c->copy1 || gi_type(c->gi, 0.5) == 1;
        if ((rc = sweep_one(c, m, fine ? g1f : g1c, kStar1, 0.5, cosi, sini, rlens1, wsum)))
            return rc;
    }

    if (hout[2] != 0.) {
        scalars[LCG_OUT_CHISQ] = hout[0];
        scalars[LCG_OUT_WNOK] = hout[1];
    }
    const double sc = sfac[0];
    if (diag) {
        double wd = 1.0 * gi_scale1(c->gi, 0.5) * wsum;
        scalars[LCG_OUT_WDWARF] = wd / 1 * sc;
        // comp_gravity1/2 (comp_gravity.cpp:20-155), comp_radius1/2 (comp_radius.cpp)
        const int64_t nb1 = (g1f.n + 8191) / 8192, nb2 = (g2f.n + 8191) / 8192;
        double gm = pow(1000. * m.velocity_scale, 3) * m.tperiod * kDay / kTwoPi;
        double a = pow(gm / sq(kTwoPi / kDay / m.tperiod), 1. / 3.);
        double gscale = 100 * gm / sq(a);
        double rr1, rr2;
        get_r1r2(m, rr1, rr2);
        const double rl1 = xl12(m.q, m.spin1), rlb2 = 1. - xl12(m.q, m.spin2);
        if (m.r2 < 0) rr2 = rlb2;
        const double ACC = m.delta_phase / 10.;
        for (int star = 0; star < 2; star++) {
            const double *b = c->h_diag.data() + (star == 0 ? 0 : 4 * nb1);
            const int64_t nb = star == 0 ? nb1 : nb2;
            double sumfg = 0., sumf = 0, sumsa = 0., sumvol = 0.;
            for (int64_t k = 0; k < nb; k++) {
                sumfg += b[4 * k];
                sumf += b[4 * k + 1];
                sumsa += b[4 * k + 2];
                sumvol += b[4 * k + 3];
            }
            double gref;
            const bool roche = star == 0 ? m.roche1 : m.roche2;
            if (roche) {
                double rref, pref, ffac = star == 0 ? rr1 / rl1 : rr2 / rlb2, rad;
                ref_sphere(star, m.q, star == 0 ? m.spin1 : m.spin2, ffac, rref, pref);
                V3 posn, dvec;
                face_scalar(star, m.q, star == 0 ? m.spin1 : m.spin2,
                            star == 0 ? v3(-1., 0., 0.) : v3(1., 0., 0.), rref, pref, ACC, posn,
                            dvec, rad, gref);
                gref *= gscale;
            } else {
                gref = star == 0 ? gscale / (1 + m.q) / sq(rr1)
                                 : gscale * m.q / (1 + m.q) / sq(rr2);
            }
            scalars[star == 0 ? LCG_OUT_LOGG1 : LCG_OUT_LOGG2] =
                ((gref > 0) & (sumfg > 0) & (sumf > 0)) ? log10(gref * sumfg / sumf) : 0.;
            scalars[star == 0 ? LCG_OUT_RV1 : LCG_OUT_RV2] = pow(sumvol / sumsa, 1. / 3.);
        }
    } else {
        scalars[LCG_OUT_WDWARF] = 0.0 * sc;
        scalars[LCG_OUT_LOGG1] = scalars[LCG_OUT_LOGG2] = 0.0;
        scalars[LCG_OUT_RV1] = scalars[LCG_OUT_RV2] = 0.0;
    }
    return LCG_OK;
}

lcg_status lcg_light_curve_batch(lcg_ctx *c, const lcg_model *models, int32_t nmodels,
                                 const lcg_datum *data, int32_t n, int32_t flags, double *sfac,
                                 double *calc, double *chisq, double *wnok, int32_t *status) {
    if (!c) return LCG_E_INVALID;
    if (!models || nmodels < 0 || !sfac || !calc || !status)
        return c->fail(LCG_E_INVALID, "null argument");
    lcg_status rs = lcg_set_data(c, data, n);
    if (rs) return rs;
    return lcg_light_curve_batch_resident(c, models, nmodels, flags, sfac, calc, chisq, wnok,
                                          status);
}

lcg_status lcg_star_face_count(lcg_ctx *c, const lcg_model *m, int32_t star, int32_t fine,
                               int32_t *nface) {
    if (!c) return LCG_E_INVALID;
    lcg_status rc = check_model(c, m);
    if (rc) return rc;
    if (!nface || (star != kStar1 && star != kStar2)) return c->fail(LCG_E_INVALID, "bad argument");
    StarSetup s;
    Fail f{0, ""};
    if (!prepare_star(*m, star, fine, s, f)) return c->fail(f.code, "%s", f.msg.c_str());
    *nface = s.nface;
    return LCG_OK;
}

lcg_status lcg_components(lcg_ctx *c, const lcg_model *m, int32_t which, int32_t cap,
                          int32_t *n, double *posn, double *dirn, float *area, float *flux,
                          int32_t *nr, double *rin, double *rout) {
    if (!c) return LCG_E_INVALID;
    c->err.clear();
    lcg_status rc = check_model(c, m);
    if (rc) return rc;
    if (!n || which < 0 || which > 2) return c->fail(LCG_E_INVALID, "bad component request");
    cudaSetDevice(c->device);
    std::vector<DiscRing> rings;
    Fail f{0, ""};
    lcg_model mm = *m;
    if (which < 2) mm.add_spot = 0;
    else mm.add_disc = 0;
    if ((which < 2 && !m->add_disc) || (which == 2 && !m->add_spot)) {
        *n = 0;
        return LCG_OK;
    }
    if (!comp_setup(mm, c->comp, rings, f)) return c->fail(f.code, "%s", f.msg.c_str());
    const int32_t total = c->comp.nd + c->comp.ne + c->comp.ns;
    const int32_t lo = which == 0 ? 0 : (which == 1 ? c->comp.nd : c->comp.nd + c->comp.ne);
    const int32_t cnt = which == 0 ? c->comp.nd : (which == 1 ? c->comp.ne : c->comp.ns);
    *n = cnt;
    cudaError_t e;
    if ((e = c->elem.ensure(total)) || (e = c->epos.ensure(total)) ||
        (e = c->drings.ensure(rings.size())))
        return c->cuda_fail(e, "component elements");
    if (!rings.empty())
        cudaMemcpyAsync(c->drings.p, rings.data(), rings.size() * sizeof(DiscRing),
                        cudaMemcpyHostToDevice, c->stream);
    c->comp.rings = c->drings.p;
    cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream);
    launch_components(c->comp, c->elem.p, c->epos.p, c->status.p, c->stream);
    if ((rc = finish_status(c))) return rc;
    if (cnt > cap || !posn || cnt == 0) return LCG_OK;
    std::vector<ElemRec> el((size_t)cnt);
    std::vector<double4> pos((size_t)cnt);
    if ((e = cudaMemcpy(el.data(), c->elem.p + lo, cnt * sizeof(ElemRec), cudaMemcpyDeviceToHost)) ||
        (e = cudaMemcpy(pos.data(), c->epos.p + lo, cnt * sizeof(double4), cudaMemcpyDeviceToHost)))
        return c->cuda_fail(e, "component copy");
    for (int32_t i = 0; i < cnt; i++) {
        posn[3 * i] = pos[i].x; posn[3 * i + 1] = pos[i].y; posn[3 * i + 2] = pos[i].z;
        dirn[3 * i] = el[i].dx; dirn[3 * i + 1] = el[i].dy; dirn[3 * i + 2] = el[i].dz;
        area[i] = (float)pos[i].w;
        flux[i] = el[i].flux;
        nr[i] = el[i].nr;
        for (int k = 0; k < kMaxRanges; k++) {
            rin[kMaxRanges * i + k] = el[i].r[k].x;
            rout[kMaxRanges * i + k] = el[i].r[k].y;
        }
    }
    return LCG_OK;
}

lcg_status lcg_star_grid(lcg_ctx *c, const lcg_model *m, int32_t star, int32_t fine,
                         int32_t nface, double *posn, double *dirn, float *area, float *gravity,
                         float *flux, int32_t *neclipse, double *ecl_in, double *ecl_out) {
    if (!c) return LCG_E_INVALID;
    lcg_status rc = check_model(c, m);
    if (rc) return rc;
    if (star != kStar1 && star != kStar2) return c->fail(LCG_E_INVALID, "bad star");
    cudaSetDevice(c->device);
    cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream);
    c->has_geom = c->has_cont = false;  // this call reuses the cache's grid slot
    Grid &g = star == kStar1 ? c->g1c : c->g2c;
    if ((rc = build_geometry(c, *m, star, fine, g, c->stream))) return rc;
    if (g.n != nface)
        return c->fail(LCG_E_INVALID, "nface = %d but the grid has %lld faces", nface,
                       (long long)g.n);
    ContParams cp = continuum_params(*m, star);
    launch_continuum(cp, g.dev(), c->stream);
    std::vector<double> px(nface), py(nface), pz(nface), nx(nface), ny(nface), nz(nface);
    std::vector<uint8_t> ne(nface);
    const size_t d8 = (size_t)nface * sizeof(double), f4 = (size_t)nface * sizeof(float);
    cudaMemcpyAsync(px.data(), g.px.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(py.data(), g.py.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(pz.data(), g.pz.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(nx.data(), g.nx.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(ny.data(), g.ny.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(nz.data(), g.nz.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(area, g.area.p, f4, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(gravity, g.grav.p, f4, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(flux, g.flux.p, f4, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(ne.data(), g.necl.p, (size_t)nface, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(ecl_in, g.ein.p, d8, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(ecl_out, g.eout.p, d8, cudaMemcpyDeviceToHost, c->stream);
    if ((rc = finish_status(c))) return rc;
    for (int i = 0; i < nface; i++) {
        posn[3 * i] = px[i]; posn[3 * i + 1] = py[i]; posn[3 * i + 2] = pz[i];
        dirn[3 * i] = nx[i]; dirn[3 * i + 1] = ny[i]; dirn[3 * i + 2] = nz[i];
        neclipse[i] = ne[i];
    }
    return LCG_OK;
}

lcg_status lcg_sum_star_multi(lcg_ctx *c, int32_t star, int64_t n, int64_t n0, const double *dx,
                              const double *dy, const double *dz, const double *px,
                              const double *py, const double *pz, const double *flux,
                              const double *in1, const double *out1, int32_t nent,
                              const double *ex, const double *ey, const double *ez,
                              const double *phin, const double *ldc, int32_t ltype, double mucrit,
                              double beam, double spin, double vfac, double xcofm,
                              int32_t glens1, double rlens1, double *out) {
    if (!c) return LCG_E_INVALID;
    if (n < 0 || n0 < 0 || n0 > n || nent < 0 || !out || !ldc)
        return c->fail(LCG_E_INVALID, "bad argument");
    cudaSetDevice(c->device);
    const int mixed = c->precision == LCG_PREC_MIXED;
    cudaError_t e;
    Grid &g = star == kStar1 ? c->g1c : c->g2c;  // scratch slot
    c->has_geom = c->has_cont = false;
    g.n = n;
    g.fast = 0;
    const bool need_pos = beam != 0. || (star == kStar2 && glens1);
    g.npad = ((n + 4095) / 4096) * 4096;
    if (g.npad == 0) g.npad = 4096;
    DBuf<double> *cols[] = {&g.fdx, &g.fdy, &g.fdz, &g.fpx, &g.fpy, &g.fpz, &g.fflux, &g.fin, &g.fout};
    for (auto *b : cols)
        if ((e = b->ensure(g.npad))) return c->cuda_fail(e, "flat columns");
    if ((e = g.n0.ensure(1))) return c->cuda_fail(e, "n0");
    if (mixed && ((e = g.geo.ensure(g.npad)) || (e = g.ecl.ensure(g.npad)) ||
                  (e = g.pos.ensure(g.npad))))
        return c->cuda_fail(e, "packed grid");
    const double *src[] = {dx, dy, dz, px, py, pz, flux};
    for (int k = 0; k < 7; k++)
        if (n) cudaMemcpyAsync(cols[k]->p, src[k], (size_t)n * 8, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(g.fin.p, 0, (size_t)g.npad * 8, c->stream);
    cudaMemsetAsync(g.fout.p, 0, (size_t)g.npad * 8, c->stream);
    if (n > n0) {
        cudaMemcpyAsync(g.fin.p + n0, in1, (size_t)(n - n0) * 8, cudaMemcpyHostToDevice, c->stream);
        cudaMemcpyAsync(g.fout.p + n0, out1, (size_t)(n - n0) * 8, cudaMemcpyHostToDevice, c->stream);
    }
    cudaMemcpyAsync(g.n0.p, &n0, sizeof(int64_t), cudaMemcpyHostToDevice, c->stream);
    if (mixed) launch_pack_flat(g.flat(), n0, need_pos, c->stream);
    if ((e = c->pex.ensure(nent)) || (e = c->pey.ensure(nent)) || (e = c->pez.ensure(nent)) ||
        (e = c->pphin.ensure(nent)) || (e = c->pef.ensure(nent)) || (e = c->ppfx.ensure(nent)))
        return c->cuda_fail(e, "phases");
    if (nent) {
        cudaMemcpyAsync(c->pex.p, ex, (size_t)nent * 8, cudaMemcpyHostToDevice, c->stream);
        cudaMemcpyAsync(c->pey.p, ey, (size_t)nent * 8, cudaMemcpyHostToDevice, c->stream);
        cudaMemcpyAsync(c->pez.p, ez, (size_t)nent * 8, cudaMemcpyHostToDevice, c->stream);
        cudaMemcpyAsync(c->pphin.p, phin, (size_t)nent * 8, cudaMemcpyHostToDevice, c->stream);
    }
    PhaseDev ph{c->pex.p, c->pey.p, c->pez.p, c->pphin.p, nullptr, nullptr, c->pef.p, nullptr, nent,
                c->ppfx.p};
    if (mixed) launch_pack_phases(ph, c->stream);
    FluxConsts k{};
    for (int i = 0; i < 4; i++) k.c[i] = ldc[i];
    k.base = 1.0 - (ldc[0] + ldc[1] + ldc[2] + ldc[3]);
    k.mucrit = mucrit;
    k.ltype = ltype;
    k.beam = beam;
    k.beam_on = beam != 0.0;
    k.glens = star == kStar2 ? glens1 : 0;
    k.spin = spin;
    k.vfac = vfac;
    k.xcofm = xcofm;
    k.rlens1 = rlens1;
    FluxPlan plan = plan_flux(mixed, 0, n, nent, c->nsm);
    const int64_t ldp = ((nent + 3) / 4) * 4;
    if ((e = c->part1f.ensure((size_t)std::max<int64_t>(plan.nchunk, 1) * std::max<int64_t>(ldp, 1))))
        return c->cuda_fail(e, "partials");
    cudaMemsetAsync(c->status.p, 0, sizeof(DevStatus), c->stream);
    {
        StageScope t(c, LCG_STAGE_FLUX);
        launch_flux(mixed, star, k, g.flat(), ph, plan, c->part1f.p, ldp, c->status.p, c->stream);
    }
    c->flux_elements += n * (int64_t)nent;
    std::vector<double> part((size_t)plan.nchunk * ldp);
    if (plan.nchunk && nent)
        cudaMemcpyAsync(part.data(), c->part1f.p, part.size() * 8, cudaMemcpyDeviceToHost,
                        c->stream);
    lcg_status rc = finish_status(c);
    if (rc) return rc;
    for (int32_t j = 0; j < nent; j++) {
        double o = 0.0;
        for (int64_t b = 0; b < plan.nchunk; b++) o += part[(size_t)b * ldp + j];
        out[j] = o;
    }
    return LCG_OK;
}

int64_t lcg_kernel_launches(int32_t reset) {
    return reset ? g_launches.exchange(0) : g_launches.load();
}

lcg_status lcg_measure_fp32_peak(lcg_ctx *c, double *tflops) {
    return measure_peak(c, tflops, [](void *sink, int blocks, int iters, double *gflop,
                                      cudaStream_t s) {
        launch_fma_probe(static_cast<float *>(sink), blocks, iters, gflop, s);
    });
}

lcg_status lcg_measure_fp64_peak(lcg_ctx *c, double *tflops) {
    return measure_peak(c, tflops, [](void *sink, int blocks, int iters, double *gflop,
                                      cudaStream_t s) {
        launch_dfma_probe(static_cast<double *>(sink), blocks, iters, gflop, s);
    });
}

}  // extern "C"
