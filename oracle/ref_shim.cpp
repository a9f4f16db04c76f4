// ref_shim.cpp — extern "C" entry points into the lcurve_re reference.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the
// reference's own, unmodified CPU sources (by oracle/Makefile, into
// oracle/_ref/) so that tests and the CPU baseline can drive the reference
// through plain C calls. It contains no reference code: it builds a
// Lcurve::Model from an lcg_model by writing the reference's own JSON
// parameter format, and calls the reference's public functions:
//   Lcurve::light_curve_comp      (src/lcurve_base/lcurve.h:669-674)
//   Lcurve::set_star_grid         (src/lcurve_base/lcurve.h:528)
//   Lcurve::set_star_continuum    (src/lcurve_base/lcurve.h:550)
//   Lcurve::flat_sum_star1_multi / flat_sum_star2_multi (lcurve.h:299-307)
//   Lcurve::set_disc_grid, set_disc_edge, set_bright_spot_grid,
//   set_disc_continuum, set_edge_continuum (lcurve.h:539-561)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "lcurve.h"
#include "../include/lcg.h"

namespace {

std::string num(double v) {
    char b[64];
    std::snprintf(b, sizeof b, "%.17g", v);
    return b;
}

// "value range dstep vary defined", the Pparam string form (lcurve.h:165-176)
std::string pp(double v, bool defined = true) {
    return num(v) + " 0 0 0 " + (defined ? "1" : "0");
}

Lcurve::Model to_model(const lcg_model &m) {
    nlohmann::json p;
    p["q"] = pp(m.q); p["iangle"] = pp(m.iangle);
    p["r1"] = pp(m.r1); p["r2"] = pp(m.r2);
    p["cphi3"] = pp(m.cphi3); p["cphi4"] = pp(m.cphi4);
    p["spin1"] = pp(m.spin1); p["spin2"] = pp(m.spin2);
    p["t1"] = pp(m.t1); p["t2"] = pp(m.t2);
    const char *l1[4] = {"ldc1_1", "ldc1_2", "ldc1_3", "ldc1_4"};
    const char *l2[4] = {"ldc2_1", "ldc2_2", "ldc2_3", "ldc2_4"};
    for (int k = 0; k < 4; k++) { p[l1[k]] = pp(m.ldc1[k]); p[l2[k]] = pp(m.ldc2[k]); }
    p["velocity_scale"] = pp(m.velocity_scale);
    p["beam_factor1"] = pp(m.beam_factor1); p["beam_factor2"] = pp(m.beam_factor2);
    p["t0"] = pp(m.t0); p["period"] = pp(m.period);
    p["pdot"] = pp(m.pdot); p["deltat"] = pp(m.deltat);
    p["gravity_dark1"] = pp(m.gravity_dark1); p["gravity_dark2"] = pp(m.gravity_dark2);
    p["absorb"] = pp(m.absorb); p["slope"] = pp(m.slope);
    p["quad"] = pp(m.quad); p["cube"] = pp(m.cube); p["third"] = pp(m.third);
    const char *disc[] = {"rdisc1", "rdisc2", "height_disc", "beta_disc", "temp_disc",
                          "texp_disc", "lin_limb_disc", "quad_limb_disc", "temp_edge",
                          "absorb_edge", "radius_spot", "length_spot", "height_spot",
                          "expon_spot", "epow_spot", "angle_spot", "yaw_spot",
                          "temp_spot", "tilt_spot", "cfrac_spot"};
    const double dv[] = {m.rdisc1, m.rdisc2, m.height_disc, m.beta_disc, m.temp_disc,
                         m.texp_disc, m.lin_limb_disc, m.quad_limb_disc, m.temp_edge,
                         m.absorb_edge, m.radius_spot, m.length_spot, m.height_spot,
                         m.expon_spot, m.epow_spot, m.angle_spot, m.yaw_spot, m.temp_spot,
                         m.tilt_spot, m.cfrac_spot};
    for (int k = 0; k < 20; k++) p[disc[k]] = pp(dv[k]);
    const char *spots[5] = {"stsp11", "stsp12", "stsp13", "stsp21", "stsp22"};
    const char *fields[4] = {"_long", "_lat", "_fwhm", "_tcen"};
    for (int s = 0; s < 5; s++)
        if (m.stsp_defined[s])
            for (int f = 0; f < 4; f++)
                p[std::string(spots[s]) + fields[f]] = pp(m.stsp[s][f]);
    if (m.uesp_defined) {
        const char *u[5] = {"uesp_long1", "uesp_long2", "uesp_lathw", "uesp_taper", "uesp_temp"};
        for (int k = 0; k < 5; k++) p[u[k]] = pp(m.uesp[k]);
    }
    p["delta_phase"] = num(m.delta_phase);
    p["nlat1f"] = std::to_string(m.nlat1f); p["nlat2f"] = std::to_string(m.nlat2f);
    p["nlat1c"] = std::to_string(m.nlat1c); p["nlat2c"] = std::to_string(m.nlat2c);
    p["npole"] = m.npole ? "1" : "0";
    p["nlatfill"] = std::to_string(m.nlatfill); p["nlngfill"] = std::to_string(m.nlngfill);
    p["lfudge"] = num(m.lfudge); p["llo"] = num(m.llo); p["lhi"] = num(m.lhi);
    p["phase1"] = num(m.phase1); p["phase2"] = num(m.phase2);
    p["wavelength"] = num(m.wavelength);
    p["roche1"] = m.roche1 ? "1" : "0"; p["roche2"] = m.roche2 ? "1" : "0";
    p["eclipse1"] = m.eclipse1 ? "1" : "0"; p["eclipse2"] = m.eclipse2 ? "1" : "0";
    p["glens1"] = m.glens1 ? "1" : "0"; p["use_radii"] = m.use_radii ? "1" : "0";
    p["tperiod"] = num(m.tperiod);
    p["gdark_bolom1"] = m.gdark_bolom1 ? "1" : "0";
    p["gdark_bolom2"] = m.gdark_bolom2 ? "1" : "0";
    p["mucrit1"] = num(m.mucrit1); p["mucrit2"] = num(m.mucrit2);
    p["limb1"] = m.limb1 == LCG_LIMB_CLARET ? "Claret" : "Poly";
    p["limb2"] = m.limb2 == LCG_LIMB_CLARET ? "Claret" : "Poly";
    p["mirror"] = m.mirror ? "1" : "0";
    p["add_disc"] = m.add_disc ? "1" : "0"; p["nrad"] = std::to_string(m.nrad);
    p["opaque"] = m.opaque ? "1" : "0";
    p["add_spot"] = m.add_spot ? "1" : "0"; p["nspot"] = std::to_string(m.nspot);
    p["iscale"] = m.iscale ? "1" : "0";
    nlohmann::json cfg;
    cfg["model_parameters"] = p;
    return Lcurve::Model(cfg);
}

int fail(const std::exception &ex, char *err, int errlen, int code) {
    if (err && errlen > 0) {
        std::strncpy(err, ex.what(), (size_t)errlen - 1);
        err[errlen - 1] = 0;
    }
    return code;
}

}  // namespace

extern "C" {

int lcref_light_curve_fast(const lcg_model *m, const lcg_datum *data, int32_t n,
                           int32_t flags, int32_t max_pts, double *sfac, double *calc,
                           double *scalars, char *err, int errlen) {
    try {
        Lcurve::Model mdl = to_model(*m);
        Lcurve::Data d(n);
        for (int i = 0; i < n; i++) {
            d[i].time = data[i].time; d[i].expose = data[i].expose;
            d[i].flux = data[i].flux; d[i].ferr = data[i].ferr;
            d[i].weight = data[i].weight; d[i].ndiv = data[i].ndiv;
        }
        std::vector<double> sf(sfac, sfac + 5), c;
        double wdwarf = scalars[LCG_OUT_WDWARF], chisq = scalars[LCG_OUT_CHISQ];
        double wnok = scalars[LCG_OUT_WNOK], logg1, logg2, rv1, rv2;
        Lcurve::light_curve_comp_fast(mdl, d, flags & LCG_FLAG_SCALE, flags & LCG_FLAG_RDATA,
                                      flags & LCG_FLAG_INFO, sf, c, wdwarf, chisq, wnok, logg1,
                                      logg2, rv1, rv2, max_pts,
                                      (flags & LCG_FLAG_DIAGNOSTICS) != 0);
        for (int i = 0; i < n; i++) calc[i] = c[i];
        for (int k = 0; k < 5; k++) sfac[k] = sf[k];
        scalars[LCG_OUT_WDWARF] = wdwarf; scalars[LCG_OUT_CHISQ] = chisq;
        scalars[LCG_OUT_WNOK] = wnok;
        return 0;
    } catch (const Lcurve::Lcurve_Error &ex) {
        return fail(ex, err, errlen, LCG_E_LOBE);
    } catch (const Roche::Roche_Error &ex) {
        return fail(ex, err, errlen, LCG_E_ROCHE);
    } catch (const std::exception &ex) {
        return fail(ex, err, errlen, LCG_E_INVALID);
    }
}

int lcref_light_curve(const lcg_model *m, const lcg_datum *data, int32_t n,
                      int32_t flags, double *sfac, double *calc,
                      double *scalars, char *err, int errlen) {
    try {
        Lcurve::Model mdl = to_model(*m);
        Lcurve::Data d(n);
        for (int i = 0; i < n; i++) {
            d[i].time = data[i].time; d[i].expose = data[i].expose;
            d[i].flux = data[i].flux; d[i].ferr = data[i].ferr;
            d[i].weight = data[i].weight; d[i].ndiv = data[i].ndiv;
        }
        std::vector<double> sf(sfac, sfac + 5), c;
        double wdwarf = scalars[LCG_OUT_WDWARF], chisq = scalars[LCG_OUT_CHISQ];
        double wnok = scalars[LCG_OUT_WNOK], logg1, logg2, rv1, rv2;
        Lcurve::light_curve_comp(mdl, d, flags & LCG_FLAG_SCALE, flags & LCG_FLAG_RDATA,
                                 flags & LCG_FLAG_INFO, sf, c, wdwarf, chisq, wnok,
                                 logg1, logg2, rv1, rv2,
                                 (flags & LCG_FLAG_DIAGNOSTICS) != 0);
        for (int i = 0; i < n; i++) calc[i] = c[i];
        for (int k = 0; k < 5; k++) sfac[k] = sf[k];
        scalars[LCG_OUT_WDWARF] = wdwarf; scalars[LCG_OUT_CHISQ] = chisq;
        scalars[LCG_OUT_WNOK] = wnok; scalars[LCG_OUT_LOGG1] = logg1;
        scalars[LCG_OUT_LOGG2] = logg2; scalars[LCG_OUT_RV1] = rv1;
        scalars[LCG_OUT_RV2] = rv2;
        return 0;
    } catch (const Lcurve::Lcurve_Error &ex) {
        return fail(ex, err, errlen, LCG_E_LOBE);
    } catch (const Roche::Roche_Error &ex) {
        return fail(ex, err, errlen, LCG_E_ROCHE);
    } catch (const std::exception &ex) {
        return fail(ex, err, errlen, LCG_E_INVALID);
    }
}

int lcref_star_grid(const lcg_model *m, int32_t star, int32_t fine, int32_t cap,
                    int32_t *nface, double *posn, double *dirn, float *area,
                    float *gravity, float *flux, int32_t *necl, double *ein,
                    double *eout, char *err, int errlen) {
    try {
        Lcurve::Model mdl = to_model(*m);
        std::vector<Lcurve::Point> g, other;
        Lcurve::set_star_grid(mdl, star == LCG_STAR1 ? Roche::PRIMARY : Roche::SECONDARY,
                              fine != 0, g);
        if (star == LCG_STAR1) Lcurve::set_star_continuum(mdl, g, other);
        else Lcurve::set_star_continuum(mdl, other, g);
        *nface = (int32_t)g.size();
        if ((int32_t)g.size() > cap || !posn) return 0;
        for (size_t i = 0; i < g.size(); i++) {
            const Lcurve::Point &p = g[i];
            posn[3 * i] = p.posn.x(); posn[3 * i + 1] = p.posn.y(); posn[3 * i + 2] = p.posn.z();
            dirn[3 * i] = p.dirn.x(); dirn[3 * i + 1] = p.dirn.y(); dirn[3 * i + 2] = p.dirn.z();
            area[i] = p.area; gravity[i] = p.gravity; flux[i] = p.flux;
            necl[i] = (int32_t)p.eclipse.size();
            ein[i] = p.eclipse.empty() ? 0. : p.eclipse[0].first;
            eout[i] = p.eclipse.empty() ? 0. : p.eclipse[0].second;
        }
        return 0;
    } catch (const Lcurve::Lcurve_Error &ex) {
        return fail(ex, err, errlen, LCG_E_LOBE);
    } catch (const Roche::Roche_Error &ex) {
        return fail(ex, err, errlen, LCG_E_ROCHE);
    } catch (const std::exception &ex) {
        return fail(ex, err, errlen, LCG_E_INVALID);
    }
}

// One component grid as light_curve_comp builds it (light_curve_comp.cpp:272-333):
// which = 0 the disc, 1 its outer edge (continua applied), 2 the bright spot.
// Up to maxr eclipse ranges per element are returned (nr holds the full count).
int lcref_components(const lcg_model *m, int32_t which, int32_t cap, int32_t maxr,
                     int32_t *nout, double *posn, double *dirn, float *area, float *flux,
                     int32_t *nr, double *rin, double *rout, char *err, int errlen) {
    try {
        Lcurve::Model mdl = to_model(*m);
        std::vector<Lcurve::Point> g;
        double r1, r2;
        mdl.get_r1r2(r1, r2);
        const double rl2 = 1. - Roche::xl12(mdl.q, mdl.spin2);
        if (r2 < 0) r2 = rl2;
        const double rdisc2 = mdl.rdisc2 > 0. ? mdl.rdisc2 : mdl.radius_spot;
        if (which == 0) {
            Lcurve::set_disc_grid(mdl, g);
            Lcurve::set_disc_continuum(rdisc2, mdl.temp_disc, mdl.texp_disc, mdl.wavelength, g);
        } else if (which == 1) {
            Lcurve::set_disc_edge(mdl, true, g, false);
            Lcurve::set_edge_continuum(mdl.temp_edge, r2, std::fabs(mdl.t2), mdl.absorb_edge,
                                       mdl.wavelength, g);
        } else {
            Lcurve::set_bright_spot_grid(mdl, g);
        }
        *nout = (int32_t)g.size();
        if ((int32_t)g.size() > cap || !posn) return 0;
        for (size_t i = 0; i < g.size(); i++) {
            const Lcurve::Point &p = g[i];
            posn[3 * i] = p.posn.x(); posn[3 * i + 1] = p.posn.y(); posn[3 * i + 2] = p.posn.z();
            dirn[3 * i] = p.dirn.x(); dirn[3 * i + 1] = p.dirn.y(); dirn[3 * i + 2] = p.dirn.z();
            area[i] = p.area; flux[i] = p.flux;
            nr[i] = (int32_t)p.eclipse.size();
            for (int k = 0; k < maxr && k < (int)p.eclipse.size(); k++) {
                rin[maxr * i + k] = p.eclipse[k].first;
                rout[maxr * i + k] = p.eclipse[k].second;
            }
        }
        return 0;
    } catch (const Lcurve::Lcurve_Error &ex) {
        return fail(ex, err, errlen, LCG_E_LOBE);
    } catch (const Roche::Roche_Error &ex) {
        return fail(ex, err, errlen, LCG_E_ROCHE);
    } catch (const std::exception &ex) {
        return fail(ex, err, errlen, LCG_E_INVALID);
    }
}

int lcref_sum_star_multi(int32_t star, int64_t n, int64_t n0, const double *dx,
                         const double *dy, const double *dz, const double *px,
                         const double *py, const double *pz, const double *flux,
                         const double *in1, const double *out1, int32_t nent,
                         const double *ex, const double *ey, const double *ez,
                         const double *phin, const double *ldc, int32_t ltype,
                         double mucrit, double beam, double spin, double vfac,
                         double xcofm, int32_t glens1, double rlens1, double *out) {
    Lcurve::FlatGrid g;
    g.n = (size_t)n; g.n0 = (size_t)n0; g.n1 = (size_t)n;
    g.dx.assign(dx, dx + n); g.dy.assign(dy, dy + n); g.dz.assign(dz, dz + n);
    g.px.assign(px, px + n); g.py.assign(py, py + n); g.pz.assign(pz, pz + n);
    g.flux.assign(flux, flux + n);
    g.in1.assign(in1, in1 + (n - n0)); g.out1.assign(out1, out1 + (n - n0));
    g.moff.assign(1, 0);
    g.generation = 1;
    Lcurve::PhaseBatch pb;
    for (int k = 0; k < nent; k++) pb.push(ex[k], ey[k], ez[k], phin[k], 1.0, k);
    Lcurve::LDC L(ldc[0], ldc[1], ldc[2], ldc[3], mucrit,
                  ltype == LCG_LIMB_CLARET ? Lcurve::LDC::CLARET : Lcurve::LDC::POLY);
    if (star == LCG_STAR1)
        Lcurve::flat_sum_star1_multi(g, pb, L, beam, spin, vfac, xcofm, out);
    else
        Lcurve::flat_sum_star2_multi(g, pb, L, beam, spin, vfac, xcofm, glens1 != 0,
                                     rlens1, out);
    return 0;
}

}  // extern "C"
