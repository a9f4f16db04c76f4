// light_curve_comp_lcg.cpp — Lcurve::light_curve_comp on the B200 engine.
//
// Link this file into lcurve_re in place of src/lcurve_base/light_curve_comp.cpp
// (and link liblcg.so): lcurve_re, mcmc_solver, simplex and levmarq_solver
// then evaluate every model on the GPU, unchanged. It implements the call
// declared at src/lcurve_base/lcurve.h:669-674 with the reference's semantics
// (light_curve_comp.cpp:119-599):
//   * calc is resized to data.size();
//   * sfac (size >= 5) is read when scale is false and all five entries are
//     written when it is true;
//   * chisq and wnok are written only when scale or rdata is set;
//   * failures throw Lcurve::Lcurve_Error with the engine's message (the
//     reference's messages for lobe overflow), which the solvers treat as a
//     rejected model (mcmc_solver.cpp:1071, levmarq_solver.cpp:682).
// One engine context per host thread: the reference keeps its caches
// thread_local too (light_curve_comp.cpp:161). Every model the reference
// evaluates runs on the engine, discs, rims, bright spots and iscale included;
// there is no CPU fallback.
//
// The environment variables the reference's CUDA path reads select the same
// things here (comp_light_cuda.cu:415,523-533): LCURVE_CUDA_PRECISION = double,
// fp64 or 64 gives FP64 contexts (every stage FP64, the sweep bit-identical
// to the CPU path); anything else, or unset, gives the mixed-precision default,
// as the reference's CUDA sweeps default to FP32. LCURVE_CUDA_DEVICE picks the
// device (default 0).
//
// The two offload counters the reference's CUDA sources define and
// levmarq_solver.cpp reports (comp_light_cuda.h:23, set_star_grid_cuda.h:24)
// are defined here too: light curves this thread evaluated on the engine (both
// stars' grids and flux sweeps run on the device for each).
#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "lcg.h"
#include "lcurve.h"

namespace {

// Every field of the model the evaluation path reads (lcurve.h:340-396).
lcg_model to_lcg(const Lcurve::Model &m) {
    lcg_model c;
    std::memset(&c, 0, sizeof c);
    c.q = m.q; c.iangle = m.iangle; c.r1 = m.r1; c.r2 = m.r2;
    c.cphi3 = m.cphi3; c.cphi4 = m.cphi4; c.spin1 = m.spin1; c.spin2 = m.spin2;
    c.t1 = m.t1; c.t2 = m.t2;
    c.ldc1[0] = m.ldc1_1; c.ldc1[1] = m.ldc1_2; c.ldc1[2] = m.ldc1_3; c.ldc1[3] = m.ldc1_4;
    c.ldc2[0] = m.ldc2_1; c.ldc2[1] = m.ldc2_2; c.ldc2[2] = m.ldc2_3; c.ldc2[3] = m.ldc2_4;
    c.velocity_scale = m.velocity_scale;
    c.beam_factor1 = m.beam_factor1; c.beam_factor2 = m.beam_factor2;
    c.t0 = m.t0; c.period = m.period; c.pdot = m.pdot; c.deltat = m.deltat;
    c.gravity_dark1 = m.gravity_dark1; c.gravity_dark2 = m.gravity_dark2;
    c.absorb = m.absorb; c.slope = m.slope; c.quad = m.quad; c.cube = m.cube;
    c.third = m.third;
    // star spots: active when all four parameters are defined
    const Lcurve::Pparam *sp[5][4] = {
        {&m.stsp11_long, &m.stsp11_lat, &m.stsp11_fwhm, &m.stsp11_tcen},
        {&m.stsp12_long, &m.stsp12_lat, &m.stsp12_fwhm, &m.stsp12_tcen},
        {&m.stsp13_long, &m.stsp13_lat, &m.stsp13_fwhm, &m.stsp13_tcen},
        {&m.stsp21_long, &m.stsp21_lat, &m.stsp21_fwhm, &m.stsp21_tcen},
        {&m.stsp22_long, &m.stsp22_lat, &m.stsp22_fwhm, &m.stsp22_tcen}};
    for (int s = 0; s < 5; s++) {
        bool all = true;
        for (int k = 0; k < 4; k++) {
            c.stsp[s][k] = sp[s][k]->value;
            all = all && sp[s][k]->defined;
        }
        c.stsp_defined[s] = all;
    }
    const Lcurve::Pparam *ue[5] = {&m.uesp_long1, &m.uesp_long2, &m.uesp_lathw, &m.uesp_taper,
                                   &m.uesp_temp};
    bool ue_all = true;
    for (int k = 0; k < 5; k++) {
        c.uesp[k] = ue[k]->value;
        ue_all = ue_all && ue[k]->defined;
    }
    c.uesp_defined = ue_all;
    c.delta_phase = m.delta_phase;
    c.nlat1f = m.nlat1f; c.nlat2f = m.nlat2f; c.nlat1c = m.nlat1c; c.nlat2c = m.nlat2c;
    c.npole = m.npole; c.nlatfill = m.nlatfill; c.nlngfill = m.nlngfill;
    c.lfudge = m.lfudge; c.llo = m.llo; c.lhi = m.lhi;
    c.phase1 = m.phase1; c.phase2 = m.phase2; c.wavelength = m.wavelength;
    c.roche1 = m.roche1; c.roche2 = m.roche2; c.eclipse1 = m.eclipse1; c.eclipse2 = m.eclipse2;
    c.glens1 = m.glens1; c.use_radii = m.use_radii; c.tperiod = m.tperiod;
    c.gdark_bolom1 = m.gdark_bolom1; c.gdark_bolom2 = m.gdark_bolom2;
    c.mucrit1 = m.mucrit1; c.mucrit2 = m.mucrit2;
    c.limb1 = m.limb1 == Lcurve::LDC::CLARET ? LCG_LIMB_CLARET : LCG_LIMB_POLY;
    c.limb2 = m.limb2 == Lcurve::LDC::CLARET ? LCG_LIMB_CLARET : LCG_LIMB_POLY;
    c.mirror = m.mirror; c.add_disc = m.add_disc; c.opaque = m.opaque;
    c.add_spot = m.add_spot; c.iscale = m.iscale;
    c.rdisc1 = m.rdisc1; c.rdisc2 = m.rdisc2; c.height_disc = m.height_disc;
    c.beta_disc = m.beta_disc; c.temp_disc = m.temp_disc; c.texp_disc = m.texp_disc;
    c.lin_limb_disc = m.lin_limb_disc; c.quad_limb_disc = m.quad_limb_disc;
    c.temp_edge = m.temp_edge; c.absorb_edge = m.absorb_edge;
    c.radius_spot = m.radius_spot; c.length_spot = m.length_spot;
    c.height_spot = m.height_spot; c.expon_spot = m.expon_spot; c.epow_spot = m.epow_spot;
    c.angle_spot = m.angle_spot; c.yaw_spot = m.yaw_spot; c.temp_spot = m.temp_spot;
    c.tilt_spot = m.tilt_spot; c.cfrac_spot = m.cfrac_spot;
    c.nrad = m.nrad; c.nspot = m.nspot;
    return c;
}

struct Context {
    lcg_ctx *ctx = nullptr;
    std::uint64_t curves = 0;
    ~Context() {
        if (ctx) lcg_destroy(ctx);
    }
};

thread_local Context t_context;

int32_t precision_from_env() {
    const char *env = std::getenv("LCURVE_CUDA_PRECISION");
    if (!env) return LCG_PREC_MIXED;
    std::string mode(env);
    std::transform(mode.begin(), mode.end(), mode.begin(),
                   [](unsigned char ch) { return (char)std::tolower(ch); });
    return (mode == "double" || mode == "fp64" || mode == "64") ? LCG_PREC_FP64 : LCG_PREC_MIXED;
}

lcg_ctx *context() {
    Context &c = t_context;
    if (!c.ctx) {
        lcg_options o;
        lcg_default_options(&o);
        o.precision = precision_from_env();
        if (const char *dev = std::getenv("LCURVE_CUDA_DEVICE")) o.device = std::atoi(dev);
        if (lcg_create(&c.ctx, &o) != LCG_OK) {
            c.ctx = nullptr;
            throw Lcurve::Lcurve_Error(std::string("light_curve_comp: ") + lcg_last_error(nullptr));
        }
    }
    return c.ctx;
}

}  // namespace

void Lcurve::light_curve_comp(const Lcurve::Model &mdl, const Lcurve::Data &data, bool scale,
                              bool rdata, bool info, std::vector<double> &sfac,
                              std::vector<double> &calc, double &wdwarf, double &chisq,
                              double &wnok, double &logg1, double &logg2, double &rv1,
                              double &rv2, bool diagnostics) {
    lcg_ctx *ctx = context();
    calc.resize(data.size());
    if (sfac.size() < 5) sfac.resize(5, 1.0);
    double s[LCG_NOUT] = {wdwarf, chisq, wnok, logg1, logg2, rv1, rv2};
    const lcg_model m = to_lcg(mdl);
    const int flags = (scale ? LCG_FLAG_SCALE : 0) | (rdata ? LCG_FLAG_RDATA : 0) |
                      (info ? LCG_FLAG_INFO : 0) | (diagnostics ? LCG_FLAG_DIAGNOSTICS : 0);
    static_assert(sizeof(Lcurve::Datum) == sizeof(lcg_datum), "Datum and lcg_datum differ");
    const lcg_status st =
        lcg_light_curve(ctx, &m, reinterpret_cast<const lcg_datum *>(data.data()),
                        (int32_t)data.size(), flags, sfac.data(), calc.data(), s);
    if (st != LCG_OK) throw Lcurve::Lcurve_Error(lcg_last_error(ctx));
    t_context.curves++;
    wdwarf = s[LCG_OUT_WDWARF];
    if (scale || rdata) {
        chisq = s[LCG_OUT_CHISQ];
        wnok = s[LCG_OUT_WNOK];
    }
    logg1 = s[LCG_OUT_LOGG1];
    logg2 = s[LCG_OUT_LOGG2];
    rv1 = s[LCG_OUT_RV1];
    rv2 = s[LCG_OUT_RV2];
}

namespace Lcurve {
std::uint64_t cuda_flux_evaluation_count() { return t_context.curves; }
std::uint64_t cuda_grid_evaluation_count() { return t_context.curves; }
}  // namespace Lcurve
