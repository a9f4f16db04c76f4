"""Parity cases shared by the CPU pinning tests and the GPU parity tests.

Each case is (name, model, data): the benchmark physics at sizes the CPU
oracle runs in well under a second, plus variants that exercise the
branches of the reference path (polynomial limb darkening, beaming,
lensing, spots, mirror, infill, coarse != fine grids, pdot/deltat, the
polynomial fudge factors, exposure subdivision, spherical stars, no
eclipses, asynchronous spin, cphi parameterisation).
"""
import numpy as np

from lcurve_re_b200 import workloads as W
from lcurve_re_b200.model import make_data


def _d(n=120, lo=-0.2, hi=1.2, ndiv=1, expose=0.0):
    return W.data(n, lo, hi, ndiv=ndiv, expose=expose)


def small_cases():
    cases = []
    cases.append(("wd_dm_small", W.model(), W.data(500)))
    cases.append(("coarse_grid", W.model(nlat1f=24, nlat2f=40, nlat1c=16, nlat2c=28), _d(160)))
    cases.append(("poly_limb", W.model(nlat1f=20, nlat2f=40, limb1="Poly", limb2="Poly",
                                       ldc1_1=0.4, ldc1_2=0.1, ldc1_3=0.0, ldc1_4=0.0,
                                       ldc2_1=0.5, ldc2_2=0.2, ldc2_3=0.0, ldc2_4=0.0), _d()))
    cases.append(("beaming", W.model(nlat1f=20, nlat2f=40, beam_factor1=1.2, beam_factor2=0.8),
                  _d()))
    cases.append(("exposure_ndiv", W.model(nlat1f=20, nlat2f=40),
                  _d(80, ndiv=7, expose=0.01)))
    cases.append(("pdot_deltat_slope", W.model(nlat1f=20, nlat2f=40, pdot=1e-4, deltat=2e-3,
                                               slope=0.01, quad=-0.003, cube=0.001, third=0.05,
                                               t0=0.01, period=1.0001), _d()))
    cases.append(("spheres", W.model(nlat1f=20, nlat2f=40, roche1=0, roche2=0), _d()))
    cases.append(("no_eclipse", W.model(nlat1f=20, nlat2f=40, iangle=60.0), _d()))
    cases.append(("spin_async", W.model(nlat1f=20, nlat2f=40, spin1=1.3, spin2=0.9), _d()))
    cases.append(("mirror_filterdark", W.model(nlat1f=20, nlat2f=40, mirror=1, gdark_bolom1=0,
                                               gdark_bolom2=0, mucrit1=0.05, mucrit2=0.02), _d()))
    cases.append(("infill", W.model(nlat1f=20, nlat2f=40, nlatfill=2, nlngfill=2, llo=90,
                                    lhi=-90, r2=0.25, r1=0.02), _d()))
    cases.append(("cphi_params", W.model(nlat1f=20, nlat2f=40, use_radii=0, cphi3=0.015,
                                         cphi4=0.06), _d()))
    m = W.model(nlat1f=20, nlat2f=40)
    m.p["stsp11_long"].value, m.p["stsp11_lat"].value = 30.0, 20.0
    m.p["stsp11_fwhm"].value, m.p["stsp11_tcen"].value = 40.0, 15000.0
    for k in ("stsp11_long", "stsp11_lat", "stsp11_fwhm", "stsp11_tcen"):
        m.p[k].defined = True
    m.p["stsp21_long"].value, m.p["stsp21_lat"].value = 180.0, -10.0
    m.p["stsp21_fwhm"].value, m.p["stsp21_tcen"].value = 30.0, 4000.0
    for k in ("stsp21_long", "stsp21_lat", "stsp21_fwhm", "stsp21_tcen"):
        m.p[k].defined = True
    cases.append(("star_spots", m, _d()))
    cases.append(("tiny_star_small", W.model(r1=0.005, q=0.2, iangle=87.0, nlat1f=60, nlat2f=30),
                  _d(200, -0.03, 0.03)))
    cases.append(("ragged_ndiv", W.model(nlat1f=16, nlat2f=32),
                  make_data(np.linspace(0.0, 1.0, 31), expose=0.004, flux=1.0, ferr=1.5e-3,
                            weight=np.r_[np.ones(30), 0.0], ndiv=np.arange(31) % 4)))
    return cases


def disc_cases():
    """Cataclysmic-variable components (set_disc_grid.cpp, set_bright_spot_grid.cpp,
    disc_eclipse.cpp, light_curve_comp.cpp:272-333, 378-414, 511-556): disc and
    rim with and without an opaque disc, the bright spot, iscale fits (with and
    without the donor's column), spherical stars, sub-exposures."""
    small = dict(nlat1f=16, nlat2f=24, nrad=16, nspot=20)
    cases = [
        ("disc_rim", W.cv_disc(opaque=0, add_spot=0, **small), _d(150)),
        ("disc_opaque", W.cv_disc(add_spot=0, **small), _d(150)),
        ("disc_spot", W.cv_disc(**small), _d(150)),
        ("spot_only", W.cv_disc(add_disc=0, **small), _d(150)),
        ("iscale", W.cv_disc(iscale=1, **small), _d(150)),
        ("iscale_no_donor", W.cv_disc(iscale=1, t2=-3000.0, **small), _d(150)),
        ("disc_spheres", W.cv_disc(roche1=0, roche2=0, **small), _d(150)),
        ("disc_ndiv", W.cv_disc(**small), _d(60, ndiv=5, expose=0.01)),
    ]
    for _, m, d in cases:
        d["flux"] = 1.0 + 0.01 * np.sin(np.arange(len(d)))
    return cases


def glens_case():
    # lensing needs a spherical star 1 (Model ctor rule, model.cpp:331-332)
    return ("lensing", W.model(nlat1f=20, nlat2f=40, roche1=0, glens1=1, eclipse2=0,
                               tperiod=0.3, velocity_scale=250.0), _d())
