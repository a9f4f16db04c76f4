"""The benchmark workloads, as seeded synthetic inputs.

No public dataset is involved: each workload is a binary-star model in the
reference's JSON parameter format plus a synthetic light curve with the
named shape (number of points, phase range, exposure subdivision) and
Gaussian noise drawn from a seeded numpy Generator.

  wd_dm_small    detached WD + dM eclipsing binary, nlat 40/80, 500 points
  wd_dm_large    same physics, nlat 200/800, 5000 points x ndiv 5
  mcmc_batch     256 models around wd_dm_small, nlat2f in 60..400, 2000 points
  tiny_star      r1 in {0.002, 0.005, 0.01}, nlat 400/200, 10000 points near eclipse
  surrogate_box  the prior box of the surrogate training set
  cv_disc        cataclysmic variable: white dwarf, Roche-filling donor, flared
                 accretion disc with its rim, and the bright spot
"""
import math

import numpy as np

from . import abi
from .model import Model, make_data

SIGMA = 1.5e-3


def _pp(v, vary=0):
    return "%.17g 0.01 0.001 %d 1" % (v, vary)


def base_parameters():
    """Detached WD+dM eclipsing binary: q=0.25, i=86 deg, r1=0.015, r2=0.20,
    T1=20000 K, T2=3200 K, 4-coefficient Claret limb darkening, gravity
    darkening 0.25/0.08, irradiation absorb=0.5; wavelength 550 nm,
    velocity_scale 300 km/s, no beaming, synchronous spins."""
    p = {
        "q": _pp(0.25, 1), "iangle": _pp(86.0, 1), "r1": _pp(0.015, 1), "r2": _pp(0.20, 1),
        "cphi3": _pp(0.01), "cphi4": _pp(0.055), "spin1": _pp(1.0), "spin2": _pp(1.0),
        "t1": _pp(20000.0, 1), "t2": _pp(3200.0, 1),
        "ldc1_1": _pp(0.10), "ldc1_2": _pp(0.60), "ldc1_3": _pp(-0.45), "ldc1_4": _pp(0.15),
        "ldc2_1": _pp(0.70), "ldc2_2": _pp(-0.60), "ldc2_3": _pp(1.00), "ldc2_4": _pp(-0.35),
        "velocity_scale": _pp(300.0), "beam_factor1": _pp(0.0), "beam_factor2": _pp(0.0),
        "t0": _pp(0.0, 1), "period": _pp(1.0), "pdot": _pp(0.0), "deltat": _pp(0.0),
        "gravity_dark1": _pp(0.25), "gravity_dark2": _pp(0.08), "absorb": _pp(0.5, 1),
        "slope": _pp(0.0), "quad": _pp(0.0), "cube": _pp(0.0), "third": _pp(0.0),
        "delta_phase": "1e-07", "nlat1f": "40", "nlat2f": "80", "nlat1c": "40", "nlat2c": "80",
        "npole": "1", "nlatfill": "0", "nlngfill": "0", "lfudge": "0", "llo": "0", "lhi": "0",
        "phase1": "0.05", "phase2": "0.45", "wavelength": "550", "roche1": "1", "roche2": "1",
        "eclipse1": "1", "eclipse2": "1", "glens1": "0", "use_radii": "1", "tperiod": "0.1",
        "gdark_bolom1": "1", "gdark_bolom2": "1", "mucrit1": "0", "mucrit2": "0",
        "limb1": "Claret", "limb2": "Claret", "mirror": "0", "add_disc": "0", "nrad": "40",
        "opaque": "0", "add_spot": "0", "nspot": "0", "iscale": "0",
    }
    for k in ("rdisc1", "rdisc2", "height_disc", "beta_disc", "temp_disc", "texp_disc",
              "lin_limb_disc", "quad_limb_disc", "temp_edge", "absorb_edge", "radius_spot",
              "length_spot", "height_spot", "expon_spot", "epow_spot", "angle_spot", "yaw_spot",
              "temp_spot", "tilt_spot", "cfrac_spot"):
        p[k] = _pp(0.0)
    return p


def model(**over):
    p = base_parameters()
    for k, v in over.items():
        if k in ("nlat1f", "nlat2f", "nlat1c", "nlat2c", "nlatfill", "nlngfill", "npole",
                 "roche1", "roche2", "eclipse1", "eclipse2", "glens1", "use_radii", "mirror",
                 "gdark_bolom1", "gdark_bolom2", "delta_phase", "phase1", "phase2", "wavelength",
                 "tperiod", "mucrit1", "mucrit2", "llo", "lhi", "lfudge", "add_disc", "opaque",
                 "add_spot", "iscale", "nrad", "nspot"):
            p[k] = str(v)
        elif k in ("limb1", "limb2"):
            p[k] = v
        else:
            p[k] = _pp(float(v), 1 if k in ("q", "iangle", "r1", "r2", "t1", "t2", "t0", "absorb") else 0)
    # keep coarse = fine unless given
    for s in ("1", "2"):
        if ("nlat%sf" % s) in over and ("nlat%sc" % s) not in over:
            p["nlat%sc" % s] = str(over["nlat%sf" % s])
    return Model({"model_parameters": p})


def times(n, lo=-0.2, hi=1.2):
    return np.linspace(lo, hi, n)


def data(n, lo=-0.2, hi=1.2, ndiv=1, expose=0.0):
    return make_data(times(n, lo, hi), expose=expose, flux=1.0, ferr=SIGMA, weight=1.0, ndiv=ndiv)


def add_noise(d, calc, seed):
    """flux = calc / median(calc) + sigma * N(0,1), from a seeded Generator."""
    rng = np.random.default_rng(seed)
    d = d.copy()
    d["flux"] = calc / np.median(calc) + SIGMA * rng.standard_normal(calc.shape[0])
    return d


def wd_dm_small():
    return model(), data(500)


def wd_dm_large():
    # ndiv 5 over one cadence of a 5000-point curve spanning 1.4 phases
    return model(nlat1f=200, nlat2f=800), data(5000, ndiv=5, expose=1.4 / 5000)


def tiny_star(r1=0.005, q=0.2, iangle=87.0):
    return (model(r1=r1, q=q, iangle=iangle, nlat1f=400, nlat2f=200),
            data(10000, lo=-0.03, hi=0.03))


def mcmc_batch(nmodels=256, seed=2024):
    """Models drawn around wd_dm_small: q~N(0.25,0.02), i~N(86,0.5),
    r1,r2 x N(1,0.05), T1,T2 x N(1,0.03); nlat2f ~ U{60..400}, nlat1f = nlat2f/2."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(nmodels):
        nl2 = int(rng.integers(60, 401))
        out.append(model(q=0.25 + 0.02 * rng.standard_normal(),
                         iangle=86.0 + 0.5 * rng.standard_normal(),
                         r1=0.015 * (1 + 0.05 * rng.standard_normal()),
                         r2=0.20 * (1 + 0.05 * rng.standard_normal()),
                         t1=20000.0 * (1 + 0.03 * rng.standard_normal()),
                         t2=3200.0 * (1 + 0.03 * rng.standard_normal()),
                         nlat1f=nl2 // 2, nlat2f=nl2))
    return out, data(2000)


CV_DISC = dict(q=0.15, iangle=84.0, r1=0.012, r2=0.25, t1=15000.0, t2=3000.0,
               add_disc=1, rdisc1=0.03, rdisc2=0.3, height_disc=0.02, beta_disc=1.3,
               temp_disc=8000.0, texp_disc=-0.8, lin_limb_disc=0.3, quad_limb_disc=0.1,
               temp_edge=6000.0, absorb_edge=0.5, nrad=40, opaque=1,
               add_spot=1, radius_spot=0.3, length_spot=0.02, height_spot=0.01,
               expon_spot=2.0, epow_spot=1.0, angle_spot=140.0, yaw_spot=10.0,
               temp_spot=12000.0, tilt_spot=60.0, cfrac_spot=0.2, nspot=50)


def cv_disc(**over):
    """A cataclysmic variable: q=0.15, i=84 deg, white dwarf r1=0.012,
    donor r2=0.25, flared opaque disc from 0.03 to 0.3 (height 0.02 r^1.3,
    T 8000 K r^-0.8, 40 radii) with its outer rim, and a 50-element bright
    spot where the stream meets r=0.3. Keyword arguments override any of
    these or the detached binary's parameters."""
    kw = dict(CV_DISC)
    kw.update(over)
    return model(**kw)


def _rings(nlat):
    """Ring count and spacing of a full star without infill: dtheta = pi / nlat
    and ceil(pi / dtheta) rings (numface.cpp:46-50, set_star_grid.cpp:249-250),
    one more than nlat where the quotient rounds above it."""
    dtheta = math.pi / nlat
    return int(math.ceil(math.pi / dtheta)), dtheta


def _numface(nlat):
    """Faces numface gives a full star without infill (numface.cpp:14-52)."""
    nl, dtheta = _rings(nlat)
    return sum(max(16, int(2 * math.pi / (dtheta / math.sin(math.pi * (i + 0.5) / nl))))
               for i in range(nl))


def _tiled(nlat):
    """Faces the ring tiling of add_faces lays on a full star without infill
    (set_star_grid.cpp:241-320): the same rings, nphi from 2 pi sin(theta) /
    dtheta, which rounds differently from numface's expression at a few nlat."""
    nl, dtheta = _rings(nlat)
    return sum(max(16, int(2 * math.pi * math.sin(math.pi * (i + 0.5) / nl) / dtheta))
               for i in range(nl))


def tiling_overflows(nlat):
    """True at the nlat (153, 297, 315, 333, 339, 549, ... up to 1200: 16
    values) where the ring tiling has more faces than numface, with which the
    reference sizes its Point vector: its add_faces then writes past the
    vector's end (set_star_grid.cpp:490,508), undefined behaviour that can
    corrupt the heap of the process running it. The engine keeps the numface
    faces the vector holds."""
    return _tiled(nlat) > _numface(nlat)


def reference_safe(m):
    """False for a model (without infill) whose fine or coarse grid of either
    star has an nlat at which the reference's grid build writes past its
    vector: such models are not run through the reference's own code."""
    c = m.to_c() if hasattr(m, "to_c") else m
    return not any(tiling_overflows(int(v)) for v in (c.nlat1f, c.nlat2f, c.nlat1c, c.nlat2c)
                   if v > 0)


def elements(nface1, nface2, nent):
    """Face x sub-phase pairs of one light curve (the flux roofline unit)."""
    return (nface1 + nface2) * nent
