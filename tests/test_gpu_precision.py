"""Precision stress of tiny hot stars (r1 in {0.002, 0.005, 0.01}, q in
0.05-0.5, i in 80-90 deg including grazing eclipses), points concentrated
within +-0.03 of primary eclipse: mixed-precision GPU vs FP64 GPU vs the C
oracle, per result.

Stated bounds, per point of the light curve (relative to the oracle):
  * FP64 GPU   <= 1e-6
  * mixed GPU  <= 1e-5
and per face, eclipse flags of the FP64 GPU grid equal the oracle's except
for faces whose eclipse interval is narrower than 1e-6 in phase (grazing
faces, where the boundary roots sit within delta_phase of each other).
Grids are nlat 160/80 here instead of the 400/200 of the full workload so
that the oracle finishes in seconds; the arithmetic per face and per
element is the same.
"""
import numpy as np
import pytest

from lcurve_re_b200 import workloads as W

pytestmark = pytest.mark.gpu

CASES = [
    # (r1, q, iangle)
    (0.002, 0.05, 89.5),
    (0.005, 0.20, 87.0),
    (0.010, 0.50, 84.0),
    (0.005, 0.10, 80.0),   # grazing: the primary's limb only is covered
    (0.002, 0.35, 82.5),
    (0.010, 0.15, 90.0),
]


def _errors(engine, oracle, m, d):
    st, err, o_calc, _, o_sc = oracle.light_curve(m, d, scale=False, rdata=False)
    assert st == 0, err
    g = engine.light_curve_comp(m, d, scale=False, rdata=False, sfac=np.ones(5))[0]
    return np.max(np.abs(g - o_calc) / np.abs(o_calc))


@pytest.mark.parametrize("r1,q,iangle", CASES)
def test_tiny_star_precision(engine_fp64, engine_mixed, oracle, r1, q, iangle):
    m = W.model(r1=r1, q=q, iangle=iangle, nlat1f=160, nlat2f=80)
    d = W.data(1500, lo=-0.03, hi=0.03)
    e64 = _errors(engine_fp64, oracle, m, d)
    emx = _errors(engine_mixed, oracle, m, d)
    assert e64 <= 1e-6, e64
    assert emx <= 1e-5, emx


@pytest.mark.parametrize("r1,q,iangle", CASES[:3])
def test_tiny_star_eclipse_flags(engine_fp64, oracle, r1, q, iangle):
    m = W.model(r1=r1, q=q, iangle=iangle, nlat1f=160, nlat2f=80)
    go = oracle.star_grid(m, 0)
    gg = engine_fp64.star_grid(m, 0)
    ne_o, ne_g = go["neclipse"], gg["neclipse"]
    assert ne_o.sum() > 0
    diff = ne_o != ne_g
    width = np.where(ne_o == 1, go["ecl_out"] - go["ecl_in"], gg["ecl_out"] - gg["ecl_in"])
    assert np.all(width[diff] < 1e-6), int(diff.sum())
    both = (ne_o == 1) & (ne_g == 1)
    assert np.max(np.abs(gg["ecl_in"][both] - go["ecl_in"][both])) <= 1e-9
    assert np.max(np.abs(gg["ecl_out"][both] - go["ecl_out"][both])) <= 1e-9
