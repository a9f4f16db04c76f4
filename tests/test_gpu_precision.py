"""Precision stress of tiny hot stars (r1 in {0.002, 0.005, 0.01}, q in
0.05-0.5, i in 80-90 deg including grazing eclipses), points concentrated
within +-0.03 of primary eclipse: mixed-precision GPU vs FP64 GPU vs the C
oracle, per result.

Stated bounds, per point of the light curve (relative to the oracle):
  * FP64 GPU   <= 1e-6
  * mixed GPU  <= 1e-5
and per face, the eclipse flags of the FP64 and the mixed GPU grids equal the
oracle's at every sub-phase of the data except within 1e-9 phase of a
boundary (tests/eclipse_flags.py), ingress and egress within 1e-9.
Grids are nlat 160/80 here instead of the 400/200 of the full workload so
that the oracle finishes in seconds; the arithmetic per face and per
element is the same.
"""
import numpy as np
import pytest

from eclipse_flags import compare
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


@pytest.mark.parametrize("r1,q,iangle", CASES)
def test_tiny_star_eclipse_flags(engine_fp64, engine_mixed, oracle, r1, q, iangle):
    m = W.model(r1=r1, q=q, iangle=iangle, nlat1f=160, nlat2f=80)
    d = W.data(1500, lo=-0.03, hi=0.03)
    phin = oracle.phase_batch(m, d)["phin"]
    go = oracle.star_grid(m, 0)
    assert go["neclipse"].sum() > 0
    for engine in (engine_fp64, engine_mixed):
        f = compare(engine.star_grid(m, 0), go, phin, 1e-9)
        assert f["outside_band"] == 0, (engine.precision, f)
        assert f["max_abs_ingress_diff"] <= 1e-9, (engine.precision, f)
        assert f["max_abs_egress_diff"] <= 1e-9, (engine.precision, f)
