"""Parity at the benchmark configurations' own sizes, through the C ABI.

The checker is lcurve_re's own FP64 CPU path, compiled from its sources
(oracle/_ref/liblcurve_ref.so, OpenMP over the host cores): the same
light_curve_comp (light_curve_comp.cpp:119-599) and set_star_grid
(set_star_grid.cpp:49-224) on identical inputs. For the five batch models
whose nlat makes the reference's ring tiling write past its own Point vector
(nlat 153, 297, 315, 333, 339: undefined behaviour in the reference, which
must not run inside the test process) the checker is the C oracle, which is
pinned bit-exact to the reference wherever the reference is defined.

Configurations:
  * wd_dm_large: nlat 200/800 (50,872 + 814,520 faces), 5000 points x
    ndiv 5 (25,000 sub-phases), exposure 1.4/5000: the workload bench.py
    times, in mixed and FP64 mode;
  * tiny stars: nlat 400/200 (203,560 + 50,872 faces), 10,000 points in
    +-0.03 around primary eclipse, r1 in {0.002, 0.005, 0.01} and a grazing
    case, mixed and FP64;
  * eight batch models drawn as the 256-model batch draws them, at nlat2f
    60, 153, 211, 297, 315, 333, 339 and 400 (nlat1f = nlat2f / 2), 2000
    points, through lcg_light_curve_batch (mixed) and one by one in FP64.

Bars: per-point relative flux error <= 1e-6 in FP64 mode and
<= 1e-5 in mixed mode; chi**2 (re_scale'd, on noisy data) within 1e-6
relative in FP64 mode and within MIXED_CHI2 relative in mixed mode; per-face
eclipse flags identical at every sub-phase of the workload except within
1e-9 phase of a boundary (tests/eclipse_flags.py), ingress and egress within
1e-9 where both see an eclipse.

With LCG_PARITY_REPORT set to a file name, every case appends its measured
figures to that file as one JSON line.
"""
import json
import os

import numpy as np
import pytest

from eclipse_flags import compare
from lcurve_re_b200 import workloads as W

pytestmark = pytest.mark.gpu

BAND = 1e-9
MIXED_CHI2 = 1e-5
REPORT = os.environ.get("LCG_PARITY_REPORT")
OVERFLOWING_NLAT = (153, 297, 315, 333, 339)


def _report(case, **kw):
    if REPORT:
        with open(REPORT, "a") as f:
            f.write(json.dumps(dict(case=case, **kw)) + "\n")


def _max_rel(a, b):
    return float(np.max(np.abs(a - b) / np.abs(b)))


class _Checked:
    """One model and its points, with the checker's unscaled curve, noisy
    data made from it and the checker's re_scale'd chi**2 on that data."""

    def __init__(self, checker, model, data, seed=1234):
        st, err, calc, _, _ = checker.light_curve(model, data, scale=False, rdata=False)
        assert st == 0, err
        self.model, self.calc = model, calc
        self.noisy = W.add_noise(data, calc, seed)
        st, err, _, sfac, sc = checker.light_curve(model, self.noisy, scale=True, rdata=True)
        assert st == 0, err
        self.chisq, self.sfac = sc[1], sfac


def _engine_errors(engine, c):
    calc = engine.light_curve_comp(c.model, c.noisy, scale=False, rdata=False, sfac=np.ones(5),
                                   diagnostics=False)[0]
    sf = np.ones(5)
    chisq = engine.light_curve_comp(c.model, c.noisy, scale=True, rdata=True, sfac=sf,
                                    diagnostics=False)[2]
    return _max_rel(calc, c.calc), abs(chisq - c.chisq) / abs(c.chisq)


def _flags(engine, checker, oracle, model, data, star):
    phin = oracle.phase_batch(model, data)["phin"]
    return compare(engine.star_grid(model, star), checker.star_grid(model, star), phin, BAND)


def _assert_flags(f, what):
    assert f["outside_band"] == 0, (what, f)
    assert f["max_abs_ingress_diff"] <= BAND and f["max_abs_egress_diff"] <= BAND, (what, f)


# ---- wd_dm_large (the benchmarked workload) -----------------------------------------------
@pytest.fixture(scope="module")
def large(reference):
    m, d = W.wd_dm_large()
    return _Checked(reference, m, d)


@pytest.mark.parametrize("precision,bar", [("mixed", 1e-5), ("fp64", 1e-6)])
def test_wd_dm_large_light_curve(large, engine_mixed, engine_fp64, precision, bar):
    engine = engine_mixed if precision == "mixed" else engine_fp64
    rel, chi = _engine_errors(engine, large)
    _report("wd_dm_large", precision=precision, max_rel_flux=rel, chi2_rel=chi,
            points=len(large.calc))
    assert rel <= bar, rel
    assert chi <= (1e-6 if precision == "fp64" else MIXED_CHI2), chi


@pytest.mark.parametrize("star", [0, 1])
def test_wd_dm_large_eclipse_flags(engine_mixed, reference, oracle, star):
    m, d = W.wd_dm_large()
    f = _flags(engine_mixed, reference, oracle, m, d, star)
    _report("wd_dm_large", star=star, flags=f)
    _assert_flags(f, star)


# ---- tiny stars ---------------------------------------------------------------------------
TINY = [(0.002, 0.05, 89.5), (0.005, 0.20, 87.0), (0.010, 0.50, 84.0), (0.005, 0.10, 80.0)]


@pytest.mark.parametrize("r1,q,iangle", TINY)
def test_tiny_star_full_size(engine_mixed, engine_fp64, reference, oracle, r1, q, iangle):
    m, d = W.tiny_star(r1=r1, q=q, iangle=iangle)
    c = _Checked(reference, m, d)
    rel64, chi64 = _engine_errors(engine_fp64, c)
    relmx, chimx = _engine_errors(engine_mixed, c)
    f = _flags(engine_mixed, reference, oracle, m, d, 0)
    _report("tiny_star r1=%g q=%g i=%g" % (r1, q, iangle), fp64_max_rel_flux=rel64,
            fp64_chi2_rel=chi64, mixed_max_rel_flux=relmx, mixed_chi2_rel=chimx, flags_star1=f)
    assert rel64 <= 1e-6 and chi64 <= 1e-6, (rel64, chi64)
    assert relmx <= 1e-5 and chimx <= MIXED_CHI2, (relmx, chimx)
    assert f["eclipsed_faces_ref"] > 0
    _assert_flags(f, "star 1")


# ---- the 256-model batch's models at full size ----------------------------------------------
BATCH_NLAT = (60, 153, 211, 297, 315, 333, 339, 400)


def _batch_models():
    drawn, d = W.mcmc_batch(len(BATCH_NLAT))
    out = []
    for m, nl in zip(drawn, BATCH_NLAT):
        c = m.to_c()
        out.append(W.model(q=c.q, iangle=c.iangle, r1=c.r1, r2=c.r2, t1=c.t1, t2=c.t2,
                           nlat1f=nl // 2, nlat2f=nl))
    return out, d


@pytest.fixture(scope="module")
def batch_checked(reference, oracle):
    ms, d = _batch_models()
    out = []
    for m, nl in zip(ms, BATCH_NLAT):
        checker = reference if W.reference_safe(m) else oracle
        assert (checker is oracle) == (nl in OVERFLOWING_NLAT)
        out.append((nl, checker, _Checked(checker, m, d)))
    return out


def test_batch_models_full_size_mixed_batch(engine_mixed, batch_checked):
    """All eight through one lcg_light_curve_batch call (the batched engine's
    graph, slot layout and autotuned flux plan), unscaled and on noisy data."""
    ms = [c.model for _, _, c in batch_checked]
    data = batch_checked[0][2].noisy
    for c in batch_checked[1:]:
        assert np.array_equal(c[2].noisy["time"], data["time"])
    calc, _, _, _, status = engine_mixed.light_curve_batch(ms, data, scale=False, rdata=False)
    assert np.all(status == 0), status
    # chi**2 per model on its own noisy data: one batch call per model's data
    for k, (nl, _, c) in enumerate(batch_checked):
        rel = _max_rel(calc[k], c.calc)
        _, chisq, _, _, st = engine_mixed.light_curve_batch([c.model], c.noisy)
        chi = abs(chisq[0] - c.chisq) / abs(c.chisq)
        _report("batch nlat2f=%d" % nl, precision="mixed (batch)", max_rel_flux=rel,
                chi2_rel=chi)
        assert st[0] == 0
        assert rel <= 1e-5, (nl, rel)
        assert chi <= MIXED_CHI2, (nl, chi)


def test_batch_models_full_size_fp64(engine_fp64, batch_checked):
    for nl, _, c in batch_checked:
        rel, chi = _engine_errors(engine_fp64, c)
        _report("batch nlat2f=%d" % nl, precision="fp64", max_rel_flux=rel, chi2_rel=chi)
        assert rel <= 1e-6 and chi <= 1e-6, (nl, rel, chi)


@pytest.mark.parametrize("star", [0, 1])
def test_batch_models_full_size_eclipse_flags(engine_mixed, batch_checked, oracle, star):
    for nl, checker, c in batch_checked:
        f = _flags(engine_mixed, checker, oracle, c.model, c.noisy, star)
        _report("batch nlat2f=%d" % nl, star=star, flags=f)
        _assert_flags(f, (nl, star))
