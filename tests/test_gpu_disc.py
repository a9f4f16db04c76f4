"""Cataclysmic-variable components on the device against the C oracle.

The oracle is pinned to the reference's own set_disc_grid / set_disc_edge /
set_bright_spot_grid / disc_eclipse / iscale path (tests/test_oracle_pin.py).

Tolerances:
  * disc and rim elements: positions and normals within 1e-12 (device sin,
    cos and pow can differ from glibc by an ulp), float areas equal, float
    fluxes within 2 float ulps (4e-7), eclipse ranges within 1e-9 and their
    counts equal except for elements grazing an eclipser;
  * bright spot: the stream is integrated on the host by the engine and by
    the oracle with the same method, positions within 1e-9;
  * light curves: FP64 mode per-point relative error <= 1e-6, mixed mode
    <= 1e-5, chi**2 and the iscale factors within 1e-6 relative.
"""
import numpy as np
import pytest

from cases import disc_cases
from lcurve_re_b200 import workloads as W
from lcurve_re_b200.engine import Engine
from lcurve_re_b200.model import LcurveError

pytestmark = pytest.mark.gpu

CASES = disc_cases()
IDS = [c[0] for c in CASES]
BAND = 1e-9


@pytest.mark.parametrize("name,model,data", CASES, ids=IDS)
def test_component_grids(engine_fp64, oracle, name, model, data):
    for which in (0, 1, 2):
        if (which < 2 and not model["add_disc"]) or (which == 2 and not model["add_spot"]):
            continue
        st, err, go = oracle.components(model, which)
        assert st == 0, err
        gg = engine_fp64.components(model, which)
        assert gg["nr"].shape == go["nr"].shape, which
        tol = 1e-12 if which < 2 else 1e-9
        np.testing.assert_allclose(gg["posn"], go["posn"], rtol=0, atol=tol)
        np.testing.assert_allclose(gg["dirn"], go["dirn"], rtol=0, atol=tol)
        np.testing.assert_array_equal(gg["area"], go["area"])
        np.testing.assert_allclose(gg["flux"], go["flux"], rtol=4e-7, atol=0)
        same = gg["nr"] == go["nr"]
        assert same.mean() > 0.995, (which, same.mean())
        live = (np.arange(4)[None, :] < go["nr"][:, None]) & same[:, None]
        np.testing.assert_allclose(gg["rin"][live], go["rin"][live], rtol=0, atol=BAND)
        np.testing.assert_allclose(gg["rout"][live], go["rout"][live], rtol=0, atol=BAND)


def _curves(engine, oracle, model, data, scale):
    sf_in = [1.1, 0.9, 1.2, 0.8, 1.05]
    st, err, co, sfo, sco = oracle.light_curve(model, data, scale=scale, sfac=sf_in)
    assert st == 0, err
    sf = np.array(sf_in)
    calc, wd, chisq, wnok, *_ = engine.light_curve_comp(model, data, scale=scale, rdata=True,
                                                        sfac=sf, diagnostics=False)
    return co, sfo, sco, calc, sf, chisq


@pytest.mark.parametrize("name,model,data", CASES, ids=IDS)
def test_light_curve_fp64(engine_fp64, oracle, name, model, data):
    for scale in (True, False):
        co, sfo, sco, calc, sf, chisq = _curves(engine_fp64, oracle, model, data, scale)
        rel = np.abs(calc - co) / np.maximum(np.abs(co), 1e-300)
        assert rel.max() <= 1e-6, (name, scale, rel.max())
        np.testing.assert_allclose(sf, sfo, rtol=1e-6)
        np.testing.assert_allclose(chisq, sco[1], rtol=1e-6)


@pytest.mark.parametrize("name,model,data", CASES, ids=IDS)
def test_light_curve_mixed(engine_mixed, oracle, name, model, data):
    co, sfo, sco, calc, sf, chisq = _curves(engine_mixed, oracle, model, data, True)
    rel = np.abs(calc - co) / np.maximum(np.abs(co), 1e-300)
    assert rel.max() <= 1e-5, (name, rel.max())


def test_opaque_disc_at_benchmark_resolution(engine_fp64, engine_mixed, oracle):
    """An opaque disc at nlat 40/80: many star faces carry two or three
    eclipse ranges (the ragged segment of the flat grids, swept by
    k_flux_ragged after the main sweeps)."""
    m = W.cv_disc(nlat1f=40, nlat2f=80, nrad=30, nspot=40)
    d = W.data(400)
    d["flux"] = 1.0
    st, err, co, _, _ = oracle.light_curve(m, d, scale=False, rdata=False)
    assert st == 0, err
    for eng, tol in ((engine_fp64, 1e-6), (engine_mixed, 1e-5)):
        calc, *_ = eng.light_curve_comp(m, d, scale=False, rdata=False, sfac=np.ones(5),
                                        diagnostics=False)
        rel = np.abs(calc - co) / np.abs(co)
        assert rel.max() <= tol, rel.max()


def test_disc_then_plain_model_reuses_nothing_stale(oracle):
    """An opaque-disc model, then the same stars without a disc, in one
    context: the second result equals a fresh context's."""
    plain = W.model(nlat1f=16, nlat2f=24, q=0.15, iangle=84.0, r1=0.012, r2=0.25,
                    t1=15000.0, t2=3000.0)
    disc = W.cv_disc(nlat1f=16, nlat2f=24, nrad=12, nspot=10)
    d = W.data(120)
    with Engine(precision="fp64") as e1, Engine(precision="fp64") as e2:
        e1.light_curve_comp(disc, d, scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)
        a, *_ = e1.light_curve_comp(plain, d, scale=False, rdata=False, sfac=np.ones(5),
                                    diagnostics=False)
        b, *_ = e2.light_curve_comp(plain, d, scale=False, rdata=False, sfac=np.ones(5),
                                    diagnostics=False)
        assert np.array_equal(a, b)


def test_component_errors(engine_fp64, oracle):
    """Lobe overflow found by the disc setup and beta < 1 with an opaque
    disc: the oracle's status and message."""
    for over in ({"r1": 0.8, "r2": 0.05}, {"beta_disc": 0.5}):
        m = W.cv_disc(nlat1f=8, nlat2f=8, nrad=6, nspot=5, **over)
        st, err, *_ = oracle.light_curve(m, W.data(20))
        assert st != 0
        with pytest.raises(LcurveError) as ex:
            engine_fp64.light_curve_comp(m, W.data(20), sfac=np.ones(5))
        assert ex.value.status == st
        assert str(ex.value).startswith(err.split(":")[0])


def test_beamed_wdwarf_uses_spin_one(engine_fp64, oracle):
    """wdwarf is comp_star1_flat at phase 0.5, which beams with spin 1 even
    when spin1 differs (light_curve_comp.cpp:504-508)."""
    m = W.model(nlat1f=20, nlat2f=40, beam_factor1=1.5, spin1=1.4)
    d = W.data(100)
    _, _, _, _, sco = oracle.light_curve(m, d, diagnostics=True)
    _, wd, *_ = engine_fp64.light_curve_comp(m, d, sfac=np.ones(5), diagnostics=True)
    np.testing.assert_allclose(wd, sco[0], rtol=1e-9)


def test_batch_routes_disc_models_one_by_one(oracle):
    """A batch mixing detached binaries and disc models: the disc models go
    through the single-model path and agree with the oracle."""
    d = W.data(150)
    d["flux"] = 1.0
    ms = [W.model(nlat1f=16, nlat2f=24), W.cv_disc(nlat1f=16, nlat2f=24, nrad=12, nspot=10),
          W.cv_disc(nlat1f=16, nlat2f=24, nrad=12, nspot=10, iscale=1)]
    with Engine(precision="mixed") as e:
        e.set_data(d)
        sf = np.ones((len(ms), 5))
        calc, chisq, wnok, sf, st = e.light_curve_batch_resident(ms, scale=True, rdata=True,
                                                                 sfac=sf)
        assert np.all(st == 0)
        for k, m in enumerate(ms):
            s, err, co, sfo, sco = oracle.light_curve(m, d)
            assert s == 0, err
            rel = np.abs(calc[k] - co) / np.abs(co)
            assert rel.max() <= 1e-5, (k, rel.max())
