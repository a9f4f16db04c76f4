"""Parity of the CUDA engine (through the C ABI) against the C oracle.

Tolerances:
  * FP64 flux sweep over the same FlatGrid and phases: bit-identical.
  * grids: positions/normals within 1e-12 relative (device sin/cos of the
    ring longitudes may differ from glibc by an ulp), float areas, gravities
    and fluxes within 2 float ulps (4e-7 relative).
  * eclipse flags identical at every sub-phase of the case's data except
    within 1e-9 phase of a boundary of either grid (tests/eclipse_flags.py);
    ingress/egress within 1e-9 where both grids see an eclipse.
  * light curves: FP64 mode per-point relative error <= 1e-6, mixed mode
    <= 1e-5; chi**2 within 1e-6 relative in FP64 mode.
"""
import numpy as np
import pytest

from cases import glens_case, small_cases
from eclipse_flags import compare
from lcurve_re_b200 import workloads as W
from lcurve_re_b200.model import LcurveError

pytestmark = pytest.mark.gpu

CASES = small_cases() + [glens_case()]
IDS = [c[0] for c in CASES]
BAND = 1e-9


def _noisy(oracle, model, data, seed=7):
    st, err, calc, _, _ = oracle.light_curve(model, data, scale=False, rdata=False)
    assert st == 0, err
    if not np.all(np.isfinite(calc)) or np.median(calc) == 0:
        return data
    return W.add_noise(data, calc, seed)


@pytest.mark.parametrize("star", [0, 1])
def test_face_counts(engine_mixed, oracle, star):
    for name, m, _ in CASES:
        for fine in (True, False):
            assert engine_mixed.face_count(m, star, fine) == oracle.face_count(m, star, fine), name


@pytest.mark.parametrize("name,model,data", CASES, ids=IDS)
def test_star_grid(engine_fp64, oracle, name, model, data):
    for star in (0, 1):
        go = oracle.star_grid(model, star)
        gg = engine_fp64.star_grid(model, star)
        np.testing.assert_allclose(gg["posn"], go["posn"], rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(gg["dirn"], go["dirn"], rtol=1e-12, atol=1e-14)
        for k in ("area", "gravity", "flux"):
            np.testing.assert_allclose(gg[k], go[k], rtol=4e-7, atol=0, err_msg=k)
        # flags identical at every sub-phase of the case's data except within
        # BAND of a boundary; ingress / egress within BAND where both eclipse
        f = compare(gg, go, oracle.phase_batch(model, data)["phin"], BAND)
        assert f["outside_band"] == 0, (name, star, f)
        assert f["max_abs_ingress_diff"] <= BAND, (name, star, f)
        assert f["max_abs_egress_diff"] <= BAND, (name, star, f)


def test_eclipse_warp_and_thread_modes_agree(oracle):
    """The warp-per-face bisection evaluates the same midpoints as the
    thread-per-face one: flags and phases are bit-identical, whichever the
    candidate count selects."""
    from lcurve_re_b200.engine import Engine
    warp = Engine(precision="fp64", eclipse_warp=1 << 30)
    thread = Engine(precision="fp64", eclipse_warp=-1)
    try:
        cases = [(n, m) for n, m, _ in CASES] + [("wd_dm_small", W.wd_dm_small()[0])]
        for name, m in cases:
            for star in (0, 1):
                a, b = warp.star_grid(m, star), thread.star_grid(m, star)
                for k in ("neclipse", "ecl_in", "ecl_out"):
                    assert np.array_equal(a[k], b[k]), (name, star, k)
    finally:
        warp.close()
        thread.close()


def test_eclipse_fp32_screen_keeps_the_fp64_decisions():
    """Mixed contexts screen the bisections' line-of-sight tests in FP32 and
    run the FP64 test only where the screen is unsure: eclipse flags and
    phases equal the FP64 context's bit for bit (thread mode, where the
    screen runs), on the parity cases and on batch models."""
    from lcurve_re_b200.engine import Engine
    fp64 = Engine(precision="fp64", eclipse_warp=-1)
    mixed = Engine(precision="mixed", eclipse_warp=-1)
    try:
        ms, _ = W.mcmc_batch(256)
        cases = [(n, m) for n, m, _ in CASES] + [("batch%d" % k, ms[k]) for k in range(0, 256, 16)]
        # a donor star beside a disc (FP32 screen on its faces) and a tiny white
        # dwarf (r1 < 0.01: its faces stay with the FP64 test alone)
        cases += [("cv_disc", W.cv_disc(nlat1f=40, nlat2f=80, nrad=12, nspot=10)),
                  ("tiny", W.model(r1=0.005, q=0.2, iangle=87.0, nlat1f=120, nlat2f=60))]
        for name, m in cases:
            for star in (0, 1):
                a, b = fp64.star_grid(m, star), mixed.star_grid(m, star)
                for k in ("neclipse", "ecl_in", "ecl_out"):
                    assert np.array_equal(a[k], b[k]), (name, star, k)
    finally:
        fp64.close()
        mixed.close()


def test_flux_fp64_bit_exact(engine_fp64, oracle):
    m, d = W.wd_dm_small()
    ph = oracle.phase_batch(m, W.data(700, ndiv=3, expose=0.002))
    for star, ldc in ((0, m.to_c().ldc1), (1, m.to_c().ldc2)):
        flat = oracle.flatten(oracle.star_grid(m, star))
        for beam, glens in ((0.0, False), (1.5, False), (0.0, True), (0.7, True)):
            kw = dict(ldc=list(ldc), ltype=1, mucrit=0.0, beam=beam, spin=1.1, vfac=1e-3,
                      xcofm=0.2, glens1=glens, rlens1=2e-6)
            a = oracle.sum_star_multi(star, flat, ph, **kw)
            b = engine_fp64.sum_star_multi(star, flat, ph, **kw)
            assert np.array_equal(a, b), (star, beam, glens, np.max(np.abs(a - b) / np.abs(a)))


def test_flux_mixed(engine_mixed, oracle):
    m, d = W.wd_dm_small()
    ph = oracle.phase_batch(m, W.data(700, ndiv=3, expose=0.002))
    for star, ldc in ((0, m.to_c().ldc1), (1, m.to_c().ldc2)):
        flat = oracle.flatten(oracle.star_grid(m, star))
        for ltype in (0, 1):
            a = oracle.sum_star_multi(star, flat, ph, ldc=list(ldc), ltype=ltype)
            b = engine_mixed.sum_star_multi(star, flat, ph, ldc=list(ldc), ltype=ltype)
            rel = np.abs(b - a) / np.max(np.abs(a))
            assert rel.max() < 1e-5, (star, ltype, rel.max())


@pytest.mark.parametrize("name,model,data", CASES, ids=IDS)
def test_light_curve_fp64(engine_fp64, oracle, name, model, data):
    d = _noisy(oracle, model, data)
    st, err, co, sfo, sco = oracle.light_curve(model, d)
    assert st == 0, err
    sf = np.ones(5)
    calc, wd, chisq, wnok, *_ = engine_fp64.light_curve_comp(model, d, scale=True, rdata=True,
                                                             sfac=sf, diagnostics=False)
    rel = np.abs(calc - co) / np.maximum(np.abs(co), 1e-300)
    assert rel.max() <= 1e-6, (name, rel.max())
    np.testing.assert_allclose(chisq, sco[1], rtol=1e-6)
    assert wnok == sco[2]
    np.testing.assert_allclose(sf, sfo, rtol=1e-6)


@pytest.mark.parametrize("name,model,data", CASES, ids=IDS)
def test_light_curve_mixed(engine_mixed, oracle, name, model, data):
    d = _noisy(oracle, model, data)
    st, err, co, sfo, sco = oracle.light_curve(model, d)
    assert st == 0, err
    calc, wd, chisq, wnok, *_ = engine_mixed.light_curve_comp(model, d, sfac=np.ones(5),
                                                              diagnostics=False)
    rel = np.abs(calc - co) / np.maximum(np.abs(co), 1e-300)
    assert rel.max() <= 1e-5, (name, rel.max())


def test_diagnostics(engine_fp64, oracle):
    m, d = W.wd_dm_small()
    d = _noisy(oracle, m, d)
    _, _, _, _, sco = oracle.light_curve(m, d, diagnostics=True)
    _, wd, chisq, wnok, logg1, logg2, rv1, rv2 = engine_fp64.light_curve_comp(
        m, d, sfac=np.ones(5), diagnostics=True)
    np.testing.assert_allclose([wd, logg1, logg2, rv1, rv2], sco[[0, 3, 4, 5, 6]], rtol=1e-9)


def test_no_scale_paths(engine_fp64, oracle):
    m, d = W.wd_dm_small()
    d = _noisy(oracle, m, d)
    for rdata in (True, False):
        sf_in = np.array([2.5, 1, 1, 1, 1.0])
        _, _, co, sfo, sco = oracle.light_curve(m, d, scale=False, rdata=rdata, sfac=sf_in)
        sf = sf_in.copy()
        calc, wd, chisq, wnok, *_ = engine_fp64.light_curve_comp(m, d, scale=False, rdata=rdata,
                                                                 sfac=sf, diagnostics=False)
        np.testing.assert_allclose(calc, co, rtol=1e-12)
        assert np.array_equal(sf, sf_in)
        if rdata:
            np.testing.assert_allclose(chisq, sco[1], rtol=1e-9)


def test_cache_reuse(engine_mixed):
    m, d = W.wd_dm_small()
    engine_mixed.set_profiling(True)
    engine_mixed.stage_times(reset=True)
    c1 = engine_mixed.light_curve_comp(m, d, diagnostics=False, no_cache=True)[0].copy()
    c2 = engine_mixed.light_curve_comp(m, d, diagnostics=False)[0].copy()
    assert np.array_equal(c1, c2)
    t = engine_mixed.stage_times(reset=True)
    assert t["grid"][1] == 2 and t["continuum"][1] == 2  # second call reused both
    m2 = m.copy()
    m2["t1"] = 21000.0  # continuum only
    engine_mixed.light_curve_comp(m2, d, diagnostics=False)
    t = engine_mixed.stage_times(reset=True)
    assert t["grid"][1] == 0 and t["continuum"][1] == 2
    engine_mixed.set_profiling(False)


def test_errors(engine_mixed):
    with pytest.raises(LcurveError, match="larger than its Roche lobe"):
        engine_mixed.light_curve_comp(W.model(nlat1f=8, nlat2f=8, r2=0.5), W.data(10))
    m = W.cv_disc(nlat1f=8, nlat2f=8, nrad=0)
    with pytest.raises(LcurveError) as ei:
        engine_mixed.light_curve_comp(m, W.data(10))
    assert ei.value.status == 1  # a disc needs nrad >= 1
    # a failure leaves the context usable
    calc = engine_mixed.light_curve_comp(W.model(nlat1f=8, nlat2f=8), W.data(10))[0]
    assert np.all(np.isfinite(calc))


def test_batch_equals_single(engine_mixed):
    # the batch chunks each grid's flux sum differently: 2e-6 (mixed mode)
    models, d = W.mcmc_batch(6, seed=3)
    models = [W.model(nlat1f=int(m["nlat1f"]) // 4 + 4, nlat2f=int(m["nlat2f"]) // 4 + 8,
                      q=m["q"], iangle=m["iangle"], r1=m["r1"], r2=m["r2"], t1=m["t1"],
                      t2=m["t2"]) for m in models]
    d = W.data(300)
    calc, chisq, wnok, sfac, status = engine_mixed.light_curve_batch(models, d)
    assert np.all(status == 0)
    for i, m in enumerate(models):
        c = engine_mixed.light_curve_comp(m, d, diagnostics=False, no_cache=True)[0]
        np.testing.assert_allclose(calc[i], c, rtol=2e-6)


def test_context_history_does_not_leak(oracle):
    """A context that has evaluated a larger grid gives a smaller one (with an
    odd face count, so the last face pair is half padding) the result of a
    fresh context, bit for bit."""
    from lcurve_re_b200.engine import Engine
    nl = next(k for k in range(17, 60) if oracle.face_count(W.model(nlat2f=k), 1) % 2)
    small = W.model(nlat1f=12, nlat2f=nl)
    big = W.model(nlat1f=40, nlat2f=90, nlat1c=20, nlat2c=45)
    d = W.data(200)
    for prec in ("mixed", "fp64"):
        fresh = Engine(precision=prec)
        used = Engine(precision=prec)
        try:
            a = fresh.light_curve_comp(small, d)[0]
            used.light_curve_comp(big, d)
            b = used.light_curve_comp(small, d)[0]
            assert np.array_equal(a, b), (prec, np.max(np.abs(a - b) / np.abs(a)))
        finally:
            fresh.close()
            used.close()


@pytest.mark.parametrize("over,star", [({"nlat1f": 20, "nlat2f": 153}, 1),
                                       ({"nlat1f": 813, "nlat2f": 40, "eclipse1": 0}, 0)],
                         ids=["tiling_long_153", "tiling_short_813"])
def test_tiling_mismatch_keeps_the_reference_face_count(engine_fp64, oracle, over, star):
    """numface and the ring tiling disagree by two faces at these nlat: the
    grid keeps numface faces, dropping the extra tiled faces (153) or ending
    in default Points (813), as the reference's vector does."""
    m = W.model(**over)
    go = oracle.star_grid(m, star)
    gg = engine_fp64.star_grid(m, star)
    assert gg["posn"].shape == go["posn"].shape
    np.testing.assert_allclose(gg["posn"], go["posn"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(gg["dirn"], go["dirn"], rtol=1e-12, atol=1e-14)
    for k in ("area", "gravity", "flux"):
        np.testing.assert_allclose(gg[k], go[k], rtol=4e-7, atol=0, err_msg=k)
    d = W.data(100)
    st, err, co, _, _ = oracle.light_curve(m, d)
    assert st == 0, err
    calc = engine_fp64.light_curve_comp(m, d, sfac=np.ones(5), diagnostics=False)[0]
    assert np.max(np.abs(calc - co) / np.abs(co)) <= 1e-6


@pytest.mark.parametrize("npts,max_pts", [(500, 120), (2000, 37), (90, 200), (300, 2)])
def test_light_curve_fast(engine_fp64, engine_mixed, oracle, npts, max_pts):
    """light_curve_comp_fast on the device against the oracle (which is pinned
    bit for bit to the reference's own function): FP64 1e-6, mixed 1e-5."""
    m = W.model(nlat1f=16, nlat2f=24)
    d = W.data(npts, ndiv=2, expose=0.003)
    d["time"] = d["time"] + 0.0007 * np.sin(np.arange(npts))
    d["flux"] = 1.0 + 1e-3 * np.cos(np.arange(npts))
    d["weight"][5] = 0.0
    for eng, tol in ((engine_fp64, 1e-6), (engine_mixed, 1e-5)):
        for scale, rdata in ((True, True), (False, True)):
            st, err, co, sfo, sco = oracle.light_curve_fast(m, d, max_pts, scale=scale,
                                                            rdata=rdata)
            assert st == 0, err
            sf = np.ones(5)
            calc, chisq, wnok = eng.light_curve_comp_fast(m, d, max_pts, scale=scale,
                                                          rdata=rdata, sfac=sf)
            assert np.max(np.abs(calc - co) / np.abs(co)) <= tol
            np.testing.assert_allclose(chisq, sco[1], rtol=100 * tol)
            assert wnok == sco[2]
            np.testing.assert_allclose(sf, sfo, rtol=tol)
