"""Pins the C oracle (oracle/lcg_oracle.c) to the reference itself.

The reference's CPU path is compiled from its own sources into
oracle/_ref/liblcurve_ref.so (oracle/Makefile, -ffp-contract=off). Both are
driven with the same lcg_model and data; with the same libm the oracle must
reproduce the reference bit for bit: grids, eclipse phases, fluxes, the
light curve and chi**2. The only exception is wdwarf, which the reference
sums with an OpenMP SIMD reduction whose order is compiler-dependent.
"""
import numpy as np
import pytest

from cases import glens_case, small_cases

CASES = small_cases() + [glens_case()]


@pytest.mark.parametrize("name,model,data", CASES, ids=[c[0] for c in CASES])
def test_light_curve_bit_exact(oracle, reference, name, model, data):
    st_o, err_o, calc_o, sf_o, sc_o = oracle.light_curve(model, data)
    st_r, err_r, calc_r, sf_r, sc_r = reference.light_curve(model, data)
    assert st_o == st_r == 0, (err_o, err_r)
    assert np.array_equal(calc_o, calc_r)
    assert np.array_equal(sf_o, sf_r)
    assert sc_o[1] == sc_r[1] and sc_o[2] == sc_r[2]  # chisq, wnok


@pytest.mark.parametrize("name,model,data", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_diagnostics(oracle, reference, name, model, data):
    _, _, _, _, sc_o = oracle.light_curve(model, data, diagnostics=True)
    _, _, _, _, sc_r = reference.light_curve(model, data, diagnostics=True)
    np.testing.assert_allclose(sc_o[0], sc_r[0], rtol=1e-12)  # wdwarf: SIMD sum order
    np.testing.assert_array_equal(sc_o[3:], sc_r[3:])         # logg1, logg2, rv1, rv2


@pytest.mark.parametrize("name,model,data", CASES, ids=[c[0] for c in CASES])
def test_grids_bit_exact(oracle, reference, name, model, data):
    for star in (0, 1):
        for fine in (True, False):
            go = oracle.star_grid(model, star, fine)
            gr = reference.star_grid(model, star, fine)
            for k in go:
                assert np.array_equal(go[k], gr[k]), (star, fine, k)


def test_flux_sweep_bit_exact(oracle, reference):
    from lcurve_re_b200 import workloads as W
    m, d = W.wd_dm_small()
    ph = oracle.phase_batch(m, d)
    for star, ldc in ((0, m.to_c().ldc1), (1, m.to_c().ldc2)):
        flat = oracle.flatten(oracle.star_grid(m, star))
        for beam, glens in ((0.0, False), (1.5, False), (0.0, True), (0.7, True)):
            kw = dict(ldc=list(ldc), ltype=1, mucrit=0.0, beam=beam, spin=1.1, vfac=1e-3,
                      xcofm=0.2, glens1=glens, rlens1=2e-6)
            a = oracle.sum_star_multi(star, flat, ph, **kw)
            b = reference.sum_star_multi(star, flat, ph, **kw)
            assert np.array_equal(a, b), (star, beam, glens)


def test_errors_match(oracle, reference):
    from lcurve_re_b200 import workloads as W
    for over, code in (({"r2": 0.5}, 2), ({"r1": 0.9, "r2": 0.05}, 2)):
        m = W.model(nlat1f=8, nlat2f=8, **over)
        st_o, err_o, *_ = oracle.light_curve(m, W.data(20))
        st_r, err_r, *_ = reference.light_curve(m, W.data(20))
        assert st_o == st_r == code
        assert err_o == err_r


def test_short_tiling_ends_in_default_points(oracle, reference):
    """At nlat 813 the ring tiling has two faces fewer than numface: the
    reference's grid ends in two default Points (zero position, normal, area
    and flux, gravity 1, never eclipsed)."""
    from lcurve_re_b200 import workloads as W
    m = W.model(nlat1f=813, nlat2f=40, eclipse1=0)
    go = oracle.star_grid(m, 0)
    gr = reference.star_grid(m, 0)
    for k in go:
        assert np.array_equal(go[k], gr[k]), k
    assert np.all(go["area"][-2:] == 0) and np.all(go["gravity"][-2:] == 1)
    assert np.all(go["posn"][-2:] == 0) and np.all(go["flux"][-2:] == 0)


@pytest.mark.parametrize("npts,max_pts", [(500, 120), (2000, 37), (90, 200), (300, 2)])
def test_light_curve_fast_bit_exact(oracle, reference, npts, max_pts):
    """light_curve_comp_fast: subsample by index, interpolate in time,
    recompute chi**2 (light_curve_comp_fast.cpp:6-84)."""
    from lcurve_re_b200 import workloads as W
    m = W.model(nlat1f=16, nlat2f=24)
    d = W.data(npts, ndiv=2, expose=0.003)
    d["time"] = d["time"] + 0.0007 * np.sin(np.arange(npts))  # uneven spacing
    d["flux"] = 1.0 + 1e-3 * np.cos(np.arange(npts))
    d["weight"][5] = 0.0
    for scale, rdata in ((True, True), (False, True), (True, False)):
        a = oracle.light_curve_fast(m, d, max_pts, scale=scale, rdata=rdata)
        b = reference.light_curve_fast(m, d, max_pts, scale=scale, rdata=rdata)
        assert a[0] == b[0] == 0, (a[1], b[1])
        assert np.array_equal(a[2], b[2])
        assert np.array_equal(a[3], b[3])
        assert np.array_equal(a[4][:3], b[4][:3])


# ---- cataclysmic-variable components ------------------------------------------
from cases import disc_cases  # noqa: E402

DISC = disc_cases()


def _spot(model):
    return model["add_spot"] != 0


@pytest.mark.parametrize("name,model,data", DISC, ids=[c[0] for c in DISC])
def test_component_grids(oracle, reference, name, model, data):
    """Disc and rim elements (positions, normals, float areas and fluxes,
    every eclipse range) are bit-exact. The bright spot sits where the gas
    stream reaches radius_spot; the oracle integrates the stream with its
    own stepper, so spot positions agree to 1e-9 and everything derived from
    them to 1e-9 relative; its fluxes do not depend on the position."""
    for which in (0, 1, 2):
        if which < 2 and not model["add_disc"] or which == 2 and not _spot(model):
            continue
        a, b = oracle.components(model, which), reference.components(model, which)
        assert a[0] == b[0] == 0, (a[1], b[1])
        ga, gb = a[2], b[2]
        assert np.array_equal(ga["nr"], gb["nr"]), which
        live = np.arange(4)[None, :] < ga["nr"][:, None]
        if which < 2:
            for k in ("posn", "dirn", "area", "flux"):
                assert np.array_equal(ga[k], gb[k]), (which, k)
            assert np.array_equal(ga["rin"][live], gb["rin"][live])
            assert np.array_equal(ga["rout"][live], gb["rout"][live])
        else:
            np.testing.assert_allclose(ga["posn"], gb["posn"], rtol=0, atol=1e-9)
            np.testing.assert_allclose(ga["dirn"], gb["dirn"], rtol=0, atol=1e-9)
            assert np.array_equal(ga["area"], gb["area"])
            np.testing.assert_allclose(ga["flux"], gb["flux"], rtol=1e-6)
            np.testing.assert_allclose(ga["rin"][live], gb["rin"][live], rtol=0, atol=1e-8)


@pytest.mark.parametrize("name,model,data", DISC, ids=[c[0] for c in DISC])
def test_component_light_curves(oracle, reference, name, model, data):
    """Light curves with a disc, rim and opaque-disc eclipses are bit-exact;
    with a bright spot (stream integration) or iscale (the SVD differs:
    one-sided Jacobi here, the reference's svdcmp there) they agree to 1e-9
    relative, the fitted scale factors included."""
    exact = not _spot(model) and not model["iscale"]
    for scale in (True, False):
        kw = dict(scale=scale, sfac=[1.1, 0.9, 1.2, 0.8, 1.05])
        a, b = oracle.light_curve(model, data, **kw), reference.light_curve(model, data, **kw)
        assert a[0] == b[0] == 0, (a[1], b[1])
        if exact:
            assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])
            assert a[4][1] == b[4][1]
        else:
            np.testing.assert_allclose(a[2], b[2], rtol=1e-9, atol=0)
            np.testing.assert_allclose(a[3], b[3], rtol=1e-9, atol=0)
            np.testing.assert_allclose(a[4][1], b[4][1], rtol=1e-9)


def test_component_errors_match(oracle, reference):
    """Lobe-overflow and disc-geometry errors: same status and message."""
    from lcurve_re_b200 import workloads as W
    for over in ({"r1": 0.8, "r2": 0.05}, {"beta_disc": 0.5}):
        m = W.cv_disc(nlat1f=8, nlat2f=8, nrad=6, nspot=5, **over)
        a, b = oracle.light_curve(m, W.data(20)), reference.light_curve(m, W.data(20))
        assert a[0] == b[0] != 0
        assert a[1] == b[1]
