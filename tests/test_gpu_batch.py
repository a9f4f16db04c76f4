"""The batched engine (lcg_light_curve_batch / _resident) against the
single-model path and the C oracle.

Tolerances:
  * grids are bit-identical to the single-model path (same kernels, same
    ring tables), but the batch chunks each grid's flux sum differently, so
    light curves agree with the single-model mixed path to 2e-6 relative and
    with the FP64 oracle to 1e-5 relative (the mixed-mode bound);
  * chi**2 within 1e-5 relative of the single-model path;
  * repeated batches on one context, with the per-model exact-reuse cache
    skipping unchanged grids, are bit-identical to a fresh context.
"""
import numpy as np
import pytest

from lcurve_re_b200 import abi
from lcurve_re_b200 import workloads as W
from lcurve_re_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _models(k=10, seed=5, lo=16, hi=48):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        nl2 = int(rng.integers(lo, hi + 1))
        out.append(W.model(q=0.25 + 0.02 * rng.standard_normal(),
                           iangle=86.0 + 0.5 * rng.standard_normal(),
                           r1=0.015 * (1 + 0.05 * rng.standard_normal()),
                           r2=0.20 * (1 + 0.05 * rng.standard_normal()),
                           t1=20000.0 * (1 + 0.03 * rng.standard_normal()),
                           t2=3200.0 * (1 + 0.03 * rng.standard_normal()),
                           nlat1f=max(nl2 // 2, 4), nlat2f=nl2))
    return out


@pytest.fixture(scope="module")
def data():
    d = W.data(300, ndiv=3, expose=0.004)
    return W.add_noise(d, np.ones(d.shape[0]), 11)


def _rel(a, b):
    return np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))


def test_batch_matches_single_path_and_oracle(data, oracle):
    ms = _models()
    e = Engine(precision="mixed")
    try:
        calc, chisq, wnok, sf, st = e.light_curve_batch(ms, data)
        assert np.all(st == 0), st
        for i, m in enumerate(ms):
            s = np.ones(5)
            ref = e.light_curve_comp(m, data, sfac=s)
            assert _rel(calc[i], ref[0]) < 2e-6, i
            assert abs(chisq[i] - ref[2]) <= 1e-5 * abs(ref[2]), i
            assert wnok[i] == ref[3]
            assert np.allclose(sf[i], s, rtol=2e-6, atol=0)
        for i in (0, len(ms) - 1):
            o_st, err, o_calc, _, _ = oracle.light_curve(ms[i], data, scale=True, rdata=True)
            assert o_st == 0, err
            assert _rel(calc[i], o_calc) < 1e-5, i
    finally:
        e.close()


def test_batch_reuse_is_bit_identical_to_a_fresh_context(data):
    ms = _models(k=8, seed=9)
    e = Engine(precision="mixed")
    try:
        e.set_data(data)
        first = e.light_curve_batch_resident(ms)
        again = e.light_curve_batch_resident(ms)  # every grid reused
        assert np.array_equal(first[0], again[0]) and np.array_equal(first[1], again[1])
        # brightness change on some models, geometry change on others
        ms2 = list(ms)
        ms2[1] = W.model(**{**_kw(ms[1]), "t1": 21000.0})
        ms2[4] = W.model(**{**_kw(ms[4]), "absorb": 0.3})
        ms2[2] = W.model(**{**_kw(ms[2]), "q": 0.27})
        ms2[6] = W.model(**{**_kw(ms[6]), "iangle": 85.0})
        got = e.light_curve_batch_resident(ms2)
        f = Engine(precision="mixed")
        try:
            f.set_data(data)
            fresh = f.light_curve_batch_resident(ms2)
        finally:
            f.close()
        assert np.all(got[4] == 0) and np.all(fresh[4] == 0)
        assert np.array_equal(got[0], fresh[0])
        assert np.array_equal(got[1], fresh[1])
        for i in (0, 3, 5, 7):
            assert np.array_equal(got[0][i], first[0][i])
    finally:
        e.close()


def _kw(m):
    """Keyword arguments rebuilding a workloads.model (the fields varied here)."""
    c = m.to_c()
    return dict(q=c.q, iangle=c.iangle, r1=c.r1, r2=c.r2, t1=c.t1, t2=c.t2,
                nlat1f=c.nlat1f, nlat2f=c.nlat2f, absorb=c.absorb)


def test_batch_failures_and_fallback_models(data):
    ms = _models(k=6, seed=3)
    ms[2] = W.model(r2=0.5)                    # overfills its Roche lobe
    ms[3] = W.model(beam_factor1=1.2)          # beaming: the one-by-one path
    ms[4] = W.model(nlat1c=10, nlat2c=20)      # coarse grids: the one-by-one path
    e = Engine(precision="mixed")
    try:
        calc, chisq, wnok, sf, st = e.light_curve_batch(ms, data)
        assert st[2] == abi.E_LOBE and np.all(calc[2] == 0)
        for i in (0, 1, 3, 4, 5):
            assert st[i] == 0, (i, st)
            ref = e.light_curve_comp(ms[i], data, sfac=np.ones(5))
            assert _rel(calc[i], ref[0]) < 2e-6, i
    finally:
        e.close()


def test_batch_chisq_only_and_layout_change(data):
    ms = _models(k=5, seed=21)
    e = Engine(precision="mixed")
    try:
        e.set_data(data)
        full = e.light_curve_batch_resident(ms)
        only = e.light_curve_batch_resident(ms, calc=False)
        assert only[0] is None and np.array_equal(only[1], full[1])
        other = _models(k=7, seed=22, lo=20, hi=30)
        res = e.light_curve_batch_resident(other)
        assert np.all(res[4] == 0)
        f = Engine(precision="mixed")
        try:
            f.set_data(data)
            assert np.array_equal(f.light_curve_batch_resident(other)[0], res[0])
        finally:
            f.close()
    finally:
        e.close()


def test_batch_profiled_run_equals_graph_run(data):
    ms = _models(k=4, seed=33)
    e = Engine(precision="mixed")
    try:
        e.set_data(data)
        a = e.light_curve_batch_resident(ms)
        e.set_profiling(True)
        b = e.light_curve_batch_resident(ms)
        t = e.stage_times(reset=True)
        e.set_profiling(False)
        assert np.array_equal(a[0], b[0])
        assert t["flux"][1] >= 1
    finally:
        e.close()


def test_batch_on_fp64_context_runs_on_concurrent_workers(data, oracle):
    """An FP64 batch takes the single-model path on up to eight concurrent
    worker contexts: 12 models (the workers take several each) give exactly
    the curves and chi**2 of single calls on the same points, within 1e-6 of
    the oracle; a model outside its lobe keeps its own status; after new
    points the workers evaluate on those."""
    ms = _models(k=12, seed=41)
    bad = ms[5].copy()
    bad["r2"] = 0.9  # past the Roche lobe
    ms[5] = bad
    e = Engine(precision="fp64")
    try:
        for pts in (data, data[: len(data) // 2].copy()):
            calc, chisq, wnok, sf, st = e.light_curve_batch(ms, pts)
            assert st[5] != 0 and calc[5].max() == 0
            for i, m in enumerate(ms):
                if i == 5:
                    continue
                assert st[i] == 0
                one = e.light_curve_comp(m, pts, scale=True, rdata=True, sfac=np.ones(5),
                                         diagnostics=False)
                assert np.array_equal(calc[i], one[0]), i
                assert chisq[i] == one[2], i
                if pts is data and i < 3:
                    o_st, err, o_calc, _, _ = oracle.light_curve(m, pts, scale=True, rdata=True)
                    assert _rel(calc[i], o_calc) < 1e-6
    finally:
        e.close()


def test_batch_skips_models_that_did_not_change(data):
    """A model identical to the previous call's model in its position (on the
    same points) is not evaluated again: its previous results come back and
    no flux work is done for it."""
    ms = _models(k=6, seed=51)
    e = Engine(precision="mixed")
    try:
        e.set_data(data)
        first = e.light_curve_batch_resident(ms)
        e.flux_elements(reset=True)
        again = e.light_curve_batch_resident(ms)
        assert e.flux_elements(reset=True) == 0
        for k in range(4):
            assert np.array_equal(first[k], again[k])
        ms2 = list(ms)
        ms2[3] = W.model(**{**_kw(ms[3]), "t2": 3300.0})
        part = e.light_curve_batch_resident(ms2)
        nent = data.shape[0] * 3  # ndiv = 3
        faces = e.face_count(ms2[3], 0) + e.face_count(ms2[3], 1)
        assert e.flux_elements(reset=True) == faces * nent
        f = Engine(precision="mixed")
        try:
            f.set_data(data)
            fresh = f.light_curve_batch_resident(ms2)
        finally:
            f.close()
        assert np.array_equal(part[0], fresh[0]) and np.array_equal(part[1], fresh[1])
        # new points (same size) invalidate every stored result
        d2 = data.copy()
        d2["flux"] = d2["flux"] * 1.01
        e.set_data(d2)
        moved = e.light_curve_batch_resident(ms2)
        assert not np.array_equal(moved[1], part[1])
    finally:
        e.close()


def test_batch_curves_returns_the_rows_of_the_last_call(data):
    ms = _models(k=5, seed=61)
    e = Engine(precision="mixed")
    try:
        e.set_data(data)
        full = e.light_curve_batch_resident(ms)[0]
        assert np.array_equal(e.batch_curves([3, 0, 3]), full[[3, 0, 3]])
        e.light_curve_batch_resident(ms, calc=False)  # all reused: rows unchanged
        assert np.array_equal(e.batch_curves(np.arange(5)), full)
        with pytest.raises(Exception):
            e.batch_curves([5])
    finally:
        e.close()


def test_batch_eclipse_modes_are_bit_identical(data):
    """The batched eclipse's warp mode (one warp per candidate) and thread mode
    (pot_min per candidate, then the two bisections on a lane pair) give the
    same light curves bit for bit: the same midpoints and decisions."""
    ms = _models(k=12, seed=21, lo=24, hi=64)
    out = []
    for mode in (1 << 30, -1):
        with Engine(precision="mixed", eclipse_warp=mode) as e:
            calc, chisq, wnok, sf, st = e.light_curve_batch(ms, data)
            assert np.all(st == 0), st
            out.append((calc.copy(), chisq.copy()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
