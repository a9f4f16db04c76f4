"""The batched finite-difference Jacobian (lcurve_re_b200.solvers) follows
levmarq_solver's compute_jacobian (new_scripts/levmarq_solver.cpp:789-886):
checked on CPU with an analytic stand-in for the light curve, then with the C
oracle as the evaluator."""
import numpy as np
import pytest

from lcurve_re_b200.model import make_data
from lcurve_re_b200.solvers import jacobian, residuals


class FakeModel(dict):
    def copy(self):
        return FakeModel(self)


def _data(n=40):
    t = np.linspace(0.0, 1.0, n)
    d = make_data(t, flux=1.0 + 0.1 * t, ferr=0.01, weight=1.0)
    d["ferr"][3] = 0.0      # sigma fallback 1e-10
    d["weight"][5] = 0.0    # weight fallback 1
    return d


def _curve(m, t):
    return m["a"] * np.sin(t) + m["b"] * t ** 2 + np.exp(0.1 * m["c"] * t)


def _evaluator(t, fail=lambda m: False, calls=None):
    def ev(models):
        if calls is not None:
            calls.append(len(models))
        calc = np.array([_curve(m, t) for m in models])
        ok = np.array([not fail(m) for m in models])
        return calc, ok
    return ev


def test_residuals_follow_the_reference_fallbacks():
    d = _data()
    r = residuals(np.zeros(len(d)), d)
    assert r[3] == d["flux"][3] / 1e-10
    assert r[5] == d["flux"][5] / d["ferr"][5]


def test_central_differences_in_one_batch():
    d = _data()
    t = d["time"]
    m = FakeModel(a=1.3, b=-0.4, c=2.0)
    calls = []
    J = jacobian(_evaluator(t, calls=calls), m, ["a", "b", "c"], d)
    assert calls == [6]  # 2 x npar models, one call
    exact = -np.stack([np.sin(t), t ** 2, 0.1 * t * np.exp(0.1 * m["c"] * t)], 1)
    scale = (residuals(np.zeros(len(d)), d) / d["flux"])[:, None]  # sqrt(w)/sigma
    np.testing.assert_allclose(J, exact * scale, rtol=1e-6, atol=1e-6 * np.abs(exact * scale).max())


def test_bounds_give_one_sided_steps():
    d = _data()
    t = d["time"]
    m = FakeModel(a=1.0, b=0.5, c=2.0)
    h = np.array([0.01, 0.01, 0.01])
    # a at its upper bound: backward; b with both sides out: half the range, forward
    lim = [(0.0, 1.0), (0.499, 0.501), (-5.0, 5.0)]
    r0 = residuals(_curve(m, t), d)
    J = jacobian(_evaluator(t), m, ["a", "b", "c"], d, steps=h, limits=lim, resid0=r0)
    # the backward step keeps the reference's divisor sign * (p' - p) = +h
    # (levmarq_solver.cpp:843-849), so this column is the derivative's negative
    ma = m.copy(); ma["a"] = 1.0 - 0.01
    np.testing.assert_allclose(J[:, 0], (residuals(_curve(ma, t), d) - r0) / (-(ma["a"] - 1.0)))
    mb = m.copy(); mb["b"] = 0.5 + 0.5 * (0.501 - 0.499)
    np.testing.assert_allclose(J[:, 1], (residuals(_curve(mb, t), d) - r0) / (mb["b"] - 0.5))


def test_failed_steps_are_halved_then_one_sided():
    d = _data()
    t = d["time"]
    m = FakeModel(a=1.0, b=0.5, c=2.0)
    h = np.full(3, 0.08)
    # every model with a moved by more than 0.015 fails: central 0.08, 0.04, 0.02
    # fail, 0.01 succeeds on the 4th attempt
    fail = lambda mm: abs(mm["a"] - 1.0) > 0.015
    J = jacobian(_evaluator(t, fail), m, ["a", "b", "c"], d, steps=h)
    mp, mm_ = m.copy(), m.copy()
    mp["a"], mm_["a"] = 1.01, 0.99
    ref = (residuals(_curve(mp, t), d) - residuals(_curve(mm_, t), d)) / 0.02
    np.testing.assert_allclose(J[:, 0], ref, rtol=1e-9)
    # a column whose every evaluation fails stays zero
    J2 = jacobian(_evaluator(t, lambda mm: mm["c"] != 2.0), m, ["a", "b", "c"], d, steps=h)
    assert np.all(J2[:, 2] == 0.0) and np.any(J2[:, 0] != 0.0)


def test_with_the_oracle_as_evaluator(oracle):
    from lcurve_re_b200 import workloads as W
    m = W.model(nlat1f=12, nlat2f=20)
    d = W.data(60)
    d["flux"] = 1.0

    def ev(models):
        out, ok = [], []
        for mm in models:
            st, err, calc, sf, sc = oracle.light_curve(mm, d)
            out.append(calc)
            ok.append(st == 0 and np.all(np.isfinite(calc)))
        return np.array(out), np.array(ok)
    J = jacobian(ev, m, ["q", "iangle", "t1"], d)
    assert J.shape == (60, 3) and np.all(np.isfinite(J)) and np.all(np.abs(J).max(0) > 0)
