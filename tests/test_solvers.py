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


def test_jacobian_reproduces_the_reference_levmarq_covariance(reference, tmp_path):
    """Pinned to the reference itself: lcurve_levmarq (new_scripts/levmarq_solver.cpp,
    built unchanged over its CPU path by tests/solvers/Makefile) prints the 1-sigma
    uncertainties of the covariance of its own finite-difference Jacobian
    (covariance_at, :1880-1921: set_fd_steps, compute_jacobian with central
    differences, data block rescaled to reduced chi**2 = 1). The model sits where
    every branch of compute_jacobian runs: iangle at its upper bound 90 (one-sided,
    backward, with the reference's divisor), r2 a hair inside its Roche lobe
    (the +h steps fail: central retries halving, then one-sided halvings, then a
    backward step), q, r1 and t0 central. jacobian() evaluated through the same
    compiled reference reproduces the printed uncertainties."""
    import json
    import os
    import re
    import subprocess
    from lcurve_re_b200 import workloads as W
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "solvers", "_build", "ref",
                       "lcurve_levmarq")
    if not os.path.exists(exe):
        pytest.skip("reference executables not built (make -C tests/solvers)")
    d = W.data(200)
    lo, hi = 0.2, 0.4  # the largest r2 the reference accepts at q = 0.25, i = 90
    for _ in range(55):
        mid = 0.5 * (lo + hi)
        st = reference.light_curve(W.model(nlat1f=20, nlat2f=40, r2=mid, iangle=90.0), d,
                                   scale=False, rdata=False)[0]
        lo, hi = (mid, hi) if st == 0 else (lo, mid)
    r2 = lo - 1e-6
    m = W.model(nlat1f=20, nlat2f=40, r2=r2, iangle=90.0)
    st, err, calc, _, _ = reference.light_curve(m, d, scale=False, rdata=False)
    assert st == 0, err
    d = W.add_noise(d, calc, 5)
    p = W.base_parameters()
    p.update(nlat1f="20", nlat1c="20", nlat2f="40", nlat2c="40")
    p["r2"] = "%.17g 0.01 0.001 1 1" % r2
    p["iangle"] = "90 0.01 0.001 1 1"
    for k in ("t1", "t2", "absorb"):  # held fixed: five free parameters
        v = p[k].split()
        v[3] = "0"
        p[k] = " ".join(v)
    cfg = {"model_parameters": p, "data_file_path": "lc.txt", "noise": 0, "seed": 42,
           "output_file_path": "out.txt", "plot_device": "none", "autoscale": True,
           "sstar1": 1, "sstar2": 1, "sdisc": 1, "sspot": 1, "ssfac": 1, "use_priors": False,
           "lm_max_iter": 0, "lm_multistart": 0, "lm_error_mcmc": False,
           "lm_continuation": False, "lm_reanchor_rounds": 0, "lm_log_path": "lm.txt",
           "priors": {}}
    (tmp_path / "cfg.json").write_text(json.dumps(cfg))
    with open(tmp_path / "lc.txt", "w") as f:
        for r in d:
            f.write("%.17g %.17g %.17g %.17g %.17g %d\n" % (r["time"], r["expose"], r["flux"],
                                                           r["ferr"], r["weight"], r["ndiv"]))
    out = subprocess.run([exe, "cfg.json"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    text = re.sub(r"\x1b\[[0-9;]*m", "", out.stdout)
    lim = re.findall(r"^\s+(\w+): \S+\s+step \S+\s+limits \[(\S+), (\S+)\]$", text, re.M)
    names = [x[0] for x in lim]
    assert names == ["q", "iangle", "r1", "r2", "t0"]
    limits = [(float(a), float(b)) for _, a, b in lim]
    printed = dict((k, float(s)) for k, s in
                   re.findall(r"^\s+(\w+)\s+= \S+ ± (\S+)$", text, re.M))
    # set_fd_steps(pars, 1.0) (levmarq_solver.cpp:766-778) with the defaults
    # fd_step_rel = eps^(1/4), fd_step_min = 1e-10
    rel, hmin = np.finfo(float).eps ** 0.25, 1e-10
    pars = np.array([m[n] for n in names])
    span = np.array([b - a for a, b in limits])
    steps = rel * np.abs(pars) + hmin
    steps = np.where(np.isfinite(span) & (span > 0), np.minimum(steps, 0.5 * span), steps)
    steps = np.maximum(steps, hmin)

    def evaluate(models):
        rows, ok = [], []
        for mk in models:
            st, _, c, _, _ = reference.light_curve(mk, d, scale=True, rdata=True)
            rows.append(c)
            ok.append(st == 0 and np.all(np.isfinite(c)))
        return np.array(rows), np.array(ok)
    J = jacobian(evaluate, m, names, d, steps=steps, limits=limits, central=True)
    st, _, c0, _, _ = reference.light_curve(m, d, scale=True, rdata=True)
    r0 = residuals(c0, d)
    s2 = float(r0 @ r0) / max(1, d.shape[0] - len(names))
    Js = J / np.sqrt(s2)
    sigma = np.sqrt(np.diag(np.linalg.inv(Js.T @ Js)))
    for k, n in enumerate(names):
        assert abs(sigma[k] - printed[n]) <= 1e-5 * abs(sigma[k]) + 1e-6, (n, sigma[k], printed[n])
    # the correlations carry the column signs (the uncertainties do not): the
    # backward step at the iangle bound divides by +h in the reference
    block = text.split("Correlation matrix:")[1].splitlines()[2:2 + len(names)]
    corr_printed = np.array([[float(v) for v in row.split()[1:]] for row in block])
    cov = np.linalg.inv(Js.T @ Js)
    corr = cov / np.outer(sigma, sigma)
    np.testing.assert_allclose(corr, corr_printed, atol=0.0051)
    assert corr_printed[0, 1] != 0.0 and np.sign(corr[0, 1]) == np.sign(corr_printed[0, 1])
