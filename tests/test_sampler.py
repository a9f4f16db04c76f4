"""The samplers and the ESS estimator on CPU, with analytic likelihoods.

ess_geyer is checked against a literal port of the reference's loop
(new_scripts/mcmc_solver.cpp:80-115). Plain and delayed-acceptance
Metropolis must both sample a known Gaussian posterior; delayed acceptance,
screened by a deliberately wrong surrogate (shifted and too wide), must
still sample the exact posterior while calling the exact model less often.
"""
import numpy as np

from lcurve_re_b200.sampler import delayed_acceptance, ess_geyer, ess_total, metropolis


def _ess_loop(x):
    # the reference's estimator, loop for loop
    n = len(x)
    mean = sum(x) / n
    c0 = sum((xi - mean) ** 2 for xi in x) / n
    tau = 1.0
    for lag in range(1, min(n // 2, 10000), 2):
        r1 = sum((x[i] - mean) * (x[i + lag] - mean) for i in range(n - lag)) / (n * c0)
        r2 = 0.0
        if lag + 1 < n:
            r2 = sum((x[i] - mean) * (x[i + lag + 1] - mean) for i in range(n - lag - 1)) / (n * c0)
        if r1 + r2 < 0.0:
            break
        tau += 2.0 * (r1 + r2)
    return n / max(tau, 1.0)


def _ar1(n, phi, seed):
    rng = np.random.default_rng(seed)
    x = np.empty(n)
    x[0] = rng.standard_normal()
    for i in range(1, n):
        x[i] = phi * x[i - 1] + np.sqrt(1 - phi * phi) * rng.standard_normal()
    return x


def test_ess_matches_the_reference_loop():
    for phi, seed in ((0.0, 1), (0.5, 2), (0.9, 3)):
        x = _ar1(400, phi, seed)
        assert abs(ess_geyer(x) - _ess_loop(list(x))) <= 1e-9 * _ess_loop(list(x))
    assert ess_geyer(np.ones(10)) == 10.0 and ess_geyer(np.arange(3.0)) == 3.0


def test_ess_of_ar1_series():
    n = 20000
    for phi in (0.0, 0.8):
        x = _ar1(n, phi, 7)
        expect = n * (1 - phi) / (1 + phi)
        assert abs(ess_geyer(x) - expect) < 0.25 * expect


MU = np.array([1.0, -2.0])
SIG = np.array([0.5, 2.0])


def _chi_exact(calls):
    # counts the rows that changed since the previous call: the batched
    # engine evaluates only those
    last = [None]

    def f(t):
        calls[0] += t.shape[0] if last[0] is None else int(np.any(t != last[0], axis=1).sum())
        last[0] = t.copy()
        return np.sum(((t - MU) / SIG) ** 2, axis=1)
    return f


def _chi_sur(t):  # wrong on purpose: shifted and too wide
    return np.sum(((t - MU - 0.3 * SIG) / (1.5 * SIG)) ** 2, axis=1)


def _everywhere(t):
    return np.ones(t.shape[0], bool)


def test_plain_and_delayed_acceptance_sample_the_posterior():
    chains, steps = 64, 3000
    theta0 = MU + SIG * np.random.default_rng(0).standard_normal((chains, 2))
    cov = np.diag((1.5 * SIG) ** 2)
    n_plain, n_da = [0], [0]
    ch, *_ = metropolis(_chi_exact(n_plain), theta0, cov, steps, seed=1, box_check=_everywhere)
    cd, _, _, acc, _, st = delayed_acceptance(_chi_exact(n_da), _chi_sur, theta0, cov, steps,
                                              seed=2, box_check=_everywhere)
    for c in (ch, cd):
        s = c[steps // 5:].reshape(-1, 2)
        assert np.all(np.abs(s.mean(axis=0) - MU) < 0.05 * SIG)
        assert np.all(np.abs(s.std(axis=0) / SIG - 1) < 0.05)
    assert n_da[0] < 0.8 * n_plain[0]
    assert 0 < st["stage2_rate"] <= 1 and 0 < acc < 1
    ess, per = ess_total(ch[steps // 5:])
    assert 0 < ess <= per.max()


class _AnchoredFake:
    """An anchored approximation for a 2-vector 'curve' c(t) = t: the curve at
    y predicted from the exact curve at x as exact(x) * s(y) / s(x), with a
    surrogate s that is off by a smooth factor."""

    def state(self, t):
        return np.asarray(t, np.float64) * (1.0 + 0.05 * np.sin(t)) + 5.0

    def chi2(self, sy, sx, anchor):
        c = (np.asarray(anchor) + 5.0) * sy / sx - 5.0
        return np.sum(((c - MU) / SIG) ** 2, axis=1)


class _CurveExact:
    def __init__(self):
        self.curves = None
        self.evals = 0
        self._last = None

    def __call__(self, t):
        t = np.asarray(t, np.float64)
        self.evals += t.shape[0] if self._last is None else int(np.any(t != self._last, 1).sum())
        self._last = t.copy()
        self.curves = t.copy()
        return np.sum(((t - MU) / SIG) ** 2, axis=1)

    def curves_of(self, rows):
        return self.curves[rows]


def test_anchored_delayed_acceptance_samples_the_posterior():
    chains, steps = 64, 3000
    theta0 = MU + SIG * np.random.default_rng(3).standard_normal((chains, 2))
    cov = np.diag((1.2 * SIG) ** 2)
    ex = _CurveExact()
    cd, _, _, acc, _, st = delayed_acceptance(ex, _AnchoredFake(), theta0, cov, steps, seed=4,
                                              box_check=_everywhere)
    s = cd[steps // 5:].reshape(-1, 2)
    assert np.all(np.abs(s.mean(axis=0) - MU) < 0.05 * SIG)
    assert np.all(np.abs(s.std(axis=0) / SIG - 1) < 0.05)
    assert st["stage2_rate"] > 0.5 and ex.evals < chains * steps


def test_between_chain_ess_matches_geyer_on_ar1_chains():
    """For AR(1) chains started in stationarity both estimators recover the
    known ESS n (1 - a) / (1 + a)."""
    from lcurve_re_b200.sampler import ess_between_chains, ess_total
    rng = np.random.default_rng(3)
    a, n, nc = 0.9, 4000, 400
    x = np.empty((n, nc, 2))
    x[0] = rng.standard_normal((nc, 2))
    for t in range(1, n):
        x[t] = a * x[t - 1] + np.sqrt(1 - a * a) * rng.standard_normal((nc, 2))
    want = nc * n * (1 - a) / (1 + a)
    g, _ = ess_total(x)
    b, _ = ess_between_chains(x)
    assert abs(g / want - 1) < 0.1 and abs(b / want - 1) < 0.25, (g, b, want)
