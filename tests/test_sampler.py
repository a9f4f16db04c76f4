"""The samplers and the ESS estimator on CPU, with analytic likelihoods.

ess_geyer is checked against a literal port of the reference's loop
(new_scripts/mcmc_solver.cpp:80-115). Plain and delayed-acceptance
Metropolis must both sample a known Gaussian posterior; delayed acceptance,
screened by a deliberately wrong surrogate (shifted and too wide), must
still sample the exact posterior while calling the exact model less often.
"""
import numpy as np
import pytest

from lcurve_re_b200.sampler import (delayed_acceptance, ess_bulk, ess_geyer, ess_mean,
                                    ess_total, mean_shift, metropolis, rhat, shift_verdict,
                                    summary)


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
    # a chain that never moved has no effective samples (the reference counts n)
    assert ess_geyer(np.ones(10)) == 0.0 and ess_geyer(np.arange(3.0)) == 3.0


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


def _ar1_chains(steps, chains, phi, seed, offsets=None):
    rng = np.random.default_rng(seed)
    x = np.empty((steps, chains))
    x[0] = rng.standard_normal(chains)
    for i in range(1, steps):
        x[i] = phi * x[i - 1] + np.sqrt(1 - phi * phi) * rng.standard_normal(chains)
    if offsets is not None:
        x += offsets[None, :]
    return x[:, :, None]


def test_multichain_ess_and_rhat_on_ar1_chains():
    """Stationary AR(1) chains: bulk and mean ESS near steps x chains x
    (1 - phi) / (1 + phi), R-hat near 1. The same chains with different
    offsets (chains that have not mixed): R-hat well above 1 and a bulk ESS
    that collapses, where the per-chain Geyer sum does not notice."""
    steps, chains = 4000, 16
    for phi in (0.0, 0.7):
        ch = _ar1_chains(steps, chains, phi, 11)
        expect = steps * chains * (1 - phi) / (1 + phi)
        assert abs(ess_bulk(ch)[0] - expect) < 0.15 * expect, (phi, ess_bulk(ch), expect)
        assert abs(ess_mean(ch)[0] - expect) < 0.15 * expect
        assert rhat(ch)[0] < 1.01
    ch = _ar1_chains(steps, chains, 0.7, 12, offsets=np.linspace(-2, 2, chains))
    assert rhat(ch)[0] > 1.5
    assert ess_bulk(ch)[0] < 0.05 * ess_total(ch)[0]


def test_summary_counts_frozen_chains_as_zero():
    ch = _ar1_chains(2000, 8, 0.5, 3)
    stuck = np.array([-1.5, -1.0, -0.5, 0.3, 0.8, 1.2, 1.6, 2.0])  # states chains stuck at
    frozen = np.concatenate([ch, np.broadcast_to(stuck[None, :, None], (2000, 8, 1))], axis=1)
    a, b = summary(ch, 1.0), summary(frozen, 1.0)
    assert b["ess_geyer"] == a["ess_geyer"]  # the frozen chains add nothing
    assert b["ess_bulk"] < a["ess_bulk"]  # and they split the distribution


def test_mean_shift_and_verdict():
    a = _ar1_chains(4000, 16, 0.5, 21)
    b = _ar1_chains(4000, 16, 0.5, 22)
    shift, mcse = mean_shift(a, b)
    assert shift[0] < 4 * mcse[0] and 0.002 < mcse[0] < 0.02
    assert shift_verdict(shift, mcse) == "within"
    c = a + 0.3
    shift, mcse = mean_shift(c, b)
    assert abs(shift[0] - 0.3) < 5 * mcse[0]
    assert shift_verdict(shift, mcse) == "outside"
    assert shift_verdict(np.array([0.09]), np.array([0.02])) == "undecided"


def test_posterior_resample_recovers_a_gaussian_posterior():
    """Importance resampling in two stages, as the delayed-acceptance
    benchmark does it: box-uniform and a wide Gaussian pool give a first
    estimate, a second Gaussian pool at 1.5x its spread is added, and the
    final weighted mean, covariance and resampled rows match the Gaussian
    posterior (chi**2 known in closed form)."""
    from lcurve_re_b200 import surrogate as S
    rng = np.random.default_rng(5)
    lo, hi = S.BOX[:, 0], S.BOX[:, 1]
    mu = (lo + hi) / 2 + 0.1 * (hi - lo)
    sd = 0.04 * (hi - lo)
    chi2 = lambda t: np.sum(((t - mu) / sd) ** 2, axis=1)
    th_u = lo + rng.random((50000, 9)) * (hi - lo)
    guess_mu, guess_cov = mu + 0.5 * sd, np.diag((1.3 * sd) ** 2)
    th_g = S.local_draws(guess_mu, guess_cov, 60000, seed=3, widen=2.0)
    pools = [(th_u, S.log_uniform_box()), (th_g, S.log_gaussian_in_box(guess_mu, guess_cov, 2.0))]
    _, m1, c1, ess1 = S.posterior_resample(pools, chi2(np.vstack([th_u, th_g])), 10, seed=1)
    th_2 = S.local_draws(m1, c1, 60000, seed=4, widen=1.5)
    pools.append((th_2, S.log_gaussian_in_box(m1, c1, 1.5)))
    rows, mean, cov, ess = S.posterior_resample(pools, chi2(np.vstack([th_u, th_g, th_2])),
                                                4000, seed=1)
    assert ess > 10 * ess1 and ess > 5000, (ess1, ess)
    assert np.all(np.abs(mean - mu) < 0.05 * sd)
    assert np.all(np.abs(np.sqrt(np.diag(cov)) / sd - 1) < 0.05)
    assert np.all(np.abs(rows.mean(0) - mu) < 0.1 * sd)


def test_adaptive_posterior_finds_a_correlated_posterior():
    """Adaptive importance sampling from a poor first estimate (offset mean,
    three times too wide, no correlation) of a strongly correlated Gaussian
    posterior (correlation 0.99 between two parameters): the rounds reach the
    target effective size and the weighted mean and covariance match."""
    from lcurve_re_b200 import surrogate as S
    rng = np.random.default_rng(9)
    lo, hi = S.BOX[:, 0], S.BOX[:, 1]
    mu = (lo + hi) / 2 + 0.05 * (hi - lo)
    sd = 0.02 * (hi - lo)
    corr = np.eye(9)
    corr[0, 3] = corr[3, 0] = 0.99
    cov = corr * np.outer(sd, sd)
    prec = np.linalg.inv(cov)
    chi2 = lambda t: np.einsum("ij,jk,ik->i", t - mu, prec, t - mu)
    th_u = lo + rng.random((50000, 9)) * (hi - lo)
    pools, chi, m, c, hist = S.adaptive_posterior(
        chi2, [(th_u, S.log_uniform_box())], chi2(th_u), mu + 2 * sd, np.diag((3 * sd) ** 2),
        rounds=8, pool=30000, target=5000, seed=4)
    assert hist[-1] >= 5000 and len(hist) <= 8, hist
    assert np.all(np.abs(m - mu) < 0.05 * sd)
    assert np.all(np.abs(np.sqrt(np.diag(c)) / sd - 1) < 0.05)
    assert abs(c[0, 3] / np.sqrt(c[0, 0] * c[3, 3]) - 0.99) < 0.003


def _banana_chi(t):
    """A curved ridge: x1 follows 0.8 x0^2 within 0.05, x2 Gaussian."""
    return (t[:, 0] ** 2 + ((t[:, 1] - 0.8 * t[:, 0] ** 2) / 0.05) ** 2 + (t[:, 2] / 0.3) ** 2)


def _banana_draws(n, seed):
    r = np.random.default_rng(seed)
    x0 = r.standard_normal(n)
    return np.c_[x0, 0.8 * x0 ** 2 + 0.05 * r.standard_normal(n), 0.3 * r.standard_normal(n)]


def test_triangular_walk_is_a_volume_preserving_bijection():
    from lcurve_re_b200.sampler import TriangularWalk
    tw = TriangularWalk(_banana_draws(20000, 1))
    x = _banana_draws(500, 2) + 0.1
    np.testing.assert_allclose(tw.inverse(tw.forward(x)), x, rtol=0, atol=1e-12)
    # Jacobian of the forward map by central differences: unit determinant
    h, x0 = 1e-6, x[:7]
    for row in x0:
        J = np.stack([(tw.forward((row + h * e)[None]) - tw.forward((row - h * e)[None]))[0]
                      / (2 * h) for e in np.eye(3)], axis=1)
        assert abs(np.linalg.det(J * tw.s[None, :]) - 1) < 1e-6
    # the fitted map straightens the ridge: u's second coordinate is the
    # ridge's width (0.05 / its spread) and uncorrelated with the first
    u = tw.forward(_banana_draws(20000, 3))
    assert abs(np.corrcoef(u.T)[0, 1]) < 0.02
    assert u[:, 1].std() < 0.1 * u[:, 0].std()


def test_triangular_walk_mixes_a_curved_ridge_where_the_gaussian_walk_does_not():
    """On a banana-shaped target, plain Metropolis with the triangular walk
    (fitted to a posterior sample, the step scale 2.38 / sqrt(d)) accepts
    0.15-0.45 of its moves (near the Gaussian optimum for 3 dimensions) and
    has at least 5x the bulk ESS of the best-scaled Gaussian walk with the
    sample's covariance; delayed acceptance with the
    same proposal and a shifted, too-wide surrogate keeps the target: both
    chains' means within 4 Monte Carlo errors of the exact ones."""
    from lcurve_re_b200.sampler import TriangularWalk
    chains, steps = 128, 1500
    sample = _banana_draws(20000, 4)
    theta0 = _banana_draws(chains, 5)
    tw = TriangularWalk(sample)
    cg = max((metropolis(_banana_chi, theta0, np.cov(sample.T) * f * f * 2.38 ** 2 / 3, steps,
                         seed=6, box_check=_everywhere) for f in (1.0, 0.5, 0.25)),
             key=lambda r: ess_bulk(r[0]).min())
    ct, _, _, acc, _ = metropolis(_banana_chi, theta0, None, steps, seed=6,
                                  box_check=_everywhere, propose=tw)
    assert 0.15 < acc < 0.45, acc
    assert ess_bulk(ct).min() >= 5 * ess_bulk(cg[0]).min(), (ess_bulk(ct), ess_bulk(cg[0]))
    sur = lambda t: _banana_chi(t - 0.05) * 0.8
    cd, _, _, acc_d, _, _ = delayed_acceptance(_banana_chi, sur, theta0, None,
                                               steps, seed=7, box_check=_everywhere,
                                               propose=tw.with_scale(1.5))
    exact_mean = np.array([0.0, 0.8, 0.0])
    for c in (ct, cd):
        s = c.reshape(-1, 3)
        mcse = s.std(0) / np.sqrt(ess_bulk(c))
        assert np.all(np.abs(s.mean(0) - exact_mean) < 4 * mcse), (s.mean(0), mcse)


def test_forming_proposals_ahead_keeps_the_chains():
    """metropolis forms the next step's proposals while the exact model runs
    (from the current states, then again for the chains that moved); the
    chains equal those of proposing in turn, with the same draws, for the
    Gaussian walk exactly and for the triangular walk to rounding (a row's
    map formed alone or among all rows)."""
    from lcurve_re_b200.sampler import GaussianWalk, TriangularWalk
    theta0 = _banana_draws(64, 8)
    tw = TriangularWalk(_banana_draws(20000, 9))
    for walk, tol in ((GaussianWalk(np.cov(_banana_draws(5000, 10).T)), 0.0), (tw, 1e-12)):
        in_turn = lambda rng, theta, w=walk: w(rng, theta)  # no delta/apply: one at a time
        a = metropolis(_banana_chi, theta0, None, 300, seed=11, box_check=_everywhere,
                       propose=walk)
        b = metropolis(_banana_chi, theta0, None, 300, seed=11, box_check=_everywhere,
                       propose=in_turn)
        np.testing.assert_allclose(a[0], b[0], rtol=0, atol=tol)
        assert a[3] == b[3]


def test_surrogate_transitions_keep_the_exact_posterior():
    """Surrogate transitions (inner Metropolis runs on the surrogate's
    posterior, one exact decision per run): with a shifted, too-wide
    surrogate the chains still hold the exact banana's first and second
    moments (within 4 Monte Carlo errors); with the exact chi**2 as its own
    surrogate every run that moved is accepted."""
    from lcurve_re_b200.sampler import TriangularWalk, surrogate_transitions
    chains, steps, inner = 128, 400, 10
    sample = _banana_draws(20000, 12)
    theta0 = _banana_draws(chains, 13)
    tw = TriangularWalk(sample)
    sur = lambda t: _banana_chi(t - 0.05) * 0.8
    n_exact = [0]

    def exact(t):
        n_exact[0] += 1
        return _banana_chi(t)
    c, _, _, acc, _, st = surrogate_transitions(exact, sur, theta0, None, steps, inner, seed=14,
                                                box_check=_everywhere, propose=tw)
    assert n_exact[0] == steps + 1
    assert 0.05 < st["exact_acceptance"] < 1.0 and 0.1 < st["inner_acceptance"] < 0.5, st
    s = c.reshape(-1, 3)
    ess = ess_bulk(c)
    for stat, truth in ((s, np.array([0.0, 0.8, 0.0])),
                        (s ** 2, np.array([1.0, 0.64 * 3 + 0.05 ** 2, 0.09]))):
        mcse = stat.std(0) / np.sqrt(ess)
        assert np.all(np.abs(stat.mean(0) - truth) < 4 * mcse), (stat.mean(0), truth, mcse)
    _, _, _, _, _, st1 = surrogate_transitions(_banana_chi, _banana_chi, theta0, None, 20, inner,
                                               seed=15, box_check=_everywhere, propose=tw)
    assert st1["exact_acceptance"] == 1.0 and st1["runs_moved"] > 0.5, st1


class _HostRunner:
    """The inner steps of surrogate_transitions for some chains, on the host
    (what DeviceTransitions does on the GPU)."""

    def __init__(self, walk, sur, inner):
        self.walk, self.sur, self.inner = walk, sur, inner

    def run(self, theta, chis, rng):
        y, chy, mv = np.array(theta), np.array(chis), 0
        for _ in range(self.inner):
            prop = self.walk.apply_rows(y, self.walk.delta(rng, y.shape))
            c = self.sur(prop)
            a = np.log(rng.random(len(y))) < -(c - chy) / 2
            y[a], chy[a] = prop[a], c[a]
            mv += int(a.sum())
        return y, chy, mv


def test_surrogate_transitions_in_two_overlapped_halves_keep_the_posterior():
    """With a pair of runners, one half's exact evaluations overlap the
    other half's inner steps; the chains keep the exact banana's moments and
    every exact call is for one half."""
    from lcurve_re_b200.sampler import TriangularWalk, surrogate_transitions
    chains, steps, inner = 128, 400, 10
    tw = TriangularWalk(_banana_draws(20000, 21))
    theta0 = _banana_draws(chains, 22)
    sur = lambda t: _banana_chi(t - 0.05) * 0.8
    sizes = []

    def exact(t):
        sizes.append(len(t))
        return _banana_chi(t)
    pair = [_HostRunner(tw, sur, inner), _HostRunner(tw.with_scale(1.0), sur, inner)]
    c, _, _, acc, _, st = surrogate_transitions(exact, sur, theta0, None, steps, inner, seed=23,
                                                box_check=_everywhere, device=pair)
    assert sizes == [chains // 2] * (2 * steps + 2)
    assert 0.05 < st["exact_acceptance"] < 1.0, st
    s = c.reshape(-1, 3)
    ess = ess_bulk(c)
    for stat, truth in ((s, np.array([0.0, 0.8, 0.0])),
                        (s ** 2, np.array([1.0, 0.64 * 3 + 0.05 ** 2, 0.09]))):
        mcse = stat.std(0) / np.sqrt(ess)
        assert np.all(np.abs(stat.mean(0) - truth) < 4 * mcse), (stat.mean(0), truth, mcse)


def _walk_from_par(par, d, y, n):
    """The proposal of lcg_walk_propose (walk.cu), restated in numpy from the
    packed layout: m, s, c0, B, A, chol, mid, half, lo, hi."""
    sizes = [d, d, d, d * d, d * d * d, d * d, d, d, d, d]
    parts, o = [], 0
    for k in sizes:
        parts.append(par[o:o + k])
        o += k
    assert o == len(par) == 7 * d + 2 * d * d + d ** 3
    m, s, c0, B, A, chol, mid, half, lo, hi = parts
    B, A, chol = B.reshape(d, d), A.reshape(d, d, d), chol.reshape(d, d)

    def poly(k, z):
        return c0[k] + sum(z[i] * (B[i, k] + sum(A[k, i, j] * z[j] for j in range(i, k)))
                           for i in range(k))
    out = np.empty_like(y)
    for r in range(len(y)):
        z = (y[r] - m) / s
        v = np.array([z[k] - poly(k, z) + chol[k, :k + 1] @ n[r, :k + 1] for k in range(d)])
        for k in range(d):
            v[k] = v[k] + poly(k, v)
        out[r] = m + v * s
    return out, (out - mid) / half, np.all((out >= lo) & (out <= hi), axis=1)


def test_walk_parameters_pack_the_maps_for_the_device_walk():
    """walk_parameters packs a TriangularWalk (and a GaussianWalk as the
    identity map) in lcg_walk_propose's layout: the kernel's arithmetic,
    restated from that layout, gives the walks' own proposals."""
    from lcurve_re_b200.sampler import GaussianWalk, TriangularWalk, walk_parameters
    box = np.array([[-3.0, 3.0], [-1.0, 9.0], [-2.0, 2.0]])
    tw = TriangularWalk(_banana_draws(5000, 31), scale=0.7)
    gw = GaussianWalk(np.diag([0.1, 0.2, 0.05]))
    y = _banana_draws(40, 32)
    n = np.random.default_rng(33).standard_normal((40, 3))
    for walk, ref in ((tw, tw.apply_rows(y, n @ tw.chol.T)), (gw, y + n @ gw.chol.T)):
        got, unit, ok = _walk_from_par(walk_parameters(walk, box), 3, y, n)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12)
        np.testing.assert_allclose(unit, (got - box.mean(1)) / ((box[:, 1] - box[:, 0]) / 2))
        assert np.array_equal(ok, np.all((got >= box[:, 0]) & (got <= box[:, 1]), axis=1))


def test_surrogate_transitions_with_a_fixed_approximation_per_chain():
    """Each chain may have its own approximation, fixed for the run (an
    anchor at its starting state, as FixedAnchorChi2 gives): the chains
    still hold the exact banana's moments."""
    from lcurve_re_b200.sampler import TriangularWalk, surrogate_transitions
    chains, steps, inner = 128, 400, 10
    tw = TriangularWalk(_banana_draws(20000, 41))
    theta0 = _banana_draws(chains, 42)
    ref = theta0.copy()
    tilt = np.random.default_rng(43).standard_normal((chains, 3))

    def sur(t):  # exact at the anchor, wrong elsewhere by a chain-specific tilt
        return _banana_chi(t) * 0.8 + 2.0 * np.sum(tilt * (t - ref), axis=1)
    c, _, _, acc, _, st = surrogate_transitions(_banana_chi, sur, theta0, None, steps, inner,
                                                seed=44, box_check=_everywhere, propose=tw)
    assert 0.05 < st["exact_acceptance"] < 1.0, st
    s = c.reshape(-1, 3)
    ess = ess_bulk(c)
    for stat, truth in ((s, np.array([0.0, 0.8, 0.0])),
                        (s ** 2, np.array([1.0, 0.64 * 3 + 0.05 ** 2, 0.09]))):
        mcse = stat.std(0) / np.sqrt(ess)
        assert np.all(np.abs(stat.mean(0) - truth) < 4 * mcse), (stat.mean(0), truth, mcse)


def test_surrogate_transitions_edge_cases():
    """An odd number of chains splits into unequal halves; without a record
    no chain is kept; the box rejects proposals outside it; zero steps are
    refused."""
    from lcurve_re_b200.sampler import TriangularWalk, surrogate_transitions
    tw = TriangularWalk(_banana_draws(5000, 61))
    theta0 = _banana_draws(7, 62)
    sizes = []

    def exact(t):
        sizes.append(len(t))
        return _banana_chi(t)
    pair = [_HostRunner(tw, _banana_chi, 3), _HostRunner(tw, _banana_chi, 3)]
    ch, th, chi, acc, _, st = surrogate_transitions(exact, _banana_chi, theta0, None, 5, 3,
                                                    seed=63, box_check=_everywhere,
                                                    device=pair, record=False)
    assert ch is None and sizes == [3, 4] * 6 and st["exact_acceptance"] == 1.0
    np.testing.assert_array_equal(chi, _banana_chi(th))
    inside = lambda t: np.all(np.abs(t) < 0.5, axis=1)  # a box the walk leaves often
    start = np.zeros((16, 3)) + [0.0, 0.1, 0.0]
    c, *_ = surrogate_transitions(_banana_chi, _banana_chi, start, None, 50, 4, seed=64,
                                  box_check=inside, propose=tw)
    assert np.all(inside(c.reshape(-1, 3)))
    with pytest.raises(ValueError):
        surrogate_transitions(_banana_chi, _banana_chi, start, None, 0, 4, propose=tw)
