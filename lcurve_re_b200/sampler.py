"""Random-walk Metropolis over many parallel chains, plain or with delayed
acceptance screened by a surrogate; the effective-sample-size estimator of
the reference sampler and the rank-normalised multi-chain ESS and R-hat.
Proposals: the Gaussian walk with one covariance (GaussianWalk), or the same
walk in coordinates that straighten a curved posterior ridge
(TriangularWalk, a volume-preserving map fitted to a posterior sample).

The likelihood is exp(-chi**2 / 2) with chi**2 from a callable over a batch
of parameter vectors (one row per chain): the exact GPU engine
(ExactChi2: every chain's model in one lcg_light_curve_batch_resident call)
or the surrogate (surrogate.SurrogateChi2). The prior is uniform over a box.

Delayed acceptance (Christen & Fox 2005): a proposal y from x first passes
the approximation's test with probability g(x, y) = min(1, pi*_x(y) / pi*_x(x));
only then is the exact chi**2 computed, and y is accepted with probability
min(1, pi(y) g(y, x) / (pi(x) g(x, y))), which leaves the exact posterior
invariant for any approximation, including one that depends on the current
state. Two are supported: the surrogate's own chi**2 (pi* = exp(-chi_s/2)),
and the anchored one, chi**2 of exact(x) * s(y) / s(x), which needs the exact
curve at the current state and, for g(y, x), at the proposal (ExactChi2.curves_of
fetches just the rows it needs from the engine). Chains whose proposal the
approximation rejects pass the engine the model it evaluated for them last,
so the batched engine skips them entirely.

Surrogate transitions (surrogate_transitions): per exact decision, a run of
inner Metropolis steps on the surrogate's own posterior, then one exact
test of the run's end point with the ratio of the two posteriors' weights;
the inner steps run on the GPU as a CUDA graph (DeviceTransitions: the walk
and decision kernels of walk.cu around the network and its chi**2 head).
"""
import copy
import ctypes as C
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .surrogate import ModelFactory, in_box


def ess_geyer(x):
    """Geyer's initial-positive-sequence ESS of one chain, as the reference
    sampler computes it (new_scripts/mcmc_solver.cpp:80-115): autocorrelations
    summed in consecutive pairs up to the first negative pair sum, lags up to
    min(n/2, 10000). Autocovariances come from an FFT (the same sums).

    One deliberate difference: a chain that never moved (zero variance) has
    no effective samples here, where the reference returns n for it. Counted
    as n, frozen chains of a sticky sampler would inflate the sum over
    chains."""
    x = np.asarray(x, np.float64)
    n = x.shape[0]
    if n < 4:
        return float(n)
    xc = x - x.mean()
    c0 = float(np.dot(xc, xc)) / n
    if c0 < 1e-30:
        return 0.0
    size = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(xc, size)
    acov = np.fft.irfft(f * np.conj(f), size)[:n]  # acov[k] = sum_i xc[i] xc[i+k]
    rho = acov / (n * c0)
    tau = 1.0
    max_lag = min(n // 2, 10000)
    for lag in range(1, max_lag, 2):
        r1 = rho[lag]
        r2 = rho[lag + 1] if lag + 1 < n else 0.0
        if r1 + r2 < 0.0:
            break
        tau += 2.0 * (r1 + r2)
    return n / max(tau, 1.0)


def ess_total(chain):
    """chain [steps x chains x params]: per parameter, the sum over chains
    of ess_geyer; the minimum over parameters (the reference reports the
    minimum)."""
    steps, nc, npar = chain.shape
    per = np.array([[ess_geyer(chain[:, c, k]) for c in range(nc)] for k in range(npar)])
    return float(per.sum(axis=1).min()), per.sum(axis=1)


def _split(chain):
    """[steps x chains] -> [2*chains x steps//2]: each chain cut in two halves
    (a chain that drifts then shows as two chains that disagree)."""
    h = chain.shape[0] // 2
    return np.concatenate([chain[:h].T, chain[chain.shape[0] - h:].T], axis=0)


def _rank_normal(x):
    """Pooled ranks of all draws mapped to normal scores,
    Phi^-1((r - 3/8) / (S + 1/4)), ties given their average rank."""
    from scipy.special import ndtri
    from scipy.stats import rankdata
    r = rankdata(x.ravel(), method="average").reshape(x.shape)
    return ndtri((r - 0.375) / (x.size + 0.25))


def _ess_chains(x):
    """Multi-chain effective sample size of x [chains x draws] (Vehtari,
    Gelman, Simpson, Carpenter & Buerkner 2021, "Rank-normalization,
    folding, and localization: an improved R-hat"): the autocorrelation at
    each lag combines the chains' mean autocovariance with the between-chain
    variance, rho_t = 1 - (W - mean_m acov_m(t)) / var_plus; the sum is cut
    by Geyer's initial positive sequence made monotone."""
    m, n = x.shape
    if n < 4:
        return float(m * n)
    xc = x - x.mean(axis=1, keepdims=True)
    size = 1 << int(np.ceil(np.log2(2 * n)))
    f = np.fft.rfft(xc, size, axis=1)
    acov = np.fft.irfft(f * np.conj(f), size, axis=1)[:, :n] / n  # biased, per chain
    w = float((acov[:, 0] * n / (n - 1)).mean())                    # within-chain variance
    var_plus = w * (n - 1) / n + (float(x.mean(axis=1).var(ddof=1)) if m > 1 else 0.0)
    if var_plus <= 0.0:
        return 0.0
    rho = 1.0 - (w - acov.mean(axis=0)) / var_plus
    rho[0] = 1.0
    # pairs (rho_2k + rho_2k+1) while positive, then made non-increasing
    pairs = []
    for t in range(0, n - 1, 2):
        p = rho[t] + rho[t + 1]
        if p <= 0.0:
            break
        pairs.append(p if not pairs else min(p, pairs[-1]))
    tau = -1.0 + 2.0 * float(np.sum(pairs))
    return float(m * n / max(tau, 1.0 / np.log10(max(m * n, 10))))


def ess_bulk(chain):
    """Bulk ESS per parameter: the multi-chain ESS of the rank-normalised
    split chains. chain [steps x chains x params] -> array [params]. Chains
    that have not mixed (different halves, different chains in different
    places) lower it through the between-chain variance, which per-chain
    estimators do not see."""
    return np.array([_ess_chains(_rank_normal(_split(chain[:, :, k])))
                     for k in range(chain.shape[2])])


def ess_mean(chain):
    """ESS for the posterior mean per parameter: the multi-chain ESS of the
    split chains on the original scale (the one the Monte Carlo standard
    error of a mean needs)."""
    return np.array([_ess_chains(_split(chain[:, :, k])) for k in range(chain.shape[2])])


def _rhat(z):
    """Potential scale reduction of z [chains x draws]: sqrt(var_plus / W)."""
    n = z.shape[1]
    w = z.var(axis=1, ddof=1).mean()
    b = n * z.mean(axis=1).var(ddof=1)
    return float(np.sqrt(((n - 1) / n * w + b / n) / w)) if w > 0 else np.inf


def _rhat_split(s, z=None):
    """Rank-normalised split R-hat of split chains s (the same paper): the
    larger of the bulk value and the folded (|x - median|) one."""
    z = _rank_normal(s) if z is None else z
    return max(_rhat(z), _rhat(_rank_normal(np.abs(s - np.median(s)))))


def rhat(chain):
    """Rank-normalised split R-hat per parameter; near 1 for chains that
    sample the same distribution."""
    return np.array([_rhat_split(_split(chain[:, :, k])) for k in range(chain.shape[2])])


def summary(chain, wall):
    """Per-sampler figures for one run (chain [steps x chains x params],
    wall seconds): bulk ESS and R-hat (rank-normalised, split chains), the
    reference's Geyer estimator (frozen chains counted as zero) and the
    between-chain estimate, each as a minimum over parameters, and ESS/s."""
    bulk, rh = [], []
    for k in range(chain.shape[2]):
        s = _split(chain[:, :, k])
        z = _rank_normal(s)
        bulk.append(_ess_chains(z))
        rh.append(_rhat_split(s, z))
    geyer, _ = ess_total(chain)
    per = [round(float(b)) for b in bulk]
    bulk = float(np.min(bulk))
    return {"ess_bulk": bulk, "ess_bulk_per_s": bulk / wall, "ess_geyer": geyer,
            "ess_geyer_per_s": geyer / wall,
            "ess_between_chains": ess_between_chains(chain)[0], "rhat_max": float(np.max(rh)),
            "wall_s": wall, "ess_bulk_per_parameter": per,
            "rhat_per_parameter": [round(float(r), 4) for r in rh]}


def mean_shift(chain_a, chain_b):
    """Posterior-mean difference of two samplers per parameter, in units of
    chain_b's posterior standard deviation, with its Monte Carlo standard
    error (the two means' errors sd / sqrt(ESS_mean) combined). Returns
    (shift, mcse) arrays [params]."""
    sa, sb = chain_a.reshape(-1, chain_a.shape[2]), chain_b.reshape(-1, chain_b.shape[2])
    sd_b = sb.std(axis=0)
    shift = np.abs(sa.mean(axis=0) - sb.mean(axis=0)) / sd_b
    mcse_a = sa.std(axis=0) / np.sqrt(np.maximum(ess_mean(chain_a), 1.0))
    mcse_b = sd_b / np.sqrt(np.maximum(ess_mean(chain_b), 1.0))
    return shift, np.sqrt(mcse_a ** 2 + mcse_b ** 2) / sd_b


def shift_verdict(shift, mcse, bar=0.1, z=2.0):
    """'within' when every parameter's shift + z * mcse is below bar,
    'outside' when some parameter's shift - z * mcse is above it,
    'undecided' otherwise (more effective samples needed)."""
    if np.all(shift + z * mcse < bar):
        return "within"
    if np.any(shift - z * mcse > bar):
        return "outside"
    return "undecided"


def ess_between_chains(chain):
    """A cross-check of ess_total that needs no autocorrelation estimate: with
    chains started from the stationary distribution, the variance of a
    chain's mean is sigma**2 / ESS_chain, so ESS = chains x sigma**2 /
    var(chain means), the minimum over parameters."""
    steps, nc, npar = chain.shape
    var_all = chain.reshape(-1, npar).var(axis=0)
    var_means = chain.mean(axis=0).var(axis=0, ddof=1)
    per = nc * var_all / np.maximum(var_means, 1e-300)
    return float(per.min()), per


class ExactChi2:
    """chi**2 of the resident data for each row of theta, from the batched
    engine (scale fitted, as re_scale does). Failed models get +inf."""

    def __init__(self, engine, data, factory=None, curves=False):
        self.engine = engine
        self.fac = factory or ModelFactory()
        engine.set_data(data)
        self.evals = 0
        self.calls = 0
        self._last = None
        self.keep_curves = curves  # curves_of() available
        self._buffers = {}  # the engine's output arrays, reused between calls

    def __call__(self, theta):
        theta = np.asarray(theta, np.float64)
        ms = self.fac(theta)
        _, chisq, _, _, st = self.engine.light_curve_batch_resident(
            ms, calc=False, buffers=self._buffers)
        if self._last is None or self._last.shape != theta.shape:
            self.evals += theta.shape[0]
        else:
            self.evals += int(np.any(theta != self._last, axis=1).sum())
        self._last = theta.copy()
        self.calls += 1
        out = chisq.copy()
        out[st != 0] = np.inf
        return out

    def curves_of(self, rows):
        """The last call's light curves (scaled) of the given chains."""
        return self.engine.batch_curves(rows)

    def curves_device(self, rows, device="cuda"):
        """The same rows as a float64 device tensor, gathered on the device."""
        import torch
        out = torch.empty((len(rows), self.engine._n), dtype=torch.float64, device=device)
        return self.engine.batch_curves_device(rows, out)

    def curves_all_device(self, out):
        """Every chain's curve of the last call into the device tensor out
        [chains x points] (one device copy)."""
        return self.engine.batch_curves_device(None, out)


class CompactExact:
    """Exact chi**2 and curves for the few chains that pass delayed
    acceptance's first stage, through a small batch of fixed size k on an
    engine context of its own: each call refills slots 0.. with those chains'
    proposals, and the slots not refilled keep their previous models, which
    the engine recognises and skips. Every engine launch is then sized for k
    models instead of every chain (the 512-chain batch costs about 0.18 ms per
    call even when nothing changed). The curves land in the rows of the
    caller's device buffer that belong to the chains evaluated."""

    def __init__(self, engine, data, k=32, factory=None):
        import torch
        self.engine, self.k = engine, k
        self.fac = factory or ModelFactory()
        engine.set_data(data)
        self.slots = None
        self.evals = 0
        self._buffers = {}
        self._rows = np.arange(k, dtype=np.int32)
        self._tmp = torch.empty((k, engine._n), dtype=torch.float64, device="cuda")

    def __call__(self, idx, theta, out):
        """chi**2 of theta[idx] (+inf for failed models); their curves into
        out[idx] (a float64 device tensor, chains x points)."""
        import torch
        idx = np.asarray(idx)
        res = np.empty(len(idx))
        if self.slots is None:
            self.slots = np.repeat(theta[idx[:1]], self.k, axis=0)
        for g0 in range(0, len(idx), self.k):
            sel = idx[g0:g0 + self.k]
            ns = len(sel)
            self.slots[:ns] = theta[sel]
            _, chisq, _, _, st = self.engine.light_curve_batch_resident(
                self.fac(self.slots), calc=False, buffers=self._buffers)
            r = chisq[:ns].copy()
            r[st[:ns] != 0] = np.inf
            res[g0:g0 + ns] = r
            self.engine.batch_curves_device(self._rows[:ns], self._tmp[:ns])
            out[torch.as_tensor(sel, device=out.device)] = self._tmp[:ns]
            self.evals += ns
        return res


class GaussianWalk:
    """The random-walk proposal y = x + N(0, cov). delta draws every row's
    step at once; apply forms the proposals of all chains from their steps,
    apply_rows those of some of them (row by row: the rows of the whole)."""

    def __init__(self, cov):
        self.chol = np.linalg.cholesky(cov)

    def delta(self, rng, shape):
        return rng.standard_normal(shape) @ self.chol.T

    def apply(self, theta, delta):
        return theta + delta

    apply_rows = apply

    def __call__(self, rng, theta):
        return self.apply(theta, self.delta(rng, theta.shape))


def _quadratic_features(z):
    """[n x (1 + k + k (k + 1) / 2)]: 1, z_i, z_i z_j (i <= j) of z [n x k]."""
    n, k = z.shape
    cols = [np.ones(n)] + [z[:, i] for i in range(k)]
    cols += [z[:, i] * z[:, j] for i in range(k) for j in range(i, k)]
    return np.stack(cols, axis=1)


class TriangularWalk:
    """Gaussian random walk in coordinates that straighten a curved
    posterior ridge. With z = (x - m) / s standardised on a sample of the
    posterior, u_1 = z_1 and u_k = z_k - P_k(z_1 .. z_{k-1}), P_k the
    least-squares quadratic in the earlier coordinates (a triangular map
    with unit diagonal: Jacobian determinant 1, inverted coordinate by
    coordinate). The proposal y = T^-1(T(x) + N(0, scale^2 2.38^2 / d
    cov(u))) is therefore symmetric in x, so Metropolis and delayed
    acceptance use it with the plain ratio pi(y) / pi(x). A random walk with
    one global covariance is limited to steps of a curved ridge's local
    width; in u the ridge is straight and its spread is the covariance."""

    def __init__(self, sample, scale=1.0):
        sample = np.asarray(sample, np.float64)
        self.m = sample.mean(0)
        self.s = sample.std(0)
        self.s[self.s == 0] = 1.0
        z = (sample - self.m) / self.s
        self.d = d = z.shape[1]
        coef = [None] + [np.linalg.lstsq(_quadratic_features(z[:, :k]), z[:, k],
                                         rcond=None)[0] for k in range(1, d)]
        # P_k(z) = c0[k] + z_<k . b[k] + z_<k^T A[k] z_<k (A upper triangular),
        # and the same for every k at once: C0 + z B + vec(z z^T) Q
        self.c0 = np.zeros(d)
        self.b = [np.zeros(0)] + [c[1:k + 1] for k, c in enumerate(coef) if k]
        self.A = [np.zeros((0, 0))]
        self.B = np.zeros((d, d))
        self.Q = np.zeros((d * d, d))
        for k in range(1, d):
            c = coef[k]
            self.c0[k] = c[0]
            self.B[:k, k] = c[1:k + 1]
            A = np.zeros((k, k))
            A[np.triu_indices(k)] = c[k + 1:]
            self.A.append(A)
            full = np.zeros((d, d))
            full[:k, :k] = A
            self.Q[:, k] = full.ravel()
        u = self._forward_z(z)
        self.mean_u = u.mean(0)
        self.cov_u = np.cov(u.T)
        self.set_scale(scale)

    def set_scale(self, scale):
        self.scale = scale
        self.chol = np.linalg.cholesky(self.cov_u * (scale * 2.38) ** 2 / self.d)
        return self

    def with_scale(self, scale):
        """A copy with another step scale (the map is shared)."""
        w = copy.copy(self)
        w._cache = (None, None)
        return w.set_scale(scale)

    def _forward_z(self, z):
        zz = (z[:, :, None] * z[:, None, :]).reshape(len(z), -1)
        return z - (self.c0 + z @ self.B + zz @ self.Q)

    def forward(self, x):
        return self._forward_z((np.asarray(x, np.float64) - self.m) / self.s)

    def inverse(self, u):
        z = np.array(u, np.float64)
        for k in range(1, self.d):
            zk = z[:, :k]
            z[:, k] = u[:, k] + self.c0[k] + zk @ self.b[k] + np.einsum(
                "ni,ni->n", zk @ self.A[k], zk)
        return self.m + z * self.s

    def draws(self, n, widen=1.0, seed=0, box_check=None):
        """n parameter vectors along the fitted posterior: u Gaussian with the
        sample's mean and widen^2 x its covariance, mapped back (the curved
        ridge's shape, widened across and along it); with box_check, redrawn
        until n lie inside."""
        rng = np.random.default_rng(seed)
        L = np.linalg.cholesky(self.cov_u) * widen
        out = np.empty((0, self.d))
        for _ in range(1000):
            if len(out) >= n:
                return out[:n]
            x = self.inverse(self.mean_u + rng.standard_normal((2 * n, self.d)) @ L.T)
            if box_check is not None:
                x = x[box_check(x)]
            out = np.r_[out, x]
        if len(out) >= n:
            return out[:n]
        raise ValueError("the box holds too few of the draws (%d of %d)" % (len(out), n))

    def delta(self, rng, shape):
        """Every row's step in the straightened coordinates."""
        return rng.standard_normal(shape) @ self.chol.T

    def apply(self, theta, delta):
        """Proposals T^-1(T(theta) + delta) of every chain. It maps only the
        rows that changed since the last call (the samplers move few chains
        per step)."""
        th, u = getattr(self, "_cache", (None, None))
        if th is None or th.shape != theta.shape:
            u = self.forward(theta)
        else:
            moved = np.any(theta != th, axis=1)
            if moved.any():
                u = u.copy()
                u[moved] = self.forward(theta[moved])
        self._cache = (theta.copy(), u)
        return self.inverse(u + delta)

    def apply_rows(self, theta, delta):
        """The same map for some of the chains, row by row, leaving apply's
        record of the last states alone."""
        return self.inverse(self.forward(theta) + delta)

    def __call__(self, rng, theta):
        return self.apply(theta, self.delta(rng, theta.shape))


def _splits(propose):
    """Whether a proposal forms its steps as delta(rng, shape) then
    apply(theta, delta) for every chain or apply_rows for some."""
    return all(hasattr(propose, a) for a in ("delta", "apply", "apply_rows"))


def _take(x, idx):
    """Rows idx of a numpy array or a device tensor."""
    if isinstance(x, np.ndarray):
        return x[idx]
    import torch
    return x[torch.as_tensor(idx, device=x.device)]


def _put(dst, idx, src):
    if isinstance(dst, np.ndarray):
        dst[idx] = src
    else:
        import torch
        dst[torch.as_tensor(idx, device=dst.device)] = src


def _delayed_acceptance_device(exact, sur, theta0, propose, steps, seed, box_check, record):
    """delayed_acceptance with the anchored surrogate kept on the device: the
    exact curves of every chain are copied from the engine in one device
    copy, the screening and reverse chi**2 run over all chains (no index
    gathers), and accepted rows are merged with masked selects. The same
    random draws and decisions as the general loop."""
    torch = sur.torch
    dev = sur.sur.dev
    rng = np.random.default_rng(seed)
    theta = np.array(theta0, np.float64)
    nc = theta.shape[0]
    chi = exact(theta)
    F = torch.empty((nc, exact.engine._n), dtype=torch.float64, device=dev)
    exact.curves_all_device(F)
    f = F.clone()  # exact curves at the states
    sx = sur.state(theta)
    last = theta.copy()
    chain = np.empty((steps,) + theta.shape) if record else None
    acc = stage1 = 0
    t0 = time.perf_counter()
    for s in range(steps):
        prop = propose(rng, theta)
        ok = box_check(prop)
        sy = sur.state(prop)
        chi_a = sur.chi2(sy, sx, f)  # chi**2 of exact(x) s(y) / s(x)
        chi_a[~ok] = np.inf
        log_g = np.minimum(0.0, -(chi_a - chi) / 2)
        a1 = ok & (np.log(rng.random(nc)) < log_g)
        u2 = np.log(rng.random(nc))
        if a1.any():
            ev = np.where(a1[:, None], prop, last)
            chi_p = exact(ev)
            last = ev
            exact.curves_all_device(F)  # F rows of a1 chains: exact(y)
            chi_rev = sur.chi2(sx, sy, F)  # exact(y) s(x) / s(y), used where a1
            log_g_rev = np.where(a1, np.minimum(0.0, -(chi_rev - chi_p) / 2), 0.0)
            with np.errstate(invalid="ignore"):
                log_rho = -(chi_p - chi) / 2 + log_g_rev - log_g
            a2 = a1 & (u2 < log_rho)
            theta[a2] = prop[a2]
            chi[a2] = chi_p[a2]
            if a2.any():
                m = torch.as_tensor(a2, device=dev)[:, None]
                f = torch.where(m, F, f)
                sx = torch.where(m, sy, sx)
            acc += int(a2.sum())
            stage1 += int(a1.sum())
        if record:
            chain[s] = theta
    wall = time.perf_counter() - t0
    n = steps * nc
    return chain, theta, chi, acc / n, wall, {"stage1_rate": stage1 / n,
                                              "stage2_rate": acc / max(stage1, 1)}


def _delayed_acceptance_graphs(exact, sur, theta0, propose, steps, seed, box_check, record,
                               compact=None):
    """The device loop with the surrogate's two per-step passes replayed as
    CUDA graphs on static buffers (sur.bind): one launch each instead of the
    network's layer-by-layer launches and allocations. Same draws and
    decisions as the other loops; with compact (a CompactExact), the
    stage-1 chains' exact evaluations go through its small batch.

    With a proposal that splits into delta and apply (both walks), the next
    step's proposals are formed on the host while a worker thread runs this
    step's exact evaluations: the next step's noise is drawn right after
    this step's two uniforms (the order of the draws of the plain loop),
    every chain's proposal is formed from its current state, and the rows of
    the chains that then move are formed again from their new states."""
    import torch
    rng = np.random.default_rng(seed)
    theta = np.array(theta0, np.float64)
    nc = theta.shape[0]
    chi = exact(theta)
    F = torch.empty((nc, exact.engine._n), dtype=torch.float64, device=sur.sur.dev)
    exact.curves_all_device(F)
    sur.bind(sur.state(theta), F)
    last = theta.copy()
    chain = np.empty((steps,) + theta.shape) if record else None
    acc = stage1 = 0
    split = _splits(propose)
    pool = ThreadPoolExecutor(max_workers=1) if split else None
    t0 = time.perf_counter()
    if split:
        prop = propose.apply(theta, propose.delta(rng, theta.shape))
    for s in range(steps):
        if not split:
            prop = propose(rng, theta)
        ok = box_check(prop)
        chi_a = sur.screen(prop)  # chi**2 of exact(x) s(y) / s(x)
        chi_a[~ok] = np.inf
        log_g = np.minimum(0.0, -(chi_a - chi) / 2)
        a1 = ok & (np.log(rng.random(nc)) < log_g)
        u2 = np.log(rng.random(nc))
        ahead = split and s + 1 < steps
        if ahead:
            d = propose.delta(rng, theta.shape)
        if a1.any():
            if compact is not None:
                idx = np.flatnonzero(a1)

                def run(idx=idx, prop=prop):
                    chi_p = np.full(nc, np.inf)
                    chi_p[idx] = compact(idx, prop, sur.g_F)  # rows of a1 chains: exact(y)
                    return chi_p
            else:
                ev = np.where(a1[:, None], prop, last)
                last = ev

                def run(ev=ev):
                    chi_p = exact(ev)
                    exact.curves_all_device(sur.g_F)  # rows of a1 chains: exact(y)
                    return chi_p
            if ahead:
                job = pool.submit(run)
                nxt = propose.apply(theta, d)
                chi_p = job.result()
            else:
                chi_p = run()
            chi_rev = sur.reverse()
            log_g_rev = np.where(a1, np.minimum(0.0, -(chi_rev - chi_p) / 2), 0.0)
            with np.errstate(invalid="ignore"):
                log_rho = -(chi_p - chi) / 2 + log_g_rev - log_g
            a2 = a1 & (u2 < log_rho)
            theta[a2] = prop[a2]
            chi[a2] = chi_p[a2]
            if a2.any():
                sur.merge(a2)
                if ahead:
                    nxt[a2] = propose.apply_rows(theta[a2], d[a2])
            acc += int(a2.sum())
            stage1 += int(a1.sum())
        elif ahead:
            nxt = propose.apply(theta, d)
        if record:
            chain[s] = theta
        if ahead:
            prop = nxt
    wall = time.perf_counter() - t0
    if pool is not None:
        pool.shutdown()
    n = steps * nc
    return chain, theta, chi, acc / n, wall, {"stage1_rate": stage1 / n,
                                              "stage2_rate": acc / max(stage1, 1)}


def metropolis(exact, theta0, cov, steps, seed=0, box_check=in_box, record=True,
               propose=None):
    """Plain Metropolis on every chain at once, with the Gaussian random walk
    of covariance cov or another symmetric proposal (propose(rng, theta) ->
    proposals, e.g. TriangularWalk). Returns (chain [steps x chains x params]
    or None, final theta, final chi**2, acceptance rate, wall seconds).

    With a proposal that splits into delta and apply (both walks), the next
    step's proposals are formed on the host while a worker thread runs this
    step's exact evaluations, as in the delayed-acceptance loop: the
    acceptance uniforms are drawn before the evaluation and the next step's
    noise after them (the same order of draws as drawing them in turn), and
    the rows of the chains that move are formed again from their new
    states. Same chains either way."""
    rng = np.random.default_rng(seed)
    propose = propose or GaussianWalk(cov)
    theta = np.array(theta0, np.float64)
    chi = exact(theta)
    last = theta.copy()
    chain = np.empty((steps,) + theta.shape) if record else None
    acc = 0
    nc = theta.shape[0]
    split = _splits(propose)
    pool = ThreadPoolExecutor(max_workers=1) if split else None
    t0 = time.perf_counter()
    if split:
        prop = propose.apply(theta, propose.delta(rng, theta.shape))
    for s in range(steps):
        if not split:
            prop = propose(rng, theta)
        ok = box_check(prop)
        ev = np.where(ok[:, None], prop, last)
        ahead = split and s + 1 < steps
        if ahead:
            u = rng.random(nc)
            d = propose.delta(rng, theta.shape)
            job = pool.submit(exact, ev)
            nxt = propose.apply(theta, d)
            chi_p = job.result()
        else:
            chi_p = exact(ev)
            u = rng.random(nc)
        chi_p[~ok] = np.inf
        a = np.log(u) < -(chi_p - chi) / 2
        theta[a] = prop[a]
        chi[a] = chi_p[a]
        last = ev
        acc += int(a.sum())
        if record:
            chain[s] = theta
        if ahead:
            if a.any():
                nxt[a] = propose.apply_rows(theta[a], d[a])
            prop = nxt
    wall = time.perf_counter() - t0
    if pool is not None:
        pool.shutdown()
    return chain, theta, chi, acc / (steps * theta.shape[0]), wall


def delayed_acceptance(exact, sur, theta0, cov, steps, seed=0, box_check=in_box, record=True,
                       compact=None, propose=None):
    """Delayed-acceptance Metropolis: the approximation screens, the exact
    model judges every step that passes. sur is either a chi**2 callable
    (state-independent approximation) or an anchored one with
    state(theta) -> s and chi2(s_y, s_x, anchor) -> chi**2 of
    anchor * s(y) / s(x); the anchored form needs exact.curves_of(rows). Returns
    (chain, final theta, final chi**2, acceptance rate, wall seconds, stats)."""
    rng = np.random.default_rng(seed)
    propose = propose or GaussianWalk(cov)
    theta = np.array(theta0, np.float64)
    anchored = hasattr(sur, "state")
    if anchored and hasattr(exact, "curves_all_device") and hasattr(sur, "bind"):
        return _delayed_acceptance_graphs(exact, sur, theta0, propose, steps, seed, box_check,
                                          record, compact)
    if anchored and hasattr(exact, "curves_all_device") and hasattr(sur, "torch"):
        return _delayed_acceptance_device(exact, sur, theta0, propose, steps, seed, box_check,
                                          record)
    place = getattr(sur, "anchor", lambda rows: np.array(rows, np.float64))
    if anchored and hasattr(exact, "curves_device") and hasattr(sur, "sur"):
        fetch = lambda rows: exact.curves_device(rows, sur.sur.dev)  # stays on the device
    else:
        fetch = lambda rows: place(exact.curves_of(rows))
    chi = exact(theta)
    if anchored:
        f = fetch(np.arange(theta.shape[0]))  # exact curves at the states
        sx = sur.state(theta)
    else:
        chi_s = sur(theta)
    last = theta.copy()
    chain = np.empty((steps,) + theta.shape) if record else None
    acc = stage1 = 0
    nc = theta.shape[0]
    t0 = time.perf_counter()
    for s in range(steps):
        prop = propose(rng, theta)
        ok = box_check(prop)
        if anchored:
            sy = sur.state(prop)
            chi_a = sur.chi2(sy, sx, f)       # chi**2 of exact(x) s(y) / s(x)
            chi_a[~ok] = np.inf
            log_g = np.minimum(0.0, -(chi_a - chi) / 2)
        else:
            chi_sp = np.full(nc, np.inf)
            if ok.any():
                chi_sp[ok] = sur(prop[ok])
            log_g = np.minimum(0.0, -(chi_sp - chi_s) / 2)
        a1 = ok & (np.log(rng.random(nc)) < log_g)
        u2 = np.log(rng.random(nc))
        if a1.any():
            ev = np.where(a1[:, None], prop, last)
            chi_p = exact(ev)
            last = ev
            if anchored:
                # only the chains that reached the engine need their new curve
                i1 = np.nonzero(a1)[0]
                fp = fetch(i1)
                chi_r = np.full(nc, np.inf)
                chi_r[i1] = sur.chi2(_take(sx, i1), _take(sy, i1), fp)  # exact(y) s(x)/s(y)
                log_g_rev = np.minimum(0.0, -(chi_r - chi_p) / 2)
            else:
                log_g_rev = np.minimum(0.0, -(chi_s - chi_sp) / 2)
            with np.errstate(invalid="ignore"):
                log_rho = -(chi_p - chi) / 2 + log_g_rev - log_g
            a2 = a1 & (u2 < log_rho)
            theta[a2] = prop[a2]
            chi[a2] = chi_p[a2]
            if anchored:
                i2 = np.nonzero(a2)[0]
                if i2.size:
                    _put(f, i2, _take(fp, np.nonzero(a2[i1])[0]))
                    _put(sx, i2, _take(sy, i2))
            else:
                chi_s[a2] = chi_sp[a2]
            acc += int(a2.sum())
            stage1 += int(a1.sum())
        if record:
            chain[s] = theta
    wall = time.perf_counter() - t0
    n = steps * nc
    return chain, theta, chi, acc / n, wall, {"stage1_rate": stage1 / n,
                                              "stage2_rate": acc / max(stage1, 1)}


def walk_parameters(walk, box):
    """The device layout of a walk (lcg_walk_propose's par): m, s, c0, B, A,
    chol, mid, half, lo, hi for a TriangularWalk, or the same with the
    identity map (m 0, s 1, no polynomial) for a GaussianWalk. box: [d x 2]
    bounds; mid and half are the network's unit coordinates as
    surrogate.to_unit forms them."""
    box = np.asarray(box, np.float64)
    lo, hi = box[:, 0], box[:, 1]
    d = box.shape[0]
    m, s, c0 = np.zeros(d), np.ones(d), np.zeros(d)
    B, A = np.zeros((d, d)), np.zeros((d, d, d))
    if isinstance(walk, TriangularWalk):
        m, s, c0, B = walk.m, walk.s, walk.c0, walk.B
        for k in range(1, d):
            A[k, :k, :k] = walk.A[k]
    elif not isinstance(walk, GaussianWalk):
        raise TypeError("the device walk takes a GaussianWalk or a TriangularWalk")
    parts = (m, s, c0, B, A, walk.chol, (lo + hi) / 2, (hi - lo) / 2, lo, hi)
    return np.ascontiguousarray(np.concatenate([np.ravel(p) for p in parts]), np.float64)


class DeviceTransitions:
    """The inner steps of surrogate_transitions on the GPU, for every chain
    at once: inner x (lcg_walk_propose, the network's forward pass, the
    chi**2 head, lcg_walk_accept), captured once as a CUDA graph and
    replayed per outer step. The chains' states and surrogate chi**2 go to
    the device and come back once per outer step. The random numbers come
    from Philox on the device; with host_draws the caller's generator fills
    them instead, in the order of the host loop (tests). anchor: None (the
    network's own chi**2) or (coefficients [nc x ncoef] FP32, exact curves
    [nc x points] FP64) of each chain's fixed anchor (FixedAnchorChi2.rows).
    """

    def __init__(self, sur_chi, walk, box, nc, inner, seed=0, host_draws=False, anchor=None):
        torch = sur_chi.torch
        self.torch, self.sur_chi, self.lib = torch, sur_chi, sur_chi.lib
        dev = sur_chi.sur.dev
        d = np.asarray(box).shape[0]
        self.nc, self.d, self.inner, self.seed = nc, d, inner, int(seed) & (2 ** 63 - 1)
        self.par = torch.as_tensor(walk_parameters(walk, box), device=dev)
        f64 = dict(dtype=torch.float64, device=dev)
        mid = np.asarray(box, np.float64).mean(axis=1)
        self.y = torch.as_tensor(np.tile(mid, (nc, 1)), **f64)  # until the first run
        self.prop = torch.zeros((nc, d), **f64)
        self.chis, self.chi = torch.zeros(nc, **f64), torch.zeros(nc, **f64)
        self.xu = torch.zeros((nc, d), dtype=torch.float32, device=dev)
        self.ok = torch.zeros(nc, dtype=torch.uint8, device=dev)
        self.moves = torch.zeros(nc, dtype=torch.int32, device=dev)
        self.ctr = torch.zeros(1, dtype=torch.int64, device=dev)
        self.h_y = torch.zeros((nc, d), dtype=torch.float64, pin_memory=True)
        self.h_c = torch.zeros(nc, dtype=torch.float64, pin_memory=True)
        self.host_draws = host_draws
        self.a_coef = self.a_f = None
        if anchor is not None:
            self.a_coef, self.a_f = (t.contiguous() for t in anchor)
            if (self.a_coef.dtype != torch.float32 or self.a_f.dtype != torch.float64 or
                    self.a_coef.shape[0] != nc or self.a_f.shape != (nc, sur_chi.npts) or
                    self.a_coef.shape[1] != sur_chi.sur.net.nout):
                raise ValueError("anchor: [nc x ncoef] FP32 coefficients and [nc x points] "
                                 "FP64 curves")
        if host_draws:
            self.noise = torch.zeros((inner, nc, d), **f64)
            self.unif = torch.zeros((inner, nc), **f64)
        self.graph = sur_chi._capture(self._steps)
        # this library's kernels per replay: propose, network, chi**2 and
        # accept per inner step, and the counter
        self.launches_per_run = 4 * inner + 1
        self.launches = 0

    def _ok(self, st, what):
        if st != 0:
            raise RuntimeError("%s failed (status %d)" % (what, st))

    def _steps(self):
        torch, lib = self.torch, self.lib
        p = lambda t: C.c_void_p(t.data_ptr())
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        net = self.sur_chi.sur.net
        for l in range(self.inner):
            noise = p(self.noise[l]) if self.host_draws else None
            unif = p(self.unif[l]) if self.host_draws else None
            self._ok(lib.lcg_walk_propose(stream, self.nc, self.d, p(self.par), p(self.y),
                                          self.seed, p(self.ctr), l, noise, p(self.prop),
                                          p(self.xu), p(self.ok)), "lcg_walk_propose")
            coef = net.forward(self.xu)
            self.sur_chi._pca(coef, self.a_coef, self.a_f, self.chi)
            self._ok(lib.lcg_walk_accept(stream, self.nc, self.d, p(self.prop), p(self.ok),
                                         p(self.chi), p(self.y), p(self.chis), p(self.moves),
                                         self.seed, p(self.ctr), l, unif), "lcg_walk_accept")
        self._ok(lib.lcg_walk_advance(stream, p(self.ctr), self.inner), "lcg_walk_advance")

    def run(self, theta, chis, rng=None):
        """inner steps from the states theta (surrogate chi**2 chis): the end
        states, their surrogate chi**2 and the number of inner moves."""
        self.h_y.numpy()[:] = theta
        self.h_c.numpy()[:] = chis
        self.y.copy_(self.h_y, non_blocking=True)
        self.chis.copy_(self.h_c, non_blocking=True)
        self.moves.zero_()
        if self.host_draws:
            for l in range(self.inner):
                self.noise[l].copy_(self.torch.as_tensor(rng.standard_normal((self.nc, self.d))))
                self.unif[l].copy_(self.torch.as_tensor(rng.random(self.nc)))
        self.graph.replay()
        self.launches += self.launches_per_run
        return self.y.cpu().numpy(), self.chis.cpu().numpy(), int(self.moves.sum())


def surrogate_transitions(exact, sur, theta0, cov, steps, inner, seed=0, box_check=in_box,
                          record=True, propose=None, device=None):
    """Delayed acceptance with surrogate transitions (Liu's surrogate
    transition method, Monte Carlo Strategies in Scientific Computing, 2001,
    sec. 9.4.3): each step runs `inner` Metropolis steps of the random walk
    on the surrogate's posterior exp(-chi_s / 2) from the chain's state x to
    y, then the exact model judges y once, accepting it with probability
    min(1, w(y) / w(x)), w = exp(-(chi - chi_s) / 2). The inner chain is
    reversible for the surrogate's posterior, so the two stages together
    are reversible for the exact one whatever the surrogate's error; a
    rejected run leaves the chain at x. sur: a chi**2 callable, a fixed
    function of the parameters (the anchored approximation of
    delayed_acceptance moves with x and does not serve).

    device: None (the inner steps on the host, with propose), a runner of
    the inner steps for every chain (DeviceTransitions: its own walk and
    inner count), or a pair of runners for the two halves of the chains:
    then a worker thread evaluates one half's run ends on the exact model
    while the GPU runs the other half's inner steps, so the two overlap.
    Chains whose run ended where it started pass the engine the model it
    evaluated for them last, so the batched engine skips them.

    Returns (chain [steps x chains x params] or None, final theta, final
    chi**2, acceptance rate of the runs, wall seconds, stats)."""
    if steps < 1 or (device is None and inner < 1):
        raise ValueError("surrogate_transitions needs at least one step and one inner step")
    rng = np.random.default_rng(seed)
    if device is None:
        propose = propose or GaussianWalk(cov)
    theta = np.array(theta0, np.float64)
    nc = theta.shape[0]
    pair = isinstance(device, (list, tuple))
    parts = [slice(0, nc // 2), slice(nc // 2, nc)] if pair else [slice(0, nc)]
    runners = list(device) if pair else [device]
    chi = np.empty(nc)
    for part in parts:  # the halves as the loop's calls will pass them
        chi[part] = exact(theta[part])
    chis = np.asarray(sur(theta), np.float64).copy()
    last = theta.copy()
    chain = np.empty((steps,) + theta.shape) if record else None
    count = {"acc": 0, "moved": 0, "inner": 0}
    inner_n = runners[0].inner if device is not None else inner

    def run(k):
        """inner steps of part k: end states, their surrogate chi**2."""
        part, dev = parts[k], runners[k]
        if dev is not None:
            y, chy, mv = dev.run(theta[part], chis[part], rng)
        else:
            y, chy, mv = theta[part].copy(), chis[part].copy(), 0
            n = y.shape[0]
            for _ in range(inner):
                prop = propose(rng, y)
                ok = box_check(prop)
                c = np.asarray(sur(prop), np.float64).copy()
                with np.errstate(invalid="ignore"):
                    a = ok & (np.log(rng.random(n)) < -(c - chy) / 2)
                y[a] = prop[a]
                chy[a] = c[a]
                mv += int(a.sum())
        count["inner"] += mv
        moved = np.any(y != theta[part], axis=1)
        ev = np.where(moved[:, None], y, last[part])
        last[part] = ev
        return y, chy, moved, ev

    def decide(k, y, chy, moved, chi_y):
        """the exact decision on part k's run ends."""
        part = parts[k]
        with np.errstate(invalid="ignore"):
            log_r = -(chi_y - chi[part]) / 2 + (chy - chis[part]) / 2
            a = moved & (np.log(rng.random(len(moved))) < log_r)
        th, c, cs = theta[part], chi[part], chis[part]
        th[a], c[a], cs[a] = y[a], chi_y[a], chy[a]
        theta[part], chi[part], chis[part] = th, c, cs
        count["acc"] += int(a.sum())
        count["moved"] += int(moved.sum())

    t0 = time.perf_counter()
    if not pair:
        for s in range(steps):
            y, chy, moved, ev = run(0)
            decide(0, y, chy, moved, exact(ev))
            if record:
                chain[s] = theta
    else:
        pool = ThreadPoolExecutor(max_workers=1)
        ra = run(0)
        for s in range(steps):
            job = pool.submit(exact, ra[3])
            rb = run(1)  # overlaps half 0's exact evaluation
            decide(0, *ra[:3], job.result())
            job = pool.submit(exact, rb[3])
            if s + 1 < steps:
                ra = run(0)  # overlaps half 1's exact evaluation
            decide(1, *rb[:3], job.result())
            if record:
                chain[s] = theta
        pool.shutdown()
    wall = time.perf_counter() - t0
    n = steps * nc
    return chain, theta, chi, count["acc"] / n, wall, {
        "inner_steps": inner_n, "inner_acceptance": count["inner"] / (n * inner_n),
        "runs_moved": count["moved"] / n,
        "exact_acceptance": count["acc"] / max(count["moved"], 1)}
