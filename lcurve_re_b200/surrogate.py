"""Learned surrogate of the light curve over the MCMC prior box.

The surrogate maps the nine sampled parameters (q, iangle, r1, r2, t1, t2,
gravity_dark2, absorb, t0) to the light curve on a fixed grid of phases
(1000 points in [-0.2, 1.2]): an MLP (lcurve_re_b200.mlp) predicts the
curve's coefficients on its leading principal components. Curves are
normalised to unit mean, since the sampler's chi**2 fits the scale factor
anyway (re_scale.cpp:16-42).

Training data come from the GPU engine itself: uniform draws over the box,
evaluated by the batched engine (lcg_light_curve_batch) at the wd_dm_small
resolution (nlat 40/80). The box is the mcmc_batch distribution's mean
+- 3 sigma, with gravity_dark2 in [0.05, 0.11], absorb in [0.3, 0.7] and t0
in [-0.005, 0.005].
"""
import ctypes as C
import time

import numpy as np

from . import abi
from . import workloads as W
from .mlp import MLP, gemm_bf16x3

PARAMS = ("q", "iangle", "r1", "r2", "t1", "t2", "gravity_dark2", "absorb", "t0")
BOX = np.array([
    (0.19, 0.31),        # q: 0.25 +- 3 x 0.02
    (84.5, 87.5),        # iangle: 86 +- 3 x 0.5
    (0.01275, 0.01725),  # r1: 0.015 x (1 +- 3 x 0.05)
    (0.17, 0.23),        # r2: 0.20 x (1 +- 3 x 0.05)
    (18200.0, 21800.0),  # t1: 20000 x (1 +- 3 x 0.03)
    (2912.0, 3488.0),    # t2: 3200 x (1 +- 3 x 0.03)
    (0.05, 0.11),        # gravity_dark2
    (0.3, 0.7),          # absorb
    (-0.005, 0.005),     # t0
])
NGRID = 1000
NCOEF = 64


def grid_times(n=NGRID):
    return np.linspace(-0.2, 1.2, n)


def to_unit(theta):
    """Parameters -> [-1, 1]^9 over the box."""
    lo, hi = BOX[:, 0], BOX[:, 1]
    return (np.asarray(theta, np.float64) - (lo + hi) / 2) / ((hi - lo) / 2)


def from_unit(u):
    lo, hi = BOX[:, 0], BOX[:, 1]
    return (lo + hi) / 2 + np.asarray(u, np.float64) * (hi - lo) / 2


def in_box(theta):
    t = np.asarray(theta)
    return np.all((t >= BOX[:, 0]) & (t <= BOX[:, 1]), axis=-1)


class ModelFactory:
    """lcg_model arrays for parameter vectors: the base model (wd_dm_small's
    physics and grids) with the nine sampled fields replaced, written through
    a structured-array view of the ctypes array (no per-model parsing)."""

    def __init__(self, base=None):
        self.base = (base if base is not None else W.model()).to_c()
        self.dtype = np.dtype(abi.LcgModel)  # the struct layout, parsed once
        self.base_row = np.frombuffer(bytes(self.base), dtype=self.dtype)[0]
        self._arr = self._view = None

    def __call__(self, theta, out=None):
        """lcg_model array for the rows of theta. Without out, the array is
        reused between calls of the same size (valid until the next call):
        it holds the base model already, so only the sampled fields are
        written."""
        theta = np.atleast_2d(np.asarray(theta, np.float64))
        n = theta.shape[0]
        if out is None:
            if self._arr is None or len(self._arr) != n:
                self._arr = (abi.LcgModel * n)()
                self._view = np.frombuffer(self._arr, dtype=self.dtype)
                self._view[:] = self.base_row
            out, view = self._arr, self._view
        else:
            view = np.frombuffer(out, dtype=self.dtype)
            view[:] = self.base_row
        for k, name in enumerate(PARAMS):
            view[name] = theta[:, k]
        return out


def training_set(engine, n, seed=0, batch=2048, npts=NGRID, theta=None):
    """n uniform draws over the box (or the given parameter vectors) and
    their unit-mean light curves on the phase grid, from the batched GPU
    engine. Returns (theta [n x 9], curves [n x npts] float32)."""
    rng = np.random.default_rng(seed)
    if theta is None:
        theta = BOX[:, 0] + rng.random((n, len(PARAMS))) * (BOX[:, 1] - BOX[:, 0])
    theta = np.asarray(theta, np.float64)
    n = theta.shape[0]
    engine.set_data(W.data(npts, -0.2, 1.2))
    fac = ModelFactory()
    curves = np.empty((n, npts), np.float32)
    for i0 in range(0, n, batch):
        i1 = min(n, i0 + batch)
        ms = fac(theta[i0:i1])
        calc, _, _, _, st = engine.light_curve_batch_resident(ms, scale=False, rdata=False,
                                                              sfac=np.ones(5 * (i1 - i0)))
        if np.any(st != 0):
            raise RuntimeError("training curves failed: statuses %s" % np.unique(st))
        curves[i0:i1] = calc / calc.mean(axis=1, keepdims=True)
    return theta, curves


class Surrogate:
    """PCA of the training curves + the MLP that predicts their coefficients."""

    def __init__(self, ncoef=NCOEF, batch=4096, seed=0, device="cuda"):
        import torch
        self.torch = torch
        self.ncoef = ncoef
        self.net = MLP(nin=len(PARAMS), nout=ncoef, batch=batch, device=device, seed=seed)
        self.dev = self.net.dev

    # -- fitting ---------------------------------------------------------------
    def fit_pca(self, curves):
        """Principal components of the centred curves. The Gram matrix, the
        coefficients and the reconstruction run on lcg_mlp_gemm (gemm_bf16x3:
        three BF16 products, FP32 accumulation per block of 8192 terms, FP64
        across blocks); the eigendecomposition of
        the npts x npts Gram matrix is torch.linalg.eigh in FP64."""
        torch = self.torch
        y = torch.as_tensor(curves, device=self.dev, dtype=torch.float64)
        self.mean = y.mean(dim=0)
        yc = y - self.mean
        cov = gemm_bf16x3(yc.T, yc.T, self.net.lib) / y.shape[0]
        cov = 0.5 * (cov + cov.T)
        evals, evecs = torch.linalg.eigh(cov)
        order = torch.argsort(evals, descending=True)[:self.ncoef]
        self.basis = evecs[:, order].T.contiguous()          # [ncoef x npts]
        coef = gemm_bf16x3(yc, self.basis, self.net.lib)       # [n x ncoef]
        self.cscale = float(coef[:, 0].std())                 # targets = coef / cscale
        resid = yc - gemm_bf16x3(coef, self.basis.T, self.net.lib)
        return float(resid.abs().max()), coef / self.cscale

    def fit(self, theta, curves, epochs=60, lr=2e-3, lr_min=2e-5, seed=1, log=None):
        """PCA, then Adam on the MSE of the scaled coefficients with a cosine
        learning-rate schedule. Returns the per-epoch mean losses."""
        torch = self.torch
        t0 = time.perf_counter()
        pca_err, target = self.fit_pca(curves)
        torch.cuda.synchronize(self.dev)
        self.pca_s = time.perf_counter() - t0
        self.pca_max_err = pca_err
        x = torch.as_tensor(to_unit(theta), device=self.dev, dtype=torch.float32)
        t = target.to(torch.float32)
        B = self.net.B
        n = (x.shape[0] // B) * B
        if n == 0:
            raise ValueError("fewer training curves than one batch")
        steps = epochs * (n // B)
        g = torch.Generator(device=self.dev).manual_seed(seed)
        net = self.net
        net.set_schedule(lr, lr_min, steps)
        losses, k = [], 0
        t0 = time.perf_counter()
        for ep in range(epochs):
            perm = torch.randperm(x.shape[0], generator=g, device=self.dev)[:n]
            tot = 0.0
            for i0 in range(0, n, B):
                idx = perm[i0:i0 + B]
                if net.fused:
                    # one graph per step, schedule and loss kept on the device
                    torch.index_select(x, 0, idx, out=net.x)
                    torch.index_select(t, 0, idx, out=net.tgt)
                    net.graph_step()
                else:
                    rate = lr_min + 0.5 * (lr - lr_min) * (1 + np.cos(np.pi * k / steps))
                    net.forward(x[idx], train=True)
                    tot += net.backward(t[idx].contiguous())
                    net.step(rate)
                k += 1
            if net.fused:
                tot = net.take_loss() * (n // B)
            losses.append(tot / (n // B))
            if log:
                log("epoch %d loss %.3e" % (ep, losses[-1]))
        torch.cuda.synchronize(self.dev)
        self.train_s = time.perf_counter() - t0
        self.train_steps = steps
        net.check()
        return losses

    # -- prediction --------------------------------------------------------------
    def coefficients(self, theta):
        """Scaled PCA coefficients [n x ncoef] (device tensor) for parameter
        vectors theta [n x 9]."""
        torch = self.torch
        x = torch.as_tensor(to_unit(theta), device=self.dev, dtype=torch.float32)
        if x.shape[0] <= self.net.B:
            return self.net.forward(x).clone()
        outs = []
        for i0 in range(0, x.shape[0], self.net.B):
            outs.append(self.net.forward(x[i0:i0 + self.net.B]).clone())
        return torch.cat(outs)

    def curves(self, theta):
        c = self.coefficients(theta).to(self.torch.float64) * self.cscale
        return (self.mean + gemm_bf16x3(c, self.basis.T, self.net.lib)).cpu().numpy()

    def head(self, index):
        """The chi**2 head restricted to the grid points index: (basis
        [ncoef x p] FP32 scaled by cscale, mean [p] FP32)."""
        torch = self.torch
        idx = torch.as_tensor(index, device=self.dev)
        return ((self.basis[:, idx] * self.cscale).to(torch.float32).contiguous(),
                self.mean[idx].to(torch.float32).contiguous())

    def save(self):
        st = self.net.state()
        st.update(mean=self.mean.cpu().numpy(), basis=self.basis.cpu().numpy(),
                  cscale=np.array(self.cscale))
        return st

    def load(self, st):
        torch = self.torch
        self.net.load_state(st)
        self.mean = torch.as_tensor(st["mean"], device=self.dev)
        self.basis = torch.as_tensor(st["basis"], device=self.dev)
        self.cscale = float(st["cscale"])


def local_draws(mean, cov, n, seed=0, widen=3.0):
    """n parameter vectors around a posterior estimate: Gaussian with the
    covariance widened by `widen` in each direction, kept inside the box
    (the region a surrogate is refined on after burn-in)."""
    rng = np.random.default_rng(seed)
    L = np.linalg.cholesky(np.asarray(cov) * widen ** 2)
    out = np.empty((0, len(PARAMS)))
    while out.shape[0] < n:
        t = np.asarray(mean) + rng.standard_normal((2 * n, len(PARAMS))) @ L.T
        out = np.vstack([out, t[in_box(t)]])
    return out[:n]


def gaussian_in_box_fraction(mean, cov, widen, n=1 << 20, seed=99):
    """Monte Carlo estimate of the probability that local_draws' Gaussian
    lands inside the box (its truncation constant)."""
    rng = np.random.default_rng(seed)
    L = np.linalg.cholesky(np.asarray(cov) * widen ** 2)
    t = np.asarray(mean) + rng.standard_normal((n, len(PARAMS))) @ L.T
    return float(in_box(t).mean())


def curves_chi2(curves, data, index):
    """Exact chi**2 of the data for unit-mean engine curves on the grid: the
    curves at the data points (index), the optimal scale as re_scale fits it
    (re_scale.cpp:16-42), and sum w ((f - s m) / sigma)**2. Rows of curves
    [n x NGRID] (float32 or float64) -> array [n]."""
    import torch
    d = np.ascontiguousarray(data)
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    f = torch.as_tensor(d["flux"].copy(), device=dev)
    wt = torch.as_tensor((d["weight"] / d["ferr"] ** 2).copy(), device=dev)
    idx = torch.as_tensor(np.asarray(index), device=dev)
    out = np.empty(curves.shape[0])
    for i0 in range(0, curves.shape[0], 65536):
        m = torch.as_tensor(curves[i0:i0 + 65536], device=dev)[:, idx].to(torch.float64)
        sc = (m * (wt * f)).sum(1) / (m * m * wt).sum(1)
        out[i0:i0 + m.shape[0]] = (((f - sc[:, None] * m) ** 2) * wt).sum(1).cpu().numpy()
    return out


def posterior_resample(pools, chi2, n, seed=0):
    """Sampling-importance-resampling of the posterior (uniform prior over the
    box, likelihood exp(-chi**2 / 2)) from parameter vectors whose exact
    chi**2 is known. pools: list of (theta [k x 9], log density of the
    distribution they were drawn from at each row); together they are one
    draw from the mixture sum_j (k_j / K) q_j, whose density weighs each row.
    Returns (n resampled rows, the weighted mean, the weighted covariance,
    the importance sample's effective size 1 / sum w**2)."""
    theta = np.vstack([p[0] for p in pools])
    K = theta.shape[0]
    logq = np.full(K, -np.inf)
    for t, logq_j in pools:
        logq = np.logaddexp(logq, logq_j(theta) + np.log(t.shape[0] / K))
    logw = -0.5 * np.asarray(chi2) - logq
    logw[~np.isfinite(logw)] = -np.inf
    w = np.exp(logw - logw.max())
    w /= w.sum()
    mean = w @ theta
    xc = theta - mean
    cov = (xc * w[:, None]).T @ xc
    rng = np.random.default_rng(seed)
    # systematic resampling
    u = (rng.random() + np.arange(n)) / n
    rows = np.minimum(np.searchsorted(np.cumsum(w), u), K - 1)
    return theta[rows].copy(), mean, cov, float(1.0 / np.sum(w ** 2))


def adaptive_posterior(chi2_of, pools, chi, mu, cov, rounds=8, pool=65536, target=2e4,
                       widen0=2.0, widen=1.3, seed=0):
    """Adaptive importance sampling of the posterior (uniform prior over the
    box, likelihood exp(-chi**2 / 2)). pools / chi: the rows already drawn
    (list of (theta, log density) as posterior_resample takes them) and their
    chi**2. Each round draws `pool` rows from the Gaussian around the current
    estimate (widen0 x the spread of (mu, cov) first, then widen x the
    weighted spread), gets their chi**2 from chi2_of(theta) (the exact engine
    in the benchmark), adds them as a pool and re-weighs every row over the
    mixture; it stops once the effective size reaches target. Returns
    (pools, chi, mean, covariance, effective size per round)."""
    jitter = np.diag(np.diag(np.asarray(cov)) * 1e-6)  # keeps estimates positive definite
    w, hist = widen0, []
    chi = np.asarray(chi, np.float64)
    for k in range(rounds):
        th = local_draws(mu, cov, pool, seed=seed + 7 * k, widen=w)
        chi = np.r_[chi, chi2_of(th)]
        pools = pools + [(th, log_gaussian_in_box(mu, cov, w))]
        _, mu, cov, ess = posterior_resample(pools, chi, 1, seed=seed)
        cov = cov + jitter
        hist.append(float(ess))
        w = widen
        if ess >= target:
            break
    return pools, chi, mu, cov, hist


def log_uniform_box():
    """Log density of uniform draws over the box."""
    vol = float(np.prod(BOX[:, 1] - BOX[:, 0]))
    return lambda theta: np.full(np.asarray(theta).shape[0], -np.log(vol))


def log_gaussian_in_box(mean, cov, widen):
    """Log density of local_draws(mean, cov, widen): the Gaussian truncated
    to the box (its normalisation from gaussian_in_box_fraction)."""
    C = np.asarray(cov) * widen ** 2
    L = np.linalg.cholesky(C)
    logdet = 2.0 * np.sum(np.log(np.diag(L)))
    z = gaussian_in_box_fraction(mean, cov, widen)
    d = len(PARAMS)

    def f(theta):
        y = np.linalg.solve(L, (np.asarray(theta) - mean).T)
        return -0.5 * (y * y).sum(0) - 0.5 * (d * np.log(2 * np.pi) + logdet) - np.log(z)
    return f


class SurrogateChi2:
    """chi**2 of the data under the surrogate, on the GPU: the MLP forward
    pass, then lcg_mlp_pca_chisq (curve at the data points, optimal scale,
    chi**2). The data points must lie on the surrogate's phase grid.

    Called with parameters, it is the surrogate's own chi**2. The anchored
    form (state / chi2) predicts the curve at y from an exact curve at x as
    exact(x) * s(y) / s(x), so only the surrogate's relative change between
    nearby points has to be right (the delayed-acceptance sampler's
    state-dependent approximation)."""

    def __init__(self, sur, data, index):
        torch = sur.torch
        self.sur, self.torch = sur, torch
        self.basis, self.mean = sur.head(index)
        d = np.ascontiguousarray(data)
        self.flux = torch.as_tensor(d["flux"].copy(), device=sur.dev)
        self.ferr = torch.as_tensor(d["ferr"].copy(), device=sur.dev)
        self.wgt = torch.as_tensor(d["weight"].copy(), device=sur.dev)
        self.npts = d.shape[0]
        self.lib = sur.net.lib

    def __call__(self, theta):
        return self.chi2(self.state(theta))

    def anchor(self, rows):
        """Exact curves (host rows) as the device tensor chi2 takes."""
        return self.torch.as_tensor(np.ascontiguousarray(rows, np.float64), device=self.sur.dev)

    def state(self, theta):
        """The surrogate's coefficients at theta (device tensor)."""
        return self.sur.coefficients(theta).contiguous()

    def _pca(self, coef, coef_x, anchor, chi):
        torch = self.torch
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        st = self.lib.lcg_mlp_pca_chisq(C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                        p(coef), coef.shape[0], coef.shape[1], p(self.basis),
                                        p(self.mean), self.npts, p(self.flux), p(self.ferr),
                                        p(self.wgt), p(coef_x), p(anchor), p(chi), None)
        if st != abi.OK:
            raise RuntimeError("lcg_mlp_pca_chisq failed")

    def chi2(self, coef, coef_x=None, anchor=None):
        """chi**2 of s(coef), or of anchor * s(coef) / s(coef_x) (anchor: exact
        curves at the data points, one row per chain)."""
        torch = self.torch
        chi = torch.empty(coef.shape[0], dtype=torch.float64, device=self.sur.dev)
        an = None
        if anchor is not None:
            an = anchor if isinstance(anchor, torch.Tensor) else self.anchor(anchor)
            an = an.contiguous()
        self._pca(coef, coef_x.contiguous() if coef_x is not None else None, an, chi)
        return chi.cpu().numpy()

    def fixed_anchor(self, theta_ref, curves_ref):
        """The anchored approximation with every chain's anchor fixed:
        FixedAnchorChi2 over the chains of theta_ref [chains x 9] with their
        exact curves curves_ref [chains x points] (float64 device tensor)."""
        return FixedAnchorChi2(self, theta_ref, curves_ref)

    # -- fixed-shape passes of the device delayed-acceptance loop -------------
    def bind(self, sx0, f0):
        """Static buffers for the chains of sx0 (their states) and f0 (their
        exact curves), and CUDA graphs of the two passes the sampler runs
        every step: screening (network forward on the proposals in g_x, then
        chi**2 of f s(y)/s(x) into g_chi) and reverse (chi**2 of F s(x)/s(y)
        into g_chr, F the exact curves of the proposals in g_F)."""
        torch = self.torch
        dev = self.sur.dev
        nc = sx0.shape[0]
        self.g_x = torch.zeros(nc, len(PARAMS), dtype=torch.float32, device=dev)
        self.h_x = torch.zeros(nc, len(PARAMS), dtype=torch.float32, pin_memory=True)
        self.g_sx, self.g_sy = sx0.clone(), torch.zeros_like(sx0)
        self.g_f, self.g_F = f0.clone(), torch.zeros_like(f0)
        self.g_chi = torch.empty(nc, dtype=torch.float64, device=dev)
        self.g_chr = torch.empty(nc, dtype=torch.float64, device=dev)

        def screen():
            self.g_sy.copy_(self.sur.net.forward(self.g_x))
            self._pca(self.g_sy, self.g_sx, self.g_f, self.g_chi)

        def reverse():
            self._pca(self.g_sx, self.g_sy, self.g_F, self.g_chr)
        self.gr_screen = self._capture(screen)
        self.gr_reverse = self._capture(reverse)
        # this library's kernels per replay (the host launch counter does not
        # see graph replays): the network and the chi**2 head, the chi**2 head
        self.graph_launches = 0

    def _capture(self, fn):
        torch = self.torch
        s = torch.cuda.Stream(device=self.sur.dev)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fn()  # first run outside the graph
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        return g

    def screen(self, theta):
        """The bound screening pass on proposals theta: chi**2 per chain."""
        self.h_x.numpy()[:] = to_unit(theta)
        self.g_x.copy_(self.h_x, non_blocking=True)
        self.gr_screen.replay()
        self.graph_launches += 2
        return self.g_chi.cpu().numpy()

    def reverse(self):
        """The bound reverse pass (g_F holds the proposals' exact curves)."""
        self.gr_reverse.replay()
        self.graph_launches += 1
        return self.g_chr.cpu().numpy()

    def merge(self, accepted):
        """Chains accepted this step take the proposal's state and curve."""
        torch = self.torch
        m = torch.as_tensor(accepted, device=self.sur.dev)[:, None]
        self.g_sx.copy_(torch.where(m, self.g_sy, self.g_sx))
        self.g_f.copy_(torch.where(m, self.g_F, self.g_f))


class FixedAnchorChi2:
    """chi**2 of exact(r_i) * s(theta_i) / s(r_i) for chain i: the anchored
    approximation of SurrogateChi2 with each chain's anchor r_i fixed before
    sampling (its exact curve at r_i), so that it is one fixed function of the
    parameters per chain, which surrogate transitions need; the network's
    error then enters only through its change between r_i and theta_i. Called
    with one row per chain, in the chains' order."""

    def __init__(self, sur_chi, theta_ref, curves_ref):
        torch = sur_chi.torch
        self.sur_chi = sur_chi
        self.coef_ref = sur_chi.state(theta_ref)  # [chains x ncoef] FP32
        f = torch.as_tensor(curves_ref, dtype=torch.float64, device=sur_chi.sur.dev)
        self.f_ref = f.contiguous()
        if self.f_ref.shape != (self.coef_ref.shape[0], sur_chi.npts):
            raise ValueError("one exact curve at the data points per chain expected")

    def __call__(self, theta):
        if len(theta) != self.coef_ref.shape[0]:
            raise ValueError("one row per chain expected")
        return self.sur_chi.chi2(self.sur_chi.state(theta), self.coef_ref, self.f_ref)

    def rows(self, part):
        """The anchors (coefficients, curves) of the chains in slice part."""
        return self.coef_ref[part].contiguous(), self.f_ref[part].contiguous()

