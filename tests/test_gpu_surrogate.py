"""The learned surrogate on the GPU: training curves from the batched engine,
the PCA + MLP fit on the tensor-core kernels, the chi**2 head, and
delayed-acceptance Metropolis driven by it.

  * training curves equal the engine's one-by-one curves (unit-mean
    normalised) to 2e-6;
  * after a short fit, the surrogate's held-out curves are at least 4x
    closer to the engine's than the mean training curve is (what the
    network gains over predicting nothing);
  * the chi**2 head agrees with chi**2 computed in numpy from the
    surrogate's own curves;
  * delayed acceptance calls the exact engine for fewer chain-steps than
    plain Metropolis on the same proposals.
"""
import numpy as np
import pytest

from lcurve_re_b200 import surrogate as S
from lcurve_re_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from lcurve_re_b200.engine import Engine
    e = Engine(precision="mixed")
    theta, curves = S.training_set(e, 12288 + 1024, seed=11, batch=2048)
    sur = S.Surrogate(batch=2048, seed=0)
    losses = sur.fit(theta[:12288], curves[:12288], epochs=40, lr=2e-3)
    yield e, sur, theta, curves, losses
    e.close()


def test_training_curves_match_the_engine(trained):
    e, sur, theta, curves, _ = trained
    fac = S.ModelFactory()
    d = W.data(S.NGRID, -0.2, 1.2)
    for i in (0, 5000):
        c = e.light_curve_comp(fac(theta[i:i + 1])[0], d, scale=False, rdata=False,
                               sfac=np.ones(5), diagnostics=False)[0]
        assert np.max(np.abs(curves[i] - c / c.mean())) <= 2e-6


def test_surrogate_beats_the_mean_curve(trained):
    e, sur, theta, curves, losses = trained
    assert losses[-1] < 0.05 * losses[0]
    held = slice(12288, 12288 + 1024)
    pred = sur.curves(theta[held])
    truth = curves[held].astype(np.float64)
    err = np.sqrt(np.mean((pred - truth) ** 2))
    base = np.sqrt(np.mean((truth - curves[:12288].mean(axis=0)) ** 2))
    assert err < 0.25 * base, (err, base)


def test_chisq_head_matches_numpy(trained):
    e, sur, theta, curves, _ = trained
    idx = np.arange(0, S.NGRID, 2)
    d = W.data(S.NGRID, -0.2, 1.2)[idx]
    d = W.add_noise(d, curves[3][idx].astype(np.float64), 5)
    f = S.SurrogateChi2(sur, d, idx)
    th = theta[:16]
    chi = f(th)
    c = sur.curves(th)[:, idx]
    w = d["weight"] / d["ferr"] ** 2
    s = (w * d["flux"] * c).sum(1) / (w * c * c).sum(1)
    ref = (d["weight"] * ((d["flux"] - s[:, None] * c) / d["ferr"]) ** 2).sum(1)
    np.testing.assert_allclose(chi, ref, rtol=2e-4)


def test_delayed_acceptance_calls_the_engine_less(trained):
    from lcurve_re_b200.sampler import ExactChi2, delayed_acceptance, metropolis
    e, sur, theta, curves, _ = trained
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    calc = e.light_curve_comp(S.ModelFactory()(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                              scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)[0]
    d = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 9)
    exact = ExactChi2(e, d)
    sur_chi = S.SurrogateChi2(sur, d, idx)
    rng = np.random.default_rng(0)
    chains = 32
    scale = (S.BOX[:, 1] - S.BOX[:, 0]) * 2e-3
    theta0 = truth + rng.standard_normal((chains, 9)) * scale
    cov = np.diag(scale ** 2)
    _, tp, chp, accp, _ = metropolis(exact, theta0, cov, 60, seed=1, record=False)
    n_plain = exact.evals
    exact2 = ExactChi2(e, d, curves=True)
    _, td, chd, accd, _, st = delayed_acceptance(exact2, sur_chi, theta0, cov, 60, seed=1,
                                                 record=False)
    assert exact2.evals < n_plain
    assert accp > 0 and accd > 0 and 0 < st["stage1_rate"] < 1
    assert np.all(np.isfinite(chd))


def test_device_delayed_acceptance_equals_the_general_loop(trained):
    """The device-resident anchored loop (whole-matrix curve copies, masked
    merges) takes the same decisions as the general loop (row gathers)."""
    from lcurve_re_b200.sampler import ExactChi2, delayed_acceptance
    e, sur, theta, curves, _ = trained
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    calc = e.light_curve_comp(S.ModelFactory()(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                              scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)[0]
    d = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 9)
    sur_chi = S.SurrogateChi2(sur, d, idx)
    rng = np.random.default_rng(4)
    scale = (S.BOX[:, 1] - S.BOX[:, 0]) * 2e-3
    theta0 = truth + rng.standard_normal((24, 9)) * scale
    cov = np.diag(scale ** 2) * 4.0

    class General:  # an ExactChi2 without the whole-matrix copy: the general loop
        def __init__(self, ex):
            self.ex = ex

        def __call__(self, theta):
            return self.ex(theta)

        def curves_of(self, rows):
            return self.ex.curves_of(rows)

        def curves_device(self, rows, device="cuda"):
            return self.ex.curves_device(rows, device)

    out = []
    for wrap in (lambda x: x, General):
        ex = wrap(ExactChi2(e, d, curves=True))
        ch, th, chi, acc, _, st = delayed_acceptance(ex, sur_chi, theta0, cov, 40, seed=3)
        out.append((ch, chi, st))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_compact_exact_matches_the_whole_chain_batch(trained):
    """CompactExact (the stage-1 chains through a small batch on a second
    context) gives the chi**2 and curves of the whole-chain batch for those
    chains, including across calls that refill only some slots, and a delayed
    acceptance run through it keeps the exact posterior's checks. The two
    batch layouts may sum their flux chunks differently (each layout's plan is
    tuned on its own), so they agree to the batch tolerances: curves 2e-6,
    chi**2 1e-5 relative."""
    from lcurve_re_b200.engine import Engine
    from lcurve_re_b200.sampler import CompactExact, ExactChi2, delayed_acceptance
    import torch
    e, sur, theta, curves, _ = trained
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    calc = e.light_curve_comp(S.ModelFactory()(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                              scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)[0]
    d = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 9)
    rng = np.random.default_rng(8)
    scale = (S.BOX[:, 1] - S.BOX[:, 0]) * 2e-3
    nc = 40
    exact = ExactChi2(e, d, curves=True)
    with Engine(precision="mixed") as ec:
        comp = CompactExact(ec, d, k=8)
        out = torch.zeros((nc, len(idx)), dtype=torch.float64, device="cuda")
        for trial in range(3):
            th = truth + rng.standard_normal((nc, 9)) * scale
            full = exact(th)
            ref = torch.empty((nc, len(idx)), dtype=torch.float64, device="cuda")
            exact.curves_all_device(ref)
            sel = np.sort(rng.choice(nc, 5 + 4 * trial, replace=False))  # one or two groups
            got = comp(sel, th, out)
            np.testing.assert_allclose(got, full[sel], rtol=1e-5)
            np.testing.assert_allclose(out[sel].cpu().numpy(), ref[sel].cpu().numpy(),
                                       rtol=2e-6, atol=0)
        assert comp.evals == 5 + 9 + 13
        sur_chi = S.SurrogateChi2(sur, d, idx)
        theta0 = truth + rng.standard_normal((24, 9)) * scale
        cov = np.diag(scale ** 2) * 4.0
        comp2 = CompactExact(ec, d, k=8)
        ch, th, chi, acc, _, st = delayed_acceptance(ExactChi2(e, d, curves=True), sur_chi,
                                                     theta0, cov, 40, seed=3, compact=comp2)
        assert 0 < st["stage1_rate"] < 1 and acc > 0 and np.all(np.isfinite(chi))
        np.testing.assert_allclose(chi, exact(th), rtol=1e-5)
