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


def _walk_case(trained, nc, seed):
    """Data around a known model, a triangular walk fitted to a cloud of
    parameters around it (narrow, so that the inner steps accept), and
    starting states."""
    from lcurve_re_b200.sampler import TriangularWalk
    e, sur, theta, curves, _ = trained
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    calc = e.light_curve_comp(S.ModelFactory()(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                              scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)[0]
    d = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 9)
    rng = np.random.default_rng(seed)
    scale = (S.BOX[:, 1] - S.BOX[:, 0]) * 2e-3
    cloud = truth + rng.standard_normal((4096, 9)) * scale
    cloud[:, 1] += 40 * (cloud[:, 0] - truth[0]) ** 2  # some curvature for the map
    tw = TriangularWalk(cloud, scale=0.5)
    theta0 = truth + rng.standard_normal((nc, 9)) * scale
    return e, sur, d, idx, tw, theta0


def test_device_walk_matches_the_host_walk(trained):
    """lcg_walk_propose with given normals forms the triangular walk's
    proposals (TriangularWalk.apply_rows) to 1e-11 of the box, the network's FP32
    input coordinates as surrogate.to_unit does, and the box test as
    surrogate.in_box; lcg_walk_accept takes the host loop's decisions."""
    import ctypes as C
    import torch
    from lcurve_re_b200.sampler import walk_parameters
    e, sur, d, idx, tw, theta0 = _walk_case(trained, 300, 16)
    lib = e.lib
    nc = theta0.shape[0]
    theta0[:40, 0] = S.BOX[0, 1] - 1e-5  # at the box's edge: some proposals leave it
    rng = np.random.default_rng(17)
    n = rng.standard_normal((nc, 9)) * 3.0
    p = lambda t: C.c_void_p(t.data_ptr())
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    par, y, nz = dev(walk_parameters(tw, S.BOX)), dev(theta0), dev(n)
    prop = torch.zeros((nc, 9), dtype=torch.float64, device="cuda")
    xu = torch.zeros((nc, 9), dtype=torch.float32, device="cuda")
    ok = torch.zeros(nc, dtype=torch.uint8, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.lcg_walk_propose(s, nc, 9, p(par), p(y), 0, None, 0, p(nz), p(prop), p(xu),
                                p(ok)) == 0
    got = prop.cpu().numpy()
    ref = tw.apply_rows(theta0, n @ tw.chol.T)
    # rounding of the map relative to the box, for the states inside the cloud the
    # map was fitted to (far outside it, 250 sd away at the box's edge, the
    # quadratic terms amplify it; there only the box test is compared)
    width = S.BOX[:, 1] - S.BOX[:, 0]
    assert np.max(np.abs(got[40:] - ref[40:]) / width) < 1e-11
    assert np.array_equal(xu.cpu().numpy(), S.to_unit(got).astype(np.float32))
    okh = ok.cpu().numpy().astype(bool)
    assert np.array_equal(okh, S.in_box(got)) and 0 < okh.sum() < nc
    # the decision: chi**2 of the proposals against the states'
    chi = rng.uniform(0, 8, nc)
    chis = rng.uniform(0, 8, nc)
    u = rng.random(nc)
    chi_d, chis_d, moves = dev(chi), dev(chis), torch.zeros(nc, dtype=torch.int32, device="cuda")
    assert lib.lcg_walk_accept(s, nc, 9, p(prop), p(ok), p(chi_d), p(y), p(chis_d), p(moves), 0,
                               None, 0, p(dev(u))) == 0
    a = okh & (np.log(u) < -(chi - chis) / 2)
    assert np.array_equal(moves.cpu().numpy().astype(bool), a) and a.any() and not a.all()
    np.testing.assert_array_equal(y.cpu().numpy(), np.where(a[:, None], got, theta0))
    np.testing.assert_array_equal(chis_d.cpu().numpy(), np.where(a, chi, chis))


def test_device_surrogate_transitions_equal_the_host_loop(trained):
    """The inner steps replayed as a CUDA graph (walk, network, chi**2 head,
    decision per step) with the host generator's normals and uniforms give
    the host loop's chains; with the device's own Philox draws the chains
    stay inside the box and the inner acceptance is that of the host loop's
    to a few percent."""
    from lcurve_re_b200.sampler import DeviceTransitions, ExactChi2, surrogate_transitions
    e, sur, d, idx, tw, theta0 = _walk_case(trained, 64, 18)
    sur_chi = S.SurrogateChi2(sur, d, idx)
    nc, steps, inner = theta0.shape[0], 12, 6
    host = surrogate_transitions(ExactChi2(e, d), sur_chi, theta0, None, steps, inner, seed=19,
                                 propose=tw.with_scale(tw.scale))
    devt = DeviceTransitions(sur_chi, tw, S.BOX, nc, inner, host_draws=True)
    got = surrogate_transitions(ExactChi2(e, d), sur_chi, theta0, None, steps, inner, seed=19,
                                device=devt)
    np.testing.assert_allclose(got[0], host[0], rtol=1e-10, atol=0)
    assert got[5] == host[5] and 0 < host[5]["inner_acceptance"] < 1, host[5]
    assert host[5]["runs_moved"] > 0 and 0 <= host[3] <= 1
    assert devt.launches == steps * (4 * inner + 1)
    philox = DeviceTransitions(sur_chi, tw, S.BOX, nc, inner, seed=5)
    ch, _, _, acc, _, st = surrogate_transitions(ExactChi2(e, d), sur_chi, theta0, None, 40,
                                                 inner, seed=20, device=philox)
    assert np.all(S.in_box(ch.reshape(-1, 9)))
    assert abs(st["inner_acceptance"] - host[5]["inner_acceptance"]) < 0.1, (st, host[5])
    assert int(philox.ctr.item()) == (40 + 1) * inner  # the capture's warm-up run, then 40
