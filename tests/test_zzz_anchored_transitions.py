"""Surrogate transitions with each chain's approximation anchored at a fixed
state (surrogate.FixedAnchorChi2) on the GPU.

  * the anchored approximation at its own anchor is the chi**2 of the
    anchor's exact curve (s(r) / s(r) = 1), and away from it equals the
    anchored chi**2 head of the delayed-acceptance screen;
  * the inner steps replayed as a CUDA graph with the anchors in the chi**2
    head, fed the host generator's normals and uniforms, give the chains of
    the host loop over the same approximation.

This file is collected last, after every other GPU test.
"""
import numpy as np
import pytest

from lcurve_re_b200 import surrogate as S
from lcurve_re_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    import torch
    from lcurve_re_b200.engine import Engine
    from lcurve_re_b200.sampler import ExactChi2, TriangularWalk
    e = Engine(precision="mixed")
    theta, curves = S.training_set(e, 8192, seed=51, batch=2048)
    sur = S.Surrogate(batch=2048, seed=0)
    sur.fit(theta, curves, epochs=30, lr=2e-3)
    idx = np.arange(0, S.NGRID, 2)
    truth = np.array([0.25, 86.0, 0.015, 0.20, 20000.0, 3200.0, 0.08, 0.5, 0.0])
    calc = e.light_curve_comp(S.ModelFactory()(truth[None])[0], W.data(S.NGRID, -0.2, 1.2),
                              scale=False, rdata=False, sfac=np.ones(5), diagnostics=False)[0]
    d = W.add_noise(W.data(S.NGRID, -0.2, 1.2)[idx], calc[idx], 52)
    rng = np.random.default_rng(53)
    scale = (S.BOX[:, 1] - S.BOX[:, 0]) * 2e-3
    tw = TriangularWalk(truth + rng.standard_normal((4096, 9)) * scale, scale=0.5)
    theta0 = truth + rng.standard_normal((48, 9)) * scale
    sur_chi = S.SurrogateChi2(sur, d, idx)
    ex = ExactChi2(e, d, curves=True)
    chi0 = ex(theta0)
    f0 = torch.empty((len(theta0), len(idx)), dtype=torch.float64, device="cuda")
    ex.curves_all_device(f0)
    yield e, d, sur_chi, tw, theta0, chi0, f0
    e.close()


def test_fixed_anchor_is_the_anchored_head(case):
    e, d, sur_chi, tw, theta0, chi0, f0 = case
    fixed = sur_chi.fixed_anchor(theta0, f0)
    at_anchor = fixed(theta0)
    # the head's own chi**2 of the exact curves (same optimal scale and sums)
    np.testing.assert_allclose(at_anchor, chi0, rtol=1e-5)
    y = tw.apply_rows(theta0, np.random.default_rng(54).standard_normal((len(theta0), 9))
                      @ tw.chol.T)
    ref = sur_chi.chi2(sur_chi.state(y), sur_chi.state(theta0), f0)
    np.testing.assert_array_equal(fixed(y), ref)
    coef, curves = fixed.rows(slice(8, 20))
    assert coef.shape == (12, fixed.coef_ref.shape[1]) and curves.shape == (12, len(d))


def test_anchored_device_transitions_equal_the_host_loop(case):
    from lcurve_re_b200.sampler import DeviceTransitions, ExactChi2, surrogate_transitions
    e, d, sur_chi, tw, theta0, chi0, f0 = case
    fixed = sur_chi.fixed_anchor(theta0, f0)
    nc, steps, inner = len(theta0), 10, 5
    host = surrogate_transitions(ExactChi2(e, d), fixed, theta0, None, steps, inner, seed=55,
                                 propose=tw.with_scale(tw.scale))
    devt = DeviceTransitions(sur_chi, tw, S.BOX, nc, inner, host_draws=True,
                             anchor=fixed.rows(slice(0, nc)))
    got = surrogate_transitions(ExactChi2(e, d), fixed, theta0, None, steps, inner, seed=55,
                                device=devt)
    np.testing.assert_allclose(got[0], host[0], rtol=1e-10, atol=0)
    assert got[5] == host[5] and 0 < host[5]["inner_acceptance"] < 1, host[5]
    assert host[5]["runs_moved"] > 0
