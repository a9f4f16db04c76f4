"""The batched Jacobian on the engine against the same scheme driven by the C
oracle: FP64 contexts, so the finite differences of the two agree to the
engine's light-curve parity (1e-6 relative per point, here far smaller)."""
import numpy as np
import pytest

from lcurve_re_b200 import workloads as W
from lcurve_re_b200.engine import Engine
from lcurve_re_b200.solvers import engine_evaluator, jacobian

pytestmark = pytest.mark.gpu


def test_engine_jacobian_matches_the_oracle(oracle):
    m = W.model(nlat1f=20, nlat2f=40)
    d = W.data(200)
    st, err, calc, _, _ = oracle.light_curve(m, d, scale=False, rdata=False)
    d = W.add_noise(d, calc, 3)
    names = ["q", "iangle", "r1", "r2", "t1", "t2"]

    def ev(models):
        out, ok = [], []
        for mm in models:
            s, e, c, sf, sc = oracle.light_curve(mm, d)
            out.append(c)
            ok.append(s == 0)
        return np.array(out), np.array(ok)
    Jo = jacobian(ev, m, names, d, limits=[(0.01, 1.0), (60.0, 90.0), (0.001, 0.1),
                                           (0.05, 0.3), (5000, 50000), (2000, 10000)])
    with Engine(precision="fp64") as e:
        Je = jacobian(engine_evaluator(e, d), m, names, d,
                      limits=[(0.01, 1.0), (60.0, 90.0), (0.001, 0.1), (0.05, 0.3),
                              (5000, 50000), (2000, 10000)])
    for j in range(len(names)):
        np.testing.assert_allclose(Je[:, j], Jo[:, j], rtol=0, atol=1e-4 * np.abs(Jo[:, j]).max(),
                                   err_msg=names[j])
