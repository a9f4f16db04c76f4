"""The drop-in shim: lcurve_re's own sources with light_curve_comp.cpp replaced
by lcurve_re_b200/shim/light_curve_comp_lcg.cpp (tests/shim/Makefile builds
tests/shim/_build/liblcurve_lcg.so where the reference sources are present;
the built library travels with the repository).

Through that library, Lcurve::Model comes from the reference's own JSON
parsing and Lcurve::light_curve_comp is called exactly as the reference's
solvers call it, but runs on the engine:
  * without a GPU the call fails with the engine's "no CUDA device" error
    (it did not fall back to the reference's CPU path);
  * on a GPU its light curves equal the oracle's to the mixed-precision bar
    (1e-5 per point), chi**2 to 1e-5 relative, and a lobe overflow raises
    Lcurve_Error with the reference's own message.
"""
import os

import numpy as np
import pytest

from cases import small_cases
from lcurve_re_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM_SO = os.path.join(HERE, "shim", "_build", "liblcurve_lcg.so")

needs_shim = pytest.mark.skipif(not os.path.exists(SHIM_SO),
                                reason="the shim library is built where the reference is")


def _shimmed():
    from oracle_lib import Reference
    return Reference(SHIM_SO)


@needs_shim
def test_shim_routes_to_the_engine_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    st, err, *_ = _shimmed().light_curve(W.model(nlat1f=8, nlat2f=8), W.data(10))
    assert st != 0 and "CUDA" in err, (st, err)


@needs_shim
@pytest.mark.gpu
def test_shim_light_curves_match_the_oracle(oracle):
    shim = _shimmed()
    for name, m, d in small_cases()[:6]:
        st, err, calc, sf, sc = shim.light_curve(m, d)
        assert st == 0, (name, err)
        so, erro, co, sfo, sco = oracle.light_curve(m, d)
        rel = np.max(np.abs(calc - co) / np.maximum(np.abs(co), 1e-300))
        assert rel <= 1e-5, (name, rel)
        assert abs(sc[1] - sco[1]) <= 1e-5 * abs(sco[1]) + 1e-12, name


@needs_shim
@pytest.mark.gpu
def test_shim_raises_the_reference_error(reference):
    m = W.model(nlat1f=8, nlat2f=8, r2=0.5)
    st, err, *_ = _shimmed().light_curve(m, W.data(20))
    st_r, err_r, *_ = reference.light_curve(m, W.data(20))
    assert st == st_r != 0 and err == err_r


@needs_shim
@pytest.mark.gpu
def test_shim_evaluates_disc_models(oracle):
    """A cataclysmic variable (opaque disc, rim, bright spot) and an iscale fit
    through the reference's own Model parsing and the shim."""
    from cases import disc_cases
    shim = _shimmed()
    for name, m, d in disc_cases()[2:5]:
        st, err, calc, sf, sc = shim.light_curve(m, d)
        assert st == 0, (name, err)
        so, erro, co, sfo, sco = oracle.light_curve(m, d)
        assert so == 0, erro
        rel = np.max(np.abs(calc - co) / np.maximum(np.abs(co), 1e-300))
        assert rel <= 1e-5, (name, rel)
