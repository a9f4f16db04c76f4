"""The C oracle against golden fixtures produced by the reference itself
(tests/golden/make_golden.py, from oracle/_ref). Runs without the reference
sources; exact equality holds with the same libm (glibc) as the fixtures."""
import json
import os

import numpy as np
import pytest

from cases import glens_case, small_cases
from lcurve_re_b200 import abi
from lcurve_re_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "reference_outputs.npz"))
META = json.load(open(os.path.join(HERE, "golden", "reference_outputs.json")))
CASES = {c[0]: c for c in small_cases() + [glens_case()]}


@pytest.mark.parametrize("name", META["cases"])
def test_light_curves_match_golden(oracle, name):
    _, model, data = CASES[name]
    gdata = GOLD[name + "/data"].view(abi.datum_dtype())
    assert np.array_equal(np.asarray(data).view(np.uint8), GOLD[name + "/data"])
    st, err, calc, sfac, sc = oracle.light_curve(model, gdata)
    assert st == 0, err
    np.testing.assert_array_equal(calc, GOLD[name + "/calc"])
    np.testing.assert_array_equal(sfac, GOLD[name + "/sfac"])
    np.testing.assert_array_equal(sc[1:3], GOLD[name + "/chisq_wnok"])


@pytest.mark.parametrize("name", META["grids"])
def test_grids_match_golden(oracle, name):
    from golden.make_golden import GRID_MODELS
    m = W.model(**GRID_MODELS[name])
    for star in (0, 1):
        g = oracle.star_grid(m, star)
        for k, v in g.items():
            np.testing.assert_array_equal(v, GOLD["%s/star%d/%s" % (name, star + 1, k)], err_msg=k)
