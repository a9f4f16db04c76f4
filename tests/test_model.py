"""Host-side Model/Data mirror: the reference's configuration rules
(model.cpp:10-360, lcurve.h:159-195, lcurve.cpp:18-85)."""
import json
import os

import numpy as np
import pytest

from lcurve_re_b200 import abi
from lcurve_re_b200 import workloads as W
from lcurve_re_b200.model import LcurveError, Model, Pparam, read_data, string_to_bool


def test_pparam_parsing():
    p = Pparam("0.25 0.01 0.001 1 1")
    assert (p.value, p.range, p.dstep, p.vary, p.defined) == (0.25, 0.01, 0.001, True, True)
    assert Pparam("1 0 0 0").defined  # defined defaults to true
    assert not Pparam("1 0 0 0 0").defined
    with pytest.raises(LcurveError):
        Pparam("1 2")


def test_string_to_bool():
    assert string_to_bool("yes") and string_to_bool("T") and not string_to_bool("0")
    with pytest.raises(LcurveError):
        string_to_bool("maybe")


def test_optional_parameters_default_to_zero():
    p = W.base_parameters()
    for k in ("pdot", "third", "temp_edge", "absorb_edge"):
        del p[k]
    m = Model({"model_parameters": p})
    assert m["pdot"] == 0.0 and m["third"] == 0.0


def test_missing_parameter_is_an_error():
    p = W.base_parameters()
    del p["q"]
    with pytest.raises(LcurveError, match="not initialised"):
        Model({"model_parameters": p})


def test_partial_spot_group_is_an_error():
    p = W.base_parameters()
    p["stsp11_long"] = "10 0 0 0 1"
    with pytest.raises(LcurveError):
        Model({"model_parameters": p})


def test_glens_with_roche1_is_an_error():
    p = W.base_parameters()
    p["glens1"] = "1"
    with pytest.raises(LcurveError, match="glens1"):
        Model({"model_parameters": p})


def test_bad_limb_law():
    p = W.base_parameters()
    p["limb1"] = "Linear"
    with pytest.raises(LcurveError, match="limb1"):
        Model({"model_parameters": p})


def test_spot_defined_flag_reaches_c_struct():
    m = W.model()
    assert m.to_c().stsp_defined[0] == 0
    p = W.base_parameters()
    for f in ("long", "lat", "fwhm", "tcen"):
        p["stsp21_" + f] = "10 0 0 0 1"
    m = Model({"model_parameters": p})
    assert list(m.to_c().stsp_defined) == [0, 0, 0, 1, 0]


def test_vary_order_and_set_param():
    m = W.model()
    names = m.vary_names()
    assert names[:4] == ["q", "iangle", "r1", "r2"]
    v = m.get_param()
    m.set_param(v * 1.01)
    assert m["q"] == pytest.approx(0.25 * 1.01)


def test_reference_example_config_parses(tmp_path):
    ref = os.path.join(os.environ.get("LCURVE_REF_DIR", "/root/reference"), "example",
                       "example.json")
    if not os.path.exists(ref):
        pytest.skip("reference example not present")
    text = open(ref).read()
    # the example file is not strict JSON (a missing comma); repair that only
    text = text.replace('"cov_epsilon": 1e-6\n', '"cov_epsilon": 1e-6,\n')
    m = Model(json.loads(text))
    assert m["q"] == 0.75 and m.c["limb1"] == abi.LIMB_POLY and m.c["nlat2f"] == 150


def test_read_data_rules(tmp_path):
    f = tmp_path / "lc.txt"
    f.write_text("# comment\n\n0.1 0.0 1.0 0.01 1 1\n0.2 0.001 1.1 -0.02 1 3\n")
    d = read_data(str(f))
    assert d.shape[0] == 2
    assert d["ferr"][1] == 0.0 and d["weight"][1] == 0.0 and d["ndiv"][1] == 3
    assert d.dtype.itemsize == 48


def test_tiling_overflow_nlat_match_numface_and_the_known_list(oracle):
    """workloads.tiling_overflows: the nlat at which the ring tiling lays more
    faces than numface sizes the reference's Point vector with. Its numface
    equals the oracle's face count (numface.cpp), and up to 1200 the overflow
    set is the one the GPU face-count tests pin."""
    for nlat in (30, 40, 80, 153, 200, 297, 306, 375, 393, 400, 813, 879):
        m = W.model(nlat1f=nlat, nlat2f=nlat)
        assert W._numface(nlat) == oracle.face_count(m, 0) == oracle.face_count(m, 1), nlat
    over = [k for k in range(1, 1201) if W.tiling_overflows(k)]
    assert over == [153, 297, 315, 333, 339, 549, 609, 621, 645, 686, 687, 705, 710, 758, 1173,
                    1191]
    assert [k for k in range(1, 1201) if W._tiled(k) < W._numface(k)] == [813, 879]
    ms, _ = W.mcmc_batch(256)
    assert sum(not W.reference_safe(m) for m in ms) == 8
