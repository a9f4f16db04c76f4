"""lcurve_re's own executables, unchanged, on the GPU engine.

tests/solvers/Makefile builds lcurve_re (main.cpp), lcurve_simplex
(new_scripts/simplex.cpp), lcurve_mcmc (new_scripts/mcmc_solver.cpp) and
lcurve_levmarq (new_scripts/levmarq_solver.cpp) from the reference's sources
twice: with the reference's light_curve_comp.cpp (its FP64 CPU path) and with
the drop-in shim linked against liblcg.so. Each pair runs here on the same
config and light curve (written by the test in the reference's JSON and
six-column text formats, plot_device "none", a few iterations), and the
numbers each prints are compared:

  lcurve_re        chi**2, scale factor, white dwarf's contribution, log g
  lcurve_simplex   best chi**2 and the fitted parameters after 20 iterations
  lcurve_mcmc      the chain file (step, parameters, chi**2) after 30 steps
  lcurve_levmarq   initial and best chi**2 after 5 iterations

With LCURVE_CUDA_PRECISION=fp64 (the shim reads the reference's own switch)
every printed number agrees to 1e-6 relative; in the mixed default the
first chi**2 of each solver agrees to 1e-5.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

from lcurve_re_b200 import workloads as W

pytestmark = pytest.mark.gpu

BUILD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "solvers", "_build")
EXES = ("lcurve_re", "lcurve_simplex", "lcurve_mcmc", "lcurve_levmarq")
NUM = r"([-+0-9.eEinfa]+)"


def _exe(variant, name):
    p = os.path.join(BUILD, variant, name)
    if not os.path.exists(p):
        pytest.skip("solver executables not built (make -C tests/solvers)")
    return p


@pytest.fixture(scope="module")
def inputs(tmp_path_factory, oracle):
    """A config JSON and a 200-point light curve (the benchmark physics at
    nlat 20/40 plus seeded noise) in the reference's formats."""
    d = tmp_path_factory.mktemp("solver_inputs")
    p = W.base_parameters()
    for k in ("nlat1f", "nlat1c"):
        p[k] = "20"
    for k in ("nlat2f", "nlat2c"):
        p[k] = "40"
    data = W.data(200)
    st, err, calc, _, _ = oracle.light_curve(W.model(nlat1f=20, nlat2f=40), data, scale=False,
                                             rdata=False)
    assert st == 0, err
    data = W.add_noise(data, calc, 3)
    with open(d / "lc.txt", "w") as f:
        for r in data:
            f.write("%.17g %.17g %.17g %.17g %.17g %d\n" % (r["time"], r["expose"], r["flux"],
                                                           r["ferr"], r["weight"], r["ndiv"]))
    cfg = {"model_parameters": p, "data_file_path": "lc.txt", "noise": 0, "seed": 42,
           "output_file_path": "out.txt", "plot_device": "none", "autoscale": True,
           "sstar1": 1, "sstar2": 1, "sdisc": 1, "sspot": 1, "ssfac": 1,
           "time1": -0.2, "time2": 1.2, "ntime": 200, "expose": 0, "ndivide": 1,
           "mcmc_steps": 30, "mcmc_burn_in": 10, "mcmc_thin": 1, "chain_out_path": "chain.txt",
           "use_priors": False, "true_period": 1.0, "adapt_enabled": False,
           "anneal_enabled": False, "simplex_max_iter": 20, "lm_max_iter": 5,
           "lm_multistart": 0, "lm_error_mcmc": False, "lm_continuation": False,
           "lm_reanchor_rounds": 0, "lm_log_path": "lm.txt", "priors": {}}
    with open(d / "cfg.json", "w") as f:
        json.dump(cfg, f, indent=1)
    return d


def _run(inputs, tmp_path, variant, name, precision=None):
    run = tmp_path / ("%s_%s_%s" % (variant, name, precision or "default"))
    run.mkdir()
    for f in ("cfg.json", "lc.txt"):
        (run / f).write_bytes((inputs / f).read_bytes())
    env = dict(os.environ)
    env.pop("LCURVE_CUDA_PRECISION", None)
    if precision:
        env["LCURVE_CUDA_PRECISION"] = precision
    r = subprocess.run([_exe(variant, name), "cfg.json"], cwd=run, capture_output=True,
                       text=True, timeout=900, env=env)
    assert r.returncode == 0, (variant, name, r.stdout[-2000:], r.stderr[-2000:])
    return r.stdout, run


def _find(pattern, text):
    m = re.findall(pattern, text)
    assert m, pattern
    return [float(x) for x in (m if isinstance(m[0], str) else m[0])]


def _numbers(name, out, run):
    """The figures each executable reports, as a flat array."""
    if name == "lcurve_re":
        return np.array(_find(r"Weighted chi\*\*2 = " + NUM, out) +
                        _find(r"Scale factor = " + NUM, out) +
                        _find(r"White dwarf's contribution = " + NUM, out) +
                        _find(r"log10\(g1 \[cgs\]\) = " + NUM, out) +
                        _find(r"log10\(g2 \[cgs\]\) = " + NUM, out))
    if name == "lcurve_simplex":
        best = _find(r"Best χ²\s+= " + NUM, out)
        pars = [float(v) for v in re.findall(r"^\w+ = " + NUM + r"$", out, re.M)]
        return np.array(best + pars)
    if name == "lcurve_mcmc":
        rows = [line.split(",") for line in open(run / "chain.txt").read().splitlines()[1:]]
        return np.array([[float(v) for v in r] for r in rows]).ravel()
    first = _find(r"Initial\s+χ²\(LC\) = " + NUM, out)
    best = re.findall(r"Best solution:.*?χ²\(LC\) = " + NUM, out, re.S)
    return np.array(first + [float(best[-1])])


def _first_chi2(name, nums):
    return nums[9] if name == "lcurve_mcmc" else nums[0]


@pytest.mark.parametrize("name", EXES)
def test_solver_runs_unchanged_on_the_engine_fp64(inputs, tmp_path, name):
    ref_out, ref_run = _run(inputs, tmp_path, "ref", name)
    lcg_out, lcg_run = _run(inputs, tmp_path, "lcg", name, precision="fp64")
    a, b = _numbers(name, ref_out, ref_run), _numbers(name, lcg_out, lcg_run)
    assert a.shape == b.shape and a.size > 0, (a, b)
    np.testing.assert_allclose(b, a, rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("name", EXES)
def test_solver_first_chi2_mixed_precision(inputs, tmp_path, name):
    ref_out, ref_run = _run(inputs, tmp_path, "ref", name)
    lcg_out, lcg_run = _run(inputs, tmp_path, "lcg", name)
    a = _first_chi2(name, _numbers(name, ref_out, ref_run))
    b = _first_chi2(name, _numbers(name, lcg_out, lcg_run))
    assert abs(b - a) <= 1e-5 * abs(a), (a, b)
