"""The FP32 screen of the eclipse bisections (ecl_screen.cuh) on the CPU.

Mixed contexts ask fblink_screen first at every bisection midpoint and run
the FP64 Roche::fblink (fblink.cpp:34-104) only where the screen is unsure.
The screen must never disagree with the FP64 test: here both bisections of
every face of real grids (built by the C oracle) run with and without the
screen, and the ingress and egress phases must be identical bit for bit.
The screen must also take most of the tests on the white dwarf's faces, or
it is not worth running.
"""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

from lcurve_re_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "screen", "screen_check.cpp")
BUILD = os.path.join(HERE, "screen", "_build")
EXE = os.path.join(BUILD, "screen_check")


@pytest.fixture(scope="module")
def checker():
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    os.makedirs(BUILD, exist_ok=True)
    deps = [SRC] + [os.path.join(HERE, "..", "lcurve_re_b200", "csrc", f)
                    for f in ("eclipse.cuh", "ecl_screen.cuh", "roche.cuh")]
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(d) for d in deps):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", EXE, SRC])
    return EXE


def _run(exe, m, star, posn):
    c = m.to_c()
    ecl = 1 - star
    ri = np.radians(c.iangle)
    hdr = struct.pack("8d", c.q, np.cos(ri), np.sin(ri), c.delta_phase,
                      c.spin2 if ecl == 1 else c.spin1, c.r2 if ecl == 1 else c.r1, 0.0,
                      float(ecl))
    blob = hdr + struct.pack("q", posn.shape[0]) + np.ascontiguousarray(posn).tobytes()
    out = subprocess.run([exe], input=blob, capture_output=True, timeout=600)
    vals = [int(v) for v in out.stdout.split()]
    return out.returncode, dict(zip(("faces", "hits", "tests", "fp64", "true", "false", "bad"),
                                    vals))


def test_screen_keeps_every_fp64_decision(checker, oracle):
    ms, _ = W.mcmc_batch(256)
    picked = [ms[k] for k in (0, 2, 5, 9)]
    picked.append(W.wd_dm_small()[0])
    tests = fp64 = 0
    for m in picked:
        for star in (0, 1):
            g = oracle.star_grid(m, star)
            rc, r = _run(checker, m, star, g["posn"])
            assert rc == 0 and r["bad"] == 0, (star, r)
            if star == 0:
                tests += r["tests"]
                fp64 += r["fp64"]
    assert tests > 100000
    assert fp64 < 0.4 * tests, (fp64, tests)
