"""The mixed sweeps' eclipse test in 64-bit fixed-point phase
(lcurve_re_b200/csrc/fixed_phase.cuh) against the reference's double test
(ecl_range, comp_light_flat.cpp:171-173), on the CPU: the device functions
are compiled for the host by tests/screen/fixed_phase_check.cpp and decide
millions of random and adversarial (phase, ingress, egress) triples exactly
as the reference does; only phases and boundaries below 2^-12 within 2^-64
of each other may differ."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "screen", "fixed_phase_check.cpp")
HDR = os.path.join(HERE, "..", "lcurve_re_b200", "csrc", "fixed_phase.cuh")
EXE = os.path.join(HERE, "screen", "_build", "fixed_phase_check")


def test_fixed_point_eclipse_test_decides_as_the_reference():
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(SRC),
                                                              os.path.getmtime(HDR)):
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-o", EXE, SRC])
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    cases, bad, tiny = (int(v) for v in r.stdout.split()[-3:])
    assert cases > 5_000_000 and bad == 0
