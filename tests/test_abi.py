"""The C ABI library without a GPU: it loads, exports every entry point that
include/lcg.h declares, and its structures have the header's layout (checked
against a C compiler's sizeof/offsetof)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from lcurve_re_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "lcg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lcg_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from lcurve_re_b200.engine import load_library
    return load_library()


def test_library_loads_and_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(abi.PROTOTYPES), set(names) ^ set(abi.PROTOTYPES)
    assert lib.lcg_abi_version() == abi.LCG_ABI_VERSION


def test_no_device_is_an_error_not_a_fallback(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    opt = abi.LcgOptions()
    lib.lcg_default_options(C.byref(opt))
    st = lib.lcg_create(C.byref(ctx), C.byref(opt))
    assert st == abi.E_CUDA
    assert lib.lcg_last_error(None)


def _c_layout():
    fields = {
        "lcg_model": [f[0] for f in abi.LcgModel._fields_],
        "lcg_datum": [f[0] for f in abi.LcgDatum._fields_],
        "lcg_options": [f[0] for f in abi.LcgOptions._fields_],
    }
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "lcg.h"', "int main(void){"]
    for st, fs in fields.items():
        src.append('printf("%s size %%zu\\n", sizeof(%s));' % (st, st))
        for f in fs:
            src.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (st, f, st, f))
    src.append("return 0;}")
    d = tempfile.mkdtemp()
    c = os.path.join(d, "layout.c")
    open(c, "w").write("\n".join(src))
    exe = os.path.join(d, "layout")
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}


def test_struct_layouts_match_header():
    lay = _c_layout()
    for name, cls in (("lcg_model", abi.LcgModel), ("lcg_datum", abi.LcgDatum),
                      ("lcg_options", abi.LcgOptions)):
        assert lay[(name, "size")] == C.sizeof(cls), name
        for f in cls._fields_:
            assert lay[(name, f[0])] == getattr(cls, f[0]).offset, (name, f[0])
    assert abi.datum_dtype().itemsize == C.sizeof(abi.LcgDatum) == 48


def test_walk_entry_points_reject_bad_arguments_before_any_launch(lib):
    """lcg_walk_propose / lcg_walk_accept / lcg_walk_advance check their
    sizes and pointers on the host and return LCG_E_INVALID without touching
    the device (the dummy addresses below are never dereferenced)."""
    P = C.c_void_p(4096)  # non-NULL, never used: every call fails its checks first
    N = None
    propose = [  # (nc, d, par, y, ctr, step, noise, prop, xunit, ok)
        (0, 9, P, P, P, 0, N, P, P, P), (8, 0, P, P, P, 0, N, P, P, P),
        (8, 17, P, P, P, 0, N, P, P, P), (8, 9, N, P, P, 0, N, P, P, P),
        (8, 9, P, P, N, 0, N, P, P, P), (8, 9, P, P, P, -1, N, P, P, P),
        (8, 9, P, P, P, 0, N, P, N, P)]
    for nc, d, par, y, ctr, step, noise, prop, xu, ok in propose:
        assert lib.lcg_walk_propose(N, nc, d, par, y, 0, ctr, step, noise, prop, xu,
                                    ok) == abi.E_INVALID
    accept = [  # (nc, d, prop, ok, chi, y, chis, ctr, step, unif)
        (0, 9, P, P, P, P, P, P, 0, N), (8, 17, P, P, P, P, P, P, 0, N),
        (8, 9, P, P, N, P, P, P, 0, N), (8, 9, P, P, P, P, P, N, 0, N),
        (8, 9, P, P, P, P, P, P, -2, N)]
    for nc, d, prop, ok, chi, y, chis, ctr, step, unif in accept:
        assert lib.lcg_walk_accept(N, nc, d, prop, ok, chi, y, chis, N, 0, ctr, step,
                                   unif) == abi.E_INVALID
    assert lib.lcg_walk_advance(N, N, 1) == abi.E_INVALID
