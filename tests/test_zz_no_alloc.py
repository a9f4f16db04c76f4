"""The allocation-free flux sweep, lcg_sum_star_multi_noalloc.

This entry point exists for callers in which the library must not allocate
device memory: programs whose device memory already belongs to another
framework's pooling allocator (an allocation from the library would fail),
and latency-critical loops where an allocation would synchronise the device.
It keeps its scratch in a fixed 16 MiB array inside the library instead.

The test calls it through the C ABI on device arrays the test owns and checks
it against the existing entry point, lcg_sum_star_multi on an FP64 context,
with the tolerance the FP64 sweep tests use (bit-identical), on two calls in
a row (star 1, then star 2: the shared scratch array holds the first call's
contents when the second runs), then repeats the first call. This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from lcurve_re_b200 import abi
from lcurve_re_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


class _Call:
    """One call's device arrays, allocated by the test (the caller) up front,
    so that the entry point itself can be run with nothing else allocating."""

    def __init__(self, torch, star, flat, ph, ldc, ltype, mucrit=0.0):
        self.torch = torch
        self.cols = {k: _dev(torch, flat[k]) for k in ("dx", "dy", "dz", "flux", "in1", "out1")}
        self.phs = {k: _dev(torch, ph[k]) for k in ("ex", "ey", "ez", "phin")}
        self.nent = self.phs["ex"].shape[0]
        self.out = torch.full((self.nent,), float("nan"), dtype=torch.float64, device="cuda")
        self.ldc = np.ascontiguousarray(ldc, dtype=np.float64)
        self.star, self.n0, self.ltype, self.mucrit = star, int(flat["n0"]), ltype, mucrit

    def run(self, lib):
        p = lambda t: C.c_void_p(t.data_ptr())
        c, q = self.cols, self.phs
        stream = C.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        return lib.lcg_sum_star_multi_noalloc(
            stream, self.star, c["dx"].shape[0], self.n0, p(c["dx"]), p(c["dy"]), p(c["dz"]),
            p(c["flux"]), p(c["in1"]), p(c["out1"]), self.nent, p(q["ex"]), p(q["ey"]),
            p(q["ez"]), p(q["phin"]), self.ldc.ctypes.data_as(C.POINTER(C.c_double)),
            self.ltype, self.mucrit, p(self.out))

    def result(self):
        self.torch.cuda.synchronize()
        return self.out.cpu().numpy()


def _noalloc(lib, torch, star, flat, ph, ldc, ltype, mucrit=0.0):
    call = _Call(torch, star, flat, ph, ldc, ltype, mucrit)
    st = call.run(lib)
    return st, call.result()


def test_noalloc_sweep_matches_existing_entry_point(engine_fp64, oracle):
    import torch
    from lcurve_re_b200.engine import load_library
    lib = load_library()
    m = W.model()
    ph = oracle.phase_batch(m, W.data(700, ndiv=3, expose=0.002))
    mc = m.to_c()
    first = None
    for star, ldc in ((abi.STAR1, list(mc.ldc1)), (abi.STAR2, list(mc.ldc2))):
        flat = oracle.flatten(oracle.star_grid(m, star))
        expected = engine_fp64.sum_star_multi(star, flat, ph, ldc=ldc, ltype=abi.LIMB_CLARET)
        st, got = _noalloc(lib, torch, star, flat, ph, ldc, abi.LIMB_CLARET)
        assert st == abi.OK
        assert np.array_equal(got, expected), (star, np.max(np.abs(got - expected)))
        if first is None:
            first = (star, flat, ldc, expected)
    star, flat, ldc, expected = first
    st, got = _noalloc(lib, torch, star, flat, ph, ldc, abi.LIMB_CLARET)
    assert st == abi.OK and np.array_equal(got, expected)


def test_noalloc_polynomial_limb_darkening_with_mucrit(engine_fp64, oracle):
    """The polynomial limb-darkening law and a critical mu above zero, on both
    stars, two calls in a row: still bit-identical to the existing sweep."""
    import torch
    from lcurve_re_b200.engine import load_library
    lib = load_library()
    m = W.model()
    ph = oracle.phase_batch(m, W.data(600, ndiv=2, expose=0.003))
    ldc = [0.4, 0.25, -0.1, 0.05]
    for star, mucrit in ((abi.STAR2, 0.12), (abi.STAR1, 0.3)):
        flat = oracle.flatten(oracle.star_grid(m, star))
        expected = engine_fp64.sum_star_multi(star, flat, ph, ldc=ldc, ltype=abi.LIMB_POLY,
                                              mucrit=mucrit)
        st, got = _noalloc(lib, torch, star, flat, ph, ldc, abi.LIMB_POLY, mucrit)
        assert st == abi.OK
        assert np.array_equal(got, expected), (star, np.max(np.abs(got - expected)))


def test_noalloc_allocates_nothing_and_keeps_the_callers_device(engine_fp64, oracle):
    """Across a second call (the first one has looked up the scratch array and
    loaded the kernels), the device's free memory does not move, and the
    caller's current device is the one it had before."""
    import torch
    from lcurve_re_b200.engine import load_library
    lib = load_library()
    m = W.model()
    ph = oracle.phase_batch(m, W.data(500))
    flat = oracle.flatten(oracle.star_grid(m, abi.STAR2))
    ldc = list(m.to_c().ldc2)
    call = _Call(torch, abi.STAR2, flat, ph, ldc, abi.LIMB_CLARET)
    dev = torch.cuda.current_device()
    assert call.run(lib) == abi.OK
    first = call.result()
    free0, _ = torch.cuda.mem_get_info()
    assert call.run(lib) == abi.OK
    second = call.result()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.current_device() == dev
    assert np.array_equal(first, second)


def test_noalloc_empty_grid_gives_zero_sums():
    """n = 0: no face block, every phase entry's sum is exactly zero."""
    import torch
    from lcurve_re_b200.engine import load_library
    lib = load_library()
    nent = 300
    ph = {k: np.linspace(-0.5, 0.5, nent) for k in ("ex", "ey", "ez", "phin")}
    flat = {k: np.zeros(0) for k in ("dx", "dy", "dz", "flux", "in1", "out1")}
    flat["n0"] = 0
    st, got = _noalloc(lib, torch, abi.STAR1, flat, ph, [0.1, 0.2, 0.3, 0.1], abi.LIMB_CLARET)
    assert st == abi.OK
    assert np.array_equal(got, np.zeros(nent))


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from lcurve_re_b200.engine import load_library
    lib = load_library()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    ldc = np.zeros(4)
    # 2048 blocks x 2048 entries = 4,194,304 partials > 2,097,152: refused before any access
    st = lib.lcg_sum_star_multi_noalloc(None, abi.STAR2, 2048 * 1024, 2048 * 1024, p, p, p, p, p,
                                        p, 2048, p, p, p, p,
                                        ldc.ctypes.data_as(C.POINTER(C.c_double)),
                                        abi.LIMB_CLARET, 0.0, p)
    assert st == abi.E_CAPACITY
    # 65,537 blocks x 1 entry fits the array but not the launch's grid.y limit
    n = 65537 * 1024
    st = lib.lcg_sum_star_multi_noalloc(None, abi.STAR2, n, n, p, p, p, p, p, p, 1, p, p, p, p,
                                        ldc.ctypes.data_as(C.POINTER(C.c_double)),
                                        abi.LIMB_CLARET, 0.0, p)
    assert st == abi.E_CAPACITY
