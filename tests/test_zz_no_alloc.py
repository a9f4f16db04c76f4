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


def _noalloc(lib, torch, star, flat, ph, ldc, ltype):
    cols = {k: _dev(torch, flat[k]) for k in ("dx", "dy", "dz", "flux", "in1", "out1")}
    phs = {k: _dev(torch, ph[k]) for k in ("ex", "ey", "ez", "phin")}
    nent = phs["ex"].shape[0]
    out = torch.full((nent,), float("nan"), dtype=torch.float64, device="cuda")
    ldc_h = np.ascontiguousarray(ldc, dtype=np.float64)
    p = lambda t: C.c_void_p(t.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = lib.lcg_sum_star_multi_noalloc(
        stream, star, cols["dx"].shape[0], int(flat["n0"]), p(cols["dx"]), p(cols["dy"]),
        p(cols["dz"]), p(cols["flux"]), p(cols["in1"]), p(cols["out1"]), nent, p(phs["ex"]),
        p(phs["ey"]), p(phs["ez"]), p(phs["phin"]), ldc_h.ctypes.data_as(C.POINTER(C.c_double)),
        ltype, 0.0, p(out))
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


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
