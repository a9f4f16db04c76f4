"""Python front end of the B200 light-curve engine (liblcg.so, include/lcg.h).

Engine.light_curve_comp mirrors Lcurve::light_curve_comp
(src/lcurve_base/lcurve.h:669-674): same arguments, same meaning of scale /
rdata / info / diagnostics, sfac read when scale is false and written when it
is true, and LcurveError where the reference throws. There is no CPU
fallback: if the library cannot be loaded or no sm_100 device is present,
construction fails.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .model import Data, LcurveError, Model

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblcg.so")
_lib = None


def load_library(path=LIB_PATH):
    """Loads liblcg.so (no GPU needed to load it)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError("liblcg.so is not built: run `python -m lcurve_re_b200.build` (%s)" % path)
        _lib = abi.bind(C.CDLL(path))
        if _lib.lcg_abi_version() != abi.LCG_ABI_VERSION:
            raise OSError("liblcg.so ABI version mismatch")
    return _lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _as_model(m):
    return m.to_c() if isinstance(m, Model) else m


def _as_data(d):
    if isinstance(d, np.ndarray) and d.dtype == abi.datum_dtype():
        return np.ascontiguousarray(d)
    raise LcurveError("data must be an lcurve_re_b200.Data / datum-dtype array")


class Engine:
    """One engine context: a CUDA stream, device buffers and the grid cache."""

    def __init__(self, device=0, precision="mixed", verbose=0, eclipse_warp=0):
        self.lib = load_library()
        opt = abi.LcgOptions()
        self.lib.lcg_default_options(C.byref(opt))
        opt.device = device
        opt.precision = {"mixed": abi.PREC_MIXED, "fp64": abi.PREC_FP64}[precision]
        opt.verbose = verbose
        opt.eclipse_warp = eclipse_warp
        ctx = C.c_void_p()
        st = self.lib.lcg_create(C.byref(ctx), C.byref(opt))
        if st != abi.OK:
            raise LcurveError("lcg_create: %s" % self.lib.lcg_last_error(None).decode(), st)
        self.ctx = ctx
        self.precision = precision

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.lcg_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        if st != abi.OK:
            raise LcurveError(self.lib.lcg_last_error(self.ctx).decode(), st)

    @property
    def stream_ptr(self):
        return self.lib.lcg_stream(self.ctx)

    # -- the hot path -------------------------------------------------------
    def light_curve_comp(self, model, data, scale=True, rdata=True, info=False, sfac=None,
                         diagnostics=True, no_cache=False, calc_out=None):
        """Returns (calc, wdwarf, chisq, wnok, logg1, logg2, rv1, rv2); sfac
        (a length-5 float64 array) is updated in place as the reference does."""
        m = _as_model(model)
        d = _as_data(data)
        n = d.shape[0]
        if sfac is None:
            sfac = np.ones(5)
        if not (isinstance(sfac, np.ndarray) and sfac.dtype == np.float64 and sfac.size >= 5):
            raise LcurveError("sfac must be a float64 array of size >= 5")
        calc = calc_out if calc_out is not None else np.empty(n)
        sc = np.zeros(abi.NOUT)
        flags = ((abi.FLAG_SCALE if scale else 0) | (abi.FLAG_RDATA if rdata else 0) |
                 (abi.FLAG_INFO if info else 0) | (abi.FLAG_DIAGNOSTICS if diagnostics else 0) |
                 (abi.FLAG_NO_CACHE if no_cache else 0))
        self._check(self.lib.lcg_light_curve(self.ctx, C.byref(m), d.ctypes.data, n, flags,
                                             _dptr(sfac), _dptr(calc), _dptr(sc)))
        return (calc, sc[abi.OUT_WDWARF], sc[abi.OUT_CHISQ], sc[abi.OUT_WNOK], sc[abi.OUT_LOGG1],
                sc[abi.OUT_LOGG2], sc[abi.OUT_RV1], sc[abi.OUT_RV2])

    def light_curve_comp_fast(self, model, data, max_model_points, scale=True, rdata=True,
                              sfac=None, diagnostics=False):
        """Lcurve::light_curve_comp_fast: above max_model_points points, the
        curve at points uniform in index, interpolated in time. Returns
        (calc, chisq, wnok); sfac updated in place."""
        m = _as_model(model)
        d = _as_data(data)
        n = d.shape[0]
        if sfac is None:
            sfac = np.ones(5)
        calc = np.empty(n)
        sc = np.zeros(abi.NOUT)
        flags = ((abi.FLAG_SCALE if scale else 0) | (abi.FLAG_RDATA if rdata else 0) |
                 (abi.FLAG_DIAGNOSTICS if diagnostics else 0))
        self._check(self.lib.lcg_light_curve_fast(self.ctx, C.byref(m), d.ctypes.data, n, flags,
                                                  max_model_points, _dptr(sfac), _dptr(calc),
                                                  _dptr(sc)))
        return calc, sc[abi.OUT_CHISQ], sc[abi.OUT_WNOK]

    def light_curve_batch(self, models, data, scale=True, rdata=True, sfac=None):
        ms = (abi.LcgModel * len(models))(*[_as_model(m) for m in models])
        d = _as_data(data)
        nm, n = len(models), d.shape[0]
        sf = np.ones(5 * nm) if sfac is None else np.ascontiguousarray(sfac, dtype=np.float64)
        calc = np.zeros((nm, n))
        chisq = np.zeros(nm)
        wnok = np.zeros(nm)
        status = np.zeros(nm, dtype=np.int32)
        flags = (abi.FLAG_SCALE if scale else 0) | (abi.FLAG_RDATA if rdata else 0)
        self._check(self.lib.lcg_light_curve_batch(
            self.ctx, ms, nm, d.ctypes.data, n, flags, _dptr(sf), _dptr(calc), _dptr(chisq),
            _dptr(wnok), status.ctypes.data_as(C.POINTER(C.c_int32))))
        return calc, chisq, wnok, sf.reshape(nm, 5), status

    def set_data(self, data):
        """Copies the points to the device once (lcg_set_data) for the
        resident calls."""
        d = _as_data(data)
        self._check(self.lib.lcg_set_data(self.ctx, d.ctypes.data, d.shape[0]))
        self._n = d.shape[0]

    def light_curve_batch_resident(self, models, scale=True, rdata=True, sfac=None, calc=True,
                                   buffers=None):
        """lcg_light_curve_batch over the points of set_data; calc=False
        returns only chi**2 (calc is None). buffers (a dict, kept by the
        caller) lets repeated calls of one size reuse their output arrays."""
        ms = models if isinstance(models, C.Array) else \
            (abi.LcgModel * len(models))(*[_as_model(m) for m in models])
        nm, n = len(ms), self._n
        b = buffers if buffers is not None else {}
        if b.get("shape") != (nm, n, bool(calc)):
            b.clear()
            b.update(shape=(nm, n, bool(calc)), out=np.zeros((nm, n)) if calc else None,
                     chisq=np.zeros(nm), wnok=np.zeros(nm), status=np.zeros(nm, np.int32),
                     sf=np.ones(5 * nm))
        out, chisq, wnok, status = b["out"], b["chisq"], b["wnok"], b["status"]
        if sfac is None:
            sf = b["sf"]
            sf[:] = 1.0
        else:
            sf = np.ascontiguousarray(sfac, dtype=np.float64)
        flags = (abi.FLAG_SCALE if scale else 0) | (abi.FLAG_RDATA if rdata else 0)
        self._check(self.lib.lcg_light_curve_batch_resident(
            self.ctx, ms, nm, flags, _dptr(sf), _dptr(out) if calc else None, _dptr(chisq),
            _dptr(wnok), status.ctypes.data_as(C.POINTER(C.c_int32))))
        return out, chisq, wnok, sf.reshape(nm, 5), status

    def batch_curves_device(self, rows, out):
        """The same rows written into a contiguous float64 device tensor out
        [len(rows) x n] on the engine's device; rows None: every model's
        row (out [nmodels x n])."""
        if rows is None:
            self._check(self.lib.lcg_batch_curves_device(self.ctx, None, out.shape[0],
                                                         C.c_void_p(out.data_ptr())))
            return out
        r = np.ascontiguousarray(rows, dtype=np.int32)
        self._check(self.lib.lcg_batch_curves_device(
            self.ctx, r.ctypes.data_as(C.POINTER(C.c_int32)), r.shape[0],
            C.c_void_p(out.data_ptr())))
        return out

    def batch_curves(self, rows):
        """Light curves of the given model indices from the last batch call."""
        r = np.ascontiguousarray(rows, dtype=np.int32)
        out = np.empty((r.shape[0], self._n))
        self._check(self.lib.lcg_batch_curves(self.ctx, r.ctypes.data_as(C.POINTER(C.c_int32)),
                                              r.shape[0], _dptr(out)))
        return out

    # -- stage seams ---------------------------------------------------------
    def face_count(self, model, star, fine=True):
        nf = C.c_int32()
        self._check(self.lib.lcg_star_face_count(self.ctx, C.byref(_as_model(model)), star,
                                                 int(fine), C.byref(nf)))
        return nf.value

    def star_grid(self, model, star, fine=True):
        """Point-order grid of one star with its continuum (set_star_grid +
        set_star_continuum): a dict of numpy arrays."""
        m = _as_model(model)
        n = self.face_count(m, star, fine)
        g = {"posn": np.zeros((n, 3)), "dirn": np.zeros((n, 3)), "area": np.zeros(n, np.float32),
             "gravity": np.zeros(n, np.float32), "flux": np.zeros(n, np.float32),
             "neclipse": np.zeros(n, np.int32), "ecl_in": np.zeros(n), "ecl_out": np.zeros(n)}
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self._check(self.lib.lcg_star_grid(
            self.ctx, C.byref(m), star, int(fine), n, _dptr(g["posn"]), _dptr(g["dirn"]),
            fp(g["area"]), fp(g["gravity"]), fp(g["flux"]),
            g["neclipse"].ctypes.data_as(C.POINTER(C.c_int32)), _dptr(g["ecl_in"]),
            _dptr(g["ecl_out"])))
        return g

    def components(self, model, which):
        """One component grid with its continuum (0 the disc, 1 its outer rim,
        2 the bright spot; set_disc_grid / set_disc_edge / set_bright_spot_grid):
        a dict of numpy arrays, rin / rout holding 4 ranges per element."""
        m = _as_model(model)
        n = C.c_int32(0)
        I = C.POINTER(C.c_int32)
        self._check(self.lib.lcg_components(self.ctx, C.byref(m), which, 0, C.byref(n), None, None,
                                            None, None, None, None, None))
        k = n.value
        g = {"posn": np.zeros((k, 3)), "dirn": np.zeros((k, 3)), "area": np.zeros(k, np.float32),
             "flux": np.zeros(k, np.float32), "nr": np.zeros(k, np.int32),
             "rin": np.zeros((k, 4)), "rout": np.zeros((k, 4))}
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self._check(self.lib.lcg_components(
            self.ctx, C.byref(m), which, k, C.byref(n), _dptr(g["posn"]), _dptr(g["dirn"]),
            fp(g["area"]), fp(g["flux"]), g["nr"].ctypes.data_as(I), _dptr(g["rin"]),
            _dptr(g["rout"])))
        return g

    def sum_star_multi(self, star, flat, phases, ldc, ltype, mucrit=0.0, beam=0.0, spin=1.0,
                       vfac=0.0, xcofm=0.0, glens1=False, rlens1=0.0):
        """flat_sum_star{1,2}_multi over a FlatGrid dict (dx,dy,dz,px,py,pz,flux,
        in1,out1,n0) and phase arrays (ex,ey,ez,phin)."""
        cols = {k: np.ascontiguousarray(flat[k], dtype=np.float64)
                for k in ("dx", "dy", "dz", "px", "py", "pz", "flux", "in1", "out1")}
        ph = {k: np.ascontiguousarray(phases[k], dtype=np.float64)
              for k in ("ex", "ey", "ez", "phin")}
        n = cols["dx"].shape[0]
        nent = ph["ex"].shape[0]
        out = np.zeros(nent)
        ldc = np.ascontiguousarray(ldc, dtype=np.float64)
        self._check(self.lib.lcg_sum_star_multi(
            self.ctx, star, n, int(flat["n0"]), *[_dptr(cols[k]) for k in
                                                 ("dx", "dy", "dz", "px", "py", "pz", "flux",
                                                  "in1", "out1")],
            nent, *[_dptr(ph[k]) for k in ("ex", "ey", "ez", "phin")], _dptr(ldc), ltype,
            mucrit, beam, spin, vfac, xcofm, int(glens1), rlens1, _dptr(out)))
        return out

    # -- measurement -----------------------------------------------------------
    def set_profiling(self, on=True):
        self.lib.lcg_set_profiling(self.ctx, int(on))

    def stage_times(self, reset=False):
        ms = np.zeros(7)
        n = np.zeros(7, dtype=np.int64)
        self.lib.lcg_stage_times(self.ctx, _dptr(ms), n.ctypes.data_as(C.POINTER(C.c_int64)),
                                 int(reset))
        return {name: (ms[i], int(n[i])) for i, name in enumerate(abi.STAGES)}

    def flux_elements(self, reset=False):
        return self.lib.lcg_flux_elements(self.ctx, int(reset))

    def fp32_peak_tflops(self):
        t = C.c_double()
        self._check(self.lib.lcg_measure_fp32_peak(self.ctx, C.byref(t)))
        return t.value

    def fp64_peak_tflops(self):
        t = C.c_double()
        self._check(self.lib.lcg_measure_fp64_peak(self.ctx, C.byref(t)))
        return t.value
