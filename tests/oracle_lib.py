"""ctypes access to the test oracles (test infrastructure only).

  Oracle      oracle/liblcg_oracle.so: the plain-C restatement (always built,
              from oracle/lcg_oracle.c, by `make -C oracle`)
  Reference   oracle/_ref/liblcurve_ref.so: lcurve_re's own CPU sources
              compiled for parity (present only where the reference
              sources were available when it was built)

Both expose the same calls, so a test can run either as the checker.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from lcurve_re_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liblcg_oracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "liblcurve_ref.so")
REF_RELEASE_SO = os.path.join(ORACLE_DIR, "_ref", "liblcurve_ref_release.so")

D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)
I32 = C.POINTER(C.c_int32)
I64 = C.POINTER(C.c_int64)
M = C.POINTER(abi.LcgModel)


def _d(a):
    return a.ctypes.data_as(D)


def ensure_oracle_built():
    src = os.path.join(ORACLE_DIR, "lcg_oracle.c")
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-C", ORACLE_DIR, "oracle"], check=True, capture_output=True)
    return ORACLE_SO


class _Lib:
    prefix = ""
    path = ""

    def __init__(self, path=None):
        self.lib = C.CDLL(path or self.path)
        p = self.prefix
        f = getattr(self.lib, p + "light_curve")
        f.restype = C.c_int
        f.argtypes = [M, C.c_void_p, C.c_int32, C.c_int32, D, D, D, C.c_char_p, C.c_int]
        f = getattr(self.lib, p + "sum_star_multi")
        f.restype = C.c_int
        f.argtypes = [C.c_int32, C.c_int64, C.c_int64] + [D] * 9 + [C.c_int32] + [D] * 5 + \
                     [C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                      C.c_int32, C.c_double, D]

    def light_curve(self, model, data, scale=True, rdata=True, diagnostics=False, sfac=None):
        m = model.to_c() if hasattr(model, "to_c") else model
        d = np.ascontiguousarray(data)
        n = d.shape[0]
        sf = np.ones(5) if sfac is None else np.array(sfac, dtype=np.float64)
        calc = np.zeros(n)
        sc = np.zeros(abi.NOUT)
        flags = (1 if scale else 0) | (2 if rdata else 0) | (8 if diagnostics else 0)
        err = C.create_string_buffer(512)
        st = getattr(self.lib, self.prefix + "light_curve")(
            C.byref(m), d.ctypes.data, n, flags, _d(sf), _d(calc), _d(sc), err, 512)
        return st, err.value.decode(), calc, sf, sc

    def light_curve_fast(self, model, data, max_pts, scale=True, rdata=True, sfac=None):
        """light_curve_comp_fast: (status, message, calc, sfac, scalars)."""
        m = model.to_c() if hasattr(model, "to_c") else model
        d = np.ascontiguousarray(data)
        n = d.shape[0]
        sf = np.ones(5) if sfac is None else np.array(sfac, dtype=np.float64)
        calc = np.zeros(n)
        sc = np.zeros(abi.NOUT)
        flags = (1 if scale else 0) | (2 if rdata else 0)
        err = C.create_string_buffer(512)
        fn = getattr(self.lib, self.prefix + "light_curve_fast")
        fn.restype = C.c_int
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, D, D, D,
                       C.c_char_p, C.c_int]
        st = fn(C.byref(m), d.ctypes.data, n, flags, max_pts, _d(sf), _d(calc), _d(sc), err, 512)
        return st, err.value.decode(), calc, sf, sc

    def components(self, model, which, maxr=4):
        """One component grid (0 disc, 1 disc edge, 2 bright spot) with its
        continuum: (status, message, dict of per-element arrays)."""
        m = model.to_c() if hasattr(model, "to_c") else model
        fn = getattr(self.lib, self.prefix + "components")
        fn.restype = C.c_int
        fn.argtypes = [M, C.c_int32, C.c_int32, C.c_int32, I32, D, D, F, F, I32, D, D,
                       C.c_char_p, C.c_int]
        err = C.create_string_buffer(512)
        n = C.c_int32(0)
        st = fn(C.byref(m), which, 0, maxr, C.byref(n), None, None, None, None, None, None,
                None, err, 512)
        if st:
            return st, err.value.decode(), None
        k = n.value
        g = dict(posn=np.zeros((k, 3)), dirn=np.zeros((k, 3)), area=np.zeros(k, np.float32),
                 flux=np.zeros(k, np.float32), nr=np.zeros(k, np.int32),
                 rin=np.zeros((k, maxr)), rout=np.zeros((k, maxr)))
        st = fn(C.byref(m), which, k, maxr, C.byref(n), _d(g["posn"]), _d(g["dirn"]),
                g["area"].ctypes.data_as(F), g["flux"].ctypes.data_as(F),
                g["nr"].ctypes.data_as(I32), _d(g["rin"]), _d(g["rout"]), err, 512)
        return st, err.value.decode(), g

    def sum_star_multi(self, star, flat, phases, ldc, ltype, mucrit=0.0, beam=0.0, spin=1.0,
                       vfac=0.0, xcofm=0.0, glens1=False, rlens1=0.0):
        cols = [np.ascontiguousarray(flat[k], dtype=np.float64)
                for k in ("dx", "dy", "dz", "px", "py", "pz", "flux")]
        n0 = int(flat["n0"])
        in1 = np.ascontiguousarray(flat["in1"][n0:] if len(flat["in1"]) == len(cols[0])
                                   else flat["in1"], dtype=np.float64)
        out1 = np.ascontiguousarray(flat["out1"][n0:] if len(flat["out1"]) == len(cols[0])
                                    else flat["out1"], dtype=np.float64)
        ph = [np.ascontiguousarray(phases[k], dtype=np.float64) for k in ("ex", "ey", "ez", "phin")]
        out = np.zeros(ph[0].shape[0])
        getattr(self.lib, self.prefix + "sum_star_multi")(
            star, cols[0].shape[0], n0, *[_d(c) for c in cols], _d(in1), _d(out1),
            ph[0].shape[0], *[_d(p) for p in ph], _d(np.asarray(ldc, dtype=np.float64)), ltype,
            mucrit, beam, spin, vfac, xcofm, int(glens1), rlens1, _d(out))
        return out


class Oracle(_Lib):
    prefix = "lco_"
    path = ORACLE_SO

    def __init__(self, path=None):
        ensure_oracle_built()
        super().__init__(path)
        L = self.lib
        L.lco_face_count.restype = C.c_int
        L.lco_face_count.argtypes = [M, C.c_int, C.c_int, I32, C.c_char_p, C.c_int]
        L.lco_star_grid.restype = C.c_int
        L.lco_star_grid.argtypes = [M, C.c_int, C.c_int, C.c_int32, D, D, F, F, F, I32, D, D,
                                    C.c_char_p, C.c_int]
        L.lco_flatten.restype = C.c_int
        L.lco_flatten.argtypes = [C.c_int32, D, D, F, I32, D, D] + [D] * 9 + [I64, I64]
        L.lco_phase_batch.restype = C.c_int64
        L.lco_phase_batch.argtypes = [M, C.c_void_p, C.c_int32, D, D, D, D, D, D, I32]
        L.lco_model_scalars.restype = C.c_int
        L.lco_model_scalars.argtypes = [M, D, C.c_char_p, C.c_int]

    def face_count(self, model, star, fine=True):
        m = model.to_c() if hasattr(model, "to_c") else model
        nf = C.c_int32()
        err = C.create_string_buffer(512)
        st = self.lib.lco_face_count(C.byref(m), star, int(fine), C.byref(nf), err, 512)
        if st:
            raise RuntimeError(err.value.decode())
        return nf.value

    def star_grid(self, model, star, fine=True):
        m = model.to_c() if hasattr(model, "to_c") else model
        n = self.face_count(m, star, fine)
        g = {"posn": np.zeros((n, 3)), "dirn": np.zeros((n, 3)), "area": np.zeros(n, np.float32),
             "gravity": np.zeros(n, np.float32), "flux": np.zeros(n, np.float32),
             "neclipse": np.zeros(n, np.int32), "ecl_in": np.zeros(n), "ecl_out": np.zeros(n)}
        err = C.create_string_buffer(512)
        st = self.lib.lco_star_grid(C.byref(m), star, int(fine), n, _d(g["posn"]), _d(g["dirn"]),
                                    g["area"].ctypes.data_as(F), g["gravity"].ctypes.data_as(F),
                                    g["flux"].ctypes.data_as(F), g["neclipse"].ctypes.data_as(I32),
                                    _d(g["ecl_in"]), _d(g["ecl_out"]), err, 512)
        if st:
            raise RuntimeError(err.value.decode())
        return g

    def flatten(self, g):
        n = g["posn"].shape[0]
        cols = {k: np.zeros(n) for k in ("dx", "dy", "dz", "px", "py", "pz", "flux", "in1", "out1")}
        n0 = C.c_int64()
        n1 = C.c_int64()
        st = self.lib.lco_flatten(n, _d(g["posn"]), _d(g["dirn"]), g["flux"].ctypes.data_as(F),
                                  g["neclipse"].ctypes.data_as(I32), _d(g["ecl_in"]),
                                  _d(g["ecl_out"]),
                                  *[_d(cols[k]) for k in ("dx", "dy", "dz", "px", "py", "pz",
                                                          "flux", "in1", "out1")],
                                  C.byref(n0), C.byref(n1))
        if st:
            raise RuntimeError("flatten failed")
        cols["n0"] = n0.value
        cols["in1"] = cols["in1"][: n - n0.value]
        cols["out1"] = cols["out1"][: n - n0.value]
        return cols

    def phase_batch(self, model, data):
        m = model.to_c() if hasattr(model, "to_c") else model
        d = np.ascontiguousarray(data)
        nent = int(np.maximum(d["ndiv"], 0).sum())
        out = {k: np.zeros(max(nent, 1)) for k in ("ex", "ey", "ez", "phin", "w1", "w2")}
        idx = np.zeros(max(nent, 1), dtype=np.int32)
        k = self.lib.lco_phase_batch(C.byref(m), d.ctypes.data, d.shape[0],
                                     *[_d(out[k]) for k in ("ex", "ey", "ez", "phin", "w1", "w2")],
                                     idx.ctypes.data_as(I32))
        out = {key: v[:k] for key, v in out.items()}
        out["idx"] = idx[:k]
        return out

    def scalars(self, model):
        m = model.to_c() if hasattr(model, "to_c") else model
        o = np.zeros(12)
        err = C.create_string_buffer(512)
        st = self.lib.lco_model_scalars(C.byref(m), _d(o), err, 512)
        if st:
            raise RuntimeError(err.value.decode())
        return o


class Reference(_Lib):
    prefix = "lcref_"
    path = REF_SO

    def __init__(self, path=None):
        super().__init__(path)
        L = self.lib
        L.lcref_star_grid.restype = C.c_int
        L.lcref_star_grid.argtypes = [M, C.c_int32, C.c_int32, C.c_int32, I32, D, D, F, F, F, I32,
                                      D, D, C.c_char_p, C.c_int]

    @staticmethod
    def available(path=REF_SO):
        return os.path.exists(path)

    def star_grid(self, model, star, fine=True):
        m = model.to_c() if hasattr(model, "to_c") else model
        nf = C.c_int32()
        err = C.create_string_buffer(512)
        nul = C.POINTER(C.c_double)()
        st = self.lib.lcref_star_grid(C.byref(m), star, int(fine), 0, C.byref(nf), nul, nul,
                                      C.POINTER(C.c_float)(), C.POINTER(C.c_float)(),
                                      C.POINTER(C.c_float)(), C.POINTER(C.c_int32)(), nul, nul,
                                      err, 512)
        if st:
            raise RuntimeError(err.value.decode())
        n = nf.value
        g = {"posn": np.zeros((n, 3)), "dirn": np.zeros((n, 3)), "area": np.zeros(n, np.float32),
             "gravity": np.zeros(n, np.float32), "flux": np.zeros(n, np.float32),
             "neclipse": np.zeros(n, np.int32), "ecl_in": np.zeros(n), "ecl_out": np.zeros(n)}
        st = self.lib.lcref_star_grid(C.byref(m), star, int(fine), n, C.byref(nf), _d(g["posn"]),
                                      _d(g["dirn"]), g["area"].ctypes.data_as(F),
                                      g["gravity"].ctypes.data_as(F), g["flux"].ctypes.data_as(F),
                                      g["neclipse"].ctypes.data_as(I32), _d(g["ecl_in"]),
                                      _d(g["ecl_out"]), err, 512)
        if st:
            raise RuntimeError(err.value.decode())
        return g
