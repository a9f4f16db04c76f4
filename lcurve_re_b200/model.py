"""Host-side mirror of lcurve_re's Model and Data types.

Model parses the reference's own JSON configuration (a "model_parameters"
object of strings, src/lcurve_base/model.cpp:10-360) with the same rules:
physical parameters are Pparam strings "value range dstep vary [defined]"
(lcurve.h:159-195); pdot, third, temp_edge and absorb_edge default to 0 when
absent; star-spot groups are optional but all-or-nothing; booleans follow
Subs::string_to_bool (new_subs.h:48-57); limb laws are "Poly" or "Claret".

Data mirrors Lcurve::Data (lcurve.h:454-472): a numpy structured array with
the byte layout of Lcurve::Datum, read from the same six-column ASCII files
(lcurve.cpp:18-31, 53-85).
"""
import copy
import json

import numpy as np

from . import abi


class LcurveError(RuntimeError):
    """Raised where the reference throws Lcurve::Lcurve_Error (lcurve.h:34-43)."""

    def __init__(self, message, status=abi.E_INVALID):
        super().__init__(message)
        self.status = status


class Pparam:
    """A physical parameter, Lcurve::Pparam (lcurve.h:159-195)."""

    __slots__ = ("value", "range", "dstep", "vary", "defined")

    def __init__(self, entry=None, value=0.0):
        if entry is None:
            self.value, self.range, self.dstep = float(value), 0.0, 0.0
            self.vary, self.defined = False, False
            return
        parts = str(entry).split()
        if len(parts) < 4:
            raise LcurveError("Pparam: could not read entry = " + str(entry))
        self.value, self.range, self.dstep = float(parts[0]), float(parts[1]), float(parts[2])
        self.vary = _int_bool(parts[3])
        self.defined = _int_bool(parts[4]) if len(parts) > 4 else True

    def __float__(self):
        return self.value

    def __repr__(self):
        return "Pparam(%r, vary=%s, defined=%s)" % (self.value, self.vary, self.defined)


def _int_bool(tok):
    try:
        return int(tok) != 0
    except ValueError:
        return string_to_bool(tok)


def string_to_bool(entry):
    """Subs::string_to_bool (new_subs.h:48-57)."""
    t = str(entry).upper()
    if t in ("T", "TRUE", "Y", "YES", "1"):
        return True
    if t in ("F", "FALSE", "N", "NO", "0"):
        return False
    raise LcurveError("string_to_bool: could not translate entry = %s to a bool" % entry)


PHYSICAL = [
    "q", "iangle", "r1", "r2", "cphi3", "cphi4", "spin1", "spin2", "t1", "t2",
    "ldc1_1", "ldc1_2", "ldc1_3", "ldc1_4", "ldc2_1", "ldc2_2", "ldc2_3", "ldc2_4",
    "velocity_scale", "beam_factor1", "beam_factor2", "t0", "period", "pdot", "deltat",
    "gravity_dark1", "gravity_dark2", "absorb", "slope", "quad", "cube", "third",
    "rdisc1", "rdisc2", "height_disc", "beta_disc", "temp_disc", "texp_disc",
    "lin_limb_disc", "quad_limb_disc", "temp_edge", "absorb_edge",
    "radius_spot", "length_spot", "height_spot", "expon_spot", "epow_spot", "angle_spot",
    "yaw_spot", "temp_spot", "tilt_spot", "cfrac_spot",
]
OPTIONAL_ZERO = ("pdot", "third", "temp_edge", "absorb_edge")
SPOT_GROUPS = [
    ["stsp11_long", "stsp11_lat", "stsp11_fwhm", "stsp11_tcen"],
    ["stsp12_long", "stsp12_lat", "stsp12_fwhm", "stsp12_tcen"],
    ["stsp13_long", "stsp13_lat", "stsp13_fwhm", "stsp13_tcen"],
    ["stsp21_long", "stsp21_lat", "stsp21_fwhm", "stsp21_tcen"],
    ["stsp22_long", "stsp22_lat", "stsp22_fwhm", "stsp22_tcen"],
]
UESP = ["uesp_long1", "uesp_long2", "uesp_lathw", "uesp_taper", "uesp_temp"]
COMP_FLOAT = ["delta_phase", "lfudge", "llo", "lhi", "phase1", "phase2", "wavelength",
              "tperiod", "mucrit1", "mucrit2"]
COMP_INT = ["nlat1f", "nlat2f", "nlat1c", "nlat2c", "nlatfill", "nlngfill", "nrad", "nspot"]
COMP_BOOL = ["npole", "roche1", "roche2", "eclipse1", "eclipse2", "glens1", "use_radii",
             "gdark_bolom1", "gdark_bolom2", "mirror", "add_disc", "opaque", "add_spot",
             "iscale"]
COMPUTATIONAL = COMP_FLOAT + COMP_INT + COMP_BOOL + ["limb1", "limb2"]

# Order of the variable-parameter vector (model.cpp:363-470, star part).
VARY_ORDER = ["q", "iangle", "r1", "r2", "spin1", "spin2", "t1", "t2",
              "ldc1_1", "ldc1_2", "ldc1_3", "ldc1_4", "ldc2_1", "ldc2_2", "ldc2_3", "ldc2_4",
              "velocity_scale", "beam_factor1", "beam_factor2", "t0", "period", "pdot",
              "deltat", "gravity_dark1", "gravity_dark2", "absorb", "slope", "quad", "cube",
              "third"]
DISC_VARY = ["rdisc1", "rdisc2", "height_disc", "beta_disc", "temp_disc", "texp_disc",
             "lin_limb_disc", "quad_limb_disc", "temp_edge", "absorb_edge"]
SPOT_VARY = ["radius_spot", "length_spot", "height_spot", "expon_spot", "epow_spot",
             "angle_spot", "yaw_spot", "temp_spot", "tilt_spot", "cfrac_spot"]


class Model:
    """Lcurve::Model built from the reference's JSON configuration."""

    def __init__(self, config):
        if isinstance(config, str):
            with open(config) as f:
                config = json.load(f)
        mp = config.get("model_parameters") if isinstance(config, dict) else None
        if not isinstance(mp, dict):
            raise LcurveError("Missing or invalid 'model_parameters'")
        pv = {}
        for k, v in mp.items():
            if not isinstance(v, str):
                raise LcurveError("Malformed model parameter value for parameter '%s'" % k)
            pv[k] = v
        missing = []
        for name in PHYSICAL + COMPUTATIONAL:
            if name not in pv:
                if name in OPTIONAL_ZERO:
                    pv[name] = "0 1.e-10 1.e-10 0 0"
                else:
                    missing.append(name)
        if missing:
            raise LcurveError("One or more parameters were not initialised: " + ", ".join(missing))
        self.p = {name: Pparam(pv[name]) for name in PHYSICAL}
        for group in SPOT_GROUPS + [UESP]:
            present = [g in pv for g in group]
            if any(present) and not all(present):
                raise LcurveError("One or more of the spot parameters %s were not initialised"
                                  % group[0][:6])
            for g in group:
                self.p[g] = Pparam(pv[g]) if g in pv else Pparam()
        self.c = {}
        for name in COMP_FLOAT:
            self.c[name] = float(pv[name])
        for name in COMP_INT:
            self.c[name] = int(pv[name])
        for name in COMP_BOOL:
            self.c[name] = string_to_bool(pv[name])
        for name in ("limb1", "limb2"):
            if pv[name] == "Poly":
                self.c[name] = abi.LIMB_POLY
            elif pv[name] == "Claret":
                self.c[name] = abi.LIMB_CLARET
            else:
                raise LcurveError("Could not recognize the value of %s = %s; should be 'Poly' "
                                  "or 'Claret'" % (name, pv[name]))
        if self.c["glens1"] and self.c["roche1"]:
            raise LcurveError("For reasons of simplicity, glens1 = 1 and roche1 = 1 are not "
                              "simultaneously allowed")

    # -- access ------------------------------------------------------------
    def __getitem__(self, name):
        if name in self.p:
            return self.p[name].value
        return self.c[name]

    def __setitem__(self, name, value):
        if name in self.p:
            self.p[name].value = float(value)
        elif name in self.c:
            self.c[name] = type(self.c[name])(value)
        else:
            raise KeyError(name)

    def copy(self):
        return copy.deepcopy(self)

    def vary_names(self):
        """Names of the varying parameters in set_param order (the star
        part, the disc and bright-spot parameters when those components are
        on, then defined star-spot parameters, model.cpp:383-457)."""
        out = []
        for n in VARY_ORDER:
            if n in ("r1", "r2") and not self.c["use_radii"]:
                n = "cphi3" if n == "r1" else "cphi4"
            if self.p[n].vary:
                out.append(n)
        if self.c["add_disc"]:
            out += [n for n in DISC_VARY if self.p[n].vary]
        if self.c["add_spot"]:
            out += [n for n in SPOT_VARY if self.p[n].vary]
        for n in sum(SPOT_GROUPS, []) + UESP:
            if self.p[n].defined and self.p[n].vary:
                out.append(n)
        return out

    def get_param(self):
        return np.array([self.p[n].value for n in self.vary_names()])

    def set_param(self, vpar):
        for n, v in zip(self.vary_names(), vpar):
            self.p[n].value = float(v)

    # -- C view ------------------------------------------------------------
    def to_c(self):
        m = abi.LcgModel()
        for n in ("q", "iangle", "r1", "r2", "cphi3", "cphi4", "spin1", "spin2", "t1", "t2",
                  "velocity_scale", "beam_factor1", "beam_factor2", "t0", "period", "pdot",
                  "deltat", "gravity_dark1", "gravity_dark2", "absorb", "slope", "quad",
                  "cube", "third"):
            setattr(m, n, self.p[n].value)
        for k in range(4):
            m.ldc1[k] = self.p["ldc1_%d" % (k + 1)].value
            m.ldc2[k] = self.p["ldc2_%d" % (k + 1)].value
        for s, group in enumerate(SPOT_GROUPS):
            for f, g in enumerate(group):
                m.stsp[s][f] = self.p[g].value
            m.stsp_defined[s] = int(all(self.p[g].defined for g in group))
        for k, g in enumerate(UESP):
            m.uesp[k] = self.p[g].value
        m.uesp_defined = int(all(self.p[g].defined for g in UESP))
        for n in COMP_FLOAT:
            setattr(m, n, self.c[n])
        for n in ("nlat1f", "nlat2f", "nlat1c", "nlat2c", "nlatfill", "nlngfill"):
            setattr(m, n, self.c[n])
        for n in ("npole", "roche1", "roche2", "eclipse1", "eclipse2", "glens1", "use_radii",
                  "gdark_bolom1", "gdark_bolom2", "mirror", "add_disc", "opaque", "add_spot",
                  "iscale"):
            setattr(m, n, int(self.c[n]))
        m.limb1, m.limb2 = self.c["limb1"], self.c["limb2"]
        for n in abi.DISC_SPOT:
            setattr(m, n, self.p[n].value)
        m.nrad, m.nspot = self.c["nrad"], self.c["nspot"]
        return m

    def geometry_key(self):
        """Parameters the star grids depend on (light_curve_comp.cpp:64-86)."""
        g = self.c["glens1"]
        return (self["q"], self["iangle"], self["r1"], self["r2"], self["cphi3"], self["cphi4"],
                self["spin1"], self["spin2"], self["velocity_scale"] if g else 0.0,
                self.c["tperiod"] if g else 0.0, self.c["llo"], self.c["lhi"], self.c["lfudge"],
                self.c["delta_phase"], self.c["phase1"], self.c["phase2"], self.c["nlat1f"],
                self.c["nlat2f"], self.c["nlat1c"], self.c["nlat2c"], self.c["nlatfill"],
                self.c["nlngfill"], self.c["use_radii"], self.c["roche1"], self.c["roche2"],
                self.c["eclipse1"], self.c["eclipse2"], g, self.c["npole"])


class Data(np.ndarray):
    """Lcurve::Data: a structured array of Datum records."""

    def __new__(cls, n_or_file=0):
        if isinstance(n_or_file, str):
            return read_data(n_or_file)
        arr = np.zeros(int(n_or_file), dtype=abi.datum_dtype())
        return arr.view(cls)

    @property
    def ptr(self):
        return self.ctypes.data


def make_data(time, expose=0.0, flux=0.0, ferr=1.0, weight=1.0, ndiv=1):
    time = np.asarray(time, dtype=np.float64)
    d = np.zeros(time.shape[0], dtype=abi.datum_dtype())
    d["time"] = time
    d["expose"] = expose
    d["flux"] = flux
    d["ferr"] = ferr
    d["weight"] = weight
    d["ndiv"] = ndiv
    return d.view(Data)


def read_data(path):
    """Data::rasc (lcurve.cpp:53-85): lines starting with '#' or blank are
    skipped; each other line is "time expose flux ferr weight ndiv"; a
    negative ferr is made zero with zero weight (lcurve.cpp:27-30)."""
    rows = []
    with open(path) as f:
        for n, line in enumerate(f, 1):
            if not line.strip() or line[0] in "# \t":
                continue
            tok = line.split()
            if len(tok) < 6:
                raise LcurveError("Data file input failure on line %d" % n)
            t, e, fl, fe, w = map(float, tok[:5])
            nd = int(tok[5])
            if fe < 0.0:
                fe -= fe
                w = 0.0
            rows.append((t, e, fl, fe, w, nd))
    d = make_data(np.array([r[0] for r in rows]))
    for k, name in enumerate(("expose", "flux", "ferr", "weight")):
        d[name] = [r[k + 1] for r in rows]
    d["ndiv"] = [r[5] for r in rows]
    return d
