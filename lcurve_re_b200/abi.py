"""ctypes mirror of include/lcg.h (the engine's C ABI).

The structures here are byte-compatible with the C declarations; a layout
test (tests/test_abi.py) checks sizes and offsets against the header.
"""
import ctypes as C

LCG_ABI_VERSION = 3

# lcg_status
OK, E_INVALID, E_LOBE, E_ROCHE, E_NOCONVERGE, E_UNSUPPORTED, E_CUDA, E_NOMEM, E_CAPACITY = range(9)
STATUS_NAMES = {
    0: "LCG_OK", 1: "LCG_E_INVALID", 2: "LCG_E_LOBE", 3: "LCG_E_ROCHE",
    4: "LCG_E_NOCONVERGE", 5: "LCG_E_UNSUPPORTED", 6: "LCG_E_CUDA",
    7: "LCG_E_NOMEM", 8: "LCG_E_CAPACITY",
}

LIMB_POLY, LIMB_CLARET = 0, 1
STAR1, STAR2 = 0, 1
PREC_FP64, PREC_MIXED = 0, 1

FLAG_SCALE, FLAG_RDATA, FLAG_INFO, FLAG_DIAGNOSTICS, FLAG_NO_CACHE = 1, 2, 4, 8, 16

OUT_WDWARF, OUT_CHISQ, OUT_WNOK, OUT_LOGG1, OUT_LOGG2, OUT_RV1, OUT_RV2 = range(7)
NOUT = 7

STAGES = ("grid", "eclipse", "continuum", "flatten", "phases", "flux", "reduce")


# disc, edge and bright-spot parameters, in lcg_model order
DISC_SPOT = ["rdisc1", "rdisc2", "height_disc", "beta_disc", "temp_disc", "texp_disc",
             "lin_limb_disc", "quad_limb_disc", "temp_edge", "absorb_edge",
             "radius_spot", "length_spot", "height_spot", "expon_spot", "epow_spot",
             "angle_spot", "yaw_spot", "temp_spot", "tilt_spot", "cfrac_spot"]


class LcgModel(C.Structure):
    _fields_ = [
        ("q", C.c_double), ("iangle", C.c_double), ("r1", C.c_double), ("r2", C.c_double),
        ("cphi3", C.c_double), ("cphi4", C.c_double), ("spin1", C.c_double), ("spin2", C.c_double),
        ("t1", C.c_double), ("t2", C.c_double),
        ("ldc1", C.c_double * 4), ("ldc2", C.c_double * 4),
        ("velocity_scale", C.c_double), ("beam_factor1", C.c_double), ("beam_factor2", C.c_double),
        ("t0", C.c_double), ("period", C.c_double), ("pdot", C.c_double), ("deltat", C.c_double),
        ("gravity_dark1", C.c_double), ("gravity_dark2", C.c_double),
        ("absorb", C.c_double), ("slope", C.c_double), ("quad", C.c_double), ("cube", C.c_double),
        ("third", C.c_double),
        ("stsp", (C.c_double * 4) * 5), ("stsp_defined", C.c_int32 * 5),
        ("uesp", C.c_double * 5), ("uesp_defined", C.c_int32),
        ("delta_phase", C.c_double),
        ("nlat1f", C.c_int32), ("nlat2f", C.c_int32), ("nlat1c", C.c_int32), ("nlat2c", C.c_int32),
        ("npole", C.c_int32), ("nlatfill", C.c_int32), ("nlngfill", C.c_int32),
        ("lfudge", C.c_double), ("llo", C.c_double), ("lhi", C.c_double),
        ("phase1", C.c_double), ("phase2", C.c_double), ("wavelength", C.c_double),
        ("roche1", C.c_int32), ("roche2", C.c_int32), ("eclipse1", C.c_int32),
        ("eclipse2", C.c_int32), ("glens1", C.c_int32), ("use_radii", C.c_int32),
        ("tperiod", C.c_double),
        ("gdark_bolom1", C.c_int32), ("gdark_bolom2", C.c_int32),
        ("mucrit1", C.c_double), ("mucrit2", C.c_double),
        ("limb1", C.c_int32), ("limb2", C.c_int32),
        ("mirror", C.c_int32), ("add_disc", C.c_int32), ("opaque", C.c_int32),
        ("add_spot", C.c_int32), ("iscale", C.c_int32), ("pad_", C.c_int32),
    ] + [(n, C.c_double) for n in DISC_SPOT] + [("nrad", C.c_int32), ("nspot", C.c_int32)]


class LcgDatum(C.Structure):
    _fields_ = [
        ("time", C.c_double), ("expose", C.c_double), ("flux", C.c_double),
        ("ferr", C.c_double), ("weight", C.c_double), ("ndiv", C.c_int32), ("pad_", C.c_int32),
    ]


class LcgOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("precision", C.c_int32), ("verbose", C.c_int32),
        ("eclipse_warp", C.c_int32), ("reserved", C.c_int32 * 4),
    ]


# numpy dtype with the lcg_datum / Lcurve::Datum layout
def datum_dtype():
    import numpy as np
    return np.dtype([("time", "<f8"), ("expose", "<f8"), ("flux", "<f8"), ("ferr", "<f8"),
                     ("weight", "<f8"), ("ndiv", "<i4"), ("pad_", "<i4")], align=True)


P = C.c_void_p
D = C.POINTER(C.c_double)
F = C.POINTER(C.c_float)
I32 = C.POINTER(C.c_int32)
I64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes)
PROTOTYPES = {
    "lcg_default_options": (None, [C.POINTER(LcgOptions)]),
    "lcg_create": (C.c_int, [C.POINTER(P), C.POINTER(LcgOptions)]),
    "lcg_destroy": (None, [P]),
    "lcg_last_error": (C.c_char_p, [P]),
    "lcg_abi_version": (C.c_int32, []),
    "lcg_stream": (P, [P]),
    "lcg_light_curve": (C.c_int, [P, C.POINTER(LcgModel), P, C.c_int32, C.c_int32, D, D, D]),
    "lcg_light_curve_batch": (C.c_int, [P, C.POINTER(LcgModel), C.c_int32, P, C.c_int32,
                                        C.c_int32, D, D, D, D, I32]),
    "lcg_star_face_count": (C.c_int, [P, C.POINTER(LcgModel), C.c_int32, C.c_int32, I32]),
    "lcg_star_grid": (C.c_int, [P, C.POINTER(LcgModel), C.c_int32, C.c_int32, C.c_int32,
                                D, D, F, F, F, I32, D, D]),
    "lcg_components": (C.c_int, [P, C.POINTER(LcgModel), C.c_int32, C.c_int32, I32, D, D, F, F,
                                 I32, D, D]),
    "lcg_sum_star_multi": (C.c_int, [P, C.c_int32, C.c_int64, C.c_int64, D, D, D, D, D, D, D, D,
                                     D, C.c_int32, D, D, D, D, D, C.c_int32, C.c_double,
                                     C.c_double, C.c_double, C.c_double, C.c_double,
                                     C.c_int32, C.c_double, D]),
    "lcg_set_profiling": (None, [P, C.c_int32]),
    "lcg_stage_times": (None, [P, D, I64, C.c_int32]),
    "lcg_flux_elements": (C.c_int64, [P, C.c_int32]),
    "lcg_measure_fp32_peak": (C.c_int, [P, D]),
    "lcg_measure_fp64_peak": (C.c_int, [P, D]),
    "lcg_set_data": (C.c_int, [P, P, C.c_int32]),
    "lcg_batch_curves": (C.c_int, [P, I32, C.c_int32, D]),
    "lcg_batch_curves_device": (C.c_int, [P, I32, C.c_int32, C.c_void_p]),
    "lcg_light_curve_fast": (C.c_int, [P, C.POINTER(LcgModel), P, C.c_int32, C.c_int32,
                                       C.c_int32, D, D, D]),
    "lcg_mlp_gemm": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P, P, P, P,
                               P, P, C.c_int32, C.c_int32, P]),
    "lcg_mlp_adam": (C.c_int, [P, P, P, P, P, C.c_int32, C.c_int32, C.c_float, C.c_float,
                               C.c_float, C.c_float, C.c_int32, P, P]),
    "lcg_mlp_adam_all": (C.c_int, [P, C.c_int32, P, P, P, P, P, P, P, P, P, P]),
    "lcg_mlp_forward": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_int32, P, P, C.c_int32,
                                  C.c_int32, P, P, P, P, P, C.c_int32, P, P, P, P, P]),
    "lcg_mlp_backward_data": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, P, P, P, P, P,
                                        C.c_int32, P]),
    "lcg_mlp_colsum": (C.c_int, [P, P, C.c_int32, C.c_int32, C.c_int32, P]),
    "lcg_mlp_input": (C.c_int, [P, P, C.c_int32, P, P, C.c_int32, C.c_int32, C.c_int32, P, P,
                                P, C.c_int32]),
    "lcg_mlp_input_grad": (C.c_int, [P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P]),
    "lcg_mlp_pca_chisq": (C.c_int, [P, P, C.c_int32, C.c_int32, P, P, C.c_int32, P, P, P, P,
                                    P, P, P]),
    "lcg_mlp_mse_grad": (C.c_int, [P, P, P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, P, P,
                                   P]),
    "lcg_light_curve_batch_resident": (C.c_int, [P, C.POINTER(LcgModel), C.c_int32, C.c_int32,
                                                 D, D, D, D, I32]),
    "lcg_light_curve_resident": (C.c_int, [P, C.POINTER(LcgModel), C.c_int32, D, D, D]),
    "lcg_device_calc": (P, [P]),
    "lcg_kernel_launches": (C.c_int64, [C.c_int32]),
    "lcg_walk_propose": (C.c_int, [P, C.c_int32, C.c_int32, P, P, C.c_uint64, P, C.c_int32,
                                   P, P, P, P]),
    "lcg_walk_accept": (C.c_int, [P, C.c_int32, C.c_int32, P, P, P, P, P, P, C.c_uint64, P,
                                  C.c_int32, P]),
    "lcg_walk_advance": (C.c_int, [P, P, C.c_int64]),
    "lcg_sum_star_multi_noalloc": (C.c_int, [P, C.c_int32, C.c_int64, C.c_int64, P, P, P, P, P,
                                             P, C.c_int32, P, P, P, P, D, C.c_int32, C.c_double,
                                             P]),
}


def bind(lib):
    """Attach restype/argtypes to every exported entry point of lib."""
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
