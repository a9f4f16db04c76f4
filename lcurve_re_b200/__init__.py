"""lcurve_re_b200 — a B200-native engine for lcurve_re's model-evaluation path.

The product is liblcg.so (CUDA kernels for sm_100a + a C++ host engine behind
the C ABI of include/lcg.h). This package is its Python front end: Model /
Data mirror lcurve_re's types and JSON configuration, Engine mirrors
Lcurve::light_curve_comp.
"""
from . import abi
from .model import Data, LcurveError, Model, Pparam, make_data, read_data

__all__ = ["abi", "Data", "Engine", "LcurveError", "Model", "Pparam", "make_data", "read_data"]


def __getattr__(name):
    if name == "Engine":
        from .engine import Engine
        return Engine
    raise AttributeError(name)
