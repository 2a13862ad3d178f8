"""Loader for the oracle's C restatement (oracle/gen_ref.c), built by oracle/build.py."""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            from . import build
            build.build()
        _lib = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.oracle_ref_spd.argtypes = [dp, ctypes.c_size_t]
        _lib.oracle_ref_spd.restype = None
        for name in ("oracle_ref_verify_lu", "oracle_ref_verify_chol"):
            fn = getattr(_lib, name)
            fn.argtypes = [dp, dp, ctypes.c_size_t]
            fn.restype = ctypes.c_double
    return _lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.c_contiguous or a.flags.f_contiguous)
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
