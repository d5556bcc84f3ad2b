"""Loader of the CUDA library (lbm_b200/_native/liblbm_b200.so).

There is no CPU fallback: if the library or a CUDA device is missing, the
product path raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(abi.native_dir(), "liblbm_b200.so")
_LIB = None


class NativeUnavailable(RuntimeError):
    pass


def load(build_if_missing: bool = True) -> C.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise NativeUnavailable(f"CUDA library not built: {LIB_PATH}")
        from .build import build
        build()
    lib = abi.declare(C.CDLL(LIB_PATH))
    abi.check_layout(lib)
    name = lib.lbm_backend_name().decode()
    if name != "cuda-sm100a":
        raise NativeUnavailable(f"unexpected backend {name!r} at {LIB_PATH}")
    _LIB = lib
    return lib
