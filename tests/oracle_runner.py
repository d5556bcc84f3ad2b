"""Test helper: drive the CPU oracle (oracle/liblbm_oracle.so) through the
same C ABI as the CUDA library.  Test infrastructure only."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from lbm_b200 import abi, state
from lbm_b200.config import load_config
from lbm_b200.hostinit import make_init_noise, prepare_initial_density

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liblbm_oracle.so")
_LIB = None


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
    return ORACLE_SO


def oracle_lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        lib = abi.declare(C.CDLL(ORACLE_SO))
        lib.lbm_oracle_create_fp64.restype = C.c_int
        lib.lbm_oracle_create_fp64.argtypes = [C.POINTER(abi.LbmParams), C.POINTER(C.c_void_p)]
        lib.lbm_oracle_tree_sum.restype = C.c_double
        lib.lbm_oracle_tree_sum.argtypes = [C.c_void_p, C.c_int64]
        abi.check_layout(lib)
        _LIB = lib
    return _LIB


class OracleSim:
    """One domain on the CPU oracle, state in numpy arrays."""

    def __init__(self, env: dict, fp64: bool = False, noise=None, rho_initial=None):
        self.cfg = load_config(env)
        self.lib = oracle_lib()
        self.params = abi.make_params(self.cfg)
        self.arrays = state.allocate_numpy(self.cfg)
        self.arrays["piecewise_bed_z"][:] = np.asarray(self.cfg.piecewise_bed_z_np, dtype=np.float32)
        self.ctx = C.c_void_p()
        create = self.lib.lbm_oracle_create_fp64 if fp64 else self.lib.lbm_create
        abi.check(self.lib, None, create(C.byref(self.params), C.byref(self.ctx)), "lbm_create")
        self.bufs = state.make_buffers(self.arrays)
        abi.check(self.lib, self.ctx, self.lib.lbm_bind(self.ctx, C.byref(self.bufs)), "lbm_bind")
        abi.check(self.lib, self.ctx, self.lib.lbm_init_geometry(self.ctx, None), "lbm_init_geometry")
        a = self.arrays
        a["init_noise"][:] = make_init_noise(self.cfg) if noise is None else noise
        if rho_initial is None:
            rho_initial = prepare_initial_density(self.cfg, a["fs_h"], a["water_h"])
        a["rho_initial"][:] = rho_initial
        abi.check(self.lib, self.ctx, self.lib.lbm_init_fields(self.ctx, None), "lbm_init_fields")

    def step(self, n: int = 1):
        abi.check(self.lib, self.ctx, self.lib.lbm_step(self.ctx, n, None), "lbm_step")

    def export(self):
        abi.check(self.lib, self.ctx, self.lib.lbm_export_diagnostics(self.ctx, None), "lbm_export_diagnostics")

    def counters(self) -> dict:
        c = abi.LbmCounters()
        abi.check(self.lib, self.ctx, self.lib.lbm_read_counters(self.ctx, C.byref(c)), "lbm_read_counters")
        return c.as_dict()

    def f(self) -> np.ndarray:
        return self.arrays["f1" if self.counters()["current_f"] else "f0"]

    def close(self):
        if self.ctx:
            self.lib.lbm_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
