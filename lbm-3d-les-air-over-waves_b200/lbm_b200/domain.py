"""One simulation domain on a CUDA device: torch-owned buffers, the C ABI.

    dom = Domain(config_or_env, device="cuda:0")
    dom.step(100)
    ux = dom.field("ux")          # torch tensor on the device
    dom.close()

Buffers are allocated by torch on the device and passed to the library as
raw pointers; the library owns only scratch (bed slots, the LES velocity
stencil, counters).  All calls are issued on the domain's CUDA stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, native, state
from .config import SolverConfig, load_config
from .hostinit import prepare_initial_density


class Domain:
    def __init__(self, cfg, device="cuda:0", stream=None, noise=None, rho_initial=None, with_diag: bool = True,
                 init: bool = True):
        import torch

        if not torch.cuda.is_available():
            raise native.NativeUnavailable("a CUDA device is required (no CPU fallback)")
        if not isinstance(cfg, SolverConfig):
            cfg = load_config(cfg)
        self.cfg = cfg
        self.device = torch.device(device)
        self.lib = native.load()
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        self.params = abi.make_params(cfg)
        # buffers belong to the domain's stream (allocation, fills, every library call)
        with torch.cuda.stream(self.stream):
            self.arrays = state.allocate_torch(cfg, self.device, with_diag=with_diag)
            self.arrays["piecewise_bed_z"].copy_(
                torch.as_tensor(np.asarray(cfg.piecewise_bed_z_np, dtype=np.float32)).to(self.device))
        self.stream.synchronize()
        self.ctx = C.c_void_p()
        self._check(self.lib.lbm_create(C.byref(self.params), C.byref(self.ctx)), "lbm_create")
        self.bufs = state.make_buffers(self.arrays)
        self._check(self.lib.lbm_bind(self.ctx, C.byref(self.bufs)), "lbm_bind")
        if init:
            self.initialize(noise=noise, rho_initial=rho_initial)

    # ------------------------------------------------------------------
    def _check(self, status, what):
        abi.check(self.lib, self.ctx, status, what)

    def _sp(self):
        return C.c_void_p(self.stream.cuda_stream)

    def initialize(self, noise=None, rho_initial=None):
        """init sequence of main() (CODEX.py:3776-3792).

        noise: the uniform [-1, 1) kick of init_fields, shape (3, nz, ny, nx);
        default: seeded (LBM_RANDOM_SEED) draws made on the device.
        rho_initial: the initial density; default: rho0 in air, the host
        prepare_initial_density_field restatement with a free surface."""
        import torch

        # everything on the domain's own stream: no device-wide synchronisation,
        # so domains can be set up while others step
        self.stream.synchronize()
        self._check(self.lib.lbm_init_geometry(self.ctx, self._sp()), "lbm_init_geometry")
        a = self.arrays
        with torch.cuda.stream(self.stream):
            if noise is None:
                # seeded uniform [-1, 1) draws made on the device
                g = torch.Generator(device=self.device)
                g.manual_seed(int(self.cfg.random_seed))
                a["init_noise"].copy_(torch.rand(a["init_noise"].shape, generator=g, device=self.device) * 2.0 - 1.0)
            else:
                a["init_noise"].copy_(torch.as_tensor(np.ascontiguousarray(noise)).to(self.device))
            if rho_initial is None and self.cfg.water_free_surface_enabled != 1:
                a["rho_initial"].fill_(float(np.float32(self.cfg.rho0)))
            else:
                if rho_initial is None:
                    rho_initial = prepare_initial_density(self.cfg, a["fs_h"].cpu().numpy(),
                                                          a["water_h"].cpu().numpy())
                a["rho_initial"].copy_(torch.as_tensor(np.ascontiguousarray(rho_initial)).to(self.device))
        self._check(self.lib.lbm_init_fields(self.ctx, self._sp()), "lbm_init_fields")
        self.stream.synchronize()

    def step(self, n: int = 1):
        self._check(self.lib.lbm_step(self.ctx, int(n), self._sp()), "lbm_step")

    def export_diagnostics(self):
        self._check(self.lib.lbm_export_diagnostics(self.ctx, self._sp()), "lbm_export_diagnostics")

    def counters(self) -> dict:
        c = abi.LbmCounters()
        self._check(self.lib.lbm_read_counters(self.ctx, C.byref(c)), "lbm_read_counters")
        return c.as_dict()

    def diagnostics(self, slice_j: int | None = None) -> dict:
        """The harness metrics of the current state reduced on the device
        (lbm_diagnostics): the health line's maximum speed with its location,
        water volume and VOF accounting, surface-line and mid-slice band
        statistics.  Only this record comes back to the host."""
        cfg = self.cfg
        inp = abi.LbmDiagInputs()
        inp.rho_phys = float(cfg.rho_phys)
        inp.gravity_phys = float(cfg.gravity_phys)
        inp.slice_j = int(cfg.Ny // 2 if slice_j is None else slice_j)
        out = abi.LbmDiag()
        self._check(self.lib.lbm_diagnostics(self.ctx, C.byref(inp), C.byref(out), self._sp()), "lbm_diagnostics")
        return out.as_dict()

    def set_kernel_timing(self, enable: bool):
        self._check(self.lib.lbm_set_kernel_timing(self.ctx, 1 if enable else 0), "lbm_set_kernel_timing")

    def kernel_timing(self):
        """(summed ms, launches, cells per launch) of the interior kernel."""
        ms, n, cells = C.c_double(), C.c_int64(), C.c_int64()
        self._check(self.lib.lbm_kernel_timing(self.ctx, C.byref(ms), C.byref(n), C.byref(cells)), "lbm_kernel_timing")
        return ms.value, n.value, cells.value

    def set_tile_chunk(self, planes: int):
        """Planes per block of the interior kernel (0: built-in choice)."""
        self._check(self.lib.lbm_set_tile_chunk(self.ctx, int(planes)), "lbm_set_tile_chunk")

    def set_step_graphs(self, enable: bool = True):
        """Run each step call as one CUDA graph launch (air mode and the
        kinematic height path; captured on first use per call shape,
        bit-identical to eager calls)."""
        self._check(self.lib.lbm_set_step_graphs(self.ctx, 1 if enable else 0), "lbm_set_step_graphs")

    def set_arithmetic(self, mode: str):
        """Arithmetic of the fused interior kernels: "exact" (the reference's
        operation order, bit-equal to the CPU oracle) or "fast" (pair-form
        collision with multiply-add contraction; differs by rounding)."""
        code = {"exact": abi.LBM_ARITH_EXACT, "fast": abi.LBM_ARITH_FAST}[mode]
        self._check(self.lib.lbm_set_arithmetic(self.ctx, code), "lbm_set_arithmetic")

    def arithmetic(self) -> str:
        v = C.c_int32()
        self._check(self.lib.lbm_get_arithmetic(self.ctx, C.byref(v)), "lbm_get_arithmetic")
        return "fast" if v.value == abi.LBM_ARITH_FAST else "exact"

    def synchronize(self):
        self.stream.synchronize()

    def f(self):
        """Current populations (the buffer the reference calls f)."""
        return self.arrays["f1" if self.counters()["current_f"] else "f0"]

    def field(self, name: str):
        return self.arrays[name]

    def close(self):
        if getattr(self, "ctx", None):
            self.stream.synchronize()
            self.lib.lbm_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
