"""Storage precision against the FP64 reference run.

The CUDA library computes in FP32 and stores populations as FP32 or as
shifted 16-bit values (f_q - w_q rho0 in FP16 or BF16).  These tests run the
same seeded case on the GPU at each storage precision and on the FP64 CPU
oracle, and bound the errors in velocity, pressure perturbation
p' = (rho - rho0)/3 and free-surface elevation.

Error measures (over open, non-gas cells, after N steps):
  velocity      max |u - u64| / max |u64|
  velocity_rms  ||u - u64||_2 / ||u64||_2
  pressure      max |p' - p'64| / max |p'64|
  elevation     max |h - h64| / max |h64 - mean initial h| (height path)

The FP32 form itself is bit-equal to the FP32 oracle (test_gpu_parity); its
distance to FP64 is the reference algorithm's own rounding sensitivity
(threshold branches next to the moving bed: link flips, the positivity
limiter, the wall model), about 2.4e-3 max / 1.4e-4 rms in the air case.
Bounds: FP32 max 5e-3, rms 5e-4; shifted FP16 rms 1.5e-3, max 5e-3;
BF16 (8 mantissa bits) rms 5e-3, max 2e-2.
"""
import json

import numpy as np
import pytest

from lbm_b200.config import air_wave_env, water_gaussian_env
from oracle_runner import OracleSim

pytestmark = pytest.mark.gpu

VEL_MAX = {"f32": 5e-3, "f16s": 5e-3, "bf16s": 2e-2}
VEL_RMS = {"f32": 5e-4, "f16s": 1.5e-3, "bf16s": 5e-3}


def _rel(a, b, mask, scale=None):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))[mask]
    s = np.abs(b.astype(np.float64))[mask].max() if scale is None else scale
    return float(d.max() / s) if s > 0 else float(d.max())


def _errors(env, storage, steps):
    from lbm_b200.domain import Domain

    ref = OracleSim(env, fp64=True)
    e = dict(env)
    e["LBM_B200_POP_STORAGE"] = storage
    dom = Domain(e, device="cuda:0", noise=ref.arrays["init_noise"], rho_initial=ref.arrays["rho_initial"])
    h0 = ref.arrays["fs_h"].astype(np.float64).copy()
    ref.step(steps)
    dom.step(steps)
    dom.synchronize()
    dom.export_diagnostics()
    dom.synchronize()
    open_ = dom.field("obstacle").cpu().numpy() == 0
    if env.get("LBM_PHYSICS_MODE") == "water":
        open_ &= dom.field("fs_type").cpu().numpy() != 0   # not gas
    out = {}
    u = np.stack([dom.field(k).cpu().numpy() for k in ("ux", "uy", "uz")]).astype(np.float64)
    u64 = np.stack([ref.arrays[k] for k in ("ux", "uy", "uz")]).astype(np.float64)
    speed64 = np.sqrt((u64 ** 2).sum(0))
    du = np.abs(u - u64).max(0)
    out["velocity"] = float(du[open_].max() / speed64[open_].max())
    out["velocity_rms"] = float(np.sqrt(((u - u64) ** 2).sum(0)[open_].mean()) / np.sqrt((speed64[open_] ** 2).mean()))
    away = open_ & (dom.field("near_obstacle").cpu().numpy() == 0)
    out["velocity_off_wall"] = float(du[away].max() / speed64[open_].max())
    kk = np.argwhere(du == du[open_].max())[0]
    out["velocity_max_at_kji"] = [int(v) for v in kk]
    rho0 = np.float64(dom.cfg.rho0)
    p = (dom.field("rho").cpu().numpy().astype(np.float64) - rho0) / 3.0
    p64 = (ref.arrays["rho"].astype(np.float64) - rho0) / 3.0
    out["pressure"] = _rel(p, p64, open_)
    if env.get("LBM_PHYSICS_MODE") == "water":
        h = dom.field("fs_h").cpu().numpy().astype(np.float64)
        h64 = ref.arrays["fs_h"].astype(np.float64)
        amp = np.abs(h64 - h0.mean()).max()
        out["elevation"] = float(np.abs(h - h64).max() / amp) if amp > 0 else float(np.abs(h - h64).max())
    dom.close()
    ref.close()
    return out


def _record(case, storage, errs):
    # one JSON line per case on stdout (pytest -s shows it)
    print(json.dumps({"case": case, "storage": storage, "errors": errs}), flush=True)


@pytest.mark.parametrize("storage", ["f32", "f16s", "bf16s"])
def test_air_storage_error_vs_fp64(storage):
    env = air_wave_env(64, 32, 40, amp=3.0, level=6.0, wavelength=32.0)
    errs = _errors(env, storage, steps=60)
    _record("air 64x32x40, 60 steps", storage, errs)
    assert errs["velocity"] <= VEL_MAX[storage], errs
    assert errs["velocity_rms"] <= VEL_RMS[storage], errs


@pytest.mark.parametrize("storage", ["f32", "f16s", "bf16s"])
def test_water_height_storage_error_vs_fp64(storage):
    env = water_gaussian_env(64, 8, 32, depth=16.0, amp=3.0, sigma=8.0, g_lb=1e-3)
    errs = _errors(env, storage, steps=60)
    _record("water height 64x8x32, 60 steps", storage, errs)
    assert errs["velocity"] <= VEL_MAX[storage], errs
    assert errs["velocity_rms"] <= VEL_RMS[storage], errs
    assert errs["elevation"] <= VEL_RMS[storage], errs
