"""Generate the render-snapshot golden with the reference's own writer.

Run where a checkout of the reference is available (it is read, never
written; GPU machines do not need it):

    python tests/golden/gen_render_golden.py --reference PATH

PATH is the reference checkout (default: the LBM_REFERENCE_DIR environment
variable).  For each case, render_inputs() builds a seeded stand-in for the
solver module (scalars and fields with .to_numpy()).  The reference's
save_render_snapshot (run_ab_case.py:140-202) writes it with the arguments
that its visualize callback passes (run_ab_case.py:291-301, 829-841).  The
result is tests/golden/render/<case>.npz.  run_ab_case.py imports
matplotlib at the top; it is absent here and the writer does not use it, so
an empty stand-in module takes its place for the import.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import shutil
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS_FILE = "run_ab_case.py"
CASES = ("air_bed", "water_height", "vof_bed_cube")


class Field:
    """A solver field as the harness reads it: .to_numpy() gives a copy."""

    def __init__(self, values):
        self._v = np.asarray(values)

    def to_numpy(self):
        return self._v.copy()


def render_inputs(case: str) -> dict:
    """The solver globals that the snapshot writer reads, for one case."""
    rng = np.random.default_rng({"air_bed": 11, "water_height": 12, "vof_bed_cube": 13}[case])
    nz, ny, nx = 6, 4, 8
    dx = 0.5
    ns = {
        "dx": dx, "Lx_m": nx * dx, "Ly_m": ny * dx, "Lz_m": nz * dx,
        "x_phys": (np.arange(nx) + 0.5) * dx, "y_phys": (np.arange(ny) + 0.5) * dx,
        "z_phys": (np.arange(nz) + 0.5) * dx,
        "water_h": Field(rng.uniform(0.5, 1.5, size=(ny, nx)).astype(np.float32)),
        "obstacle": Field((rng.uniform(size=(nz, ny, nx)) < 0.25).astype(np.int32)),
        "water_free_surface_enabled": 0 if case == "air_bed" else 1,
        "free_surface_tracking_mode": "vof" if case == "vof_bed_cube" else "height",
        "include_cube_geometry": 1 if case == "vof_bed_cube" else 0,
        "cube_side_m": 1.5, "cube_size_x_m": 1.5, "cube_size_y_m": 1.0, "cube_size_z_m": 1.25,
        "cube_center_x_m": 2.0, "cube_center_y_m": 1.0, "cube_center_z_m": 1.75,
        "cube_yaw_deg": 20.0, "cube_pitch_deg": -5.0,
    }
    if case != "air_bed":
        ns["free_surface_h"] = Field(rng.uniform(1.0, 2.0, size=(ny, nx)).astype(np.float32))
        ns["free_surface_fill"] = Field(rng.uniform(0.0, 1.0, size=(nz, ny, nx)).astype(np.float32))
    return ns


STEP, TIME = 40, 12.5


def write_with_reference(reference: str, case: str, folder: Path) -> Path:
    if "matplotlib" not in sys.modules:
        mpl = types.ModuleType("matplotlib")
        mpl.pyplot = types.ModuleType("matplotlib.pyplot")
        sys.modules["matplotlib"] = mpl
        sys.modules["matplotlib.pyplot"] = mpl.pyplot
    sys.path.insert(0, reference)
    try:
        spec = importlib.util.spec_from_file_location("ref_harness", os.path.join(reference, HARNESS_FILE))
        harness = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(harness)
    finally:
        sys.path.remove(reference)
    module = types.SimpleNamespace(**render_inputs(case))
    obs_np = module.obstacle.to_numpy().astype(bool)
    water_h_np = module.water_h.to_numpy()
    enabled = getattr(module, "water_free_surface_enabled", 0) == 1
    tracking = getattr(module, "free_surface_tracking_mode", "height")
    fill = module.free_surface_fill.to_numpy() if enabled else None
    height = module.free_surface_h.to_numpy() if enabled else None
    saved = os.environ.get("LBM_SAVE_RENDER_SNAPSHOT")
    os.environ["LBM_SAVE_RENDER_SNAPSHOT"] = "1"
    try:
        return harness.save_render_snapshot(
            module, label=case, step=STEP, time_phys=TIME, output_dir=folder, free_surface_enabled=enabled,
            tracking_mode=tracking, fs_fill_np=fill, free_surface_h_np=height, water_h_np=water_h_np,
            obs_np=obs_np)
    finally:
        if saved is None:
            del os.environ["LBM_SAVE_RENDER_SNAPSHOT"]
        else:
            os.environ["LBM_SAVE_RENDER_SNAPSHOT"] = saved


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LBM_REFERENCE_DIR", ""),
                    help="reference checkout (default: $LBM_REFERENCE_DIR)")
    args = ap.parse_args()
    reference = os.path.abspath(args.reference) if args.reference else ""
    if not reference or not os.path.exists(os.path.join(reference, HARNESS_FILE)):
        raise SystemExit(f"{HARNESS_FILE} not found: pass --reference PATH or set LBM_REFERENCE_DIR")
    os.makedirs(os.path.join(HERE, "render"), exist_ok=True)
    with tempfile.TemporaryDirectory() as folder:
        for case in CASES:
            path = write_with_reference(reference, case, Path(folder))
            out = os.path.join(HERE, "render", f"{case}.npz")
            shutil.copyfile(path, out)
            print(f"wrote {out} ({os.path.getsize(out)} B)")


if __name__ == "__main__":
    main()
