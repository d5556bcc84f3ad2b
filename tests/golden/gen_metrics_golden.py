"""Generate the metric-row golden with the reference's own make_visualize.

Run where a checkout of the reference is available (it is read, never
written; GPU machines do not need it):

    python tests/golden/gen_metrics_golden.py --reference PATH

PATH is the reference checkout (default: the LBM_REFERENCE_DIR environment
variable).  For each case, metrics_inputs() builds seeded fields and options:
an air domain over a wavy bed, height-function water in the hydrostatic-
balanced and the total-pressure formulation, and VOF with the component-
balanced one; metrics_counters() gives seeded counter values.  The
reference's visualize callback (run_ab_case.py:283-679) runs on a stand-in
solver module that serves those fields as float64 copies (so its formulas
run in float64, like the restatement they pin) and the counters through
[None]; the row it hands to the metrics writer is kept and the plotting
after it is skipped.
The rows go to tests/golden/metrics_rows.json.  run_ab_case.py imports
matplotlib at the top; it is absent here and the row does not use it, so an
empty stand-in module takes its place for the import.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS_FILE = "run_ab_case.py"
OUT = os.path.join(HERE, "metrics_rows.json")
CASES = ("air_periodic", "water_height_solid_balanced", "water_height_periodic_total", "vof_component_balanced")
CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0]
CY = [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1]
CZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1]


def metrics_inputs(case: str):
    """(fields, options) of one case.  Fields use the library's names and
    layout ([nz][ny][nx] cells, [ny][nx] columns) in float32 / int32; every
    option is exactly representable in float32."""
    seed = {"air_periodic": 21, "water_height_solid_balanced": 22, "water_height_periodic_total": 23,
            "vof_component_balanced": 24}[case]
    rng = np.random.default_rng(seed)
    nz, ny, nx, dx = 14, 5, 16, 0.5
    fs = case != "air_periodic"
    vof = case == "vof_component_balanced"
    z = (np.arange(nz) + 0.5) * dx
    x = (np.arange(nx) + 0.5) * dx
    if fs:
        bed = np.full((ny, nx), 1.0)
    else:
        bed = 1.25 + 0.75 * np.sin(2.0 * np.pi * x / (nx * dx))[None, :] * np.ones((ny, 1))
    obstacle = (z[:, None, None] < bed[None, :, :]).astype(np.int32)
    obstacle[rng.uniform(size=obstacle.shape) < 0.02] = 1
    phi = (z[:, None, None] - bed[None, :, :]).astype(np.float32)
    g = {
        "rho": (1.0 + 2e-3 * rng.uniform(-1.0, 1.0, size=(nz, ny, nx))).astype(np.float32),
        "ux": (0.05 + 0.03 * rng.uniform(-1.0, 1.0, size=(nz, ny, nx))).astype(np.float32),
        "uy": (0.02 * rng.uniform(-1.0, 1.0, size=(nz, ny, nx))).astype(np.float32),
        "uz": (0.02 * rng.uniform(-1.0, 1.0, size=(nz, ny, nx))).astype(np.float32),
        "obstacle": obstacle,
        "phi": phi,
        "water_h": bed.astype(np.float32),
    }
    base = 4.25
    opts = {
        "dx": dx, "Nx": nx, "Ny": ny, "Nz": nz, "Lx_m": nx * dx, "vel_scale": 2.5, "rho0": 1.0,
        "water_free_surface_enabled": 1 if fs else 0,
        "free_surface_tracking_mode": "vof" if vof else "height",
        "x_boundary_mode": "solid" if case == "water_height_solid_balanced" else "periodic",
        "free_surface_base_m": base, "vof_empty_fill_threshold": 0.125,
        "rho_phys": 998.0 if fs else 1.25, "gravity_phys": 9.75 if fs else 0.0,
        "use_hydrostatic_balanced_pressure": 1 if case in ("water_height_solid_balanced",
                                                          "vof_component_balanced") else 0,
        "use_component_balanced_pressure": 1 if vof else 0,
    }
    if fs:
        h = (base + 0.4 * rng.uniform(-1.0, 1.0, size=(ny, nx))).astype(np.float32)
        t = np.where(z[:, None, None] < h[None, :, :] - 0.5 * dx, 1, 0).astype(np.int32)
        near = np.abs(z[:, None, None] - h[None, :, :]) <= 0.5 * dx
        t[near] = 2
        fill = np.where(t == 1, 1.0, 0.0)
        fill = np.where(t == 2, rng.uniform(0.0, 1.0, size=t.shape), fill)
        fill[(t == 2) & (rng.uniform(size=t.shape) < 0.2)] = 0.0625   # below the empty threshold
        g.update(
            fs_h=h,
            fs_type=t,
            fs_fill=fill.astype(np.float32),
            fs_mass=(fill * g["rho"]).astype(np.float32),
            fs_mass_excess=np.where(rng.uniform(size=t.shape) < 0.3,
                                    1e-3 * rng.uniform(-1.0, 1.0, size=t.shape), 0.0).astype(np.float32),
            pressure_reference_head=np.maximum(base - z[:, None, None] + 0.0 * h[None, :, :], 0.0)
            .astype(np.float32),
        )
    else:
        g.update(fs_h=np.zeros((ny, nx), np.float32), fs_type=np.zeros((nz, ny, nx), np.int32),
                 fs_fill=np.zeros((nz, ny, nx), np.float32), fs_mass=np.zeros((nz, ny, nx), np.float32),
                 fs_mass_excess=np.zeros((nz, ny, nx), np.float32),
                 pressure_reference_head=np.zeros((nz, ny, nx), np.float32))
    return g, opts


COUNTER_INTS = ("boundary_cut_link_count", "free_surface_cut_link_count", "boundary_refill_count",
                "free_surface_refill_count", "free_surface_coalescence_repair_count",
                "free_surface_thin_gap_bridge_count", "free_surface_vof_excess_count", "free_surface_vof_orphan_count",
                "free_surface_vof_collapse_cell_count", "free_surface_vof_detached_advect_count",
                "free_surface_vof_detached_compress_count")
COUNTER_FLOATS = ("free_surface_vof_collapse_candidate_volume_m3", "free_surface_vof_collapse_applied_volume_m3",
                  "free_surface_vof_detached_advect_mass", "free_surface_vof_detached_compress_mass")


def metrics_counters(case: str) -> dict:
    """Seeded values of the solver's scalar counters (floats exact in float32)."""
    rng = np.random.default_rng(100 + CASES.index(case))
    out = {k: int(rng.integers(0, 500)) for k in COUNTER_INTS}
    out.update({k: float(rng.integers(1, 4096)) / 256.0 for k in COUNTER_FLOATS})
    return out


class _Scalar:
    """A scalar counter as the harness reads it: counter[None]."""

    def __init__(self, value):
        self._v = value

    def __getitem__(self, index):
        assert index is None
        return self._v


class _Field:
    def __init__(self, values):
        self._v = np.asarray(values)

    def to_numpy(self):
        return self._v.copy()


class _RowTaken(Exception):
    pass


def reference_row(reference: str, case: str) -> dict:
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
    g, o = metrics_inputs(case)
    nz, ny, nx, dx = o["Nz"], o["Ny"], o["Nx"], o["dx"]
    f64 = {k: v.astype(np.float64) if v.dtype == np.float32 else v for k, v in g.items()}
    z = (np.arange(nz) + 0.5) * dx
    m = types.SimpleNamespace(**o)
    m.Ly_m, m.Lz_m = ny * dx, nz * dx
    m.x_phys, m.y_phys, m.z_phys = (np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dx, z
    m.Z_phys = z[:, None, None] * np.ones((1, ny, nx))
    m.X_phys = m.x_phys[None, None, :] * np.ones((nz, ny, 1))
    m.FS_GAS, m.FS_INTERFACE = 0, 2
    m.rho_air_phys = o["rho_phys"]
    m.cx, m.cy, m.cz = _Field(CX), _Field(CY), _Field(CZ)
    for ours, theirs in (("rho", "rho"), ("ux", "ux"), ("uy", "uy"), ("uz", "uz"), ("obstacle", "obstacle"),
                         ("phi", "phi"), ("water_h", "water_h")):
        setattr(m, theirs, _Field(f64[ours]))
    if o["water_free_surface_enabled"]:
        for ours, theirs in (("fs_h", "free_surface_h"), ("fs_type", "free_surface_type"),
                             ("fs_fill", "free_surface_fill"), ("fs_mass", "free_surface_mass"),
                             ("fs_mass_excess", "free_surface_mass_excess"),
                             ("pressure_reference_head", "pressure_reference_head")):
            setattr(m, theirs, _Field(f64[ours]))
    for name, value in metrics_counters(case).items():
        setattr(m, name, _Scalar(value))
    rows = []

    class Writer:
        def writerow(self, row):
            rows.append(dict(row))
            raise _RowTaken()

    with tempfile.TemporaryDirectory() as folder:
        visualize = harness.make_visualize(m, case, Path(folder), Writer())
        try:
            visualize(40, 12.5, 1.0e6, 1.0e4)
        except _RowTaken:
            pass
    row = rows[0]
    out = {}
    for k, v in row.items():
        if isinstance(v, (np.floating, float)):
            out[k] = None if math.isnan(float(v)) else float(v)
        elif isinstance(v, (np.integer, int)):
            out[k] = int(v)
        else:
            out[k] = v
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LBM_REFERENCE_DIR", ""),
                    help="reference checkout (default: $LBM_REFERENCE_DIR)")
    args = ap.parse_args()
    reference = os.path.abspath(args.reference) if args.reference else ""
    if not reference or not os.path.exists(os.path.join(reference, HARNESS_FILE)):
        raise SystemExit(f"{HARNESS_FILE} not found: pass --reference PATH or set LBM_REFERENCE_DIR")
    rows = {case: reference_row(reference, case) for case in CASES}
    with open(OUT, "w", encoding="utf-8") as fh:
        json.dump(rows, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"wrote {OUT} ({os.path.getsize(OUT)} B)")


if __name__ == "__main__":
    main()
