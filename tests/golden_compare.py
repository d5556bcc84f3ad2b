"""Test helper: map golden snapshots (reference field names) onto the ABI
field names and compare.  Test infrastructure only."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# golden name -> (ABI array name, kind) ; kind: "state" (bound buffer) or "diag"
FIELD_MAP = {
    "rho": ("rho", "state"), "ux": ("ux", "state"), "uy": ("uy", "state"), "uz": ("uz", "state"),
    "omegaLoc": ("omega", "state"),
    "water_h": ("water_h", "state"), "water_h_last": ("water_h_last", "state"), "u_wave": ("u_wave", "state"),
    "v_wave": ("v_wave", "state"), "w_wave": ("w_wave", "state"), "free_surface_h": ("fs_h", "state"),
    "free_surface_h_last": ("fs_h_last", "state"), "free_surface_flux_x": ("fs_flux_x", "state"),
    "free_surface_flux_y": ("fs_flux_y", "state"), "u_inlet_profile": ("u_inlet_profile", "state"),
    "free_surface_fill": ("fs_fill", "state"), "free_surface_type": ("fs_type", "state"),
    "free_surface_type_prev": ("fs_type_prev", "state"), "free_surface_mass": ("fs_mass", "state"),
    "free_surface_mass_excess": ("fs_mass_excess", "state"), "free_surface_mass_excess_dir": ("fs_excess_dir", "state"),
    "phi": ("phi", "diag"), "obstacle": ("obstacle", "diag"), "near_obstacle": ("near_obstacle", "diag"),
    "lattice_open": ("lattice_open", "diag"), "lattice_open_frac": ("lattice_open_frac", "diag"),
    "lattice_wall_type": ("lattice_wall_type", "diag"),
    "pressure_reference_head": ("pressure_reference_head", "diag"),
    "gravity_body_fraction": ("gravity_body_fraction", "diag"), "vof_exterior_gas": ("vof_exterior_gas", "diag"),
}
EXACT = {"obstacle", "near_obstacle", "lattice_open", "lattice_wall_type", "free_surface_type",
         "free_surface_type_prev", "free_surface_mass_excess_dir", "vof_exterior_gas"}


# options that name a file stored beside the goldens
FILE_OPTIONS = ("LBM_BOTTOM_FILE",)


def load_golden(name: str):
    data = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
    env = json.loads(str(data["env"]))
    for key in FILE_OPTIONS:
        if key in env and not os.path.isabs(env[key]):
            env[key] = os.path.join(GOLDEN_DIR, env[key])
    return data, env


def is_injected(data) -> bool:
    """The case's state was edited after the reference's init; a run starts
    from its s0 snapshot instead of its own init."""
    return "injected" in data and bool(int(data["injected"]))


def golden_state(data, tag: str = "s0") -> dict:
    """ABI name -> array of the state buffers in snapshot `tag` (plus "f",
    the current populations), in the ABI's dtypes."""
    out = {"f": np.ascontiguousarray(data[f"{tag}_f"], dtype=np.float32)}
    for gname, (aname, kind) in FIELD_MAP.items():
        key = f"{tag}_{gname}"
        if kind != "state" or key not in data:
            continue
        v = data[key]
        if aname in ("fs_type", "fs_type_prev", "fs_excess_dir"):
            v = v.astype(np.int8)
        else:
            v = v.astype(np.float32)
        out[aname] = np.ascontiguousarray(v)
    return out


def load_state_numpy(arrays: dict, current_f: str, state: dict):
    """Write a golden state into numpy state arrays (the oracle's)."""
    for name, v in state.items():
        dst = arrays[current_f] if name == "f" else arrays[name]
        dst[...] = v.reshape(dst.shape)


def golden_cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN_DIR) if f.endswith(".npz"))


def compare_snapshot(data, tag: str, sim, rtol: float, atol: float, skip=()):
    """Return a list of mismatch descriptions (empty = agreement)."""
    problems = []
    arrays = dict(sim.arrays)
    arrays["f"] = sim.f()
    names = ["f"] + list(FIELD_MAP)
    for gname in names:
        if gname in skip or f"{tag}_{gname}" not in data:
            continue
        ref = data[f"{tag}_{gname}"]
        mine = arrays[FIELD_MAP[gname][0] if gname != "f" else "f"]
        mine = np.asarray(mine).reshape(ref.shape)
        if gname in EXACT:
            bad = np.count_nonzero(mine.astype(np.int64) != ref.astype(np.int64))
            if bad:
                problems.append(f"{tag}:{gname}: {bad} exact mismatches")
        else:
            r = ref.astype(np.float64)
            m = mine.astype(np.float64)
            err = np.abs(m - r)
            lim = atol + rtol * np.abs(r)
            bad = np.count_nonzero(~(err <= lim))
            if bad:
                problems.append(f"{tag}:{gname}: {bad} values out of tol, max abs err {np.nanmax(err):.3e}")
    return problems
