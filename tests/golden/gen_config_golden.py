"""Generate the option-surface golden: the reference module's own globals
for a set of LBM_* environments, or the exception its import raises.

Run where a checkout of the reference is available (it is read, never
written; GPU machines do not need it):

    python tests/golden/gen_config_golden.py --reference PATH

PATH is the reference checkout (default: the LBM_REFERENCE_DIR environment
variable).  Each case imports LBM_3D_LES_air_over_waves_CODEX.py with
taichi_shim standing in for Taichi and the case's options as the only LBM_*
variables.  The import evaluates the option surface (CODEX.py:35-529,
lbm_env.py:9-22) and stops before main().  tests/golden/config_cases.json
then holds, per case, either every scalar module global (numbers, flags,
strings; the piecewise bed and its metadata when the bed is piecewise) or
the exception's class and message; for valid cases also the lines the
import printed (without Taichi's cache line) and, on the small grids, the
lines main() prints when it has no steps to run (its initialisation and
configuration summary).  A case's "files" are written to a
scratch folder first and "{name}" in an option value or a message stands
for that file's absolute path, so the fixture does not depend on where it
was made.
"""
from __future__ import annotations

import argparse
import contextlib
import importlib.util
import io
import json
import os
import sys
import tempfile
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SOLVER_FILE = "LBM_3D_LES_air_over_waves_CODEX.py"
OUT = os.path.join(HERE, "config_cases.json")

sys.path.insert(0, HERE)
import taichi_shim  # noqa: E402

AIR = {"LBM_PHYSICS_MODE": "air", "LBM_DX_M": "1", "LBM_LX_M": "12", "LBM_LY_M": "4", "LBM_LZ_M": "10"}
WATER = {"LBM_PHYSICS_MODE": "water", "LBM_DX_M": "1", "LBM_LX_M": "40", "LBM_LY_M": "2", "LBM_LZ_M": "16",
         "LBM_WATER_DEPTH_M": "8"}
VOF = dict(WATER, LBM_FREE_SURFACE_TRACKING="vof", LBM_VOF_INITIAL_SHAPE="block", LBM_LZ_M="20")
PIECEWISE = dict(AIR, LBM_BED_PROFILE="piecewise_linear", LBM_BOTTOM_FILE="{bottom}")

# name -> (options, files written beside the case, {file name: text})
CASES = {
    # the reference's own defaults (300 x 10 x 20 m at dx 0.5)
    "defaults_air": ({}, {}),
    "defaults_water": ({"LBM_PHYSICS_MODE": "water"}, {}),
    "air_small": (AIR, {}),
    "air_regularized_no_les_no_drive": (dict(AIR, LBM_COLLISION="regularized", LBM_USE_LES="0",
                                             LBM_ENABLE_TOP_DRIVE="0", LBM_ENABLE_X_FRINGE="0",
                                             LBM_ENABLE_TOP_SPONGE="0", LBM_BACKSCATTER="0"), {}),
    "air_solid_x_cell_sampling": (dict(AIR, LBM_X_BOUNDARY="solid", LBM_WALL_VELOCITY_SAMPLING="cell",
                                       LBM_U_TOP_MPS="12"), {}),
    "air_cube_yaw_pitch": (dict(AIR, LBM_OBSTACLE_MODE="cube", LBM_CUBE_SIZE_X_M="3", LBM_CUBE_SIZE_Y_M="2",
                                LBM_CUBE_SIZE_Z_M="2.5", LBM_CUBE_YAW_DEG="30", LBM_CUBE_PITCH_DEG="10"), {}),
    "air_bed_cube_placed": (dict(AIR, LBM_OBSTACLE_MODE="bed_cube", LBM_CUBE_SIDE_M="2", LBM_CUBE_CENTER_X_M="5",
                                 LBM_CUBE_CENTER_Y_M="1.5", LBM_CUBE_CENTER_Z_M="6"), {}),
    "air_phi_fraction": (dict(AIR, LBM_BOUNDARY_GEOMETRY="phi_fraction", LBM_BED_AMP_M="0.75",
                              LBM_BED_WAVELENGTH_M="6", LBM_WATER_DEPTH_M="4", LBM_BED_LEVEL_M="2.5"), {}),
    "air_phi_flags_gravity": (dict(AIR, LBM_BOUNDARY_GEOMETRY="phi", LBM_GRAVITY_MPS2="9.81"), {}),
    "air_flat_bed_upper_case": (dict(AIR, LBM_BED_PROFILE="FLAT", LBM_COLLISION="KBC", LBM_USE_LES="True",
                                     LBM_X_BOUNDARY="Solid"), {}),
    "air_piecewise_bed": (PIECEWISE, {"bottom": "# x z\n10, 3.5\n0 2.0\n\n4.5 1.25  # dip\n12 2.75\n"}),
    "air_fine_dx": (dict(AIR, LBM_DX_M="0.25", LBM_LX_M="4", LBM_LY_M="1", LBM_LZ_M="3"), {}),
    "steps_and_plots": (dict(AIR, LBM_STEPS="123", LBM_PLOT_FREQ="7", LBM_PLOT_START="3"), {}),
    "ti_arch_cpu": (dict(AIR, LBM_TI_ARCH="CPU"), {}),
    "water_solitary": (WATER, {}),
    "water_solitary_ratio_leftward": (dict(WATER, LBM_SOLITARY_HEIGHT_DEPTH_RATIO="0.2",
                                           LBM_SOLITARY_DIRECTION="-3", LBM_SOLITARY_X0_M="30",
                                           LBM_SOLITARY_INITIAL_VELOCITY="shallow_water"), {}),
    "water_gaussian_hydrostatic_boundary": (dict(WATER, LBM_FREE_SURFACE_INITIAL="gaussian",
                                                 LBM_FREE_SURFACE_BOUNDARY="hydrostatic",
                                                 LBM_GAUSSIAN_AMPLITUDE_M="1.5", LBM_GAUSSIAN_SIGMA_M="4",
                                                 LBM_GAUSSIAN_CENTER_X_M="20"), {}),
    "water_prescribed_solitary": (dict(WATER, LBM_FREE_SURFACE_MODE="prescribed_solitary",
                                       LBM_SOLITARY_AMPLITUDE_M="0.8",
                                       LBM_SOLITARY_INITIAL_VELOCITY="none"), {}),
    "water_static_flat_total_pressure": (dict(WATER, LBM_FREE_SURFACE_MODE="height_static",
                                              LBM_PRESSURE_FORMULATION="total_pressure",
                                              LBM_FREE_SURFACE_DEPTH_M="6", LBM_FREE_SURFACE_LEVEL_M="7"), {}),
    "water_linear_wave_current": (dict(WATER, LBM_INITIAL_PRESSURE_MODE="linear_wave",
                                       LBM_WATER_CURRENT_MPS="0.3", LBM_GRAVITY_MPS2="5", LBM_WATER_NU_M2S="1e-5",
                                       LBM_WATER_RHO_KGM3="1000"), {}),
    "water_without_free_surface": (dict(WATER, LBM_FREE_SURFACE_MODE="none"), {}),
    "water_moving_bed": (dict(WATER, LBM_BED_PROFILE="moving_sine", LBM_BED_AMP_M="0.5",
                              LBM_BED_WAVELENGTH_M="10"), {}),
    "vof_block": (VOF, {}),
    "vof_block_total_pressure_corrected": (dict(VOF, LBM_PRESSURE_FORMULATION="total_pressure"), {}),
    "vof_block_total_pressure_allowed": (dict(VOF, LBM_PRESSURE_FORMULATION="total_pressure",
                                              LBM_ALLOW_TOTAL_PRESSURE_VOF_DIAGNOSTIC="yes"), {}),
    "vof_options": (dict(VOF, LBM_VOF_BLOCK_SIZE_M="3", LBM_VOF_BLOCK_SIZE_X_M="5", LBM_VOF_BLOCK_CENTER_X_M="12",
                         LBM_VOF_BLOCK_BOTTOM_M="12", LBM_FREE_SURFACE_REFILL="directional",
                         LBM_INIT_FREE_SURFACE_POPULATIONS="1", LBM_VOF_LINK_APERTURE="0",
                         LBM_VOF_EMPTY_FILL_THRESHOLD="0.1", LBM_VOF_ORPHAN_EMPTY_THRESHOLD="0.3",
                         LBM_VOF_ORPHAN_SEARCH_RADIUS="2", LBM_VOF_ORPHAN_MAX_WEAK_NEIGHBORS="3",
                         LBM_VOF_DETACHED_ADVECTION="0", LBM_VOF_DETACHED_MAX_WET_NEIGHBORS="6",
                         LBM_VOF_DETACHED_MAX_RESOLVED_NEIGHBORS="2",
                         LBM_VOF_DETACHED_RESIDUAL_FILL_THRESHOLD="0.05", LBM_VOF_THIN_GAP_BRIDGE="true",
                         LBM_VOF_THIN_GAP_BRIDGE_STRENGTH="0.5", LBM_VOF_COLLAPSE_TRAPPED_GAS="1",
                         LBM_VOF_COLLAPSE_INTERVAL="3", LBM_VOF_COLLAPSE_MAX_VOLUME_M3="2.5",
                         LBM_VOF_COLLAPSE_FLOOD_SWEEPS="9"), {}),
    "vof_centered_block": (dict(VOF, LBM_VOF_BLOCK_CENTER_Z_M="15", LBM_VOF_BLOCK_SIZE_Y_M="1"), {}),
    # invalid options: the import raises
    "bad_ti_arch": (dict(AIR, LBM_TI_ARCH="tpu"), {}),
    "bad_physics_mode": (dict(AIR, LBM_PHYSICS_MODE="plasma"), {}),
    "bad_free_surface_mode": (dict(WATER, LBM_FREE_SURFACE_MODE="wild"), {}),
    "bad_free_surface_initial": (dict(WATER, LBM_FREE_SURFACE_INITIAL="square"), {}),
    "bad_vof_shape": (dict(WATER, LBM_VOF_INITIAL_SHAPE="sphere"), {}),
    "bad_initial_pressure_mode": (dict(WATER, LBM_INITIAL_PRESSURE_MODE="cold"), {}),
    "bad_pressure_formulation": (dict(WATER, LBM_PRESSURE_FORMULATION="gauge"), {}),
    "bad_tracking": (dict(WATER, LBM_FREE_SURFACE_TRACKING="level_set"), {}),
    "bad_free_surface_boundary": (dict(WATER, LBM_FREE_SURFACE_BOUNDARY="open"), {}),
    "bad_refill": (dict(WATER, LBM_FREE_SURFACE_REFILL="zero"), {}),
    "bad_empty_fill": (dict(WATER, LBM_VOF_EMPTY_FILL_THRESHOLD="0.5"), {}),
    "bad_orphan_empty": (dict(WATER, LBM_VOF_ORPHAN_EMPTY_THRESHOLD="-0.01"), {}),
    "bad_orphan_radius": (dict(WATER, LBM_VOF_ORPHAN_SEARCH_RADIUS="5"), {}),
    "bad_orphan_radius_text": (dict(WATER, LBM_VOF_ORPHAN_SEARCH_RADIUS="two"), {}),
    "bad_orphan_weak": (dict(WATER, LBM_VOF_ORPHAN_MAX_WEAK_NEIGHBORS="19"), {}),
    "bad_detached_wet": (dict(WATER, LBM_VOF_DETACHED_MAX_WET_NEIGHBORS="-1"), {}),
    "bad_detached_resolved": (dict(WATER, LBM_VOF_DETACHED_MAX_RESOLVED_NEIGHBORS="19"), {}),
    "bad_detached_residual": (dict(WATER, LBM_VOF_DETACHED_RESIDUAL_FILL_THRESHOLD="0.5"), {}),
    "bad_bridge_strength": (dict(WATER, LBM_VOF_THIN_GAP_BRIDGE_STRENGTH="-0.5"), {}),
    "bad_collapse_interval": (dict(WATER, LBM_VOF_COLLAPSE_INTERVAL="0"), {}),
    "bad_collapse_volume": (dict(WATER, LBM_VOF_COLLAPSE_MAX_VOLUME_M3="-1"), {}),
    "bad_collapse_sweeps": (dict(WATER, LBM_VOF_COLLAPSE_FLOOD_SWEEPS="0"), {}),
    "bad_dx_text": (dict(AIR, LBM_DX_M="half"), {}),
    "bad_boundary_geometry": (dict(AIR, LBM_BOUNDARY_GEOMETRY="curved"), {}),
    "bad_x_boundary": (dict(AIR, LBM_X_BOUNDARY="open"), {}),
    "bad_wall_sampling": (dict(AIR, LBM_WALL_VELOCITY_SAMPLING="face"), {}),
    "bad_bed_profile": (dict(AIR, LBM_BED_PROFILE="step"), {}),
    "bad_bottom_missing": (dict(PIECEWISE, LBM_BOTTOM_FILE="{missing}"), {}),
    "bad_bottom_three_values": (PIECEWISE, {"bottom": "0 1\n4 1 2\n"}),
    "bad_bottom_number": (PIECEWISE, {"bottom": "0 1\n4 a\n"}),
    "bad_bottom_non_finite": (PIECEWISE, {"bottom": "0 1\nnan 2\n"}),
    "bad_bottom_one_pair": (PIECEWISE, {"bottom": "# one point only\n0 1\n"}),
    "bad_bottom_duplicate_x": (PIECEWISE, {"bottom": "0 1\n5 2\n5 3\n"}),
    "bad_free_surface_depth": (dict(WATER, LBM_FREE_SURFACE_DEPTH_M="0"), {}),
    "bad_solitary_ratio": (dict(WATER, LBM_SOLITARY_HEIGHT_DEPTH_RATIO="0"), {}),
    "bad_solitary_amplitude": (dict(WATER, LBM_SOLITARY_AMPLITUDE_M="-0.1"), {}),
    "bad_solitary_direction": (dict(WATER, LBM_SOLITARY_DIRECTION="0"), {}),
    "bad_solitary_velocity": (dict(WATER, LBM_SOLITARY_INITIAL_VELOCITY="deep"), {}),
    "bad_vof_shape_without_vof": (dict(WATER, LBM_VOF_INITIAL_SHAPE="block"), {}),
    "bad_vof_hydrostatic_balanced": (dict(VOF, LBM_PRESSURE_FORMULATION="hydrostatic_balanced"), {}),
    "bad_vof_hydrostatic_boundary": (dict(VOF, LBM_FREE_SURFACE_BOUNDARY="hydrostatic"), {}),
    "bad_obstacle_mode": (dict(AIR, LBM_OBSTACLE_MODE="sphere"), {}),
    "bad_cube_size": (dict(AIR, LBM_OBSTACLE_MODE="cube", LBM_CUBE_SIZE_Y_M="0"), {}),
    "bad_collision": (dict(AIR, LBM_COLLISION="bgk"), {}),
}


def materialize(env: dict, files: dict, folder: str):
    """The case's options with "{name}" replaced by the path of its file in
    `folder` (written from `files`; "{missing}" names a file never written).
    Returns (options, {path: "{name}"})."""
    paths = {}
    for name, text in files.items():
        path = os.path.join(folder, f"{name}.txt")
        with open(path, "w", encoding="utf-8") as fh:
            fh.write(text)
        paths[name] = path
    paths.setdefault("missing", os.path.join(folder, "missing.txt"))
    out = {}
    for key, value in env.items():
        for name, path in paths.items():
            value = value.replace("{" + name + "}", path)
        out[key] = value
    return out, {path: "{" + name + "}" for name, path in paths.items()}


def unplace(text: str, placeholders: dict) -> str:
    for path, mark in placeholders.items():
        text = text.replace(path, mark)
    return text


def scalar_globals(mod, placeholders: dict) -> dict:
    """Every scalar module global, as plain JSON values."""
    out = {}
    for name, value in vars(mod).items():
        if name.startswith("_"):
            continue
        if isinstance(value, (bool, np.bool_)):
            out[name] = bool(value)
        elif isinstance(value, (int, np.integer)):
            out[name] = int(value)
        elif isinstance(value, (float, np.floating)):
            out[name] = float(value)
        elif isinstance(value, str):
            out[name] = unplace(value, placeholders)
    if getattr(mod, "bed_profile", "") == "piecewise_linear":
        out["piecewise_bed_z_np"] = [float(v) for v in np.asarray(mod.piecewise_bed_z_np, dtype=np.float32)]
        out["piecewise_bed_metadata"] = {k: unplace(v, placeholders) if isinstance(v, str) else v
                                         for k, v in mod.piecewise_bed_metadata.items()}
    return out


def import_reference(reference: str, env: dict):
    """Import the reference module with `env` as its only LBM_* options.
    Returns the module and what the import printed."""
    saved = dict(os.environ)
    try:
        for key in list(os.environ):
            if key.startswith("LBM_"):
                del os.environ[key]
        os.environ.update(env)
        os.environ["LBM_TI_CACHE_DIR"] = tempfile.mkdtemp(prefix="ticache_")
        sys.modules["taichi"] = taichi_shim
        sys.path.insert(0, reference)
        spec = importlib.util.spec_from_file_location("ref_options", os.path.join(reference, SOLVER_FILE))
        mod = importlib.util.module_from_spec(spec)
        printed = io.StringIO()
        with warnings.catch_warnings(), contextlib.redirect_stdout(printed):
            warnings.simplefilter("ignore")
            spec.loader.exec_module(mod)
        return mod, printed.getvalue()
    finally:
        os.environ.clear()
        os.environ.update(saved)
        if reference in sys.path:
            sys.path.remove(reference)


def main_stdout(mod) -> str:
    """What the module's main() prints with no steps to run: its
    initialisation and configuration summary (CODEX.py:3757-3871).  The
    initial kick's random draws are fixed at 0.5; they print nothing."""
    taichi_shim._state["random_hook"] = lambda kernel, cell: 0.5
    taichi_shim._state["calls"] = {}
    mod.steps, mod.plot_freq, mod.plot_step_start = 0, 1, 0
    printed = io.StringIO()
    with warnings.catch_warnings(), contextlib.redirect_stdout(printed), np.errstate(all="ignore"):
        warnings.simplefilter("ignore")
        mod.main()
    return printed.getvalue()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LBM_REFERENCE_DIR", ""),
                    help="reference checkout (default: $LBM_REFERENCE_DIR)")
    args = ap.parse_args()
    reference = os.path.abspath(args.reference) if args.reference else ""
    if not reference or not os.path.exists(os.path.join(reference, SOLVER_FILE)):
        raise SystemExit(f"{SOLVER_FILE} not found: pass --reference PATH or set LBM_REFERENCE_DIR")
    cases = []
    for name, (env, files) in CASES.items():
        with tempfile.TemporaryDirectory() as folder:
            options, placeholders = materialize(env, files, folder)
            case = {"name": name, "env": env, "files": files}
            try:
                mod, printed = import_reference(reference, options)
            except Exception as exc:  # noqa: BLE001 - the exception is the expected output
                case["error"] = {"type": type(exc).__name__, "message": unplace(str(exc), placeholders)}
            else:
                case["values"] = scalar_globals(mod, placeholders)
                case["import_stdout"] = [ln for ln in unplace(printed, placeholders).splitlines()
                                         if not ln.startswith("Taichi offline cache:")]
                if not name.startswith("defaults_"):   # the defaults' grids are too large for the numpy stand-in
                    case["main_stdout"] = unplace(main_stdout(mod), placeholders).splitlines()
        cases.append(case)
        print(f"{name}: {'error ' + case['error']['type'] if 'error' in case else len(case['values'])}", flush=True)
    with open(OUT, "w", encoding="utf-8") as fh:
        json.dump({"solver": SOLVER_FILE, "cases": cases}, fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"wrote {OUT} ({os.path.getsize(OUT) / 1024:.0f} KiB)")


if __name__ == "__main__":
    main()
