"""Generate golden vectors by running the reference solver's own kernels.

Run where a checkout of the reference is available (it is read, never
written; GPU machines do not need it):

    python tests/golden/gen_golden.py --reference PATH [--only NAME]

PATH is the reference checkout (default: the LBM_REFERENCE_DIR environment
variable).

Each case sets LBM_* options, imports LBM_3D_LES_air_over_waves_CODEX.py
with taichi_shim standing in for Taichi, runs main() for a few steps on a
tiny grid and saves tests/golden/<case>.npz with:
  env            the options (JSON)
  noise          the initial kick fed to ti.random() in init_fields
  rho_initial    the reference's prepare_initial_density_field output
  s<k>_<field>   snapshots after init (k = 0) and after step k
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import sys
import tempfile
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SOLVER_FILE = "LBM_3D_LES_air_over_waves_CODEX.py"
REFERENCE = os.environ.get("LBM_REFERENCE_DIR", "")

sys.path.insert(0, HERE)
import taichi_shim  # noqa: E402

MASK64 = (1 << 64) - 1


def splitmix64(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK64
    return x ^ (x >> 31)


def uniform01(seed: int, step: int, cell: int) -> float:
    h = splitmix64(seed ^ splitmix64(step ^ splitmix64((cell + 0x632BE59BD9B4E019) & MASK64)))
    return float(np.float32(np.float32(h >> 40) * np.float32(1.0 / 16777216.0)))


BASE_AIR = {"LBM_PHYSICS_MODE": "air", "LBM_DX_M": "1"}

CASES = {
    # reference air defaults (KBC + LES + backscatter + fringe + top drive + sponge)
    "air_kbc_default": dict(BASE_AIR, LBM_LX_M="12", LBM_LY_M="4", LBM_LZ_M="10",
                            LBM_BED_AMP_M="1.0", LBM_BED_WAVELENGTH_M="8", LBM_WATER_DEPTH_M="6"),
    # benchmark air configuration: regularized + LES, single-sine bed, free-slip top
    "air_regularized_sine": dict(BASE_AIR, LBM_LX_M="12", LBM_LY_M="4", LBM_LZ_M="10",
                                 LBM_COLLISION="regularized", LBM_BACKSCATTER="0", LBM_ENABLE_X_FRINGE="0",
                                 LBM_ENABLE_TOP_DRIVE="0", LBM_ENABLE_TOP_SPONGE="0",
                                 LBM_BED_LEVEL_M="3", LBM_BED_AMP_M="1.5", LBM_BED_WAVELENGTH_M="12",
                                 LBM_U_TOP_MPS="0.6"),
    # cube obstacle over the moving bed, solid x walls, cell wall sampling
    "air_bed_cube_solidx": dict(BASE_AIR, LBM_LX_M="12", LBM_LY_M="6", LBM_LZ_M="10",
                                LBM_OBSTACLE_MODE="bed_cube", LBM_CUBE_SIDE_M="3", LBM_CUBE_CENTER_Z_M="6",
                                LBM_CUBE_YAW_DEG="20", LBM_X_BOUNDARY="solid", LBM_WALL_VELOCITY_SAMPLING="cell",
                                LBM_BED_AMP_M="1.0", LBM_BED_WAVELENGTH_M="8", LBM_WATER_DEPTH_M="6",
                                LBM_BACKSCATTER="0"),
    # phi-based geometry
    "air_phi_geometry": dict(BASE_AIR, LBM_LX_M="10", LBM_LY_M="4", LBM_LZ_M="8",
                             LBM_BOUNDARY_GEOMETRY="phi", LBM_BED_AMP_M="1.0", LBM_BED_WAVELENGTH_M="10",
                             LBM_WATER_DEPTH_M="6", LBM_COLLISION="regularized"),
    # water, height-function kinematic path, Gaussian, hydrostatic balanced
    "water_height_gaussian": {"LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_INITIAL": "gaussian",
                              "LBM_DX_M": "1", "LBM_LX_M": "16", "LBM_LY_M": "3", "LBM_LZ_M": "10",
                              "LBM_WATER_DEPTH_M": "5", "LBM_GAUSSIAN_AMPLITUDE_M": "1.5",
                              "LBM_GAUSSIAN_SIGMA_M": "3", "LBM_WATER_NU_M2S": "0.05"},
    # water, solitary wave, periodic, total pressure, noneq refill, LES on
    "water_height_solitary": {"LBM_PHYSICS_MODE": "water", "LBM_DX_M": "1", "LBM_LX_M": "16",
                              "LBM_LY_M": "3", "LBM_LZ_M": "10", "LBM_WATER_DEPTH_M": "5",
                              "LBM_SOLITARY_AMPLITUDE_M": "1.5", "LBM_PRESSURE_FORMULATION": "total_pressure",
                              "LBM_FREE_SURFACE_REFILL": "noneq", "LBM_USE_LES": "1",
                              "LBM_WATER_NU_M2S": "0.05", "LBM_INIT_FREE_SURFACE_POPULATIONS": "1"},
    # VOF falling block with KBC, collapse each 2 steps, bridge
    "vof_block_kbc": {"LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_TRACKING": "vof",
                      "LBM_FREE_SURFACE_INITIAL": "gaussian", "LBM_X_BOUNDARY": "solid", "LBM_COLLISION": "kbc",
                      "LBM_VOF_INITIAL_SHAPE": "block", "LBM_GAUSSIAN_AMPLITUDE_M": "0",
                      "LBM_WATER_DEPTH_M": "4", "LBM_VOF_BLOCK_SIZE_M": "3", "LBM_VOF_BLOCK_SIZE_Y_M": "2",
                      "LBM_VOF_BLOCK_BOTTOM_M": "6", "LBM_PRESSURE_FORMULATION": "vof_component_balanced",
                      "LBM_VOF_COLLAPSE_TRAPPED_GAS": "1", "LBM_VOF_COLLAPSE_INTERVAL": "2",
                      "LBM_VOF_COLLAPSE_MAX_VOLUME_M3": "64", "LBM_VOF_THIN_GAP_BRIDGE": "1",
                      "LBM_VOF_THIN_GAP_BRIDGE_STRENGTH": "4", "LBM_DX_M": "1", "LBM_LX_M": "10",
                      "LBM_LY_M": "3", "LBM_LZ_M": "12", "LBM_WATER_NU_M2S": "0.05",
                      "LBM_VOF_EMPTY_FILL_THRESHOLD": "0.02"},
    # VOF with hydrostatic refill / directional refill and a Gaussian surface
    "vof_gaussian_directional": {"LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_TRACKING": "vof",
                                 "LBM_FREE_SURFACE_INITIAL": "gaussian", "LBM_FREE_SURFACE_REFILL": "directional",
                                 "LBM_DX_M": "1", "LBM_LX_M": "12", "LBM_LY_M": "3", "LBM_LZ_M": "10",
                                 "LBM_WATER_DEPTH_M": "5", "LBM_GAUSSIAN_AMPLITUDE_M": "2",
                                 "LBM_GAUSSIAN_SIGMA_M": "2", "LBM_WATER_NU_M2S": "0.05"},
}

# VOF pool whose initial state is edited after the reference's own init
# (inject_vof_features below) so that the rarely reached VOF kernels act in
# the first steps: trapped-gas collapse (every step), the thin-gap bridge,
# orphan removal, detached-cell advection and residual compression
VOF_FEATURES = {"LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_TRACKING": "vof",
                "LBM_FREE_SURFACE_INITIAL": "gaussian", "LBM_GAUSSIAN_AMPLITUDE_M": "0",
                "LBM_X_BOUNDARY": "solid", "LBM_DX_M": "1", "LBM_LX_M": "16", "LBM_LY_M": "4", "LBM_LZ_M": "16",
                "LBM_WATER_DEPTH_M": "4.5", "LBM_PRESSURE_FORMULATION": "vof_component_balanced",
                "LBM_VOF_COLLAPSE_TRAPPED_GAS": "1", "LBM_VOF_COLLAPSE_INTERVAL": "1",
                "LBM_VOF_COLLAPSE_MAX_VOLUME_M3": "64", "LBM_VOF_THIN_GAP_BRIDGE": "1",
                "LBM_VOF_THIN_GAP_BRIDGE_STRENGTH": "4", "LBM_WATER_NU_M2S": "0.05"}
CASES["vof_features_kbc"] = dict(VOF_FEATURES, LBM_COLLISION="kbc")
CASES["vof_features_regularized"] = dict(VOF_FEATURES, LBM_COLLISION="regularized", LBM_X_BOUNDARY="periodic",
                                         LBM_FREE_SURFACE_REFILL="noneq")
# piecewise-linear bed profile from a bottom file (x_m z_m pairs)
CASES["air_piecewise_bed"] = dict(BASE_AIR, LBM_LX_M="16", LBM_LY_M="4", LBM_LZ_M="10",
                                  LBM_BED_PROFILE="piecewise_linear", LBM_BOTTOM_FILE="bottom_piecewise.txt",
                                  LBM_COLLISION="regularized", LBM_BACKSCATTER="0")
# linear-wave initial pressure (cosine modes with solid x walls, FFT modes when periodic)
CASES["water_linear_wave_solid"] = {"LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_INITIAL": "gaussian",
                                    "LBM_INITIAL_PRESSURE_MODE": "linear_wave", "LBM_DX_M": "1",
                                    "LBM_LX_M": "16", "LBM_LY_M": "3", "LBM_LZ_M": "10", "LBM_WATER_DEPTH_M": "5",
                                    "LBM_GAUSSIAN_AMPLITUDE_M": "1.5", "LBM_GAUSSIAN_SIGMA_M": "3",
                                    "LBM_WATER_NU_M2S": "0.05", "LBM_PRESSURE_FORMULATION": "total_pressure"}
CASES["water_linear_wave_periodic"] = dict(CASES["water_linear_wave_solid"], LBM_X_BOUNDARY="periodic",
                                           LBM_PRESSURE_FORMULATION="hydrostatic_balanced")

STEPS = {"air_kbc_default": 3, "air_regularized_sine": 3, "air_bed_cube_solidx": 2, "air_phi_geometry": 2,
         "water_height_gaussian": 3, "water_height_solitary": 3, "vof_block_kbc": 4, "vof_gaussian_directional": 3,
         "vof_features_kbc": 4, "vof_features_regularized": 4, "air_piecewise_bed": 3,
         "water_linear_wave_solid": 2, "water_linear_wave_periodic": 2}

# files a case reads, stored beside the goldens (the env holds the bare name)
CASE_FILES = {"air_piecewise_bed": {"LBM_BOTTOM_FILE": "bottom_piecewise.txt"}}


def inject_vof_features(mod):
    """Edit the VOF state after the reference's init (before its first column
    height update), in place on the reference's own fields:
      - a trapped gas pocket one cell thick in z (2 x 1 cells at k = 2):
        non-exterior gas, so the collapse applies; the liquid cells around it
        stream through a one-cell gas gap, so the thin-gap bridge acts;
      - a lone interface cell (fill 0.3) two cells above the surface layer:
        no wet neighbour, resolved cells within reach -> orphan removal;
      - a lone interface cell (fill 0.6) far above the pool (no resolved cell
        within the search radius) -> detached-cell advection;
      - a lone interface cell of fill 0.005 far above the pool -> advection,
        then residual compression.
    The reference's interface-layer kernel then re-establishes its invariant
    around the edits, and the previous types follow the new ones."""
    t = mod.free_surface_type.arr
    fill = mod.free_surface_fill.arr
    mass = mod.free_surface_mass.arr
    rho = mod.rho.arr
    gas, iface = int(mod.FS_GAS), int(mod.FS_INTERFACE)

    def put(k, j, i, ctype, fl):
        t[k, j, i] = ctype
        fill[k, j, i] = np.float32(fl)
        mass[k, j, i] = np.float32(np.float32(fl) * rho[k, j, i])

    nx = t.shape[2]
    put(2, 1, 5, gas, 0.0)
    put(2, 1, 6, gas, 0.0)
    put(6, 2, nx - 5, iface, 0.3)
    put(12, 1, 3, iface, 0.6)
    put(12, 2, nx - 6, iface, 0.005)
    mod.enforce_vof_interface_layer()
    mod.free_surface_type_prev.arr[...] = t


INJECT = {"vof_features_kbc": inject_vof_features, "vof_features_regularized": inject_vof_features}

SCALAR_FIELDS = ["rho", "ux", "uy", "uz", "omegaLoc", "phi", "obstacle", "near_obstacle", "free_surface_fill",
                 "free_surface_type", "free_surface_type_prev", "free_surface_mass", "free_surface_mass_excess",
                 "free_surface_mass_excess_dir", "pressure_reference_head", "gravity_body_fraction",
                 "vof_exterior_gas"]
PLANE_FIELDS = ["water_h", "water_h_last", "u_wave", "v_wave", "w_wave", "free_surface_h", "free_surface_h_last",
                "free_surface_flux_x", "free_surface_flux_y", "u_inlet_profile"]
VECTOR_FIELDS = ["f", "lattice_open", "lattice_open_frac", "lattice_wall_type"]
COUNTERS = ["boundary_refill_count", "free_surface_refill_count", "free_surface_coalescence_repair_count",
            "free_surface_thin_gap_bridge_count", "free_surface_cut_link_count", "free_surface_vof_excess_count",
            "free_surface_vof_orphan_count", "free_surface_vof_collapse_cell_count",
            "free_surface_vof_collapse_candidate_volume_m3", "free_surface_vof_collapse_applied_volume_m3",
            "free_surface_vof_collapse_removal_scale", "free_surface_vof_collapse_candidate_mass",
            "free_surface_vof_collapse_exterior_capacity", "free_surface_vof_detached_advect_count",
            "free_surface_vof_detached_advect_mass", "free_surface_vof_detached_compress_count",
            "free_surface_vof_detached_compress_mass", "boundary_cut_link_count"]


def snapshot(mod, tag, out):
    for name in SCALAR_FIELDS + PLANE_FIELDS:
        out[f"{tag}_{name}"] = getattr(mod, name).to_numpy()
    for name in VECTOR_FIELDS:
        arr = getattr(mod, name).to_numpy()          # (Nz, Ny, Nx, 19)
        out[f"{tag}_{name}"] = np.ascontiguousarray(np.moveaxis(arr, -1, 0))  # (19, Nz, Ny, Nx)
    for name in COUNTERS:
        out[f"{tag}_{name}"] = np.array(getattr(mod, name)[None])


def run_case(name: str, env: dict, seed: int = 12345) -> dict:
    saved = dict(os.environ)
    cache = tempfile.mkdtemp(prefix="ticache_")
    try:
        for key in list(os.environ):
            if key.startswith("LBM_"):
                del os.environ[key]
        os.environ.update(env)
        for key, fname in CASE_FILES.get(name, {}).items():
            os.environ[key] = os.path.join(HERE, fname)
        os.environ["LBM_TI_CACHE_DIR"] = cache
        sys.modules["taichi"] = taichi_shim
        sys.path.insert(0, REFERENCE)
        spec = importlib.util.spec_from_file_location(f"ref_{name}", os.path.join(REFERENCE, SOLVER_FILE))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        shape = (mod.Nz, mod.Ny, mod.Nx)
        rng = np.random.default_rng(seed)
        noise = rng.uniform(-1.0, 1.0, size=(3,) + shape).astype(np.float32)
        state = {"kick": 0}

        def hook(kernel, cell):
            if kernel == "init_fields":
                v = float(noise[0].reshape(-1)[state["kick"]])
                state["kick"] += 1
                return v / 2.0 + 0.5
            if kernel == "collide_KBC":
                step = taichi_shim._state["calls"].get("collide_KBC", 0)
                return uniform01(seed, step, cell)
            raise RuntimeError(f"unexpected ti.random in {kernel}")

        taichi_shim._state["random_hook"] = hook
        taichi_shim._state["calls"] = {}
        out = {"env": np.array(json.dumps(env)), "noise": noise, "seed": np.array(seed)}
        captured = {"init": False}
        orig_height = mod.update_free_surface_height_from_vof

        def height_then_snapshot():
            if not captured["init"] and name in INJECT:
                INJECT[name](mod)
            orig_height()
            if not captured["init"]:
                captured["init"] = True
                snapshot(mod, "s0", out)
                out["rho_initial"] = mod.rho_initial.to_numpy()

        mod.update_free_surface_height_from_vof = height_then_snapshot

        def visualize(step, time_phys, re_a, re_b):
            snapshot(mod, f"s{step}", out)

        mod.visualize = visualize
        mod.steps = STEPS[name]
        mod.plot_freq = 1
        mod.plot_step_start = 0
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            with np.errstate(all="ignore"):
                mod.main()
        out["nsteps"] = np.array(STEPS[name])
        out["injected"] = np.array(1 if name in INJECT else 0)
        return out
    finally:
        os.environ.clear()
        os.environ.update(saved)
        if REFERENCE in sys.path:
            sys.path.remove(REFERENCE)


def main():
    global REFERENCE
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=REFERENCE, help="reference checkout (default: $LBM_REFERENCE_DIR)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    REFERENCE = os.path.abspath(args.reference) if args.reference else ""
    if not REFERENCE or not os.path.exists(os.path.join(REFERENCE, SOLVER_FILE)):
        raise SystemExit(f"{SOLVER_FILE} not found: pass --reference PATH or set LBM_REFERENCE_DIR")
    for name, env in CASES.items():
        if args.only and name != args.only:
            continue
        out = run_case(name, env)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB)", flush=True)


if __name__ == "__main__":
    main()
