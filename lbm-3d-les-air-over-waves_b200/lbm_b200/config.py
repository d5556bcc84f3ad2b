"""LBM_* environment options -> solver configuration.

Re-implements the option surface of the reference solver module
(LBM_3D_LES_air_over_waves_CODEX.py:35-529 and lbm_env.py:9-22): every
LBM_* variable it reads, with the same defaults, the same cross-option
corrections (CODEX.py:343-363) and the same ValueError messages, evaluated
once when a configuration is loaded (the reference evaluates it at import).

The result is a :class:`SolverConfig` whose attributes carry the
reference's global names (``Nx``, ``dx``, ``tau0``, ``vel_scale``,
``free_surface_base_m`` ...), so the drop-in module can re-export them.

Build extensions (not in the reference, all default to its behaviour) are
read from ``LBM_B200_*`` variables; they exist because the benchmark
configurations specify lattice-unit values the reference only hard-codes:

  LBM_B200_LATTICE_UNITS=1     dt_phys = 1 s and vel_scale = 1 (lattice units)
  LBM_B200_TAU0, LBM_B200_CS   override tau0 (nu0 = (tau0-1/2)/3) and Cs
  LBM_B200_G_LB                override the lattice gravity g_lb
  LBM_B200_BED_MODEL=single_sine  one bed harmonic A sin(2 pi (x - c t)/L)
      with LBM_B200_BED_SPEED (c), LBM_B200_BED_RAMP (0/1) and
      LBM_B200_BED_ORBITAL (0/1: wall velocity u_s from the orbital term)
  LBM_B200_TOP=free_slip       specular top wall for air runs
  LBM_B200_INIT_VELOCITY=uniform with LBM_B200_INIT_U0="ux,uy,uz" and
      LBM_B200_INIT_NOISE (amplitude of uniform noise per component)
  LBM_B200_POP_STORAGE=f32|f16s|bf16s   population storage precision
  LBM_RANDOM_SEED              seed of the host noise and the counter RNG
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Mapping

import numpy as np

FS_GAS = 0
FS_LIQUID = 1
FS_INTERFACE = 2
WALL_NONE = 0
WALL_BED = 1
WALL_CUBE = 2
WALL_XMIN = 3
WALL_XMAX = 4


def _truthy(value: str) -> bool:
    return value.lower() in ("1", "true", "yes")


class _Env:
    """Typed reads of an environment mapping (lbm_env.py:9-22)."""

    def __init__(self, environ: Mapping[str, str]):
        self.environ = environ

    def get(self, name, default):
        return self.environ.get(name, default)

    def choice(self, name: str, default: str, choices: tuple) -> str:
        value = str(self.environ.get(name, default)).lower()
        if value not in choices:
            allowed = ", ".join(repr(choice) for choice in choices)
            raise ValueError(f"{name} must be one of: {allowed}")
        return value

    def int(self, name: str, default: int) -> int:
        return int(self.environ.get(name, default))

    def float(self, name: str, default) -> float:
        return float(self.environ.get(name, default))

    def flag(self, name: str, default: str) -> bool:
        return _truthy(str(self.environ.get(name, default)))


@dataclass
class SolverConfig:
    """All reference globals relevant to the step path, plus extensions."""

    values: dict = field(default_factory=dict)

    def __getattr__(self, name):
        try:
            return self.values[name]
        except KeyError as exc:
            raise AttributeError(name) from exc

    def __setattr__(self, name, value):
        if name == "values":
            object.__setattr__(self, name, value)
        else:
            self.values[name] = value


def _load_piecewise_bed(path: str, Nx: int, dx: float, Lx_m: float):
    """Piecewise-linear bed sampled at x cell centres (CODEX.py:223-276)."""
    resolved = path if os.path.isabs(path) else os.path.abspath(path)
    if not os.path.exists(resolved):
        raise FileNotFoundError(f"LBM_BOTTOM_FILE not found: {resolved}")
    pairs = []
    with open(resolved, "r", encoding="utf-8") as handle:
        for number, raw in enumerate(handle, start=1):
            line = raw.split("#", 1)[0].replace(",", " ").strip()
            if not line:
                continue
            parts = line.split()
            if len(parts) != 2:
                raise ValueError(
                    f"Invalid bottom profile line {number} in {resolved}: "
                    "expected exactly two values: x_m z_m"
                )
            try:
                xv, zv = float(parts[0]), float(parts[1])
            except ValueError as exc:
                raise ValueError(f"Invalid numeric value on bottom profile line {number} in {resolved}") from exc
            if not (np.isfinite(xv) and np.isfinite(zv)):
                raise ValueError(f"Non-finite bottom profile value on line {number} in {resolved}")
            pairs.append((xv, zv))
    if len(pairs) < 2:
        raise ValueError(f"LBM_BOTTOM_FILE must contain at least two x z pairs: {resolved}")
    pairs.sort(key=lambda item: item[0])
    xs = np.array([p[0] for p in pairs], dtype=np.float64)
    zs = np.array([p[1] for p in pairs], dtype=np.float64)
    if np.any(np.diff(xs) <= 0.0):
        raise ValueError(f"LBM_BOTTOM_FILE contains duplicate x coordinates: {resolved}")
    centres = (np.arange(Nx, dtype=np.float64) + 0.5) * dx
    z_c = np.interp(centres, xs, zs, left=zs[0], right=zs[-1]).astype(np.float32)
    meta = {
        "path": resolved, "point_count": len(pairs), "first_x": float(xs[0]), "last_x": float(xs[-1]),
        "min_z": float(np.min(z_c)), "max_z": float(np.max(z_c)),
        "z_at_lx": float(np.interp(Lx_m, xs, zs, left=zs[0], right=zs[-1])),
    }
    return z_c, meta


def load_config(environ: Mapping[str, str] | None = None) -> SolverConfig:
    """Evaluate the option surface in the reference's order (CODEX.py:49-529)."""
    env = _Env(os.environ if environ is None else environ)
    c = SolverConfig()

    c.taichi_arch_name = env.choice("LBM_TI_ARCH", "gpu", ("gpu", "cpu"))
    physics_mode = c.physics_mode = env.choice("LBM_PHYSICS_MODE", "air", ("air", "water"))

    fsm = str(env.get("LBM_FREE_SURFACE_MODE", "none" if physics_mode == "air" else "height_kinematic")).lower()
    if fsm not in ("none", "height_static", "height_kinematic", "prescribed_solitary"):
        raise ValueError(
            "LBM_FREE_SURFACE_MODE must be 'none', 'height_static', "
            "'height_kinematic', or 'prescribed_solitary'"
        )
    c.free_surface_mode = fsm
    c.water_free_surface_enabled = 1 if fsm != "none" else 0
    fsi = str(env.get(
        "LBM_FREE_SURFACE_INITIAL",
        "solitary" if (physics_mode == "water" and fsm in ("height_kinematic", "prescribed_solitary")) else "flat",
    )).lower()
    if fsi not in ("flat", "solitary", "gaussian"):
        raise ValueError("LBM_FREE_SURFACE_INITIAL must be 'flat', 'solitary', or 'gaussian'")
    c.free_surface_initial_condition = fsi
    vis = str(env.get("LBM_VOF_INITIAL_SHAPE", "none")).lower()
    if vis not in ("none", "block"):
        raise ValueError("LBM_VOF_INITIAL_SHAPE must be 'none' or 'block'")
    c.vof_initial_shape = vis
    c.initial_pressure_mode = env.choice("LBM_INITIAL_PRESSURE_MODE", "hydrostatic", ("hydrostatic", "linear_wave"))
    default_pf = "hydrostatic_balanced" if physics_mode == "water" else "total_pressure"
    if physics_mode == "water" and vis != "none":
        default_pf = "vof_component_balanced"
    c.default_pressure_formulation = default_pf
    c.pressure_formulation = env.choice(
        "LBM_PRESSURE_FORMULATION", default_pf,
        ("total_pressure", "hydrostatic_balanced", "vof_component_balanced"),
    )
    c.pressure_formulation_auto_corrected = False
    fst = str(env.get("LBM_FREE_SURFACE_TRACKING", "height")).lower()
    if fst not in ("height", "vof"):
        raise ValueError("LBM_FREE_SURFACE_TRACKING must be 'height' or 'vof'")
    c.free_surface_tracking_mode = fst
    fsb = str(env.get("LBM_FREE_SURFACE_BOUNDARY", "cell")).lower()
    if fsb not in ("cell", "hydrostatic"):
        raise ValueError("LBM_FREE_SURFACE_BOUNDARY must be 'cell' or 'hydrostatic'")
    c.free_surface_boundary_mode = fsb
    fsr = str(env.get("LBM_FREE_SURFACE_REFILL", "equilibrium")).lower()
    if fsr not in ("equilibrium", "noneq", "directional"):
        raise ValueError("LBM_FREE_SURFACE_REFILL must be 'equilibrium', 'noneq', or 'directional'")
    c.free_surface_refill_mode = fsr
    c.initialize_free_surface_populations = env.flag("LBM_INIT_FREE_SURFACE_POPULATIONS", "0")
    c.vof_link_aperture_enabled = 1 if env.flag("LBM_VOF_LINK_APERTURE", "1") else 0
    c.vof_empty_fill_threshold = env.float("LBM_VOF_EMPTY_FILL_THRESHOLD", "0.0")
    if not (0.0 <= c.vof_empty_fill_threshold < 0.5):
        raise ValueError("LBM_VOF_EMPTY_FILL_THRESHOLD must be in [0, 0.5)")
    c.vof_orphan_empty_threshold = env.float("LBM_VOF_ORPHAN_EMPTY_THRESHOLD", "0.49")
    if not (0.0 <= c.vof_orphan_empty_threshold < 0.5):
        raise ValueError("LBM_VOF_ORPHAN_EMPTY_THRESHOLD must be in [0, 0.5)")
    c.vof_orphan_search_radius = env.int("LBM_VOF_ORPHAN_SEARCH_RADIUS", "4")
    if c.vof_orphan_search_radius < 1 or c.vof_orphan_search_radius > 4:
        raise ValueError("LBM_VOF_ORPHAN_SEARCH_RADIUS must be in [1, 4]")
    c.vof_orphan_max_weak_neighbors = env.int("LBM_VOF_ORPHAN_MAX_WEAK_NEIGHBORS", "1")
    if c.vof_orphan_max_weak_neighbors < 0 or c.vof_orphan_max_weak_neighbors > 18:
        raise ValueError("LBM_VOF_ORPHAN_MAX_WEAK_NEIGHBORS must be in [0, 18]")
    c.vof_detached_advection_enabled = env.flag("LBM_VOF_DETACHED_ADVECTION", "1")
    c.vof_detached_max_wet_neighbors = env.int("LBM_VOF_DETACHED_MAX_WET_NEIGHBORS", "18")
    if c.vof_detached_max_wet_neighbors < 0 or c.vof_detached_max_wet_neighbors > 18:
        raise ValueError("LBM_VOF_DETACHED_MAX_WET_NEIGHBORS must be in [0, 18]")
    c.vof_detached_max_resolved_neighbors = env.int("LBM_VOF_DETACHED_MAX_RESOLVED_NEIGHBORS", "0")
    if c.vof_detached_max_resolved_neighbors < 0 or c.vof_detached_max_resolved_neighbors > 18:
        raise ValueError("LBM_VOF_DETACHED_MAX_RESOLVED_NEIGHBORS must be in [0, 18]")
    c.vof_detached_residual_fill_threshold = env.float("LBM_VOF_DETACHED_RESIDUAL_FILL_THRESHOLD", "0.01")
    if not (0.0 <= c.vof_detached_residual_fill_threshold < 0.5):
        raise ValueError("LBM_VOF_DETACHED_RESIDUAL_FILL_THRESHOLD must be in [0, 0.5)")
    c.vof_thin_gap_bridge_enabled = env.flag("LBM_VOF_THIN_GAP_BRIDGE", "0")
    c.vof_thin_gap_bridge_strength = env.float("LBM_VOF_THIN_GAP_BRIDGE_STRENGTH", "1.0")
    if c.vof_thin_gap_bridge_strength < 0.0:
        raise ValueError("LBM_VOF_THIN_GAP_BRIDGE_STRENGTH must be nonnegative")
    c.vof_collapse_trapped_gas_enabled = env.flag("LBM_VOF_COLLAPSE_TRAPPED_GAS", "0")

    U_top_phys = 30.0 if physics_mode == "air" else 0.0
    U_top_phys = c.U_top_phys = env.float("LBM_U_TOP_MPS", U_top_phys)
    c.water_current_phys = env.float("LBM_WATER_CURRENT_MPS", 0.0 if physics_mode == "water" else U_top_phys)
    c.Lx_m = env.float("LBM_LX_M", 300.0)
    c.Ly_m = env.float("LBM_LY_M", 10.0)
    c.Lz_m = env.float("LBM_LZ_M", 20.0)
    dx = c.dx = env.float("LBM_DX_M", 0.5)
    c.nu_air = 1.516e-5
    c.rho_air_standard_phys = 1.2
    c.nu_water = env.float("LBM_WATER_NU_M2S", 1.004e-6)
    c.rho_water_phys = env.float("LBM_WATER_RHO_KGM3", 998.2)
    c.fluid_name = "water" if physics_mode == "water" else "air"
    c.nu_phys = c.nu_water if physics_mode == "water" else c.nu_air
    c.rho_phys = c.rho_water_phys if physics_mode == "water" else c.rho_air_standard_phys
    c.rho_air_phys = c.rho_phys
    c.gravity_phys = env.float("LBM_GRAVITY_MPS2", 9.81 if physics_mode == "water" else 0.0)

    Nx = c.Nx = int(c.Lx_m / dx)
    Ny = c.Ny = int(c.Ly_m / dx)
    Nz = c.Nz = int(c.Lz_m / dx)
    c.vof_collapse_interval = env.int("LBM_VOF_COLLAPSE_INTERVAL", 200)
    if c.vof_collapse_interval < 1:
        raise ValueError("LBM_VOF_COLLAPSE_INTERVAL must be positive")
    c.vof_collapse_max_volume_m3 = env.float("LBM_VOF_COLLAPSE_MAX_VOLUME_M3", "8.0")
    if c.vof_collapse_max_volume_m3 < 0.0:
        raise ValueError("LBM_VOF_COLLAPSE_MAX_VOLUME_M3 must be nonnegative")
    c.vof_collapse_flood_sweeps = env.int("LBM_VOF_COLLAPSE_FLOOD_SWEEPS", max(1, Nx + Ny + Nz))
    if c.vof_collapse_flood_sweeps < 1:
        raise ValueError("LBM_VOF_COLLAPSE_FLOOD_SWEEPS must be positive")

    c.steps = env.int("LBM_STEPS", 400000)
    c.plot_freq = env.int("LBM_PLOT_FREQ", 100)
    c.plot_step_start = env.int("LBM_PLOT_START", 0)
    bgm = str(env.get("LBM_BOUNDARY_GEOMETRY", "vertical")).lower()
    if bgm not in ("vertical", "phi_fraction", "phi"):
        raise ValueError("LBM_BOUNDARY_GEOMETRY must be 'vertical', 'phi_fraction', or 'phi'")
    c.boundary_geometry_mode = bgm
    c.use_phi_open_fraction = 1 if bgm in ("phi_fraction", "phi") else 0
    c.use_phi_open_flags = 1 if bgm == "phi" else 0
    default_xb = c.default_x_boundary_mode = "solid" if (physics_mode == "water" and fsi == "gaussian") else "periodic"
    c.x_boundary_mode = env.choice("LBM_X_BOUNDARY", default_xb, ("periodic", "solid"))
    c.wall_velocity_sampling = env.choice("LBM_WALL_VELOCITY_SAMPLING", "link", ("cell", "link"))
    c.use_link_wall_velocity = 1 if c.wall_velocity_sampling == "link" else 0

    bp = str(env.get("LBM_BED_PROFILE", "moving_sine" if physics_mode == "air" else "flat")).lower()
    if bp not in ("moving_sine", "flat", "piecewise_linear"):
        raise ValueError("LBM_BED_PROFILE must be 'moving_sine', 'flat', or 'piecewise_linear'")
    c.bed_profile = bp
    c.bed_is_moving = 1 if bp == "moving_sine" else 0
    c.bottom_file_path = str(env.get("LBM_BOTTOM_FILE", "bottom.txt"))
    c.bed_amp_m = env.float("LBM_BED_AMP_M", 1.5 if bp == "moving_sine" else 0.0)
    c.depth_swl_m = env.float("LBM_WATER_DEPTH_M", 10.0)
    g = c.gravity_phys
    c.wave_speed = float(np.sqrt(g * c.depth_swl_m) if g > 0.0 else np.sqrt(9.81 * c.depth_swl_m))
    c.bed_wavelength_m = env.float("LBM_BED_WAVELENGTH_M", 30.0)
    c.wave_period = c.bed_wavelength_m / max(c.wave_speed, 1e-12)
    offset_m = 2.0 * c.bed_amp_m + 3.0 * dx if bp == "moving_sine" else 0.0
    c.offset_m = env.float("LBM_BED_LEVEL_M", offset_m)
    c.U_wave_phys = c.wave_speed if c.bed_is_moving == 1 else 0.0

    if bp == "piecewise_linear":
        c.piecewise_bed_z_np, c.piecewise_bed_metadata = _load_piecewise_bed(c.bottom_file_path, Nx, dx, c.Lx_m)
    else:
        c.piecewise_bed_z_np = np.full(Nx, c.offset_m, dtype=np.float32)
        c.piecewise_bed_metadata = {
            "path": "", "point_count": 0, "first_x": 0.0, "last_x": c.Lx_m,
            "min_z": float(c.offset_m), "max_z": float(c.offset_m), "z_at_lx": float(c.offset_m),
        }

    c.free_surface_depth_m = env.float("LBM_FREE_SURFACE_DEPTH_M", c.depth_swl_m)
    c.free_surface_base_m = env.float("LBM_FREE_SURFACE_LEVEL_M", c.offset_m + c.free_surface_depth_m)
    if c.free_surface_depth_m <= 0.0:
        raise ValueError("LBM_FREE_SURFACE_DEPTH_M must be positive")
    ratio_env = c.solitary_height_depth_ratio_env = env.get("LBM_SOLITARY_HEIGHT_DEPTH_RATIO", None)
    if ratio_env is not None:
        c.solitary_height_depth_ratio = float(ratio_env)
        if c.solitary_height_depth_ratio <= 0.0:
            raise ValueError("LBM_SOLITARY_HEIGHT_DEPTH_RATIO must be positive")
        c.solitary_amp_m = c.solitary_height_depth_ratio * c.free_surface_depth_m
    else:
        c.solitary_amp_m = env.float("LBM_SOLITARY_AMPLITUDE_M", 0.5)
        if c.solitary_amp_m <= 0.0:
            raise ValueError("LBM_SOLITARY_AMPLITUDE_M must be positive")
        c.solitary_height_depth_ratio = c.solitary_amp_m / c.free_surface_depth_m
    c.solitary_x0_m = env.float("LBM_SOLITARY_X0_M", 0.25 * c.Lx_m)
    sd = env.float("LBM_SOLITARY_DIRECTION", 1.0)
    if sd == 0.0:
        raise ValueError("LBM_SOLITARY_DIRECTION must be nonzero")
    c.solitary_direction = 1.0 if sd > 0.0 else -1.0
    siv = str(env.get("LBM_SOLITARY_INITIAL_VELOCITY", "shallow_water_divfree")).lower()
    if siv not in ("none", "shallow_water", "shallow_water_divfree"):
        raise ValueError(
            "LBM_SOLITARY_INITIAL_VELOCITY must be 'none', 'shallow_water', "
            "or 'shallow_water_divfree'"
        )
    c.solitary_initial_velocity_mode = siv
    h = c.free_surface_depth_m
    c.solitary_celerity_phys = float(np.sqrt(g * (h + c.solitary_amp_m))) if g > 0.0 else 0.0
    c.solitary_kappa_m_inv = float(np.sqrt(3.0 * c.solitary_amp_m / (4.0 * h ** 3)))
    c.solitary_length_scale_m = 1.0 / c.solitary_kappa_m_inv
    c.gaussian_amp_m = env.float("LBM_GAUSSIAN_AMPLITUDE_M", 3.0)
    c.gaussian_center_x_m = env.float("LBM_GAUSSIAN_CENTER_X_M", 0.5 * c.Lx_m)
    c.gaussian_sigma_m = env.float("LBM_GAUSSIAN_SIGMA_M", 12.5)
    c.gaussian_celerity_phys = float(np.sqrt(g * (h + c.gaussian_amp_m))) if g > 0.0 else 0.0
    c.vof_block_size_m = env.float("LBM_VOF_BLOCK_SIZE_M", 4.0)
    c.vof_block_size_x_m = env.float("LBM_VOF_BLOCK_SIZE_X_M", c.vof_block_size_m)
    c.vof_block_size_y_m = env.float("LBM_VOF_BLOCK_SIZE_Y_M", min(c.vof_block_size_m, c.Ly_m))
    c.vof_block_size_z_m = env.float("LBM_VOF_BLOCK_SIZE_Z_M", c.vof_block_size_m)
    c.vof_block_center_x_m = env.float("LBM_VOF_BLOCK_CENTER_X_M", 0.5 * c.Lx_m)
    c.vof_block_center_y_m = env.float("LBM_VOF_BLOCK_CENTER_Y_M", 0.5 * c.Ly_m)
    bottom_default = c.vof_block_bottom_default_m = min(c.Lz_m - c.vof_block_size_z_m - dx,
                                                        c.free_surface_base_m + 2.0 * dx)
    c.vof_block_bottom_m = env.float("LBM_VOF_BLOCK_BOTTOM_M", bottom_default)
    c.vof_block_center_z_m = env.float("LBM_VOF_BLOCK_CENTER_Z_M", c.vof_block_bottom_m + 0.5 * c.vof_block_size_z_m)
    if vis != "none" and fst != "vof":
        raise ValueError("LBM_VOF_INITIAL_SHAPE requires LBM_FREE_SURFACE_TRACKING=vof")
    c.vof_has_disconnected_feature = vis != "none"
    c.allow_total_pressure_vof = env.flag("LBM_ALLOW_TOTAL_PRESSURE_VOF_DIAGNOSTIC", "0")
    if c.vof_has_disconnected_feature and c.pressure_formulation == "total_pressure" and not c.allow_total_pressure_vof:
        c.pressure_formulation = "vof_component_balanced"
        c.pressure_formulation_auto_corrected = True
    if c.vof_has_disconnected_feature and c.pressure_formulation == "hydrostatic_balanced":
        raise ValueError(
            "Disconnected VOF features with LBM_PRESSURE_FORMULATION=hydrostatic_balanced are not supported; "
            "use vof_component_balanced so the flat pool is balanced while detached water still falls."
        )
    if c.vof_has_disconnected_feature and fsb == "hydrostatic":
        raise ValueError(
            "Disconnected VOF features require LBM_FREE_SURFACE_BOUNDARY=cell; "
            "the hydrostatic option still uses a column-height surface."
        )
    c.vof_block_drop_height_m = max(c.vof_block_center_z_m - c.free_surface_base_m, 0.0)
    c.vof_reference_speed_phys = (
        float(np.sqrt(2.0 * g * c.vof_block_drop_height_m)) if (g > 0.0 and vis != "none") else 0.0
    )

    om = str(env.get("LBM_OBSTACLE_MODE", "bed")).lower()
    if om not in ("bed", "bed_cube", "cube"):
        raise ValueError("LBM_OBSTACLE_MODE must be 'bed', 'bed_cube', or 'cube'")
    c.obstacle_mode = om
    c.include_bed_geometry = 1 if om in ("bed", "bed_cube") else 0
    c.include_cube_geometry = 1 if om in ("bed_cube", "cube") else 0
    c.cube_side_m = env.float("LBM_CUBE_SIDE_M", 6.0)
    c.cube_size_x_m = env.float("LBM_CUBE_SIZE_X_M", c.cube_side_m)
    c.cube_size_y_m = env.float("LBM_CUBE_SIZE_Y_M", c.cube_side_m)
    c.cube_size_z_m = env.float("LBM_CUBE_SIZE_Z_M", c.cube_side_m)
    if c.cube_size_x_m <= 0.0 or c.cube_size_y_m <= 0.0 or c.cube_size_z_m <= 0.0:
        raise ValueError("LBM_CUBE_SIZE_X_M, LBM_CUBE_SIZE_Y_M, and LBM_CUBE_SIZE_Z_M must be positive")
    c.cube_half_x_m = 0.5 * c.cube_size_x_m
    c.cube_half_y_m = 0.5 * c.cube_size_y_m
    c.cube_half_z_m = 0.5 * c.cube_size_z_m
    c.cube_center_x_m = env.float("LBM_CUBE_CENTER_X_M", 0.5 * c.Lx_m)
    c.cube_center_y_m = env.float("LBM_CUBE_CENTER_Y_M", 0.5 * c.Ly_m)
    c.cube_yaw_deg = env.float("LBM_CUBE_YAW_DEG", 0.0)
    yaw = c.cube_yaw_rad = float(np.deg2rad(c.cube_yaw_deg))
    c.cube_yaw_cos, c.cube_yaw_sin = float(np.cos(yaw)), float(np.sin(yaw))
    c.cube_pitch_deg = env.float("LBM_CUBE_PITCH_DEG", 0.0)
    pitch = c.cube_pitch_rad = float(np.deg2rad(c.cube_pitch_deg))
    c.cube_pitch_cos, c.cube_pitch_sin = float(np.cos(pitch)), float(np.sin(pitch))
    c.cube_vertical_half_extent_m = c.cube_half_z_m * abs(c.cube_pitch_cos) + c.cube_half_x_m * abs(c.cube_pitch_sin)
    cz_default = c.cube_center_z_default = min(
        c.Lz_m - c.cube_vertical_half_extent_m - dx,
        max(0.5 * c.Lz_m, c.offset_m + 2.0 * c.bed_amp_m + c.cube_vertical_half_extent_m + dx),
    )
    c.cube_center_z_m = env.float("LBM_CUBE_CENTER_Z_M", cz_default)

    c.WALL_NONE, c.WALL_BED, c.WALL_CUBE, c.WALL_XMIN, c.WALL_XMAX = 0, 1, 2, 3, 4
    c.FS_GAS, c.FS_LIQUID, c.FS_INTERFACE = FS_GAS, FS_LIQUID, FS_INTERFACE
    c.rho0 = 1.0
    c.u_lid = 0.075
    c.U_ref_phys = max(
        abs(U_top_phys), abs(c.U_wave_phys), abs(c.water_current_phys), abs(c.solitary_celerity_phys),
        abs(c.gaussian_celerity_phys), abs(c.vof_reference_speed_phys), 1e-6,
    )
    c.vel_scale = c.U_ref_phys / c.u_lid
    c.dt_phys = c.u_lid * dx / c.U_ref_phys

    # ---- build extension: lattice units (dt = 1, velocity scale = 1) ----
    c.lattice_units = env.flag("LBM_B200_LATTICE_UNITS", "0")
    if c.lattice_units:
        c.vel_scale = 1.0
        c.dt_phys = 1.0

    c.u_top_lb = U_top_phys / c.vel_scale
    c.u_bed_lb = c.wave_speed / c.vel_scale
    c.u_current_lb = c.water_current_phys / c.vel_scale
    c.g_lb = g * c.dt_phys * c.dt_phys / dx
    if env.get("LBM_B200_G_LB", None) is not None:
        c.g_lb = env.float("LBM_B200_G_LB", 0.0)
    c.use_component_balanced_pressure = 1 if (
        c.water_free_surface_enabled == 1 and c.pressure_formulation == "vof_component_balanced") else 0
    c.use_hydrostatic_balanced_pressure = 1 if (
        c.water_free_surface_enabled == 1
        and c.pressure_formulation in ("hydrostatic_balanced", "vof_component_balanced")) else 0
    c.g_body_lb = 0.0 if (c.water_free_surface_enabled == 1 and c.pressure_formulation == "hydrostatic_balanced") else c.g_lb

    c.Re_phys_air = c.U_ref_phys * c.Lz_m / c.nu_phys
    c.Re_phys = c.Re_phys_air
    c.nu0 = c.u_lid * Nz / c.Re_phys_air
    c.tau0 = 0.5 + 3 * c.nu0
    if env.get("LBM_B200_TAU0", None) is not None:
        c.tau0 = env.float("LBM_B200_TAU0", 0.0)
        if not c.tau0 > 0.5:
            raise ValueError("LBM_B200_TAU0 must be greater than 0.5")
        c.nu0 = (c.tau0 - 0.5) / 3.0
    c.Re_lb_base = c.u_lid * Nz / c.nu0 if c.nu0 > 0 else float("inf")

    c.use_LES = env.flag("LBM_USE_LES", "1" if physics_mode == "air" else "0")
    col = str(env.get("LBM_COLLISION", "regularized" if physics_mode == "water" else "kbc")).lower()
    if col not in ("kbc", "regularized"):
        raise ValueError("LBM_COLLISION must be 'kbc' or 'regularized'")
    c.collision_model = col
    c.Cs = 0.2
    if env.get("LBM_B200_CS", None) is not None:
        c.Cs = env.float("LBM_B200_CS", 0.2)
    c.Delta = 1.0
    c.nu_t_max = 10.0
    c.TI = 0.1
    c.Correlation = 0.0
    c.kappa = 0.41
    c.z0_phys = 0.01
    c.C_backscatter = env.float("LBM_BACKSCATTER", 0.02 if physics_mode == "air" else 0.0)
    c.enable_top_drive = 1 if (physics_mode == "air" and str(env.get("LBM_ENABLE_TOP_DRIVE", "1")) != "0") else 0
    c.enable_x_fringe = 1 if (
        physics_mode == "air" and c.x_boundary_mode == "periodic" and str(env.get("LBM_ENABLE_X_FRINGE", "1")) != "0") else 0
    c.enable_top_sponge = 1 if (physics_mode == "air" and str(env.get("LBM_ENABLE_TOP_SPONGE", "1")) != "0") else 0

    # ---- remaining build extensions ----
    bm = env.choice("LBM_B200_BED_MODEL", "reference", ("reference", "single_sine"))
    c.bed_model = bm
    c.bed_speed = env.float("LBM_B200_BED_SPEED", c.wave_speed)
    c.bed_ramp = env.flag("LBM_B200_BED_RAMP", "1" if bm == "reference" else "0")
    c.bed_orbital = env.flag("LBM_B200_BED_ORBITAL", "1" if bm == "reference" else "0")
    c.top_mode = env.choice("LBM_B200_TOP", "reference", ("reference", "free_slip"))
    c.init_velocity = env.choice("LBM_B200_INIT_VELOCITY", "reference", ("reference", "uniform"))
    u0 = [float(v) for v in str(env.get("LBM_B200_INIT_U0", "0,0,0")).split(",")]
    if len(u0) != 3:
        raise ValueError("LBM_B200_INIT_U0 must be three comma-separated numbers")
    c.init_u0 = tuple(u0)
    c.init_noise_amp = env.float("LBM_B200_INIT_NOISE", 0.0)
    c.pop_storage = env.choice("LBM_B200_POP_STORAGE", "f32", ("f32", "f16s", "bf16s"))
    c.random_seed = env.int("LBM_RANDOM_SEED", 12345)
    if c.top_mode == "free_slip" and (c.enable_top_drive or physics_mode != "air"):
        raise ValueError("LBM_B200_TOP=free_slip requires LBM_PHYSICS_MODE=air and LBM_ENABLE_TOP_DRIVE=0")
    return c


# ---------------------------------------------------------------------------
# benchmark configurations (lattice-unit restatements of the five workloads)
# ---------------------------------------------------------------------------

def air_wave_env(nx: int, ny: int, nz: int, *, storage: str = "f32", seed: int = 12345,
                 amp: float = 4.0, level: float = 8.0, wavelength: float = 64.0, speed: float = 0.02,
                 inflow: float = 0.05, tau0: float = 0.52, cs: float = 0.16) -> dict:
    """Air over a moving sinusoidal bed in lattice units: regularized
    collision, Smagorinsky LES, periodic x/y, free-slip top, bed
    z = level + amp sin(2 pi (x - speed t)/wavelength), u0 = (inflow,0,0)
    plus uniform noise of 1e-3 per component."""
    return {
        "LBM_PHYSICS_MODE": "air", "LBM_DX_M": "1", "LBM_LX_M": str(nx), "LBM_LY_M": str(ny), "LBM_LZ_M": str(nz),
        "LBM_COLLISION": "regularized", "LBM_USE_LES": "1", "LBM_BACKSCATTER": "0",
        "LBM_ENABLE_X_FRINGE": "0", "LBM_ENABLE_TOP_DRIVE": "0", "LBM_ENABLE_TOP_SPONGE": "0",
        "LBM_BED_PROFILE": "moving_sine", "LBM_BED_LEVEL_M": repr(level), "LBM_BED_AMP_M": repr(amp),
        "LBM_BED_WAVELENGTH_M": repr(wavelength), "LBM_B200_BED_MODEL": "single_sine",
        "LBM_B200_BED_SPEED": repr(speed), "LBM_B200_BED_RAMP": "0", "LBM_B200_BED_ORBITAL": "0",
        "LBM_B200_LATTICE_UNITS": "1", "LBM_B200_TAU0": repr(tau0), "LBM_B200_CS": repr(cs),
        "LBM_B200_TOP": "free_slip", "LBM_B200_INIT_VELOCITY": "uniform",
        "LBM_B200_INIT_U0": f"{inflow!r},0,0", "LBM_B200_INIT_NOISE": "1e-3",
        "LBM_B200_POP_STORAGE": storage, "LBM_RANDOM_SEED": str(seed),
    }


def water_gaussian_env(nx: int, ny: int, nz: int, *, storage: str = "f32", depth: float = 48.0,
                       amp: float = 8.0, sigma: float = 16.0, g_lb: float = 1e-5, tau0: float = 0.51) -> dict:
    """Water free surface, height-function kinematic path: hydrostatic
    balanced pressure, cell boundary, solid x walls, flat pool with a
    Gaussian ridge at the domain centre (the reference's Gaussian is
    uniform in y, CODEX.py:1184-1194), lattice units."""
    return {
        "LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_INITIAL": "gaussian", "LBM_X_BOUNDARY": "solid",
        "LBM_DX_M": "1", "LBM_LX_M": str(nx), "LBM_LY_M": str(ny), "LBM_LZ_M": str(nz),
        "LBM_WATER_DEPTH_M": repr(depth), "LBM_GAUSSIAN_AMPLITUDE_M": repr(amp),
        "LBM_GAUSSIAN_SIGMA_M": repr(sigma), "LBM_PRESSURE_FORMULATION": "hydrostatic_balanced",
        "LBM_FREE_SURFACE_BOUNDARY": "cell", "LBM_B200_LATTICE_UNITS": "1", "LBM_B200_G_LB": repr(g_lb),
        "LBM_B200_TAU0": repr(tau0), "LBM_B200_POP_STORAGE": storage,
    }


def vof_block_env(nx: int, ny: int, nz: int, *, storage: str = "f16s", depth: float = 64.0,
                  block: float = 32.0, bottom: float = 96.0, g_lb: float | None = None) -> dict:
    """VOF falling block with KBC collision, component-balanced pressure,
    trapped-gas collapse every 200 steps (max 512 cells), thin-gap bridge
    strength 4, solid x walls."""
    env = {
        "LBM_PHYSICS_MODE": "water", "LBM_FREE_SURFACE_TRACKING": "vof", "LBM_FREE_SURFACE_INITIAL": "gaussian",
        "LBM_X_BOUNDARY": "solid", "LBM_COLLISION": "kbc", "LBM_VOF_INITIAL_SHAPE": "block",
        "LBM_GAUSSIAN_AMPLITUDE_M": "0", "LBM_WATER_DEPTH_M": repr(depth), "LBM_VOF_BLOCK_SIZE_M": repr(block),
        "LBM_VOF_BLOCK_BOTTOM_M": repr(bottom), "LBM_PRESSURE_FORMULATION": "vof_component_balanced",
        "LBM_VOF_COLLAPSE_TRAPPED_GAS": "1", "LBM_VOF_COLLAPSE_INTERVAL": "200",
        "LBM_VOF_COLLAPSE_MAX_VOLUME_M3": "512", "LBM_VOF_THIN_GAP_BRIDGE": "1",
        "LBM_VOF_THIN_GAP_BRIDGE_STRENGTH": "4", "LBM_DX_M": "1", "LBM_LX_M": str(nx), "LBM_LY_M": str(ny),
        "LBM_LZ_M": str(nz), "LBM_B200_POP_STORAGE": storage,
    }
    if g_lb is not None:
        env["LBM_B200_G_LB"] = repr(g_lb)
    return env
