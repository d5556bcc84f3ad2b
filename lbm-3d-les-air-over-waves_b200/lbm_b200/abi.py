"""ctypes mirror of include/lbm_b200.h and the params builder.

Both the CUDA library (lbm_b200/_native/liblbm_b200.so) and the CPU oracle
export the same ABI; this module describes the structs once and loads
either library.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LBM_ABI_VERSION = 1
LBM_PARAMS_MAGIC = 0x1B200D19

LBM_OK = 0
LBM_ERR_BAD_ARG = -1
LBM_ERR_CUDA = -2
LBM_ERR_NOT_CONVERGED = -3
LBM_ERR_NONFINITE = -4
LBM_ERR_UNSUPPORTED = -5
LBM_ERR_NOT_BOUND = -6
LBM_ARITH_EXACT = 0
LBM_ARITH_FAST = 1
ERRORS = {
    -1: "bad argument", -2: "CUDA error", -3: "not converged", -4: "non-finite value",
    -5: "unsupported configuration", -6: "buffers not bound",
}

_I = C.c_int32
_F = C.c_float

PARAM_FIELDS = [
    ("abi_version", _I), ("nx", _I), ("ny", _I), ("nz", _I),
    ("physics_water", _I), ("fs_mode", _I), ("fs_tracking", _I), ("fs_boundary", _I), ("fs_refill", _I),
    ("fs_initial", _I), ("init_fs_populations", _I), ("vof_link_aperture", _I), ("vof_initial_block", _I),
    ("pressure_formulation", _I), ("use_hydrostatic_balanced_pressure", _I), ("use_component_balanced_pressure", _I),
    ("x_solid", _I), ("use_phi_open_fraction", _I), ("use_phi_open_flags", _I), ("use_link_wall_velocity", _I),
    ("bed_profile", _I), ("include_bed", _I), ("include_cube", _I), ("use_les", _I), ("collision", _I),
    ("enable_top_drive", _I), ("enable_x_fringe", _I), ("enable_top_sponge", _I), ("solitary_velocity_mode", _I),
    ("top_free_slip", _I), ("init_velocity_mode", _I), ("bed_orbital_velocity", _I), ("pop_storage", _I),
    ("vof_orphan_search_radius", _I), ("vof_orphan_max_weak_neighbors", _I), ("vof_detached_advection", _I),
    ("vof_detached_max_wet_neighbors", _I), ("vof_detached_max_resolved_neighbors", _I),
    ("vof_thin_gap_bridge", _I), ("vof_collapse_enabled", _I), ("vof_collapse_interval", _I),
    ("vof_collapse_flood_sweeps", _I), ("pad0", _I),
    ("seed", C.c_uint64),
    ("dx", _F), ("rho0", _F), ("tau0", _F), ("nu0", _F), ("cs_delta_sq", _F), ("nu_t_max", _F), ("kappa", _F),
    ("z0_phys", _F), ("wall_dist_floor", _F), ("ti_kick", _F), ("c_backscatter", _F), ("u_top_lb", _F),
    ("u_current_lb", _F), ("g_lb", _F), ("g_body_lb", _F), ("vel_scale", _F), ("dt_phys_f", _F),
    ("dt_phys", C.c_double),
    ("bed_offset_m", _F), ("bed_amp1", _F), ("bed_k1", _F), ("bed_c1", _F), ("bed_amp2", _F), ("bed_k2", _F),
    ("bed_c2", _F), ("bed_ramp_time", _F), ("bed_h0", _F),
    ("cube_cx", _F), ("cube_cy", _F), ("cube_cz", _F), ("cube_hx", _F), ("cube_hy", _F), ("cube_hz", _F),
    ("cube_yaw_cos", _F), ("cube_yaw_sin", _F), ("cube_pitch_cos", _F), ("cube_pitch_sin", _F),
    ("fs_base_m", _F), ("fs_depth_m", _F), ("solitary_amp_m", _F), ("solitary_x0_m", _F),
    ("solitary_direction", _F), ("solitary_celerity", _F), ("solitary_kappa_inv", _F),
    ("gaussian_amp_m", _F), ("gaussian_center_x_m", _F), ("gaussian_sigma_m", _F),
    ("vof_block_xmin", _F), ("vof_block_xmax", _F), ("vof_block_ymin", _F), ("vof_block_ymax", _F),
    ("vof_block_zmin", _F), ("vof_block_zmax", _F),
    ("vof_empty_fill_threshold", _F), ("vof_orphan_empty_threshold", _F),
    ("vof_detached_residual_fill_threshold", _F), ("vof_thin_gap_bridge_strength", _F),
    ("vof_collapse_max_volume_m3", _F),
    ("init_u0x", _F), ("init_u0y", _F), ("init_u0z", _F), ("init_noise_amp", _F),
    ("omega0", _F), ("half_inv_dx", _F), ("solitary_dir_cel", _F), ("nu_lbm_init", _F), ("u_tau_init", _F),
    ("inv_kappa", _F), ("one_third", _F), ("magic_end", _I),
]


class LbmDiagInputs(C.Structure):
    _fields_ = [("rho_phys", C.c_double), ("gravity_phys", C.c_double), ("slice_j", C.c_int32), ("pad", C.c_int32)]


_D, _I64 = C.c_double, C.c_int64
DIAG_FIELDS = [
    ("max_speed_lb", _D), ("max_speed_phys", _D), ("max_speed_x", _D), ("max_speed_y", _D), ("max_speed_z", _D),
    ("max_k", _I), ("max_j", _I), ("max_i", _I), ("max_speed_fs_type", _I), ("max_speed_fs_fill", _D),
    ("max_speed_wet_neighbors", _I), ("max_speed_full_neighbors", _I), ("max_speed_gas_neighbors", _I),
    ("pad0", _I), ("active_cells", _I64),
    ("water_volume", _D), ("vof_mass_total", _D), ("vof_min_interface_fill", _D),
    ("vof_tiny_interface_count", _I64), ("vof_pending_excess_mass", _D), ("vof_pending_excess_count", _I64),
    ("surface_min", _D), ("surface_max", _D), ("surface_symmetry_l2", _D), ("surface_eta_hp_rms", _D),
    ("surface_left_max", _D), ("surface_right_max", _D),
    ("p_rms", _D), ("p_hp_rms", _D), ("p_total_rms", _D), ("p_total_hp_rms", _D), ("vort_rms", _D),
    ("vort_hp_rms", _D), ("fs_p_rms", _D), ("fs_p_hp_rms", _D), ("fs_p_total_rms", _D), ("fs_p_total_hp_rms", _D),
    ("fs_vort_rms", _D), ("fs_vort_hp_rms", _D), ("band_cells", _I64), ("fs_band_cells", _I64),
]


class LbmDiag(C.Structure):
    """lbm_diag: the harness metrics reduced on the device."""
    _fields_ = DIAG_FIELDS

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("pad")}


class LbmParams(C.Structure):
    _fields_ = PARAM_FIELDS


_P = C.c_void_p
BUFFER_FIELDS = [
    ("f0", _P), ("f1", _P), ("rho", _P), ("ux", _P), ("uy", _P), ("uz", _P), ("omega", _P),
    ("water_h", _P), ("water_h_last", _P), ("u_wave", _P), ("v_wave", _P), ("w_wave", _P),
    ("fs_h", _P), ("fs_h_last", _P), ("fs_flux_x", _P), ("fs_flux_y", _P), ("piecewise_bed_z", _P),
    ("u_inlet_profile", _P), ("rho_initial", _P), ("init_noise", _P),
    ("fs_fill", _P), ("fs_type", _P), ("fs_type_prev", _P), ("fs_mass", _P), ("fs_mass_excess", _P),
    ("fs_excess_dir", _P),
    ("phi", _P), ("obstacle", _P), ("near_obstacle", _P), ("lattice_open", _P), ("lattice_open_frac", _P),
    ("lattice_wall_type", _P), ("pressure_reference_head", _P), ("gravity_body_fraction", _P),
    ("vof_exterior_gas", _P),
]


class LbmBuffers(C.Structure):
    _fields_ = BUFFER_FIELDS


COUNTER_INT_NAMES = [
    "boundary_refill_count", "free_surface_refill_count", "free_surface_coalescence_repair_count",
    "free_surface_thin_gap_bridge_count", "free_surface_cut_link_count", "free_surface_vof_excess_count",
    "free_surface_vof_orphan_count", "free_surface_vof_collapse_cell_count",
    "free_surface_vof_detached_advect_count", "free_surface_vof_detached_compress_count",
    "boundary_cut_link_count", "status_flags",
]
COUNTER_FLOAT_NAMES = [
    "free_surface_vof_collapse_candidate_volume_m3", "free_surface_vof_collapse_applied_volume_m3",
    "free_surface_vof_collapse_removal_scale", "free_surface_vof_collapse_candidate_mass",
    "free_surface_vof_collapse_exterior_capacity", "free_surface_vof_detached_advect_mass",
    "free_surface_vof_detached_compress_mass",
]


class LbmCounters(C.Structure):
    _fields_ = (
        [(n, _I) for n in COUNTER_INT_NAMES]
        + [(n, _F) for n in COUNTER_FLOAT_NAMES]
        + [("pad", _F), ("step", C.c_int64), ("current_f", _I), ("flood_sweeps_used", _I)]
    )

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


def f32(x) -> float:
    """Round a Python float to the nearest f32 (how Taichi captures constants)."""
    return float(np.float32(x))


def make_params(cfg) -> LbmParams:
    """Fill lbm_params from a SolverConfig (see config.load_config)."""
    p = LbmParams()
    p.abi_version = LBM_ABI_VERSION
    p.magic_end = LBM_PARAMS_MAGIC
    p.nx, p.ny, p.nz = cfg.Nx, cfg.Ny, cfg.Nz
    p.physics_water = 1 if cfg.physics_mode == "water" else 0
    p.fs_mode = {"none": 0, "height_static": 1, "height_kinematic": 2, "prescribed_solitary": 3}[cfg.free_surface_mode]
    p.fs_tracking = 1 if cfg.free_surface_tracking_mode == "vof" else 0
    p.fs_boundary = 1 if cfg.free_surface_boundary_mode == "hydrostatic" else 0
    p.fs_refill = {"equilibrium": 0, "noneq": 1, "directional": 2}[cfg.free_surface_refill_mode]
    p.fs_initial = {"flat": 0, "solitary": 1, "gaussian": 2}[cfg.free_surface_initial_condition]
    p.init_fs_populations = int(bool(cfg.initialize_free_surface_populations))
    p.vof_link_aperture = int(cfg.vof_link_aperture_enabled)
    p.vof_initial_block = 1 if cfg.vof_initial_shape == "block" else 0
    p.pressure_formulation = {"total_pressure": 0, "hydrostatic_balanced": 1, "vof_component_balanced": 2}[
        cfg.pressure_formulation]
    p.use_hydrostatic_balanced_pressure = cfg.use_hydrostatic_balanced_pressure
    p.use_component_balanced_pressure = cfg.use_component_balanced_pressure
    p.x_solid = 1 if cfg.x_boundary_mode == "solid" else 0
    p.use_phi_open_fraction = cfg.use_phi_open_fraction
    p.use_phi_open_flags = cfg.use_phi_open_flags
    p.use_link_wall_velocity = cfg.use_link_wall_velocity
    p.bed_profile = {"moving_sine": 0, "flat": 1, "piecewise_linear": 2}[cfg.bed_profile]
    p.include_bed = cfg.include_bed_geometry
    p.include_cube = cfg.include_cube_geometry
    p.use_les = int(bool(cfg.use_LES))
    p.collision = 1 if cfg.collision_model == "regularized" else 0
    p.enable_top_drive = cfg.enable_top_drive
    p.enable_x_fringe = cfg.enable_x_fringe
    p.enable_top_sponge = cfg.enable_top_sponge
    p.solitary_velocity_mode = {"none": 0, "shallow_water": 1, "shallow_water_divfree": 2}[
        cfg.solitary_initial_velocity_mode]
    p.top_free_slip = 1 if cfg.top_mode == "free_slip" else 0
    p.init_velocity_mode = 1 if cfg.init_velocity == "uniform" else 0
    p.bed_orbital_velocity = int(bool(cfg.bed_orbital))
    p.pop_storage = {"f32": 0, "f16s": 1, "bf16s": 2}[cfg.pop_storage]
    p.vof_orphan_search_radius = cfg.vof_orphan_search_radius
    p.vof_orphan_max_weak_neighbors = cfg.vof_orphan_max_weak_neighbors
    p.vof_detached_advection = int(bool(cfg.vof_detached_advection_enabled))
    p.vof_detached_max_wet_neighbors = cfg.vof_detached_max_wet_neighbors
    p.vof_detached_max_resolved_neighbors = cfg.vof_detached_max_resolved_neighbors
    p.vof_thin_gap_bridge = int(bool(cfg.vof_thin_gap_bridge_enabled))
    p.vof_collapse_enabled = int(bool(cfg.vof_collapse_trapped_gas_enabled))
    p.vof_collapse_interval = cfg.vof_collapse_interval
    p.vof_collapse_flood_sweeps = cfg.vof_collapse_flood_sweeps
    p.seed = cfg.random_seed & 0xFFFFFFFFFFFFFFFF

    dx = cfg.dx
    p.dx = f32(dx)
    p.rho0 = f32(cfg.rho0)
    p.tau0 = f32(cfg.tau0)
    p.nu0 = f32(cfg.nu0)
    p.cs_delta_sq = f32((cfg.Cs * cfg.Delta) ** 2)
    p.nu_t_max = f32(cfg.nu_t_max)
    p.kappa = f32(cfg.kappa)
    p.z0_phys = f32(cfg.z0_phys)
    p.wall_dist_floor = f32(0.001 * dx)
    p.ti_kick = f32(cfg.TI)
    p.c_backscatter = f32(cfg.C_backscatter)
    p.u_top_lb = f32(cfg.u_top_lb)
    p.u_current_lb = f32(cfg.u_current_lb)
    p.g_lb = f32(cfg.g_lb)
    p.g_body_lb = f32(cfg.g_body_lb)
    p.vel_scale = f32(cfg.vel_scale)
    p.dt_phys_f = f32(cfg.dt_phys)
    p.dt_phys = float(cfg.dt_phys)

    # bed kinematics (CODEX.py:1107-1160); the reference's harmonics are
    # (amp, k/2, c) and (amp, k, c/2) with k = 2 pi / wavelength
    k = 2.0 * 3.141592653589793 / cfg.bed_wavelength_m
    p.bed_offset_m = f32(cfg.offset_m)
    p.bed_h0 = f32(cfg.depth_swl_m)
    if cfg.bed_model == "single_sine":
        p.bed_amp1, p.bed_k1, p.bed_c1 = f32(cfg.bed_amp_m), f32(k), f32(cfg.bed_speed)
        p.bed_amp2, p.bed_k2, p.bed_c2 = 0.0, 0.0, 0.0
    else:
        c = f32(cfg.wave_speed)
        p.bed_amp1, p.bed_k1, p.bed_c1 = f32(cfg.bed_amp_m), 0.5 * f32(k), c
        p.bed_amp2, p.bed_k2, p.bed_c2 = f32(cfg.bed_amp_m), f32(k), 0.5 * c
    p.bed_ramp_time = f32(2.0 * cfg.wave_period) if cfg.bed_ramp else 0.0

    p.cube_cx, p.cube_cy, p.cube_cz = f32(cfg.cube_center_x_m), f32(cfg.cube_center_y_m), f32(cfg.cube_center_z_m)
    p.cube_hx, p.cube_hy, p.cube_hz = f32(cfg.cube_half_x_m), f32(cfg.cube_half_y_m), f32(cfg.cube_half_z_m)
    p.cube_yaw_cos, p.cube_yaw_sin = f32(cfg.cube_yaw_cos), f32(cfg.cube_yaw_sin)
    p.cube_pitch_cos, p.cube_pitch_sin = f32(cfg.cube_pitch_cos), f32(cfg.cube_pitch_sin)

    p.fs_base_m = f32(cfg.free_surface_base_m)
    p.fs_depth_m = f32(cfg.free_surface_depth_m)
    p.solitary_amp_m = f32(cfg.solitary_amp_m)
    p.solitary_x0_m = f32(cfg.solitary_x0_m)
    p.solitary_direction = f32(cfg.solitary_direction)
    p.solitary_celerity = f32(cfg.solitary_celerity_phys)
    p.solitary_kappa_inv = f32(cfg.solitary_kappa_m_inv)
    p.solitary_dir_cel = f32(cfg.solitary_direction * cfg.solitary_celerity_phys)
    p.gaussian_amp_m = f32(cfg.gaussian_amp_m)
    p.gaussian_center_x_m = f32(cfg.gaussian_center_x_m)
    p.gaussian_sigma_m = f32(cfg.gaussian_sigma_m)
    p.vof_block_xmin = f32(cfg.vof_block_center_x_m - 0.5 * cfg.vof_block_size_x_m)
    p.vof_block_xmax = f32(cfg.vof_block_center_x_m + 0.5 * cfg.vof_block_size_x_m)
    p.vof_block_ymin = f32(cfg.vof_block_center_y_m - 0.5 * cfg.vof_block_size_y_m)
    p.vof_block_ymax = f32(cfg.vof_block_center_y_m + 0.5 * cfg.vof_block_size_y_m)
    p.vof_block_zmin = f32(cfg.vof_block_center_z_m - 0.5 * cfg.vof_block_size_z_m)
    p.vof_block_zmax = f32(cfg.vof_block_center_z_m + 0.5 * cfg.vof_block_size_z_m)
    p.vof_empty_fill_threshold = f32(cfg.vof_empty_fill_threshold)
    p.vof_orphan_empty_threshold = f32(cfg.vof_orphan_empty_threshold)
    p.vof_detached_residual_fill_threshold = f32(cfg.vof_detached_residual_fill_threshold)
    p.vof_thin_gap_bridge_strength = f32(cfg.vof_thin_gap_bridge_strength)
    p.vof_collapse_max_volume_m3 = f32(cfg.vof_collapse_max_volume_m3)
    p.init_u0x, p.init_u0y, p.init_u0z = (f32(v) for v in cfg.init_u0)
    p.init_noise_amp = f32(cfg.init_noise_amp)

    p.omega0 = f32(1.0 / cfg.tau0)
    p.half_inv_dx = f32(0.5 / dx)
    p.nu_lbm_init = f32((cfg.tau0 - 0.5) / 3.0)
    p.u_tau_init = f32(0.1 * cfg.u_top_lb)
    p.inv_kappa = f32(1.0 / cfg.kappa)
    p.one_third = f32(1.0 / 3.0)
    return p


def declare(lib: C.CDLL) -> C.CDLL:
    """Attach argtypes/restype to the ABI entry points of a loaded library."""
    vp = C.c_void_p
    lib.lbm_backend_name.restype = C.c_char_p
    lib.lbm_backend_name.argtypes = []
    lib.lbm_abi_version.restype = C.c_int
    lib.lbm_struct_size.restype = C.c_int64
    lib.lbm_struct_size.argtypes = [C.c_int32]
    lib.lbm_create.restype = C.c_int
    lib.lbm_create.argtypes = [C.POINTER(LbmParams), C.POINTER(vp)]
    lib.lbm_bind.restype = C.c_int
    lib.lbm_bind.argtypes = [vp, C.POINTER(LbmBuffers)]
    for name in ("lbm_init_geometry", "lbm_init_fields", "lbm_export_diagnostics"):
        fn = getattr(lib, name)
        fn.restype = C.c_int
        fn.argtypes = [vp, vp]
    lib.lbm_step.restype = C.c_int
    lib.lbm_step.argtypes = [vp, C.c_int32, vp]
    lib.lbm_read_counters.restype = C.c_int
    lib.lbm_read_counters.argtypes = [vp, C.POINTER(LbmCounters)]
    lib.lbm_destroy.restype = C.c_int
    lib.lbm_destroy.argtypes = [vp]
    lib.lbm_last_error.restype = C.c_char_p
    lib.lbm_last_error.argtypes = [vp]
    lib.lbm_set_kernel_timing.restype = C.c_int
    lib.lbm_set_kernel_timing.argtypes = [vp, C.c_int32]
    lib.lbm_kernel_timing.restype = C.c_int
    lib.lbm_kernel_timing.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.lbm_launch_count.restype = C.c_int
    lib.lbm_launch_count.argtypes = [C.POINTER(C.c_int64)]
    lib.lbm_set_tile_chunk.restype = C.c_int
    lib.lbm_set_tile_chunk.argtypes = [vp, C.c_int32]
    lib.lbm_set_step_graphs.restype = C.c_int
    lib.lbm_set_step_graphs.argtypes = [vp, C.c_int32]
    lib.lbm_batch_create.restype = C.c_int
    lib.lbm_batch_create.argtypes = [C.POINTER(vp), C.c_int32, C.POINTER(vp)]
    lib.lbm_batch_step.restype = C.c_int
    lib.lbm_batch_step.argtypes = [vp, C.c_int32, vp]
    lib.lbm_batch_destroy.restype = C.c_int
    lib.lbm_batch_destroy.argtypes = [vp]
    lib.lbm_batch_last_error.restype = C.c_char_p
    lib.lbm_batch_last_error.argtypes = [vp]
    lib.lbm_diagnostics.restype = C.c_int
    lib.lbm_diagnostics.argtypes = [vp, C.POINTER(LbmDiagInputs), C.POINTER(LbmDiag), vp]
    lib.lbm_set_arithmetic.restype = C.c_int
    lib.lbm_set_arithmetic.argtypes = [vp, C.c_int32]
    lib.lbm_get_arithmetic.restype = C.c_int
    lib.lbm_get_arithmetic.argtypes = [vp, C.POINTER(C.c_int32)]
    lib.lbm_link_geometry_noalloc.restype = C.c_int
    lib.lbm_link_geometry_noalloc.argtypes = [C.POINTER(LbmParams), vp, vp, vp, vp, vp, vp, vp, vp, C.c_char_p,
                                              C.c_size_t]
    return lib


ABI_SYMBOLS = (
    "lbm_backend_name", "lbm_abi_version", "lbm_struct_size", "lbm_create", "lbm_bind", "lbm_init_geometry",
    "lbm_init_fields", "lbm_step", "lbm_export_diagnostics", "lbm_read_counters", "lbm_destroy", "lbm_last_error",
    "lbm_set_kernel_timing", "lbm_kernel_timing", "lbm_launch_count", "lbm_link_geometry_noalloc",
    "lbm_set_tile_chunk", "lbm_set_step_graphs", "lbm_set_arithmetic", "lbm_get_arithmetic", "lbm_diagnostics",
    "lbm_batch_create", "lbm_batch_step", "lbm_batch_destroy", "lbm_batch_last_error",
)


def check_layout(lib: C.CDLL) -> None:
    """Raise if the library's struct sizes differ from this binding's."""
    for which, cls in enumerate((LbmParams, LbmBuffers, LbmCounters, LbmDiag, LbmDiagInputs)):
        got = lib.lbm_struct_size(which)
        if got != C.sizeof(cls):
            raise RuntimeError(f"ABI layout mismatch for {cls.__name__}: library {got} vs binding {C.sizeof(cls)}")


class LbmError(RuntimeError):
    pass


def check(lib, ctx, status: int, what: str) -> None:
    if status != LBM_OK:
        msg = lib.lbm_last_error(ctx) if ctx else None
        detail = msg.decode() if msg else ERRORS.get(status, "unknown")
        raise LbmError(f"{what} failed ({status}): {detail}")


def native_dir() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "_native")
