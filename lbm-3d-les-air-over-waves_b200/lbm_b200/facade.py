"""The solver module surface of LBM_3D_LES_air_over_waves_CODEX.py on top of
the B200 engine, so that the reference's drivers use it as a drop-in.

run_ab_case.py loads a solver file by path, sets `steps`, `plot_freq`,
`plot_step_start` and `visualize`, and calls `main()`; its metrics read
module globals, fields through `.to_numpy()` and counters through `[None]`
(run_ab_case.py:261-280, 283-679, 899-912).  `install(namespace)` fills a
module namespace with:

  - the configuration globals, evaluated from the LBM_* environment at
    import exactly as the reference evaluates them (dx, Nx, Ny, Nz, Lx_m ...,
    x_phys/y_phys/z_phys, X_phys/Y_phys/Z_phys, vel_scale, rho0, U_ref_phys,
    FS_GAS/FS_LIQUID/FS_INTERFACE, cube parameters, mode flags);
  - field objects (rho, ux, uy, uz, obstacle, phi, water_h, free_surface_*,
    pressure_reference_head, cx, cy, cz) whose to_numpy() returns the
    current values in the reference's (Nz, Ny, Nx) layout;
  - counter objects (boundary_cut_link_count, free_surface_* ...) read with
    `[None]`;
  - main(): the reference's initialisation and time loop (CODEX.py:3757-3954):
    `visualize(step, time_phys, Re_phys_air, Re_lb_base)` every plot_freq
    steps after plot_step_start, the health line every 100 steps (its
    maximum speed reduced on the device).  Steps between those events run as
    one call of the engine;
  - device_metrics(): the run_ab_case.py metric row of the current state,
    reduced on the device (lbm_diagnostics), for harnesses that do not want
    to pull whole fields; save_render_snapshot(): the render-snapshot npz of
    run_ab_case.py:140-202.

The seed of the initial kick and of the random backscatter is the one a
harness hands to taichi.init (run_ab_case.py:261-273), else LBM_RANDOM_SEED.
The engine itself (buffers on the device, kernels) is created on first use.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from .config import load_config

D3Q19_CX = (0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0)
D3Q19_CY = (0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1)
D3Q19_CZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1)

# reference field name -> (engine buffer, dtype of the reference field, needs export_diagnostics)
FIELDS = {
    "rho": ("rho", np.float32, False), "ux": ("ux", np.float32, False), "uy": ("uy", np.float32, False),
    "uz": ("uz", np.float32, False), "omega": ("omega", np.float32, False),
    "water_h": ("water_h", np.float32, False), "water_h_last": ("water_h_last", np.float32, False),
    "u_wave": ("u_wave", np.float32, False), "v_wave": ("v_wave", np.float32, False),
    "w_wave": ("w_wave", np.float32, False),
    "free_surface_h": ("fs_h", np.float32, False), "free_surface_h_last": ("fs_h_last", np.float32, False),
    "free_surface_fill": ("fs_fill", np.float32, False), "free_surface_type": ("fs_type", np.int32, False),
    "free_surface_type_prev": ("fs_type_prev", np.int32, False), "free_surface_mass": ("fs_mass", np.float32, False),
    "free_surface_mass_excess": ("fs_mass_excess", np.float32, False),
    "phi": ("phi", np.float32, True), "obstacle": ("obstacle", np.int32, True),
    "near_obstacle": ("near_obstacle", np.int32, True), "lattice_open": ("lattice_open", np.int32, True),
    "lattice_open_frac": ("lattice_open_frac", np.float32, True),
    "pressure_reference_head": ("pressure_reference_head", np.float32, True),
    "gravity_body_fraction": ("gravity_body_fraction", np.float32, True),
    "free_surface_vof_exterior_gas": ("vof_exterior_gas", np.int32, True),
}
COUNTERS = (
    "boundary_cut_link_count", "free_surface_cut_link_count", "boundary_refill_count", "free_surface_refill_count",
    "free_surface_coalescence_repair_count", "free_surface_thin_gap_bridge_count", "free_surface_vof_excess_count",
    "free_surface_vof_orphan_count", "free_surface_vof_collapse_cell_count",
    "free_surface_vof_collapse_candidate_volume_m3", "free_surface_vof_collapse_applied_volume_m3",
    "free_surface_vof_detached_advect_count", "free_surface_vof_detached_advect_mass",
    "free_surface_vof_detached_compress_count", "free_surface_vof_detached_compress_mass",
)


# The columns of the harness's metrics CSV, in its order (run_ab_case.py:15-35).
METRIC_FIELDNAMES = (
    "label", "step", "time_phys", "max_speed_phys", "max_speed_x", "max_speed_y", "max_speed_z", "max_speed_fs_type",
    "max_speed_fs_fill", "max_speed_wet_neighbors", "max_speed_full_neighbors", "max_speed_gas_neighbors", "p_rms",
    "p_hp_rms", "p_total_rms", "p_total_hp_rms", "p_linear_resid_rms", "p_linear_resid_hp_rms", "vort_rms",
    "vort_hp_rms", "fs_p_rms", "fs_p_hp_rms", "fs_p_total_rms", "fs_p_total_hp_rms", "fs_p_linear_resid_rms",
    "fs_p_linear_resid_hp_rms", "fs_vort_rms", "fs_vort_hp_rms", "cut_links", "fs_cut_links", "refill", "fs_refill",
    "fs_coalesce", "fs_bridge", "vof_detached_count", "vof_detached_mass", "vof_compact_count", "vof_compact_mass",
    "surface_min", "surface_max", "water_volume", "vof_mass_total", "vof_excess_count", "vof_orphan_count",
    "vof_collapse_cells", "vof_collapse_candidate_volume", "vof_collapse_applied_volume", "vof_min_interface_fill",
    "vof_tiny_interface_count", "vof_pending_excess_mass", "vof_pending_excess_count", "surface_symmetry_l2",
    "surface_eta_hp_rms", "surface_left_max", "surface_right_max",
)

# metric column -> engine counter, for the counters the row carries in every mode
_ROW_COUNTERS = {
    "cut_links": "boundary_cut_link_count", "fs_cut_links": "free_surface_cut_link_count",
    "refill": "boundary_refill_count", "fs_refill": "free_surface_refill_count",
    "fs_coalesce": "free_surface_coalescence_repair_count", "fs_bridge": "free_surface_thin_gap_bridge_count",
    "vof_detached_count": "free_surface_vof_detached_advect_count",
    "vof_detached_mass": "free_surface_vof_detached_advect_mass",
    "vof_compact_count": "free_surface_vof_detached_compress_count",
    "vof_compact_mass": "free_surface_vof_detached_compress_mass",
}
# metric column -> engine counter, reported with VOF tracking only
_VOF_COUNTERS = {
    "vof_excess_count": "free_surface_vof_excess_count", "vof_orphan_count": "free_surface_vof_orphan_count",
    "vof_collapse_cells": "free_surface_vof_collapse_cell_count",
    "vof_collapse_candidate_volume": "free_surface_vof_collapse_candidate_volume_m3",
    "vof_collapse_applied_volume": "free_surface_vof_collapse_applied_volume_m3",
}
_ALWAYS = ("max_speed_phys", "p_rms", "p_hp_rms", "p_total_rms", "p_total_hp_rms", "vort_rms", "vort_hp_rms")
_FREE_SURFACE = ("max_speed_fs_fill", "fs_p_rms", "fs_p_hp_rms", "fs_p_total_rms", "fs_p_total_hp_rms", "fs_vort_rms",
                 "fs_vort_hp_rms", "surface_min", "surface_max", "water_volume", "surface_symmetry_l2",
                 "surface_eta_hp_rms", "surface_left_max", "surface_right_max")
_FREE_SURFACE_COUNTS = ("max_speed_fs_type", "max_speed_wet_neighbors", "max_speed_full_neighbors",
                        "max_speed_gas_neighbors")
_VOF = ("vof_mass_total", "vof_min_interface_fill", "vof_pending_excess_mass")
_VOF_COUNTS = ("vof_tiny_interface_count", "vof_pending_excess_count")


LINEAR_RESIDUAL_COLUMNS = ("p_linear_resid_rms", "p_linear_resid_hp_rms", "fs_p_linear_resid_rms",
                           "fs_p_linear_resid_hp_rms")


def _high_pass_xz(field: np.ndarray, x_periodic: bool) -> np.ndarray:
    """Grid-scale residual of an xz slice (run_ab_case.py:111-137): the value
    minus the mean of its four neighbours, with linear extrapolation past
    the top and bottom rows and past solid x ends, wrap-around in periodic x."""
    zp, zm = np.empty_like(field), np.empty_like(field)
    zp[:-1], zp[-1] = field[1:], 2.0 * field[-1] - field[-2]
    zm[1:], zm[0] = field[:-1], 2.0 * field[0] - field[1]
    if x_periodic:
        xp, xm = np.roll(field, -1, axis=1), np.roll(field, 1, axis=1)
    else:
        xp, xm = np.empty_like(field), np.empty_like(field)
        xp[:, :-1], xp[:, -1] = field[:, 1:], 2.0 * field[:, -1] - field[:, -2]
        xm[:, 1:], xm[:, 0] = field[:, :-1], 2.0 * field[:, 0] - field[:, 1]
    return field - 0.25 * (zp + zm + xp + xm)


def linear_residual_metrics(cfg, rho_xz, phi_xz, inactive_xz, surface_line, bed_line) -> dict:
    """The four linear-wave residual columns of the metric row
    (run_ab_case.py:52-108, 505-595) from the mid-y xz slice: the lattice
    pressure minus the pressure of linear finite-depth theory under the
    instantaneous surface line (hostinit.linear_wave_heads, plus the still-
    water head unless the formulation is hydrostatic-balanced), as RMS over
    the near-bed band 0 < phi <= 10 dx and over the free-surface band, plain
    and high-passed.  NaN where the harness has none: no free surface, VOF
    tracking, or a bed line that is not flat.  One slice, on the host."""
    from .hostinit import linear_wave_heads

    out = dict.fromkeys(LINEAR_RESIDUAL_COLUMNS, float("nan"))
    if int(cfg.water_free_surface_enabled) != 1 or str(cfg.free_surface_tracking_mode) == "vof":
        return out
    bed_line = np.asarray(bed_line, dtype=np.float64)
    if not np.allclose(bed_line, bed_line[0], atol=1.0e-12, rtol=0.0):
        return out
    rho_xz = np.asarray(rho_xz, dtype=np.float64)
    nz, nx = rho_xz.shape
    dx, base = float(cfg.dx), float(cfg.free_surface_base_m)
    rho_phys, gravity = float(cfg.rho_phys), float(cfg.gravity_phys)
    z = (np.arange(nz, dtype=np.float64) + 0.5) * dx
    bed = float(bed_line[0])
    surface = np.asarray(surface_line, dtype=np.float64)
    heads = np.array(linear_wave_heads(surface - base, dx, bed, max(base - bed, dx), z,
                                       str(cfg.x_boundary_mode) == "solid"))
    if int(cfg.use_hydrostatic_balanced_pressure) != 1:
        heads = np.maximum(base - z, 0.0)[:, None] + heads
    p_lattice = rho_phys * float(cfg.vel_scale) ** 2 * ((1.0 / 3.0) * (rho_xz - float(cfg.rho0)))
    resid = p_lattice - rho_phys * gravity * heads
    resid_hp = _high_pass_xz(resid, str(cfg.x_boundary_mode) == "periodic")
    inactive = np.asarray(inactive_xz, dtype=bool)
    zz = z[:, None]
    bands = {"": (np.asarray(phi_xz) > 0.0) & (np.asarray(phi_xz) <= 10.0 * dx) & ~inactive,
             "fs_": (zz <= surface[None, :] + 0.5 * dx) & (zz >= surface[None, :] - 3.0 * dx) & ~inactive}
    for prefix, band in bands.items():
        if band.any():
            v, h = resid[band], resid_hp[band]
            if np.isfinite(v).any():
                out[prefix + "p_linear_resid_rms"] = float(np.sqrt(np.nanmean((v - np.nanmean(v)) ** 2)))
                out[prefix + "p_linear_resid_hp_rms"] = float(np.sqrt(np.nanmean(h ** 2)))
    return out


def metric_row(cfg, label: str, step: int, time_phys: float, diag: dict, counters: dict,
               linear: dict | None = None) -> dict:
    """One row of the harness's metrics CSV (make_visualize,
    run_ab_case.py:283-679) from a device diagnostics record (lbm_diagnostics),
    the engine's counters and the linear-wave residual columns
    (linear_residual_metrics; NaN when not given): the same columns, and per
    mode the same not-applicable values (-1 for counts, NaN for values) the
    harness writes."""
    nan = float("nan")
    fs = int(cfg.water_free_surface_enabled) == 1
    vof = fs and str(cfg.free_surface_tracking_mode) == "vof"
    dx = float(cfg.dx)
    row = dict.fromkeys(METRIC_FIELDNAMES, nan)
    row.update(label=label, step=step, time_phys=time_phys)
    for k in _ALWAYS:
        row[k] = float(diag[k])
    row.update(max_speed_x=(int(diag["max_i"]) + 0.5) * dx, max_speed_y=(int(diag["max_j"]) + 0.5) * dx,
               max_speed_z=(int(diag["max_k"]) + 0.5) * dx)
    for col, key in _ROW_COUNTERS.items():
        row[col] = counters[key]
    for k in _FREE_SURFACE_COUNTS:
        row[k] = int(diag[k]) if fs else -1
    if fs:
        for k in _FREE_SURFACE:
            row[k] = float(diag[k])
    for k in _VOF_COUNTS:
        row[k] = int(diag[k]) if vof else -1
    for col, key in _VOF_COUNTERS.items():
        row[col] = counters[key] if vof else (-1 if col in ("vof_excess_count", "vof_orphan_count",
                                                            "vof_collapse_cells") else nan)
    if vof:
        for k in _VOF:
            row[k] = float(diag[k])
    if linear:
        for k in LINEAR_RESIDUAL_COLUMNS:
            row[k] = float(linear[k])
    return row


def _linear_residual_from_device(eng, cfg) -> dict | None:
    """linear_residual_metrics from the mid-y slices of the device fields
    (a few rows copied to the host), or None where the harness has none."""
    if int(cfg.water_free_surface_enabled) != 1 or str(cfg.free_surface_tracking_mode) == "vof":
        return None
    mj = int(cfg.Ny) // 2

    def row(name, diag=False):
        return eng.buffer(name, diag)[..., mj, :].detach().cpu().numpy()

    bed_line = row("water_h")
    if not np.allclose(bed_line, bed_line[0], atol=1.0e-12, rtol=0.0):
        return None
    obstacle = row("obstacle", True) != 0
    inactive = obstacle | ((row("fs_type") == 0) & ~obstacle)
    return linear_residual_metrics(cfg, row("rho"), row("phi", True), inactive, row("fs_h"), bed_line)


def make_device_visualize(ns: dict, label: str, output_dir, metrics_writer):
    """A visualize callback like the harness's make_visualize
    (run_ab_case.py:283-880) that needs no plotting: each call writes the
    metric row of the current state, reduced on the device, to
    `metrics_writer` (a csv.DictWriter over METRIC_FIELDNAMES), writes the
    render snapshot when LBM_SAVE_RENDER_SNAPSHOT is set, and prints the
    harness's frame line.  The linear-wave residual columns come from one
    mid-y slice of the fields on the host.  The frame PNGs are not drawn."""
    from pathlib import Path

    out = Path(output_dir)
    out.mkdir(parents=True, exist_ok=True)

    def visualize(step, time_phys, Re_phys_air, Re_lb_base):
        dom = ns["_engine"].domain()
        r = metric_row(dom.cfg, label, step, time_phys, dom.diagnostics(), dom.counters(),
                       _linear_residual_from_device(ns["_engine"], dom.cfg))
        metrics_writer.writerow(r)
        note = ""
        if str(os.environ.get("LBM_SAVE_RENDER_SNAPSHOT", "")).strip().lower() in ("1", "true", "yes", "on"):
            note = f", render_snapshot={write_render_snapshot(ns, label=label, step=step, time_phys=time_phys, output_dir=out)}"
        surface = "column_surface" if str(dom.cfg.free_surface_tracking_mode) == "vof" else "surface"
        print(
            f"[{label}] Boundary band <=10 cells: p_dyn_rms={r['p_rms']:.3e} Pa, "
            f"p_dyn_hp_rms={r['p_hp_rms']:.3e} Pa, p_total_hp_rms={r['p_total_hp_rms']:.3e} Pa, "
            f"p_lin_resid_hp={r['p_linear_resid_hp_rms']:.3e} Pa, vort_rms={r['vort_rms']:.3e}, "
            f"vort_hp_rms={r['vort_hp_rms']:.3e}, cut_links={r['cut_links']}, fs_cut_links={r['fs_cut_links']}, "
            f"refill={r['refill']}, fs_refill={r['fs_refill']}, fs_coalesce={r['fs_coalesce']}, "
            f"fs_bridge={r['fs_bridge']}, {surface}=[{r['surface_min']:.3f},{r['surface_max']:.3f}] m, "
            f"volume={r['water_volume']:.3f} m^3, vof_mass={r['vof_mass_total']:.3f}, "
            f"vof_excess={r['vof_excess_count']}, vof_orphans={r['vof_orphan_count']}, "
            f"vof_detached={r['vof_detached_count']} ({r['vof_detached_mass']:.3e}), "
            f"vof_compact={r['vof_compact_count']} ({r['vof_compact_mass']:.3e}), "
            f"vof_collapse={r['vof_collapse_applied_volume']:.3f}/{r['vof_collapse_candidate_volume']:.3f} m^3 "
            f"({r['vof_collapse_cells']} cells), vof_min_fill={r['vof_min_interface_fill']:.3f}, "
            f"vof_tiny={r['vof_tiny_interface_count']}, vof_pending={r['vof_pending_excess_mass']:.3e} "
            f"({r['vof_pending_excess_count']}), sym_l2={r['surface_symmetry_l2']:.3e} m, "
            f"eta_hp={r['surface_eta_hp_rms']:.3e} m, fs_p_dyn_hp={r['fs_p_hp_rms']:.3e} Pa, "
            f"fs_p_total_hp={r['fs_p_total_hp_rms']:.3e} Pa, fs_p_lin_resid_hp={r['fs_p_linear_resid_hp_rms']:.3e} Pa, "
            f"fs_vort_hp={r['fs_vort_hp_rms']:.3e}, "
            f"Umax_loc=({r['max_speed_x']:.2f},{r['max_speed_y']:.2f},{r['max_speed_z']:.2f}) m, "
            f"Umax_type={r['max_speed_fs_type']}, Umax_fill={r['max_speed_fs_fill']:.3f}, "
            f"Umax_nbrs(wet/full/gas)={r['max_speed_wet_neighbors']}/{r['max_speed_full_neighbors']}/"
            f"{r['max_speed_gas_neighbors']}, "
            f"L/R max=[{r['surface_left_max']:.3f},{r['surface_right_max']:.3f}] m{note}",
            flush=True,
        )

    return visualize


def configure_direct_visualization(ns: dict):
    """Direct runs of the solver file (CODEX.py:3735-3753): the metrics CSV
    <LBM_RUN_LABEL>_metrics.csv (label default "direct") in LBM_OUTPUT_DIR
    (default "frames"), written by make_device_visualize.  Returns the open
    file, which the caller closes after main()."""
    import csv
    from pathlib import Path

    label = os.environ.get("LBM_RUN_LABEL", "direct")
    output_dir = Path(os.environ.get("LBM_OUTPUT_DIR", "frames")).resolve()
    output_dir.mkdir(parents=True, exist_ok=True)
    metrics_file = (output_dir / f"{label}_metrics.csv").open("w", newline="")
    writer = csv.DictWriter(metrics_file, fieldnames=list(METRIC_FIELDNAMES))
    writer.writeheader()
    ns["visualize"] = make_device_visualize(ns, label, output_dir, writer)
    return metrics_file


def tau_line(cfg) -> str:
    """The line the reference prints when it is imported (CODEX.py:471)."""
    return f"tau used in current simulation: {cfg.tau0:.10f}"


def run_summary(cfg) -> list:
    """The configuration summary the reference's main() prints after its
    initialisation (CODEX.py:3794-3871), line for line, from the same
    globals, so that logs of either solver read alike."""
    c = cfg
    out = [f"Grid Size (Nx, Ny, Nz):  {c.Nx} {c.Ny} {c.Nz}",
           f"Physics mode: {c.physics_mode} ({c.fluid_name})",
           f"Free-surface mode: {c.free_surface_mode}, initial={c.free_surface_initial_condition}, "
           f"tracking={c.free_surface_tracking_mode}"]
    if int(c.water_free_surface_enabled) == 1:
        out.append(
            f"Free surface: base={c.free_surface_base_m:.3f} m, depth={c.free_surface_depth_m:.3f} m, "
            f"solitary_amp={c.solitary_amp_m:.3f} m, H/h={c.solitary_height_depth_ratio:.3f}, "
            f"solitary_c={c.solitary_celerity_phys:.3f} m/s, "
            f"solitary_dir={c.solitary_direction:+.0f}, solitary_1/kappa={c.solitary_length_scale_m:.3f} m, "
            f"solitary_u0={c.solitary_initial_velocity_mode}, "
            f"boundary={c.free_surface_boundary_mode}, refill={c.free_surface_refill_mode}, "
            f"initial_pressure={c.initial_pressure_mode}, pressure_formulation={c.pressure_formulation}")
        if c.pressure_formulation_auto_corrected:
            out.append("Pressure formulation auto-corrected from total_pressure to vof_component_balanced for "
                       "disconnected VOF. Set LBM_ALLOW_TOTAL_PRESSURE_VOF_DIAGNOSTIC=1 only for a known-bad "
                       "full-pressure diagnostic.")
        if c.free_surface_tracking_mode == "vof":
            out.append(
                f"VOF state change: empty_fill_threshold={c.vof_empty_fill_threshold:.4f}, "
                f"orphan_empty_threshold={c.vof_orphan_empty_threshold:.4f}, "
                f"orphan_search_radius={c.vof_orphan_search_radius}, "
                f"orphan_max_weak_neighbors={c.vof_orphan_max_weak_neighbors}, "
                f"detached_advection={bool(c.vof_detached_advection_enabled)}, "
                f"detached_max_wet_neighbors={c.vof_detached_max_wet_neighbors}, "
                f"detached_max_resolved_neighbors={c.vof_detached_max_resolved_neighbors}, "
                f"detached_residual_fill_threshold={c.vof_detached_residual_fill_threshold:.4f}, "
                f"link_aperture={int(c.vof_link_aperture_enabled) == 1}, "
                f"thin_gap_bridge={bool(c.vof_thin_gap_bridge_enabled)}, "
                f"bridge_strength={c.vof_thin_gap_bridge_strength:.3f}, "
                f"collapse_trapped_gas={bool(c.vof_collapse_trapped_gas_enabled)}, "
                f"collapse_interval={c.vof_collapse_interval}, "
                f"collapse_max_volume={c.vof_collapse_max_volume_m3:.3f} m^3, "
                f"collapse_flood_sweeps={c.vof_collapse_flood_sweeps}")
            if c.vof_initial_shape == "block":
                out.append(
                    f"VOF initial block: center=({c.vof_block_center_x_m:.3f}, {c.vof_block_center_y_m:.3f}, "
                    f"{c.vof_block_center_z_m:.3f}) m, size=({c.vof_block_size_x_m:.3f}, "
                    f"{c.vof_block_size_y_m:.3f}, {c.vof_block_size_z_m:.3f}) m")
        if c.free_surface_initial_condition == "gaussian":
            out.append(f"Gaussian hump: amp={c.gaussian_amp_m:.3f} m, center_x={c.gaussian_center_x_m:.3f} m, "
                       f"sigma={c.gaussian_sigma_m:.3f} m, zero initial velocity")
    out.append(f"Bed profile: {c.bed_profile}, bed_level={c.offset_m:.3f} m")
    if c.bed_profile == "piecewise_linear":
        m = c.piecewise_bed_metadata
        out.append(f"Piecewise bottom: file={m['path']}, points={m['point_count']}, x_first={m['first_x']:.3f} m, "
                   f"x_last={m['last_x']:.3f} m, z_min={m['min_z']:.3f} m, z_max={m['max_z']:.3f} m, "
                   f"z_at_Lx={m['z_at_lx']:.3f} m")
    out.append(f"Obstacle mode: {c.obstacle_mode}")
    if int(c.include_cube_geometry) == 1:
        out.append(f"Cube size/center/yaw/pitch: size=({c.cube_size_x_m:.3f}, {c.cube_size_y_m:.3f}, "
                   f"{c.cube_size_z_m:.3f}) m, center=({c.cube_center_x_m:.3f}, {c.cube_center_y_m:.3f}, "
                   f"{c.cube_center_z_m:.3f}) m, yaw={c.cube_yaw_deg:.3f} deg, pitch={c.cube_pitch_deg:.3f} deg")
    out += [f"Boundary geometry mode: {c.boundary_geometry_mode}",
            f"X boundary mode: {c.x_boundary_mode}",
            f"Wall velocity sampling: {c.wall_velocity_sampling}",
            f"Initial free-surface population projection: {bool(c.initialize_free_surface_populations)}",
            f"Collision model: {c.collision_model}",
            f"Fluid rho={c.rho_phys:.3f} kg/m^3, nu={c.nu_phys:.6e} m^2/s, gravity={c.gravity_phys:.3f} m/s^2",
            f"Reference speed={c.U_ref_phys:.3f} m/s, dt={c.dt_phys:.6e} s, g_lb={c.g_lb:.6e}, "
            f"g_body_lb={c.g_body_lb:.6e}",
            f"Physical Re ({c.fluid_name}): {c.Re_phys_air:.3e}",
            f"Lattice Re (base): {c.Re_lb_base:.2f}"]
    return out


def _visualize_unbound(step, time_phys, Re_phys_air, Re_lb_base):
    """The solver's visualize before a harness binds one (CODEX.py:3728-3732)."""
    raise RuntimeError(
        "Visualization has not been configured. Use run_ab_case.py or run "
        "this solver as a script so direct-run visualization can be bound."
    )


class _Engine:
    """Lazily created Domain shared by the field and counter views."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.dom = None
        self.export_step = -1

    def domain(self):
        if self.dom is None:
            from .domain import Domain

            self.dom = Domain(self.cfg, device=os.environ.get("LBM_B200_DEVICE", "cuda:0"), with_diag=True,
                              init=False)
        return self.dom

    def buffer(self, name, diag):
        dom = self.domain()
        if diag:
            step = dom.counters()["step"]
            if step != self.export_step:
                dom.export_diagnostics()
                self.export_step = step
        dom.synchronize()
        return dom.field(name)


class Field:
    """A reference field: to_numpy() gives the current values."""

    def __init__(self, engine, name, buf, dtype, diag):
        self._engine, self.name, self._buf, self._dtype, self._diag = engine, name, buf, dtype, diag

    def to_numpy(self):
        arr = self._engine.buffer(self._buf, self._diag).detach().cpu().numpy().astype(self._dtype)
        if arr.ndim == 4 and arr.shape[0] == 19:
            # per-link fields: the reference's ti.Vector.field(19) layout (Nz, Ny, Nx, 19)
            arr = np.ascontiguousarray(np.moveaxis(arr, 0, -1))
        return arr

    @property
    def shape(self):
        return tuple(self._engine.domain().field(self._buf).shape)


class _Const:
    """A small constant field (the lattice vectors)."""

    def __init__(self, values):
        self._v = np.asarray(values, dtype=np.int32)

    def to_numpy(self):
        return self._v.copy()

    def __getitem__(self, i):
        return int(self._v[i])

    @property
    def shape(self):
        return self._v.shape


class Counter:
    """A scalar counter of the reference, read as counter[None]."""

    def __init__(self, engine, key):
        self._engine, self._key = engine, key

    def __getitem__(self, idx):
        if idx is not None:
            raise IndexError("scalar fields are indexed with [None]")
        if self._engine.dom is None:
            return 0
        return self._engine.dom.counters()[self._key]


def harness_seed():
    """The seed a harness hands to taichi.init, or None.

    run_ab_case.py seeds a solver by replacing taichi.init with a wrapper
    that adds random_seed=<its --random-seed> to every call, before it
    loads the solver file (run_ab_case.py:261-273).  This module never
    starts Taichi, so the wrapper is not called: the value is read from the
    wrapper's closure."""
    init = getattr(sys.modules.get("taichi"), "init", None)
    code, cells = getattr(init, "__code__", None), getattr(init, "__closure__", None)
    if code is None or not cells:
        return None
    for name, cell in zip(code.co_freevars, cells):
        if name == "random_seed":
            try:
                value = cell.cell_contents
            except ValueError:   # an empty cell
                return None
            return value if isinstance(value, int) and not isinstance(value, bool) else None
    return None


def install(ns: dict, environ=None) -> None:
    """Fill `ns` with the solver module surface.  The seed of the initial
    kick and of the random backscatter is the harness's (harness_seed())
    when a harness wrapped taichi.init, else LBM_RANDOM_SEED."""
    env = dict(os.environ if environ is None else environ)
    seed = harness_seed()
    if seed is not None:
        env["LBM_RANDOM_SEED"] = str(seed)
    cfg = load_config(env)
    print(tau_line(cfg), flush=True)
    for k, v in cfg.values.items():
        if not k.startswith("_"):
            ns[k] = v
    Nx, Ny, Nz, dx = cfg.Nx, cfg.Ny, cfg.Nz, cfg.dx
    ns.update(dx=dx, Nx=Nx, Ny=Ny, Nz=Nz, rho0=cfg.rho0, FS_GAS=0, FS_LIQUID=1, FS_INTERFACE=2)
    x_phys = (np.arange(Nx) + 0.5) * dx
    y_phys = (np.arange(Ny) + 0.5) * dx
    z_phys = (np.arange(Nz) + 0.5) * dx
    Z_phys, Y_phys, X_phys = np.meshgrid(z_phys, y_phys, x_phys, indexing="ij")
    ns.update(x_phys=x_phys, y_phys=y_phys, z_phys=z_phys, X_phys=X_phys, Y_phys=Y_phys, Z_phys=Z_phys)
    ns.setdefault("Re_phys_air", cfg.Re_phys_air)
    ns.setdefault("Re_lb_base", cfg.Re_lb_base)
    eng = _Engine(cfg)
    ns["_engine"] = eng
    for name, (buf, dt, diag) in FIELDS.items():
        ns[name] = Field(eng, name, buf, dt, diag)
    ns["cx"], ns["cy"], ns["cz"] = _Const(D3Q19_CX), _Const(D3Q19_CY), _Const(D3Q19_CZ)
    for key in COUNTERS:
        ns[key] = Counter(eng, key)
    ns.setdefault("visualize", _visualize_unbound)

    def main():
        """Initialisation and time loop of the reference (CODEX.py:3757-3954)."""
        dom = eng.domain()
        dom.initialize()
        eng.export_step = -1
        print("\n".join(run_summary(cfg)), flush=True)
        steps = int(ns["steps"])
        plot_freq = max(1, int(ns["plot_freq"]))
        plot_start = int(ns["plot_step_start"])
        dt_phys = float(cfg.dt_phys)
        step = 0
        while step < steps:
            # next step with an event: a plot, a health report, or the end
            nxt = min(steps, (step // plot_freq + 1) * plot_freq, (step // 100 + 1) * 100)
            dom.step(nxt - step)
            step = nxt
            time_phys = (step + 1) * dt_phys
            if step % plot_freq == 0 and step > plot_start:
                ns["visualize"](step, time_phys, ns["Re_phys_air"], ns["Re_lb_base"])
            if step % 100 == 0:
                _health(ns, dom, step)
        print("Simulation Complete.")

    ns["main"] = main

    def device_metrics(slice_j=None) -> dict:
        """The metric row of run_ab_case.py's make_visualize for the current
        state (max speed and location, volume and VOF accounting, surface
        line and mid-slice band statistics), reduced on the device."""
        return eng.domain().diagnostics(slice_j)

    ns["device_metrics"] = device_metrics

    def save_render_snapshot(label, step, time_phys, output_dir):
        """Write <output_dir>/<label>_render_<step:05d>.npz in the format of
        run_ab_case.py:140-202 (grid, bed, obstacle mask, free-surface height
        and fill, cube description).  Returns the path."""
        return write_render_snapshot(ns, label=label, step=step, time_phys=time_phys, output_dir=output_dir)

    ns["save_render_snapshot"] = save_render_snapshot


def write_render_snapshot(ns, *, label: str, step: int, time_phys: float, output_dir) -> str:
    """The render-snapshot writer of run_ab_case.py:140-202: one compressed
    npz per call with the arrays a renderer needs, in the reference's names,
    dtypes and shapes.  Only the format is reproduced; nothing is rendered."""
    from pathlib import Path

    out = Path(output_dir)
    out.mkdir(parents=True, exist_ok=True)
    fs_enabled = int(ns.get("water_free_surface_enabled", 0)) == 1
    tracking = str(ns.get("free_surface_tracking_mode", "height"))
    water_h = ns["water_h"].to_numpy()
    obstacle = ns["obstacle"].to_numpy()
    side = float(ns.get("cube_side_m", 0.0))
    data = {
        "time_phys": np.array(time_phys, dtype=np.float64),
        "dx": np.array(ns["dx"], dtype=np.float64),
        "lx_m": np.array(ns["Lx_m"], dtype=np.float64),
        "ly_m": np.array(ns["Ly_m"], dtype=np.float64),
        "lz_m": np.array(ns["Lz_m"], dtype=np.float64),
        "x_phys": np.asarray(ns["x_phys"]).astype(np.float32),
        "y_phys": np.asarray(ns["y_phys"]).astype(np.float32),
        "z_phys": np.asarray(ns["z_phys"]).astype(np.float32),
        "water_h": water_h.astype(np.float32),
        "obstacle": obstacle.astype(bool).astype(np.uint8),
        "free_surface_enabled": np.array(int(fs_enabled), dtype=np.int8),
        "tracking_mode": np.array(tracking),
        "include_cube_geometry": np.array(int(ns.get("include_cube_geometry", 0)), dtype=np.int8),
        "cube_size_m": np.array([float(ns.get("cube_size_x_m", side)), float(ns.get("cube_size_y_m", side)),
                                 float(ns.get("cube_size_z_m", side))], dtype=np.float32),
        "cube_center_m": np.array([float(ns.get("cube_center_x_m", 0.0)), float(ns.get("cube_center_y_m", 0.0)),
                                   float(ns.get("cube_center_z_m", 0.0))], dtype=np.float32),
        "cube_yaw_pitch_deg": np.array([float(ns.get("cube_yaw_deg", 0.0)), float(ns.get("cube_pitch_deg", 0.0))],
                                       dtype=np.float32),
    }
    if fs_enabled:   # without a free surface the reference's caller passes neither array
        data["free_surface_h"] = ns["free_surface_h"].to_numpy().astype(np.float32)
        data["free_surface_fill"] = ns["free_surface_fill"].to_numpy().astype(np.float32)
    path = out / f"{label}_render_{int(step):05d}.npz"
    np.savez_compressed(path, **data)
    return str(path)


def health_line(step: int, max_u, vel_scale: float, c: dict) -> str:
    """The reference's periodic health line (CODEX.py:3930-3954) from the
    maximum speed over active cells (lattice units, float32 as the
    reference reduces it) and the counters."""
    max_u = np.float32(max_u)
    return (
        f"Time Step {step}, Max |U| (LB units) = {max_u:.4f}, "
        f"Max U (phys) ~ {max_u * np.float32(vel_scale):.2f} m/s, "
        f"cut_links={c['boundary_cut_link_count']}, refill={c['boundary_refill_count']}, "
        f"fs_refill={c['free_surface_refill_count']}, fs_coalesce={c['free_surface_coalescence_repair_count']}, "
        f"fs_bridge={c['free_surface_thin_gap_bridge_count']}, "
        f"vof_excess={c['free_surface_vof_excess_count']}, "
        f"vof_orphans={c['free_surface_vof_orphan_count']}, "
        f"vof_detached={c['free_surface_vof_detached_advect_count']} "
        f"({c['free_surface_vof_detached_advect_mass']:.3e}), "
        f"vof_compact={c['free_surface_vof_detached_compress_count']} "
        f"({c['free_surface_vof_detached_compress_mass']:.3e}), "
        f"vof_collapse_cells={c['free_surface_vof_collapse_cell_count']}, "
        f"vof_collapse_vol={c['free_surface_vof_collapse_applied_volume_m3']:.3f} m^3"
    )


def _health(ns, dom, step):
    """The health line of the current state.  The maximum speed over active
    cells is reduced on the device (lbm_diagnostics); only scalars come back
    to the host."""
    print(health_line(step, dom.diagnostics()["max_speed_lb"], ns["vel_scale"], dom.counters()), flush=True)
