"""Test helper: run the CUDA library and the CPU oracle side by side on the
same inputs and compare their state.  Test infrastructure only."""
from __future__ import annotations

import numpy as np

from oracle_runner import OracleSim

STATE = ["rho", "ux", "uy", "uz", "omega", "water_h", "water_h_last", "u_wave", "v_wave", "w_wave", "fs_h",
         "fs_h_last", "fs_flux_x", "fs_flux_y", "u_inlet_profile", "fs_fill", "fs_type", "fs_type_prev",
         "fs_mass", "fs_mass_excess", "fs_excess_dir"]
DIAG = ["phi", "obstacle", "near_obstacle", "lattice_open", "lattice_open_frac", "lattice_wall_type",
        "pressure_reference_head", "gravity_body_fraction", "vof_exterior_gas"]
COUNTERS = ["boundary_cut_link_count", "free_surface_cut_link_count", "free_surface_thin_gap_bridge_count",
            "free_surface_refill_count", "free_surface_coalescence_repair_count", "free_surface_vof_excess_count",
            "free_surface_vof_orphan_count", "free_surface_vof_collapse_cell_count",
            "free_surface_vof_detached_advect_count", "free_surface_vof_detached_compress_count", "flood_sweeps_used",
            "free_surface_vof_collapse_candidate_volume_m3", "free_surface_vof_collapse_applied_volume_m3",
            "free_surface_vof_collapse_removal_scale", "free_surface_vof_collapse_candidate_mass",
            "free_surface_vof_collapse_exterior_capacity", "free_surface_vof_detached_advect_mass",
            "free_surface_vof_detached_compress_mass", "step", "status_flags"]


def gpu_f32(dom, name):
    t = dom.field(name)
    return t.detach().cpu().numpy()


def populations(dom):
    import torch
    f = dom.f()
    if f.dtype == torch.float32:
        return f.detach().cpu().numpy()
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, dtype=np.float32)
    v = f.detach().float().cpu().numpy()
    if f.dtype == torch.float16:
        v = v * np.float32(1.0 / 256.0)   # FP16 holds the shifted value times 2^8
    return v + (w * np.float32(dom.cfg.rho0))[:, None, None, None]


def compare_states(dom, ref: OracleSim, tag: str, diag: bool = True, exact: bool = True, rtol=0.0, atol=0.0):
    problems = []
    mine_f = populations(dom)
    ref_f = ref.f()

    def cmp(name, a, b):
        if exact:
            bad = np.count_nonzero(a != b) if a.dtype.kind in "iu" else np.count_nonzero(
                a.view(np.uint32) != b.view(np.uint32)) if a.dtype == np.float32 else np.count_nonzero(a != b)
            if bad:
                problems.append(f"{tag}:{name}: {bad} differ (max abs {np.nanmax(np.abs(a.astype(np.float64) - b)):.3e})")
        else:
            err = np.abs(a.astype(np.float64) - b.astype(np.float64))
            bad = np.count_nonzero(~(err <= atol + rtol * np.abs(b.astype(np.float64))))
            if bad:
                problems.append(f"{tag}:{name}: {bad} out of tolerance (max abs {np.nanmax(err):.3e})")

    cmp("f", mine_f, ref_f)
    for name in STATE:
        cmp(name, gpu_f32(dom, name), ref.arrays[name])
    if diag:
        dom.export_diagnostics()
        ref.export()
        dom.synchronize()
        for name in DIAG:
            cmp(name, gpu_f32(dom, name), ref.arrays[name])
    c_gpu, c_ref = dom.counters(), ref.counters()
    for key in COUNTERS:
        if c_gpu[key] != c_ref[key]:
            problems.append(f"{tag}: counter {key}: gpu {c_gpu[key]} oracle {c_ref[key]}")
    return problems
