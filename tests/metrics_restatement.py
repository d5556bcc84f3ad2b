"""Test helper: a numpy restatement of the metric row that run_ab_case.py
computes on the host from whole fields (make_visualize, run_ab_case.py:283-596):
the maximum speed over active cells with its location and neighbourhood,
water volume and VOF accounting, surface-line statistics, and band RMS of
pressure, total pressure and vorticity on the mid-y xz slice.  Sums run in
float64; the maximum speed is taken in float32, as the reference takes it
from Taichi's float32 fields.  tests/test_metrics_golden.py pins it to the
reference's own make_visualize; tests/test_gpu_diagnostics.py checks the
device reductions against it."""
import math

import numpy as np

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1])


def high_pass_xz(field, x_periodic):
    """run_ab_case.py:111-137."""
    zp = np.empty_like(field); zm = np.empty_like(field); xp = np.empty_like(field); xm = np.empty_like(field)
    zp[:-1] = field[1:]; zp[-1] = 2.0 * field[-1] - field[-2]
    zm[1:] = field[:-1]; zm[0] = 2.0 * field[0] - field[1]
    if x_periodic:
        xp[:] = np.roll(field, -1, axis=1); xm[:] = np.roll(field, 1, axis=1)
    else:
        xp[:, :-1] = field[:, 1:]; xp[:, -1] = 2.0 * field[:, -1] - field[:, -2]
        xm[:, 1:] = field[:, :-1]; xm[:, 0] = 2.0 * field[:, 0] - field[:, 1]
    return field - 0.25 * (zp + zm + xp + xm)


def metrics_from_fields(g: dict, cfg) -> dict:
    """The metric row of run_ab_case.py:283-596 in float64 from the fields `g`
    (rho, ux, uy, uz, obstacle, phi, fs_h, fs_type, fs_fill, fs_mass,
    fs_mass_excess, pressure_reference_head; [nz][ny][nx] and [ny][nx]) and
    the options `cfg` (attributes of the solver's global names)."""
    nz, ny, nx = g["rho"].shape
    dx = float(cfg.dx)
    fs = int(cfg.water_free_surface_enabled) == 1
    vof = fs and cfg.free_surface_tracking_mode == "vof"
    xper = cfg.x_boundary_mode == "periodic"
    obs = g["obstacle"].astype(bool)
    inactive = obs.copy()
    if fs:
        inactive |= (g["fs_type"] == 0) & ~obs
    out = {}
    a, b, c = (g[k] for k in ("ux", "uy", "uz"))
    speed = np.sqrt(a * a + b * b + c * c)                        # float32, as the reference
    sp = speed * np.float32(cfg.vel_scale)
    sp = np.where(inactive, np.float32(np.nan), sp)
    idx = int(np.nanargmax(sp))
    k, j, i = np.unravel_index(idx, sp.shape)
    out.update(max_speed_phys=float(np.nanmax(sp)), max_k=int(k), max_j=int(j), max_i=int(i),
               max_speed_lb=float(speed[k, j, i]))
    if fs:
        t, f = g["fs_type"], g["fs_fill"]
        out["max_speed_fs_type"] = int(t[k, j, i])
        wet = full = gas = 0
        for q in range(1, 19):
            ni, valid = i + CX[q], True
            if xper:
                ni %= nx
            elif ni < 0 or ni >= nx:
                valid = False
            nj, nk = (j + CY[q]) % ny, k + CZ[q]
            if nk < 0 or nk >= nz:
                valid = False
            if valid and not obs[nk, nj, ni]:
                if t[nk, nj, ni] == 0:
                    gas += 1
                else:
                    wet += 1
                    full += int(f[nk, nj, ni] > 0.5)
        out.update(max_speed_wet_neighbors=wet, max_speed_full_neighbors=full, max_speed_gas_neighbors=gas)
        out["water_volume"] = float(np.where(obs, 0.0, f.astype(np.float64)).sum()) * dx ** 3
        h = g["fs_h"].astype(np.float64)
        out["surface_min"], out["surface_max"] = float(h.min()), float(h.max())
        eta = h.mean(axis=0) - float(cfg.free_surface_base_m)
        out["surface_symmetry_l2"] = float(np.sqrt(np.mean((eta - eta[::-1]) ** 2)))
        xc = (np.arange(nx) + 0.5) * dx
        left = xc < 0.5 * nx * dx
        out["surface_left_max"], out["surface_right_max"] = float(eta[left].max()), float(eta[~left].max())
        if not xper:
            hp = eta.copy()
            hp[1:-1] = eta[1:-1] - 0.5 * (eta[:-2] + eta[2:])
            hp[0] = eta[0] - eta[1]
            hp[-1] = eta[-1] - eta[-2]
        else:
            hp = eta - 0.5 * (np.roll(eta, 1) + np.roll(eta, -1))
        out["surface_eta_hp_rms"] = float(np.sqrt(np.mean(hp ** 2)))
        if vof:
            out["vof_mass_total"] = float(np.where(obs, 0.0, g["fs_mass"].astype(np.float64)).sum())
            iface = (t == 2) & ~obs
            out["vof_min_interface_fill"] = float(f[iface].min()) if iface.any() else math.nan
            thr = float(cfg.vof_empty_fill_threshold)
            out["vof_tiny_interface_count"] = int(np.count_nonzero(iface & (f > 0) & (f < thr)))
            ex = np.where(obs, 0.0, g["fs_mass_excess"].astype(np.float64))
            out["vof_pending_excess_mass"] = float(ex.sum())
            out["vof_pending_excess_count"] = int(np.count_nonzero(np.abs(ex) > 1e-12))
    # the xz slice at Ny // 2
    mj = ny // 2
    obs_xz = inactive[:, mj, :]
    ux_xz, uz_xz = a[:, mj, :].astype(np.float64), c[:, mj, :].astype(np.float64)
    if not xper:
        dv = np.empty_like(uz_xz)
        dv[:, 1:-1] = (uz_xz[:, 2:] - uz_xz[:, :-2]) / 2.0
        dv[:, 0] = uz_xz[:, 1] - uz_xz[:, 0]
        dv[:, -1] = uz_xz[:, -1] - uz_xz[:, -2]
    else:
        dv = (np.roll(uz_xz, -1, axis=1) - np.roll(uz_xz, 1, axis=1)) / 2.0
    du = (np.roll(ux_xz, -1, axis=0) - np.roll(ux_xz, 1, axis=0)) / 2.0
    vort = dv - du
    z = ((np.arange(nz) + 0.5) * dx)[:, None] * np.ones((1, nx))
    rho_phys, grav = float(cfg.rho_phys), float(cfg.gravity_phys)
    plb = rho_phys * float(np.float32(cfg.vel_scale)) ** 2 * ((g["rho"][:, mj, :].astype(np.float64) -
                                                               float(np.float32(cfg.rho0))) / 3.0)
    column = fs and not vof
    if fs:
        surf = g["fs_h"][mj, :].astype(np.float64)[None, :]
        if cfg.use_component_balanced_pressure == 1:
            pt = plb + rho_phys * grav * g["pressure_reference_head"][:, mj, :].astype(np.float64)
            pp = pt
        elif cfg.use_hydrostatic_balanced_pressure == 1:
            pt = plb + rho_phys * grav * (float(np.float32(cfg.free_surface_base_m)) - z)
            pp = plb if column else pt
        else:
            pt = plb
            pp = pt - rho_phys * grav * np.maximum(surf - z, 0.0) if column else pt
    else:
        pt = pp = plb
    phi = g["phi"][:, mj, :]
    band = (phi > 0.0) & (phi <= 10.0 * dx) & ~obs_xz
    vals = {"p": pp, "p_hp": high_pass_xz(pp, xper), "p_total": pt, "p_total_hp": high_pass_xz(pt, xper),
            "vort": vort, "vort_hp": high_pass_xz(vort, xper)}

    def rms(v, centred):
        return float(np.sqrt(np.mean((v - v.mean()) ** 2))) if centred else float(np.sqrt(np.mean(v ** 2)))

    def stats(mask, prefix):
        for name, v in vals.items():
            key = prefix + (name + "_rms" if not name.endswith("_hp") else name + "_rms")
            out[key] = rms(v[mask], not name.endswith("_hp")) if mask.any() else math.nan

    stats(band, "")
    out["band_cells"] = int(np.count_nonzero(band))
    if fs:
        if vof:
            fill_xz = g["fs_fill"][:, mj, :]
            seed = (fill_xz > 0.0) & (fill_xz < 1.0) & ~obs_xz
            fsb = seed.copy()
            fsb[1:, :] |= seed[:-1, :]
            fsb[:-1, :] |= seed[1:, :]
            fsb[:, 1:] |= seed[:, :-1]
            fsb[:, :-1] |= seed[:, 1:]
            fsb &= ~obs_xz
        else:
            fsb = (z <= surf + 0.5 * dx) & (z >= surf - 3.0 * dx) & ~obs_xz
        stats(fsb, "fs_")
        out["fs_band_cells"] = int(np.count_nonzero(fsb))
    return out
