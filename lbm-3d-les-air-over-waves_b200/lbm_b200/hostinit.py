"""Host-side initial-condition helpers (setup, runs once, not timed).

prepare_initial_density restates the reference's host numpy routine
prepare_initial_density_field (LBM_3D_LES_air_over_waves_CODEX.py:743-818):
the initial density column from the free-surface height, including the
linear-wave (finite-depth FFT / cosine-series) pressure mode.

make_init_noise produces the uniform [-1, 1) draws that replace the
reference's ti.random() kick in init_fields (CODEX.py:2747); with
LBM_B200_INIT_VELOCITY=uniform the three components are the velocity
noise of the benchmark configurations.
"""
from __future__ import annotations

import numpy as np


def make_init_noise(cfg, seed: int | None = None) -> np.ndarray:
    seed = cfg.random_seed if seed is None else seed
    rng = np.random.default_rng(seed)
    return rng.uniform(-1.0, 1.0, size=(3, cfg.Nz, cfg.Ny, cfg.Nx)).astype(np.float32)


def linear_wave_heads(eta: np.ndarray, dx: float, bed: float, depth: float, z, solid_x: bool) -> list:
    """Pressure heads of linear finite-depth wave theory under the surface
    elevation eta(x) (cell centres, spacing dx), at each height in z: the
    modes of eta (a cosine series for walls at x = 0 and Lx, Fourier modes for
    periodic x), each scaled by cosh(k z_rel) / cosh(k depth) with z_rel =
    z - bed clipped to [0, depth].  One row of len(eta) per height; the
    reference evaluates the same theory for its linear-wave initial pressure
    (CODEX.py:754-803) and its linear-pressure diagnostic
    (run_ab_case.py:52-108)."""
    nx = len(eta)
    x = (np.arange(nx, dtype=np.float64) + 0.5) * dx

    def vertical_factor(wavenumbers, zc):
        z_rel = min(max(zc - bed, 0.0), depth)
        factor = np.ones_like(wavenumbers)
        active = wavenumbers > 0.0
        kh = wavenumbers[active] * depth
        kz = wavenumbers[active] * z_rel
        # cosh(k z_rel) / cosh(k h), written with decaying exponentials
        factor[active] = (np.exp(kz - kh) + np.exp(-kz - kh)) / (1.0 + np.exp(-2.0 * kh))
        return factor

    if solid_x:
        # cosine series for walls at x = 0 and x = Lx
        kx = np.arange(nx, dtype=np.float64) * np.pi / (nx * dx)
        basis = np.cos(np.outer(kx, x))
        coeff = (2.0 / nx) * (basis @ eta)
        coeff[0] = np.mean(eta)
        return [coeff @ (vertical_factor(kx, zc)[:, None] * basis) for zc in z]
    modes = np.fft.rfftfreq(nx, d=dx) * 2.0 * np.pi
    eta_hat = np.fft.rfft(eta)
    return [np.fft.irfft(eta_hat * vertical_factor(modes, zc), n=nx) for zc in z]


def prepare_initial_density(cfg, fs_h: np.ndarray, water_h: np.ndarray) -> np.ndarray:
    """rho_initial[k, j, i] (float32) from the column heights at t = 0."""
    Nx, Ny, Nz, dx = cfg.Nx, cfg.Ny, cfg.Nz, cfg.dx
    rho0, g_lb = cfg.rho0, cfg.g_lb
    base = cfg.free_surface_base_m
    rho_np = np.full((Nz, Ny, Nx), rho0, dtype=np.float32)
    if cfg.water_free_surface_enabled != 1:
        return rho_np
    h_np = np.asarray(fs_h, dtype=np.float64)
    bed_np = np.asarray(water_h, dtype=np.float64)
    z = (np.arange(Nz, dtype=np.float64) + 0.5) * dx
    balanced = cfg.use_hydrostatic_balanced_pressure == 1
    use_linear = (
        cfg.initial_pressure_mode == "linear_wave"
        and cfg.free_surface_initial_condition == "gaussian"
        and np.allclose(bed_np, bed_np[0, 0], atol=1.0e-12, rtol=0.0)
    )
    if use_linear:
        bed = float(bed_np[0, 0])
        depth0 = max(base - bed, dx)
        eta = h_np.mean(axis=0) - base
        heads = linear_wave_heads(eta, dx, bed, depth0, z, cfg.x_boundary_mode == "solid")
        for kk, zc in enumerate(z):
            head = heads[kk]
            if not balanced:
                head = np.maximum((base - zc) + head, 0.0)
            line = rho0 + g_lb * head / dx / (1.0 / 3.0)
            rho_np[kk, :, :] = line.astype(np.float32)[None, :]
        return rho_np
    for kk, zc in enumerate(z):
        if balanced:
            head = h_np - base
        else:
            head = np.maximum(h_np - zc, 0.0)
        plane = rho0 + g_lb * head / dx / (1.0 / 3.0)
        rho_np[kk, :, :] = np.asarray(plane, dtype=np.float32)
    return rho_np
