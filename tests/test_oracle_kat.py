"""Known-answer tests of the oracle, derived from the mathematics of the
scheme rather than from the reference's outputs:

  - populations set to equilibrium carry the prescribed moments: sum f = rho,
    sum f c = rho u, sum f c c = rho (u u + I/3) (Hermite equilibrium,
    CODEX.py:623-643, and the D3Q19 weights and velocities of
    lbm_lattice.py:3-43);
  - a flat bed at height h gives open fraction 0.5 + (0 - h)/dx on every
    downward link of the bottom plane (the half-link endpoint sits at z = 0;
    CODEX.py:2492-2686);
  - still water under gravity with a hydrostatic-balanced pressure stays at
    rest with its volume (height-function path);
  - a flat VOF pool has no trapped gas: the collapse finds candidate volume
    0 at every step, and the mass exchange conserves the pool's mass.

The GPU library is bit-equal to the oracle on the golden and parity cases,
so these hold for it too."""
import numpy as np
import pytest

from lbm_b200.config import air_wave_env, vof_block_env, water_gaussian_env
from oracle_runner import OracleSim

CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, -1, 1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1])


def _flat_air(level: float, inflow=(0.05, 0.01, -0.02)):
    env = air_wave_env(32, 16, 24, amp=0.0, level=level, speed=0.0)
    env.update(LBM_BED_PROFILE="flat", LBM_B200_INIT_NOISE="0",
               LBM_B200_INIT_U0=",".join(repr(float(v)) for v in inflow))
    return env


def test_lattice_tables_are_a_d3q19_set():
    c = np.stack([CX, CY, CZ], axis=1)
    opp = [int(np.flatnonzero((c == -c[q]).all(axis=1))[0]) for q in range(19)]
    assert all(opp[opp[q]] == q for q in range(19)) and len(set(map(tuple, c))) == 19
    assert sorted(np.abs(c).sum(axis=1).tolist()) == [0] + [1] * 6 + [2] * 12


def test_equilibrium_populations_carry_their_moments():
    u0 = np.array([0.05, 0.01, -0.02])
    sim = OracleSim(_flat_air(0.0, tuple(u0)))
    try:
        f = sim.f().astype(np.float64)
        rho = sim.arrays["rho"].astype(np.float64)
        assert np.abs(f.sum(0) / rho - 1.0).max() <= 1e-6
        c = (CX, CY, CZ)
        for a in range(3):
            ja = np.tensordot(c[a], f, 1)
            assert np.abs(ja / rho - u0[a]).max() <= 1e-6 * max(abs(u0[a]), 1e-2)
            for b in range(a, 3):
                pab = np.tensordot(c[a] * c[b], f, 1)
                want = rho * (u0[a] * u0[b] + (1.0 / 3.0 if a == b else 0.0))
                assert np.abs(pab - want).max() <= 1e-6, (a, b)
    finally:
        sim.close()


@pytest.mark.parametrize("level", [0.0, 0.25])
def test_flat_bed_open_fraction_of_the_bottom_links(level):
    sim = OracleSim(_flat_air(level))
    try:
        sim.export()
        frac = sim.arrays["lattice_open_frac"]
        for q in np.flatnonzero(CZ == -1):
            assert np.all(frac[q, 0] == np.float32(0.5 - level)), (q, np.unique(frac[q, 0]))
    finally:
        sim.close()


def test_still_water_stays_at_rest():
    env = water_gaussian_env(32, 4, 32, depth=16.0, amp=0.0, sigma=4.0, g_lb=1e-5, tau0=0.51)
    sim = OracleSim(env)
    try:
        a = sim.arrays
        h0 = a["fs_h"].astype(np.float64).sum()
        sim.step(100)
        speed = np.sqrt(a["ux"].astype(np.float64) ** 2 + a["uy"] ** 2 + a["uz"] ** 2)
        # free fall over the run would reach g t = 1e-3
        assert speed.max() <= 1e-5
        assert abs(a["fs_h"].astype(np.float64).sum() / h0 - 1.0) <= 1e-5
        assert np.abs(a["fs_h"] - 16.0).max() <= 1e-4
    finally:
        sim.close()


def test_flat_vof_pool_has_no_trapped_gas_and_keeps_its_mass():
    env = vof_block_env(32, 4, 48, storage="f32", depth=16.0)
    env.update(LBM_VOF_INITIAL_SHAPE="none", LBM_VOF_COLLAPSE_INTERVAL="1",
               LBM_PRESSURE_FORMULATION="hydrostatic_balanced")
    sim = OracleSim(env)
    try:
        a = sim.arrays
        m0 = a["fs_mass"].astype(np.float64).sum()
        for _ in range(4):
            sim.step(5)
            c = sim.counters()
            assert c["free_surface_vof_collapse_candidate_volume_m3"] == 0.0
            assert c["free_surface_vof_collapse_cell_count"] == 0
        assert abs(a["fs_mass"].astype(np.float64).sum() / m0 - 1.0) <= 1e-5
        speed = np.sqrt(a["ux"].astype(np.float64) ** 2 + a["uy"] ** 2 + a["uz"] ** 2)
        assert speed.max() <= 1e-5
    finally:
        sim.close()
