"""The oracle against the reference's own kernels after 100 to 1000 steps.

tests/golden/long/<case>.npz were made by tests/golden/gen_long_golden.py:
the reference's main() runs 100 steps of every golden case, and up to 1000
steps of a few (among them air with the reference's defaults: KBC, LES,
backscatter, fringe, top drive and sponge; height-function water; the VOF
falling block with collapse and bridge; the edited VOF pools whose orphan,
detached-cell and collapse kernels act), and keeps the final state and the
health line it printed.  The oracle must reproduce the state bit for bit
(the scalar FP64 tallies to f32 rounding, as in the short goldens), and the
drop-in module's health-line formatter must print the same line from the
oracle's state.  The GPU library is bit-equal to the oracle, so this pins it
over such runs too."""
import json
import os

import numpy as np
import pytest

from golden_compare import EXACT, FIELD_MAP, FILE_OPTIONS, GOLDEN_DIR, golden_state, is_injected, load_state_numpy
from lbm_b200.facade import health_line
from oracle_runner import OracleSim

LONG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "long")
LONG = sorted(f[:-4] for f in os.listdir(LONG_DIR) if f.endswith(".npz")) if os.path.isdir(LONG_DIR) else []
INT_COUNTERS = ["boundary_cut_link_count", "free_surface_cut_link_count", "free_surface_refill_count",
                "free_surface_thin_gap_bridge_count", "free_surface_coalescence_repair_count",
                "free_surface_vof_excess_count", "free_surface_vof_orphan_count",
                "free_surface_vof_collapse_cell_count", "free_surface_vof_detached_advect_count",
                "free_surface_vof_detached_compress_count"]
FLOAT_COUNTERS = ["free_surface_vof_collapse_candidate_volume_m3", "free_surface_vof_collapse_applied_volume_m3",
                  "free_surface_vof_detached_advect_mass", "free_surface_vof_detached_compress_mass"]


def test_long_goldens_present():
    assert {"air_kbc_default", "water_height_gaussian", "vof_block_kbc"} <= set(LONG)


@pytest.mark.parametrize("name", LONG)
def test_oracle_matches_the_reference_after_a_long_run(name):
    data = np.load(os.path.join(LONG_DIR, f"{name}.npz"))
    env = json.loads(str(data["env"]))
    for key in FILE_OPTIONS:   # files stored beside the short goldens
        if key in env and not os.path.isabs(env[key]):
            env[key] = os.path.join(GOLDEN_DIR, env[key])
    n = int(data["nsteps"])
    sim = OracleSim(env, noise=data["noise"])
    try:
        if is_injected(data):
            # state edited after the reference's init: start from its s0 snapshot
            load_state_numpy(sim.arrays, "f1" if sim.counters()["current_f"] else "f0", golden_state(data, "s0"))
        sim.step(n)
        sim.export()
        arrays = dict(sim.arrays)
        arrays["f"] = sim.f()
        tag = f"s{n}"
        compared = 0
        for gname in ["f"] + list(FIELD_MAP):
            key = f"{tag}_{gname}"
            if key not in data:
                continue
            ref = data[key]
            mine = np.asarray(arrays[FIELD_MAP[gname][0] if gname != "f" else "f"]).reshape(ref.shape)
            if gname in EXACT:
                np.testing.assert_array_equal(mine.astype(np.int64), ref.astype(np.int64), err_msg=key)
            else:
                np.testing.assert_array_equal(mine.astype(np.float32), ref.astype(np.float32), err_msg=key)
            compared += 1
        assert compared >= 10
        c = sim.counters()
        for key in INT_COUNTERS:
            assert c[key] == int(data[f"{tag}_{key}"]), key
        for key in FLOAT_COUNTERS:
            np.testing.assert_allclose(c[key], float(data[f"{tag}_{key}"]), rtol=1e-5, atol=1e-9, err_msg=key)
        # the health line at step n (CODEX.py:3930-3954): maximum speed over active cells
        cfg = sim.cfg
        a = sim.arrays
        active = a["obstacle"] == 0
        if int(cfg.water_free_surface_enabled) == 1:
            active &= a["fs_type"] != 0
        speed = np.sqrt(a["ux"] ** 2 + a["uy"] ** 2 + a["uz"] ** 2)
        # a run that diverged would match vacuously (NaN states): the reference's run must still be finite
        assert np.isfinite(speed[active]).all() and np.isfinite(data[f"{tag}_f"]).all()
        line = health_line(n, np.nanmax(speed[active]), cfg.vel_scale, c)
        assert len(data["health"]) == n // 100 and line == str(data["health"][-1])
    finally:
        sim.close()
