"""The drop-in solver module: loaded by path the way run_ab_case.py loads a
solver (run_ab_case.py:261-280), driven through steps / plot_freq /
plot_step_start / visualize / main() (899-912), read through module globals,
.to_numpy() fields and [None] counters (283-679)."""
import importlib.util
import math
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODULE = os.path.join(ROOT, "lbm-3d-les-air-over-waves_b200", "LBM_3D_LES_air_over_waves_B200.py")


def _load(env, monkeypatch, label="t"):
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    spec = importlib.util.spec_from_file_location(f"lbm_ab_{label}", MODULE)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_module_surface_matches_the_reference_globals(monkeypatch):
    from lbm_b200.config import air_wave_env

    m = _load(air_wave_env(64, 16, 32), monkeypatch)
    assert (m.Nx, m.Ny, m.Nz) == (64, 16, 32) and m.dx == 1.0
    assert m.FS_GAS == 0 and m.FS_INTERFACE == 2
    assert np.allclose(m.x_phys, (np.arange(64) + 0.5) * m.dx)
    assert m.X_phys.shape == (32, 16, 64) and m.Z_phys[3, 0, 0] == 3.5
    assert list(m.cx.to_numpy()) == [0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0]
    assert m.boundary_cut_link_count[None] == 0
    for name in ("Lx_m", "Ly_m", "Lz_m", "vel_scale", "U_ref_phys", "rho0", "rho_air_phys", "free_surface_base_m",
                 "water_free_surface_enabled", "free_surface_tracking_mode", "x_boundary_mode",
                 "use_hydrostatic_balanced_pressure", "use_component_balanced_pressure", "vof_empty_fill_threshold",
                 "include_cube_geometry", "cube_side_m", "cube_yaw_sin", "cube_pitch_cos", "steps", "plot_freq",
                 "plot_step_start", "Re_phys_air", "Re_lb_base", "gravity_phys"):
        assert hasattr(m, name), name
    assert callable(m.main) and callable(m.visualize)


def _harness_wrap(ti, random_seed):
    """What run_ab_case.py:261-273 does to taichi.init before loading a solver."""
    original_init = ti.init

    def init_with_seed(*args, **kwargs):
        kwargs.setdefault("random_seed", random_seed)
        return original_init(*args, **kwargs)

    ti.init = init_with_seed


def test_seed_comes_from_the_harness_when_it_wrapped_taichi_init(monkeypatch):
    import sys
    import types

    from lbm_b200.config import air_wave_env

    def never(*args, **kwargs):
        raise AssertionError("the module must not start Taichi")

    fake = types.ModuleType("taichi")
    fake.init = never
    _harness_wrap(fake, 777)
    monkeypatch.setitem(sys.modules, "taichi", fake)
    env = dict(air_wave_env(32, 16, 16), LBM_RANDOM_SEED="5")
    assert _load(env, monkeypatch, "harness_seed").random_seed == 777
    monkeypatch.delitem(sys.modules, "taichi")
    assert _load(env, monkeypatch, "env_seed").random_seed == 5


def test_visualize_before_a_harness_binds_one_raises_like_the_reference(monkeypatch):
    from lbm_b200.config import air_wave_env

    m = _load(air_wave_env(32, 16, 16), monkeypatch, "unbound")
    with pytest.raises(RuntimeError, match="Visualization has not been configured"):
        m.visualize(100, 1.0, 1.0, 1.0)


def test_direct_run_writes_the_harness_metrics_csv(monkeypatch, tmp_path, capsys):
    """configure_direct_visualization binds a visualize that writes one CSV row
    per plot in the harness's columns (the device record comes from a
    stand-in engine here; its values are checked in test_metrics_golden)."""
    import csv
    import types

    from lbm_b200 import facade
    from lbm_b200.abi import COUNTER_FLOAT_NAMES, COUNTER_INT_NAMES, DIAG_FIELDS
    from lbm_b200.config import water_gaussian_env

    import torch

    m = _load(water_gaussian_env(32, 8, 16), monkeypatch, "direct")
    rec = {name: 0 if ctype.__name__.startswith("c_int") else 0.25 for name, ctype in DIAG_FIELDS}
    rec.update(max_i=3, max_j=1, max_k=5)
    counters = dict({k: 7 for k in COUNTER_INT_NAMES}, **{k: 0.5 for k in COUNTER_FLOAT_NAMES}, step=100)
    nz, ny, nx = m.Nz, m.Ny, m.Nx
    gen = torch.Generator().manual_seed(3)
    z = (torch.arange(nz) + 0.5) * m.dx
    level = 0.6 * nz * float(m.dx)
    fields = {  # a flat bed at 2 m, a surface at 0.6 of the height, a perturbed density
        "water_h": torch.full((ny, nx), 2.0),
        "fs_h": level + 0.2 * torch.rand(ny, nx, generator=gen),
        "rho": 1.0 + 1e-3 * torch.rand(nz, ny, nx, generator=gen),
        "phi": (z - 2.0)[:, None, None].expand(nz, ny, nx).clone(),
        "obstacle": (z < 2.0)[:, None, None].expand(nz, ny, nx).to(torch.int32),
        "fs_type": (z < level)[:, None, None].expand(nz, ny, nx).to(torch.int32),
    }
    dom = types.SimpleNamespace(cfg=m._engine.cfg, diagnostics=lambda: rec, counters=lambda: counters,
                                field=fields.__getitem__, synchronize=lambda: None, export_diagnostics=lambda: None)
    monkeypatch.setattr(m._engine, "domain", lambda: dom)
    monkeypatch.setenv("LBM_OUTPUT_DIR", str(tmp_path))
    monkeypatch.setenv("LBM_RUN_LABEL", "direct_t")
    fh = facade.configure_direct_visualization(vars(m))
    m.visualize(100, 1.5, 1.0, 1.0)
    m.visualize(200, 3.0, 1.0, 1.0)
    fh.close()
    with open(tmp_path / "direct_t_metrics.csv", newline="") as f:
        rows = list(csv.DictReader(f))
    assert [r["step"] for r in rows] == ["100", "200"]
    assert tuple(rows[0]) == facade.METRIC_FIELDNAMES
    dx = float(m.dx)
    assert float(rows[0]["max_speed_x"]) == 3.5 * dx and float(rows[0]["max_speed_z"]) == 5.5 * dx
    assert rows[0]["cut_links"] == "7" and rows[0]["vof_excess_count"] == "-1" and rows[0]["vof_mass_total"] == "nan"
    assert all(math.isfinite(float(rows[0][k])) for k in facade.LINEAR_RESIDUAL_COLUMNS)
    assert capsys.readouterr().out.count("[direct_t] Boundary band <=10 cells:") == 2


class _OracleEngine:
    """The CPU oracle behind the drop-in module's engine interface (test
    stand-in for the CUDA Domain): same state arrays, same step calls; the
    health line's maximum speed is reduced on the host as the reference does."""

    def __init__(self, env, noise):
        from oracle_runner import OracleSim

        self.sim = OracleSim(env, noise=noise)
        self.cfg = self.sim.cfg

    def initialize(self):
        pass   # OracleSim ran the init sequence

    def step(self, n):
        self.sim.step(n)

    def counters(self):
        return self.sim.counters()

    def diagnostics(self, slice_j=None):
        a = self.sim.arrays
        active = a["obstacle"] == 0
        if int(self.cfg.water_free_surface_enabled) == 1:
            active &= a["fs_type"] != 0
        speed = np.sqrt(a["ux"] ** 2 + a["uy"] ** 2 + a["uz"] ** 2)
        return {"max_speed_lb": float(np.nanmax(speed[active]))}

    def export_diagnostics(self):
        self.sim.export()

    def synchronize(self):
        pass


@pytest.mark.parametrize("case", ["air_kbc_default", "vof_block_kbc"])
def test_main_loop_prints_the_reference_health_line(monkeypatch, capsys, case):
    """The drop-in module's main() driven like the reference's loop, with the
    CPU oracle as its engine, prints at step 100 the health line the
    reference printed for the same case (tests/golden/long)."""
    import json

    from golden_compare import GOLDEN_DIR

    data = np.load(os.path.join(GOLDEN_DIR, "long", f"{case}.npz"))
    env = json.loads(str(data["env"]))
    m = _load(env, monkeypatch, f"oracle_{case}")
    m._engine.dom = _OracleEngine(env, data["noise"])
    m.steps, m.plot_freq, m.plot_step_start = 100, 1000, 0
    m.main()
    out = capsys.readouterr().out.splitlines()
    assert [ln for ln in out if ln.startswith("Time Step")] == [str(data["health"][0])]
    assert out[-1] == "Simulation Complete."
    m._engine.dom.sim.close()


@pytest.mark.gpu
def test_main_drives_the_engine_like_the_reference_loop(monkeypatch, capsys):
    from lbm_b200.config import air_wave_env
    from lbm_b200.domain import Domain

    env = air_wave_env(64, 16, 32, amp=2.0, level=6.0, wavelength=32.0)
    m = _load(env, monkeypatch, "main")
    m.steps, m.plot_freq, m.plot_step_start = 120, 40, 0
    seen = []

    def visualize(step, time_phys, re_phys, re_lb):
        seen.append((step, m.ux.to_numpy().copy(), m.obstacle.to_numpy().copy(), m.boundary_cut_link_count[None]))

    m.visualize = visualize
    m.main()
    out = capsys.readouterr().out
    assert [s[0] for s in seen] == [40, 80, 120]
    assert "Time Step 100, Max |U|" in out and "Simulation Complete." in out
    assert seen[-1][1].shape == (32, 16, 64) and seen[-1][2].dtype == np.int32
    assert seen[-1][3] > 0
    # the same 120 steps through the engine directly: identical fields
    dom = Domain(env, device="cuda:0")
    dom.step(40)
    dom.step(40)
    dom.step(40)
    dom.synchronize()
    a = dom.field("ux").cpu().numpy()
    assert np.array_equal(a.view(np.uint32), seen[-1][1].view(np.uint32))
    dom.close()
    m._engine.dom.close()
