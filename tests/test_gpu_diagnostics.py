"""Device-side harness metrics (lbm_diagnostics) against the host formulas.

run_ab_case.py computes its per-plot metric row on the host from whole
fields (make_visualize, run_ab_case.py:283-596) and main() its health line
(CODEX.py:3930-3937).  metrics_restatement.py restates those formulas in
numpy, in float64 (pinned to the reference's own make_visualize by
tests/test_metrics_golden.py); here it runs on the fields pulled from the
device, and the device reductions must agree: exactly for locations, types and counts, to 1e-9
relative for sums and statistics (both sides are FP64 over the same float32
fields; the reference's own float32 numpy differs by rounding only).
"""
import math

import pytest

from golden_compare import golden_state, load_golden
from metrics_restatement import metrics_from_fields
from lbm_b200.config import air_wave_env, vof_block_env, water_gaussian_env

pytestmark = pytest.mark.gpu


def host_metrics(dom):
    """The restated metric row from the device fields."""
    dom.export_diagnostics()
    dom.synchronize()
    g = {k: dom.field(k).cpu().numpy() for k in ("rho", "ux", "uy", "uz", "obstacle", "phi", "water_h", "fs_h",
                                                 "fs_type", "fs_fill", "fs_mass", "fs_mass_excess",
                                                 "pressure_reference_head")}
    return metrics_from_fields(g, dom.cfg)


EXACT = {"max_k", "max_j", "max_i", "max_speed_fs_type", "max_speed_wet_neighbors", "max_speed_full_neighbors",
         "max_speed_gas_neighbors", "vof_tiny_interface_count", "vof_pending_excess_count", "band_cells",
         "fs_band_cells", "max_speed_phys", "max_speed_lb", "surface_min", "surface_max"}


def _check(dom):
    dev = dom.diagnostics()
    host = host_metrics(dom)
    for key, v in host.items():
        d = dev[key]
        if key in EXACT or (isinstance(v, float) and math.isnan(v)):
            assert (d == v) or (math.isnan(d) and math.isnan(v)), (key, d, v)
        else:
            assert abs(d - v) <= 1e-9 * max(1.0, abs(v)), (key, d, v)
    return dev


def test_diagnostics_air():
    from lbm_b200.domain import Domain

    dom = Domain(air_wave_env(64, 32, 40, amp=3.0, level=6.0, wavelength=32.0), device="cuda:0")
    dom.step(20)
    dev = _check(dom)
    assert dev["band_cells"] > 0 and math.isnan(dev["water_volume"]) and dev["max_speed_fs_type"] == -1
    dom.close()


def test_diagnostics_water_height():
    from lbm_b200.domain import Domain

    dom = Domain(water_gaussian_env(48, 8, 24, depth=12.0, amp=3.0, sigma=6.0, g_lb=1e-3), device="cuda:0")
    dom.step(15)
    dev = _check(dom)
    assert dev["fs_band_cells"] > 0 and dev["water_volume"] > 0
    dom.close()


def test_diagnostics_vof_block_and_features():
    from lbm_b200.domain import Domain
    from test_gpu_parity import load_state_torch

    env = vof_block_env(32, 8, 40, storage="f32", depth=10.0, block=8.0, bottom=20.0)
    dom = Domain(env, device="cuda:0")
    dom.step(12)
    _check(dom)
    dom.close()
    # the edited VOF state (trapped gas, droplets), after one step
    data, env = load_golden("vof_features_kbc")
    dom = Domain(env, device="cuda:0")
    load_state_torch(dom, golden_state(data, "s0"))
    dom.step(1)
    dev = _check(dom)
    assert dev["vof_mass_total"] > 0
    dom.close()


def test_health_line_pulls_no_fields(monkeypatch, capsys):
    """The facade's health line takes its maximum speed from the device
    reduction: no field is copied to the host for it."""
    import types

    from lbm_b200 import facade

    env = air_wave_env(32, 16, 24, amp=3.0, level=6.0, wavelength=32.0)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    mod = types.ModuleType("solver")
    facade.install(mod.__dict__)
    pulled = []
    orig = facade.Field.to_numpy
    monkeypatch.setattr(facade.Field, "to_numpy", lambda self: pulled.append(self.name) or orig(self))
    mod.steps, mod.plot_freq, mod.plot_step_start = 100, 1000, 0
    mod.main()
    assert pulled == []
    assert "Time Step 100, Max |U| (LB units) =" in capsys.readouterr().out
    mod._engine.dom.close()
