"""The metric-row restatement against the reference's own make_visualize.

tests/golden/metrics_rows.json holds the rows that run_ab_case.py's
visualize callback (run_ab_case.py:283-596) computed from the seeded fields
of metrics_inputs() (gen_metrics_golden.py beside it).  The restatement in
metrics_restatement.py, which the device diagnostics are checked against,
must give the same values from the same fields: locations, types and counts
exactly, the maximum speed to float32 rounding (the restatement takes it in
float32 as Taichi's fields give it; the golden ran on float64 copies), and
sums and band statistics to 1e-9 relative.  A metric the restatement does not
produce for a mode must be the reference's not-applicable value there (NaN
or -1)."""
import json
import math
import os
import sys
import types

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from gen_metrics_golden import CASES, metrics_counters, metrics_inputs  # noqa: E402
from metrics_restatement import metrics_from_fields  # noqa: E402

from lbm_b200.abi import DIAG_FIELDS  # noqa: E402
from lbm_b200.facade import METRIC_FIELDNAMES, linear_residual_metrics, metric_row  # noqa: E402

with open(os.path.join(HERE, "golden", "metrics_rows.json"), encoding="utf-8") as _fh:
    ROWS = json.load(_fh)

RESTATED = ("max_speed_phys", "max_speed_x", "max_speed_y", "max_speed_z", "max_speed_fs_type",
            "max_speed_wet_neighbors", "max_speed_full_neighbors", "max_speed_gas_neighbors", "water_volume",
            "vof_mass_total", "vof_min_interface_fill", "vof_tiny_interface_count", "vof_pending_excess_mass",
            "vof_pending_excess_count", "surface_min", "surface_max", "surface_symmetry_l2", "surface_eta_hp_rms",
            "surface_left_max", "surface_right_max", "p_rms", "p_hp_rms", "p_total_rms", "p_total_hp_rms",
            "vort_rms", "vort_hp_rms", "fs_p_rms", "fs_p_hp_rms", "fs_p_total_rms", "fs_p_total_hp_rms",
            "fs_vort_rms", "fs_vort_hp_rms")
INTEGER = {"max_speed_fs_type", "max_speed_wet_neighbors", "max_speed_full_neighbors", "max_speed_gas_neighbors",
           "vof_tiny_interface_count", "vof_pending_excess_count"}


def test_golden_rows_cover_every_case():
    assert sorted(ROWS) == sorted(CASES)


@pytest.mark.parametrize("case", CASES)
def test_restatement_matches_the_reference_row(case):
    g, opts = metrics_inputs(case)
    ours = metrics_from_fields(g, types.SimpleNamespace(**opts))
    dx = opts["dx"]
    for axis, index in (("x", "max_i"), ("y", "max_j"), ("z", "max_k")):
        ours[f"max_speed_{axis}"] = (ours[index] + 0.5) * dx
    row = ROWS[case]
    compared = 0
    for key in RESTATED:
        ref = row[key]
        if key not in ours:
            assert ref is None or ref == -1, (key, ref)
            continue
        v = ours[key]
        if ref is None:
            assert isinstance(v, float) and math.isnan(v), (key, v)
        elif key in INTEGER:
            assert v == ref, (key, v, ref)
        elif key == "max_speed_phys":
            assert abs(v - ref) <= 2e-7 * abs(ref), (key, v, ref)
        else:
            assert abs(v - ref) <= 1e-9 * max(1.0, abs(ref)), (key, v, ref)
        compared += 1
    # every metric of the mode is compared: air has no free-surface metrics, the height path no VOF ones
    assert compared == {"air_periodic": 10, "vof_component_balanced": 32}.get(case, 27), compared


def _device_record(case):
    """A diagnostics record as lbm_diagnostics returns it, with the values of
    the restatement (every field present, whatever the mode)."""
    g, opts = metrics_inputs(case)
    ours = metrics_from_fields(g, types.SimpleNamespace(**opts))
    rec = {name: -1 if ctype.__name__.startswith("c_int") else float("nan") for name, ctype in DIAG_FIELDS}
    rec.update(ours)
    rec["max_speed_fs_fill"] = float(g["fs_fill"][ours["max_k"], ours["max_j"], ours["max_i"]])
    return rec, opts


def _linear(case):
    """linear_residual_metrics on the mid-y slices of the case's fields."""
    g, opts = metrics_inputs(case)
    mj = opts["Ny"] // 2
    obstacle = g["obstacle"][:, mj, :] != 0
    inactive = obstacle
    if opts["water_free_surface_enabled"]:
        inactive = obstacle | ((g["fs_type"][:, mj, :] == 0) & ~obstacle)
    return linear_residual_metrics(types.SimpleNamespace(**opts), g["rho"][:, mj, :], g["phi"][:, mj, :], inactive,
                                   g["fs_h"][mj, :], g["water_h"][mj, :])


@pytest.mark.parametrize("case", CASES)
def test_linear_residual_matches_the_reference_row(case):
    """The harness's finite-depth linear pressure residual (run_ab_case.py:52-108,
    505-595): present for the height-function cases, NaN for air and VOF."""
    ours, ref = _linear(case), ROWS[case]
    for key, v in ours.items():
        if ref[key] is None:
            assert math.isnan(v), (key, v)
        else:
            assert abs(v - ref[key]) <= 1e-9 * max(1.0, abs(ref[key])), (key, v, ref[key])
    assert (ref["p_linear_resid_rms"] is not None) == case.startswith("water_height")


@pytest.mark.parametrize("case", CASES)
def test_metric_row_matches_the_reference_row(case):
    """The CSV row the drop-in module writes (facade.metric_row over a device
    record, the counters and the linear-wave residual of one slice) against
    the harness's row: every column, with the same not-applicable values per
    mode."""
    rec, opts = _device_record(case)
    row = metric_row(types.SimpleNamespace(**opts), case, 40, 12.5, rec, metrics_counters(case), _linear(case))
    ref = ROWS[case]
    assert tuple(row) == METRIC_FIELDNAMES and sorted(ref) == sorted(METRIC_FIELDNAMES)
    for key in METRIC_FIELDNAMES:
        v, r = row[key], ref[key]
        if r is None:
            assert isinstance(v, float) and math.isnan(v), (key, v)
        elif isinstance(r, str) or isinstance(r, int) and not isinstance(r, bool) and key != "time_phys":
            assert v == r and type(v) is type(r), (key, v, r)
        elif key == "max_speed_phys":
            assert abs(v - r) <= 2e-7 * abs(r), (key, v, r)
        else:
            assert abs(v - r) <= 1e-9 * max(1.0, abs(r)), (key, v, r)
