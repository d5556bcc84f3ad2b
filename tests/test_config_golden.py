"""The LBM_* option surface against the reference's own module globals.

tests/golden/config_cases.json holds, for each set of options, the scalar
globals that importing LBM_3D_LES_air_over_waves_CODEX.py produced (or the
exception the import raised); gen_config_golden.py beside it made the file.
load_config must give every one of those globals under the same name with
the same value, and raise the same exception class with the same message
for every invalid set (CODEX.py:35-529, lbm_env.py:9-22)."""
import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from gen_config_golden import CASES, materialize, unplace  # noqa: E402

from lbm_b200.config import load_config  # noqa: E402
from lbm_b200.facade import run_summary, tau_line  # noqa: E402

with open(os.path.join(HERE, "golden", "config_cases.json"), encoding="utf-8") as _fh:
    GOLDEN = json.load(_fh)["cases"]

# the fixture covers every valid and invalid case the generator defines
assert sorted(c["name"] for c in GOLDEN) == sorted(CASES)


def _ours(value):
    if hasattr(value, "tolist"):
        return value.tolist()
    return value


def _equal(ref, ours) -> bool:
    if isinstance(ref, bool) or isinstance(ours, bool):
        return bool(ref) == bool(ours) and int(ref) == int(ours)
    if isinstance(ref, float) and isinstance(ours, (int, float)):
        # same operations in the same order: equal to the last bit
        return ref == float(ours) or (ref != ref and ours != ours)
    if isinstance(ref, list):
        return isinstance(ours, list) and len(ref) == len(ours) and all(_equal(a, b) for a, b in zip(ref, ours))
    if isinstance(ref, dict):
        return isinstance(ours, dict) and ref.keys() == ours.keys() and all(_equal(ref[k], ours[k]) for k in ref)
    return ref == ours


@pytest.mark.parametrize("case", GOLDEN, ids=[c["name"] for c in GOLDEN])
def test_options_match_the_reference_module(case, tmp_path):
    options, placeholders = materialize(case["env"], case["files"], str(tmp_path))
    if "error" in case:
        kind = {"ValueError": ValueError, "FileNotFoundError": FileNotFoundError}[case["error"]["type"]]
        with pytest.raises(Exception) as info:
            load_config(options)
        assert type(info.value) is kind
        assert unplace(str(info.value), placeholders) == case["error"]["message"]
        return
    cfg = load_config(options)
    missing = sorted(set(case["values"]) - set(cfg.values))
    assert not missing, f"reference globals without a counterpart: {missing}"
    wrong = []
    for name, ref in case["values"].items():
        ours = _ours(cfg.values[name])
        if isinstance(ours, str):
            ours = unplace(ours, placeholders)
        if isinstance(ours, dict):
            ours = {k: unplace(v, placeholders) if isinstance(v, str) else _ours(v) for k, v in ours.items()}
        if not _equal(ref, ours):
            wrong.append((name, ref, ours))
    assert not wrong, wrong


def test_golden_covers_every_error_message_of_the_option_surface():
    """Each distinct ValueError text of load_config occurs in some invalid case."""
    import inspect
    import re

    from lbm_b200 import config

    src = inspect.getsource(config.load_config) + inspect.getsource(config._load_piecewise_bed)
    fixed = set(re.findall(r'raise ValueError\(\s*"(LBM_[A-Z0-9_]+) must', src))
    seen = {c["error"]["message"].split(" ")[0] for c in GOLDEN if "error" in c}
    ours_only = {"LBM_B200_TAU0", "LBM_B200_INIT_U0", "LBM_B200_TOP"}   # build options, not in the reference
    assert fixed - ours_only <= seen, sorted(fixed - ours_only - seen)


PRINTED = [c for c in GOLDEN if "main_stdout" in c]


@pytest.mark.parametrize("case", PRINTED, ids=[c["name"] for c in PRINTED])
def test_printed_lines_match_the_reference(case, tmp_path):
    """The line the module prints at import and the configuration summary
    its main() prints after initialisation (CODEX.py:471, 3794-3871, 3957),
    line for line, as the reference printed them for the same options."""
    options, placeholders = materialize(case["env"], case["files"], str(tmp_path))
    cfg = load_config(options)
    assert [tau_line(cfg)] == case["import_stdout"]
    ours = [unplace(ln, placeholders) for ln in run_summary(cfg)] + ["Simulation Complete."]
    assert ours == case["main_stdout"]


def test_printed_cases_cover_every_mode():
    names = {c["name"] for c in PRINTED}
    assert {"air_piecewise_bed", "air_cube_yaw_pitch", "water_gaussian_hydrostatic_boundary", "vof_options",
            "vof_block_total_pressure_corrected"} <= names
