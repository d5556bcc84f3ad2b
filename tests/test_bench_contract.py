"""bench.py's reference arm (the CPU restatement of the step on the host
cores) keeps the bench line's contract: one JSON line with the metric, the
configuration of the GPU arm, "impl": "reference", a cpu_baseline object
describing the run and an e2e object with no copies; under torchrun only
rank 0 works and prints."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(extra_env=None):
    env = dict(os.environ)
    env.update(extra_env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)


def test_reference_arm_prints_one_contract_line():
    p = _run()
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, p.stdout
    rec = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config"):
        assert key in rec, key
    assert rec["impl"] == "reference" and rec["metric"] == "MLUPS" and rec["unit"] == "MLUPS"
    assert rec["higher_is_better"] is True and rec["steps"] == 1 and rec["warmup"] == 0 and rec["value"] > 0
    assert rec["config"]["workload"].startswith("air over moving wave") and rec["config"]["cells"] == 512 * 256 * 256
    cb = rec["cpu_baseline"]
    assert cb["value"] == rec["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["sample"]
    assert rec["e2e"] == {"value": rec["value"], "unit": rec["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    p = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert not [ln for ln in p.stdout.splitlines() if ln.strip().startswith("{")]


def test_reference_arm_times_the_stated_configs():
    """--mode configs on the reference arm: the oracle on each stated-size
    configuration, one JSON line with MLUPS per configuration."""
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--mode", "configs",
                        "--only", "C1", "--steps", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    rec = json.loads([ln for ln in p.stdout.splitlines() if ln.strip().startswith("{")][-1])
    assert rec["impl"] == "reference" and rec["mode"] == "configs" and rec["cpu_baseline"]["cores"] >= 1
    c1 = rec["configs"]["C1"]
    assert c1["cells"] == 128 * 64 * 64 and c1["steps"] == 1 and c1["value"] > 0 and c1["unit"] == "MLUPS"
