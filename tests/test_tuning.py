"""The interior kernel's autotuner: it times candidate planes-per-block on a
live domain, applies the fastest, and the solution stays the one the CPU
oracle computes (the chunk length changes the work split, not the result)."""
import pytest

pytestmark = pytest.mark.gpu


def test_autotuned_chunk_keeps_the_oracle_result():
    from gpu_compare import compare_states
    from lbm_b200.config import air_wave_env
    from lbm_b200.domain import Domain
    from lbm_b200.tuning import autotune_tile_chunk
    from oracle_runner import OracleSim

    env = air_wave_env(64, 32, 48, amp=3.0, level=6.0, wavelength=32.0)
    ref = OracleSim(env)
    dom = Domain(env, device="cuda:0", noise=ref.arrays["init_noise"], rho_initial=ref.arrays["rho_initial"])
    res = autotune_tile_chunk(dom, candidates=(8, 16, 32), steps=2, repeats=1)
    assert res["chunk"] in (8, 16, 32) and set(res["ms_per_step"]) == {8, 16, 32}
    steps = dom.counters()["step"]
    ref.step(steps)
    dom.step(4)
    ref.step(4)
    dom.synchronize()
    problems = compare_states(dom, ref, "tuned")
    assert not problems, "\n".join(problems[:10])
    dom.close()
