"""CUDA library vs CPU oracle, bit for bit, through the C ABI.

Both backends start from identical inputs (the same initial noise and
initial density) and are advanced in calls of 1, 3 and 4 steps (the CUDA
library's rotated step loop has distinct first/middle/last passes).  After
each call every state buffer, the exported link geometry and the counters
must be identical: the library is compiled with -fmad=false and follows the
oracle's operation order, so f32 results agree exactly.
"""
import pytest

import numpy as np

from golden_compare import golden_cases, golden_state, is_injected, load_golden, load_state_numpy
from gpu_compare import compare_states
from lbm_b200.config import air_wave_env, vof_block_env, water_gaussian_env
from oracle_runner import OracleSim

pytestmark = pytest.mark.gpu

GOLDEN_ENVS = golden_cases()
# golden cases built so that a rarely reached reference kernel acts: the
# counters that must be non-zero in the GPU run as well
TRIGGERED = {
    "vof_features_kbc": ("free_surface_vof_orphan_count", "free_surface_vof_detached_advect_count",
                         "free_surface_vof_detached_compress_count", "free_surface_vof_collapse_cell_count",
                         "free_surface_thin_gap_bridge_count"),
    "vof_features_regularized": ("free_surface_vof_orphan_count", "free_surface_vof_detached_advect_count",
                                 "free_surface_vof_detached_compress_count", "free_surface_vof_collapse_cell_count",
                                 "free_surface_thin_gap_bridge_count"),
}


def load_state_torch(dom, state: dict):
    """Write a golden state into a domain's device buffers."""
    import torch

    cur = "f1" if dom.counters()["current_f"] else "f0"
    for name, v in state.items():
        dst = dom.arrays[cur] if name == "f" else dom.arrays[name]
        dst.copy_(torch.from_numpy(np.ascontiguousarray(v.reshape(tuple(dst.shape)))).to(dst.dtype))
    torch.cuda.synchronize(dom.device)


def _run_pair(env, chunks=(1, 3, 4), state=None, watch=()):
    """Run the CUDA library and the oracle from the same inputs (or from
    `state`, a golden snapshot written into both after init) and compare
    after each call; `watch` counters are summed over the calls."""
    from lbm_b200.domain import Domain

    ref = OracleSim(env)
    dom = Domain(env, device="cuda:0", noise=ref.arrays["init_noise"], rho_initial=ref.arrays["rho_initial"])
    if state is not None:
        load_state_numpy(ref.arrays, "f1" if ref.counters()["current_f"] else "f0", state)
        load_state_torch(dom, state)
    # an edited state has no geometry pass of its own yet: the derived fields
    # (pressure reference of the last step) are compared from the first step on
    problems = compare_states(dom, ref, "init", diag=state is None)
    seen = {k: 0 for k in watch}
    for n in chunks:
        for _ in range(n if watch else 1):
            k = 1 if watch else n
            ref.step(k)
            dom.step(k)
            dom.synchronize()
            c = dom.counters()
            for key in watch:
                seen[key] += c[key]
        problems += compare_states(dom, ref, f"after+{n}")
    dom.close()
    ref.close()
    return problems, seen


@pytest.mark.parametrize("name", GOLDEN_ENVS)
def test_gpu_matches_oracle_golden_configs(name):
    data, env = load_golden(name)
    state = golden_state(data, "s0") if is_injected(data) else None
    watch = TRIGGERED.get(name, ())
    problems, seen = _run_pair(env, state=state, watch=watch)
    assert not problems, "\n".join(problems[:20])
    for key in watch:
        assert seen[key] > 0, f"{key} never acted on the GPU ({seen})"


def test_gpu_matches_oracle_air_wave_benchmark_shape():
    # the benchmark's air configuration at a small size
    problems, _ = _run_pair(air_wave_env(48, 16, 24, amp=3.0, level=6.0, wavelength=24.0), chunks=(1, 5, 10))
    assert not problems, "\n".join(problems[:20])


def test_gpu_matches_oracle_water_gaussian_benchmark_shape():
    problems, _ = _run_pair(water_gaussian_env(48, 8, 24, depth=12.0, amp=3.0, sigma=6.0, g_lb=1e-3),
                         chunks=(1, 4, 7))
    assert not problems, "\n".join(problems[:20])


def test_gpu_matches_oracle_vof_block_benchmark_shape():
    """The VOF falling-block configuration at a small size, FP32 storage,
    with the trapped-gas collapse every 3 steps (flood fill, FP64 sums)."""
    env = vof_block_env(32, 8, 40, storage="f32", depth=10.0, block=8.0, bottom=20.0)
    env["LBM_VOF_COLLAPSE_INTERVAL"] = "3"
    problems, _ = _run_pair(env, chunks=(1, 3, 5))
    assert not problems, "\n".join(problems[:20])


def test_gpu_matches_oracle_c1_air_1000_steps():
    """The plain air configuration at its stated size and length: 128x64x64,
    regularized + Smagorinsky, moving sinusoidal bed z = 8 + 4 sin(2 pi (x -
    0.02 t)/64), uniform u = (0.05, 0, 0) plus seeded noise of 1e-3, 1000
    steps.  Populations, moments, flags and counters bit-equal to the oracle
    after steps 1, 10, 100 and 1000."""
    env = air_wave_env(128, 64, 64, amp=4.0, level=8.0, wavelength=64.0, speed=0.02, inflow=0.05)
    problems, _ = _run_pair(env, chunks=(1, 9, 90, 900))
    assert not problems, "\n".join(problems[:20])


def test_gpu_matches_oracle_vof_falling_block_400_steps():
    """A falling-block VOF case shaped like the benchmark's (KBC, component-
    balanced pressure, solid x walls, thin-gap bridge 4), reduced so that the
    block reaches the pool within the run: 48x16x64, pool depth 16, block of
    8 cells from 24, g = 1e-3, trapped-gas collapse every 20 steps, 400 steps.
    The collapse applies, orphans are removed, detached cells are advected and
    the bridge acts (counters summed over the run); flags, fills, masses,
    flood-fill labels and populations are bit-equal to the oracle after steps
    1, 10, 100, 200 and 400."""
    env = vof_block_env(48, 16, 64, storage="f32", depth=16.0, block=8.0, bottom=24.0, g_lb=1e-3)
    env["LBM_VOF_COLLAPSE_INTERVAL"] = "20"
    watch = ("free_surface_vof_collapse_cell_count", "free_surface_vof_orphan_count",
             "free_surface_vof_detached_advect_count", "free_surface_thin_gap_bridge_count")
    problems, seen = _run_pair(env, chunks=(1, 9, 90, 100, 200), watch=watch)
    assert not problems, "\n".join(problems[:20])
    for key in watch:
        assert seen[key] > 0, f"{key} never acted ({seen})"


@pytest.mark.parametrize("variant", ["les", "no_les", "kbc", "small_chunks", "classic", "classic_no_les", "tile_copies",
                                     "tile_copies_kbc", "cp_async"])
def test_gpu_tile_path_matches_oracle(variant, monkeypatch):
    """nx, ny multiples of 16 and periodic x: interior planes run on the
    tile kernel (the pipelined one for FP32, or the classic one), the planes
    next to the bed and the top on the general kernels."""
    env = air_wave_env(64, 32, 48, amp=3.0, level=6.0, wavelength=32.0)
    if variant.startswith("tile_copies") or variant == "cp_async":
        # 4 x 4 tiles: the inner 2 x 2 are staged by tile copies (TMA), the
        # edge tiles by cp.async (or every tile by cp.async)
        env = air_wave_env(64, 64, 40, amp=3.0, level=6.0, wavelength=32.0)
        if variant == "tile_copies_kbc":
            env["LBM_COLLISION"] = "kbc"
        if variant == "cp_async":
            monkeypatch.setenv("LBM_B200_TILE_KERNEL", "pipe")
    if variant == "no_les":
        env["LBM_USE_LES"] = "0"
    elif variant == "kbc":
        env["LBM_COLLISION"] = "kbc"
    elif variant == "small_chunks":
        monkeypatch.setenv("LBM_B200_TILE_CHUNK", "7")
    if variant.startswith("classic"):
        monkeypatch.setenv("LBM_B200_TILE_KERNEL", "classic")
        if variant == "classic_no_les":
            env["LBM_USE_LES"] = "0"
    problems, _ = _run_pair(env, chunks=(1, 2, 6))
    assert not problems, "\n".join(problems[:20])


def test_tile_copy_wait_timeout_reports_status_and_recovers(monkeypatch):
    """The bounded mbarrier wait of the tile-copy kernel.  With the test
    switch set, the first wait of every block gives up at once: the block
    waits (bounded) for the copies it has in flight, leaves, and the launch
    reports status bit 2.  No copy is skipped, so the GPU and the process
    stay usable: a fresh domain then matches the oracle bit for bit."""
    from lbm_b200.domain import Domain

    env = air_wave_env(64, 64, 40, amp=3.0, level=6.0, wavelength=32.0)   # 2 x 2 tiles on tile copies
    monkeypatch.setenv("LBM_B200_TEST_TMA_TIMEOUT", "1")
    dom = Domain(env, device="cuda:0")
    dom.step(3)       # steps 2 and 3 are fused steps: tile-copy launches
    dom.synchronize()
    flags = dom.counters()["status_flags"]
    dom.close()
    assert flags & 4, flags
    monkeypatch.delenv("LBM_B200_TEST_TMA_TIMEOUT")
    problems, _ = _run_pair(env, chunks=(1, 3))
    assert not problems, "\n".join(problems[:20])


def test_gpu_step_chunking_is_invisible():
    """Ten steps in one call equal ten calls of one step."""
    from lbm_b200.domain import Domain
    import torch

    env = air_wave_env(32, 8, 16, amp=2.0, level=4.0, wavelength=16.0)
    a = Domain(env)
    b = Domain(env)
    a.step(10)
    for _ in range(10):
        b.step(1)
    a.synchronize()
    b.synchronize()
    assert torch.equal(a.f(), b.f())
    for name in ("rho", "ux", "uy", "uz", "omega", "water_h"):
        assert torch.equal(a.field(name), b.field(name)), name


@pytest.mark.parametrize("les", [True, False])
@pytest.mark.parametrize("storage", ["f16s", "bf16s"])
def test_gpu_16bit_pipelined_kernel_equals_classic(storage, les, monkeypatch):
    """The pipelined 16-bit interior kernel (pair-wise staging) and the
    unpipelined one compute the same arithmetic on the same stored values:
    their results must be identical bit for bit."""
    import numpy as np
    import torch

    from lbm_b200.domain import Domain

    env = air_wave_env(64, 32, 48, amp=3.0, level=6.0, wavelength=32.0, storage=storage)
    env["LBM_USE_LES"] = "1" if les else "0"
    out = {}
    for kernel in ("pipelined", "classic"):
        if kernel == "classic":
            monkeypatch.setenv("LBM_B200_TILE_KERNEL", "classic")
        else:
            monkeypatch.delenv("LBM_B200_TILE_KERNEL", raising=False)
        dom = Domain(env, device="cuda:0")
        dom.step(1)
        dom.step(5)
        dom.synchronize()
        out[kernel] = {k: dom.field(k).cpu().numpy().copy() for k in ("rho", "ux", "uy", "uz", "omega")}
        f = dom.f()
        out[kernel]["f"] = (f.view(torch.int16) if f.element_size() == 2 else f).cpu().numpy().copy()
        assert dom.counters()["status_flags"] == 0
        dom.close()
    for k in out["classic"]:
        a, b = out["pipelined"][k], out["classic"][k]
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k


@pytest.mark.parametrize("storage", ["f32", "f16s", "bf16s"])
def test_gpu_tile_copy_kernel_equals_cp_async_kernel(storage, monkeypatch):
    """The interior kernel staged by tile copies (TMA) and the one staged by
    cp.async compute the same arithmetic: identical results, bit for bit,
    on a domain with 6 x 5 tiles (12 staged by tile copies) over 12 steps,
    for FP32 and for 16-bit population storage."""
    import numpy as np
    import torch

    from lbm_b200.domain import Domain

    env = air_wave_env(96, 80, 56, amp=3.0, level=6.0, wavelength=48.0, storage=storage)
    out = {}
    for kernel in ("tile_copies", "pipe"):
        if kernel == "pipe":
            monkeypatch.setenv("LBM_B200_TILE_KERNEL", "pipe")
        else:
            monkeypatch.delenv("LBM_B200_TILE_KERNEL", raising=False)
        dom = Domain(env, device="cuda:0")
        dom.step(2)
        dom.step(10)
        dom.synchronize()
        out[kernel] = {k: dom.field(k).cpu().numpy().copy() for k in ("rho", "ux", "uy", "uz", "omega")}
        f = dom.f()
        out[kernel]["f"] = (f.view(torch.int16) if f.element_size() == 2 else f).cpu().numpy().copy()
        assert dom.counters()["status_flags"] == 0
        dom.close()
        torch.cuda.synchronize()
    for k in out["pipe"]:
        assert np.array_equal(out["tile_copies"][k].view(np.uint8), out["pipe"][k].view(np.uint8)), k


@pytest.mark.parametrize("variant", ["tiles", "small", "backscatter", "water", "water_kbc_backscatter"])
def test_gpu_step_graphs_equal_eager_calls(variant):
    """Calls replayed from captured step graphs equal eager calls bit for
    bit.  The call lengths cover both step parities and both population
    buffers, first captures and later replays; the backscatter variants
    take their random-kick key from the device step clock.  The water
    variants run the kinematic height path (solid x walls)."""
    import numpy as np
    import torch

    from lbm_b200.domain import Domain

    if variant == "small":
        env = air_wave_env(32, 16, 24, amp=2.0, level=5.0, wavelength=16.0)
    elif variant.startswith("water"):
        env = water_gaussian_env(64, 16, 32, depth=16.0, amp=2.0, sigma=6.0, g_lb=1e-3)
        if variant == "water_kbc_backscatter":
            env["LBM_COLLISION"] = "kbc"
            env["LBM_BACKSCATTER"] = "0.02"
    else:
        env = air_wave_env(64, 64, 40, amp=3.0, level=6.0, wavelength=32.0)
    if variant == "backscatter":
        env["LBM_BACKSCATTER"] = "0.02"
    eager, graphed = Domain(env), Domain(env)
    graphed.set_step_graphs(True)
    for n in (1, 5, 6, 5, 4, 5, 6, 5, 1, 1):
        eager.step(n)
        graphed.step(n)
        eager.synchronize()
        graphed.synchronize()
        ce, cg = eager.counters(), graphed.counters()
        assert ce["step"] == cg["step"] and ce["current_f"] == cg["current_f"], n
        assert cg["status_flags"] == 0
        assert torch.equal(eager.f(), graphed.f()), (n, ce["step"])
        names = ("rho", "ux", "uy", "uz", "omega", "water_h")
        if variant.startswith("water"):
            names += ("fs_h", "fs_fill")
        for k in names:
            a, b = eager.field(k).cpu().numpy(), graphed.field(k).cpu().numpy()
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (n, k)
    eager.close()
    graphed.close()


@pytest.mark.parametrize("storage", ["f32", "f16s", "bf16s"])
def test_gpu_general_stash_equals_recomputed_stream(storage, monkeypatch):
    """The general planes' collide reads the pre-pass's post-condition
    populations back (FP32: from the destination slots; 16-bit storage:
    from an FP32 stash) instead of repeating the stream and bed conditions.
    Both give the same populations, bit for bit."""
    import numpy as np
    import torch

    from lbm_b200.domain import Domain

    env = air_wave_env(64, 32, 40, amp=3.0, level=6.0, wavelength=32.0, storage=storage)
    out = {}
    for mode in ("stash", "recompute"):
        if mode == "recompute":
            monkeypatch.setenv("LBM_B200_NO_STASH", "1")
        else:
            monkeypatch.delenv("LBM_B200_NO_STASH", raising=False)
        dom = Domain(env, device="cuda:0")
        dom.step(1)
        dom.step(7)
        dom.synchronize()
        f = dom.f()
        out[mode] = [(f.view(torch.int16) if f.element_size() == 2 else f).cpu().numpy().copy()]
        out[mode] += [dom.field(k).cpu().numpy().copy() for k in ("rho", "ux", "uy", "uz", "omega")]
        assert dom.counters()["status_flags"] == 0
        dom.close()
    for a, b in zip(out["stash"], out["recompute"]):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))
