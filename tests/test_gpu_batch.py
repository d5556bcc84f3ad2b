"""Ensembles stepped with one launch per phase (lbm_batch_*) against the same
domains stepped one by one.

The batched kernels run the same per-block bodies as a domain's own launches
(the interior planes through the cp.async-staged tile bodies, taken from a
work queue), so the populations, moments, relaxation rates and counters of
every domain must be bit-equal to stepping it alone with lbm_step.
"""
import pytest
import torch

from lbm_b200.batch import Batch, ensemble_envs
from lbm_b200.config import air_wave_env, water_gaussian_env
from lbm_b200.domain import Domain

pytestmark = pytest.mark.gpu


def _small_ensemble(n, storage, seed=11):
    envs = ensemble_envs(n, seed=seed, storage=storage)
    for e in envs:   # small versions of the ensemble shapes, whole waves in x
        nx = min(int(e["LBM_LX_M"]), 96)
        e["LBM_LX_M"] = str(nx)
        e["LBM_LY_M"] = str(min(int(e["LBM_LY_M"]), 64))
        e["LBM_LZ_M"] = str(min(int(e["LBM_LZ_M"]), 48))
        e["LBM_BED_WAVELENGTH_M"] = repr(nx / max(1, round(nx / float(e["LBM_BED_WAVELENGTH_M"]))))
        e["LBM_BED_AMP_M"] = repr(min(float(e["LBM_BED_AMP_M"]), 0.07 * float(e["LBM_BED_WAVELENGTH_M"])))
    return envs


def _same(a, b):
    assert torch.equal(a.f(), b.f())
    for name in ("rho", "ux", "uy", "uz", "omega", "water_h", "u_wave", "w_wave"):
        assert torch.equal(a.field(name), b.field(name)), name
    ca, cb = a.counters(), b.counters()
    for key in ("boundary_cut_link_count", "status_flags", "step", "current_f"):
        assert ca[key] == cb[key], key


@pytest.mark.parametrize("storage", ["f32", "f16s"])
def test_batched_ensemble_equals_domains_alone(storage):
    envs = _small_ensemble(6, storage)
    batch = Batch(envs, chunk=10, graphs=False, queue=True)
    alone = [Domain(e, device="cuda:0", with_diag=False) for e in envs]
    for k in (1, 3, 4):
        batch.step(k)
        batch.synchronize()
        for d in alone:
            d.step(k)
            d.synchronize()
        for a, b in zip(batch.domains, alone):
            _same(a, b)
    # the domains' own calls between batch calls keep them in step (same call
    # boundaries on both sides: with 16-bit storage the post-stream state is
    # rounded to its storage at the end of each call)
    batch.step_each(2)
    batch.synchronize()
    batch.step(5)
    batch.synchronize()
    for d in alone:
        d.step(2)
        d.step(5)
        d.synchronize()
    for a, b in zip(batch.domains, alone):
        _same(a, b)
        assert a.counters()["step"] == 15
    batch.close()
    for d in alone:
        d.close()


def test_batch_refuses_unsupported_domains():
    envs = [air_wave_env(64, 32, 32), water_gaussian_env(64, 16, 32, depth=16.0, amp=2.0, sigma=6.0, g_lb=1e-3)]
    with pytest.raises(RuntimeError, match="air domains only"):
        Batch(envs, queue=True)


def _stable_mixed_envs():
    """Four uneven air domains with moderate beds, one of them KBC; each
    stays finite on the CPU oracle over 40 steps (maximum speed 0.04-0.07,
    minimum density above 0.98)."""
    envs = [air_wave_env(96, 64, 48, amp=3.0, level=8.0, wavelength=48.0, speed=0.02, inflow=0.05, seed=21),
            air_wave_env(64, 48, 40, amp=2.0, level=8.0, wavelength=32.0, speed=0.01, inflow=0.03, seed=22),
            air_wave_env(80, 64, 32, amp=4.0, level=9.0, wavelength=80.0, speed=0.015, inflow=0.06, seed=23),
            air_wave_env(128, 32, 48, amp=1.5, level=8.0, wavelength=64.0, speed=0.025, inflow=0.04, seed=24)]
    envs[2]["LBM_COLLISION"] = "kbc"
    return envs


def test_batched_fast_arithmetic_within_rounding_of_exact():
    """An ensemble on the fast arithmetic of the interior planes stays within
    rounding of the same ensemble on the exact arithmetic (the bound of the
    FP32 form, 1e-5 relative to the flow's maximum), with the same geometry,
    for regularized and KBC domains in one work queue."""
    envs = _stable_mixed_envs()
    exact = Batch(envs, chunk=10, graphs=False, queue=True, arith="exact")
    fast = Batch(envs, chunk=10, graphs=False, queue=True, arith="fast")
    assert all(d.arithmetic() == "fast" for d in fast.domains)
    exact.step(20)
    fast.step(20)
    exact.synchronize()
    fast.synchronize()
    for a, b in zip(exact.domains, fast.domains):
        assert a.counters()["status_flags"] == 0
        assert b.counters()["status_flags"] == 0
        u = torch.stack([a.field(k) for k in ("ux", "uy", "uz")]).double()
        v = torch.stack([b.field(k) for k in ("ux", "uy", "uz")]).double()
        assert float(u.abs().max()) < 0.2
        rel = float((u - v).abs().max() / u.abs().max())
        assert rel <= 1e-5, rel
        assert torch.equal(a.field("water_h"), b.field("water_h"))
    exact.close()
    fast.close()
