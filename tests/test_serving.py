"""Batched ensemble and the continuous-batching request loop.

CPU tests drive the server's admission and round logic with stand-in
domains and a stand-in clock.  The GPU tests run real solves: a small
ensemble steps as one batch, and every request of a mixed trace gives the
same result alone as in the mix (bit for bit: solves share no state).
"""
import numpy as np
import pytest

from lbm_b200.batch import domain_bytes, ensemble_envs
from lbm_b200.config import load_config
from lbm_b200.serving import Request, Server, poisson_trace


class _Clock:
    def __init__(self, dt=0.001):
        self.t = 0.0
        self.dt = dt

    def __call__(self):
        self.t += self.dt
        return self.t


class _FakeDomain:
    live = 0
    peak = 0
    live_bytes = 0
    peak_bytes = 0

    def __init__(self, env):
        self.cfg = load_config(env)
        self.steps = 0
        self.bytes = domain_bytes(self.cfg)
        _FakeDomain.live += 1
        _FakeDomain.peak = max(_FakeDomain.peak, _FakeDomain.live)
        _FakeDomain.live_bytes += self.bytes
        _FakeDomain.peak_bytes = max(_FakeDomain.peak_bytes, _FakeDomain.live_bytes)

    def step(self, k):
        self.steps += k

    def synchronize(self):
        pass

    def result(self):
        return {"steps": self.steps}

    def close(self):
        _FakeDomain.live -= 1
        _FakeDomain.live_bytes -= self.bytes


def test_ensemble_is_seeded_and_uneven():
    a, b = ensemble_envs(96, seed=7), ensemble_envs(96, seed=7)
    assert a == b
    shapes = {(e["LBM_LX_M"], e["LBM_LY_M"], e["LBM_LZ_M"]) for e in a}
    assert len(shapes) > 50
    for e in a:
        assert all(int(e[k]) % 16 == 0 for k in ("LBM_LX_M", "LBM_LY_M", "LBM_LZ_M"))
    cells = sum(int(e["LBM_LX_M"]) * int(e["LBM_LY_M"]) * int(e["LBM_LZ_M"]) for e in a)
    assert 60e6 < cells < 250e6


def test_trace_is_seeded_and_poisson_like():
    t1, t2 = poisson_trace(200, seed=3), poisson_trace(200, seed=3)
    assert [(q.arrival_s, q.steps) for q in t1] == [(q.arrival_s, q.steps) for q in t2]
    gaps = np.diff([0.0] + [q.arrival_s for q in t1])
    assert 0.03 < gaps.mean() < 0.08          # rate 20/s
    assert all(500 <= q.steps <= 5000 for q in t1)


def test_server_admits_by_budget_and_finishes_every_request():
    reqs = poisson_trace(12, rate_hz=200.0, seed=5, cells_range=(2e4, 6e4), steps_range=(40, 200))
    need = max(domain_bytes(load_config(q.env)) for q in reqs)
    _FakeDomain.live = _FakeDomain.peak = _FakeDomain.live_bytes = _FakeDomain.peak_bytes = 0
    budget = 2.2 * need
    srv = Server(budget_bytes=budget, chunk=25, domain_factory=_FakeDomain, clock=_Clock())
    rep = srv.run(reqs, idle_sleep_s=0.0)
    assert rep["requests"] == 12
    assert _FakeDomain.peak_bytes <= budget and _FakeDomain.live == 0
    assert _FakeDomain.peak >= 2          # solves overlap
    for q in rep["finished"]:
        assert q.result["steps"] == q.steps
        assert q.admitted_s >= q.arrival_s and q.done_s > q.admitted_s
    # arrival order is admission order
    adm = sorted(rep["finished"], key=lambda q: q.admitted_s)
    assert [q.rid for q in adm] == sorted(q.rid for q in adm)
    assert rep["p99_s"] >= rep["p50_s"] > 0


def test_a_failing_solve_fails_its_request_alone():
    """A set-up that raises and a step call that raises each fail their own
    request (error recorded, memory released); the other requests finish."""
    reqs = poisson_trace(8, rate_hz=200.0, seed=9, cells_range=(2e4, 6e4), steps_range=(40, 200))
    bad_build, bad_step = reqs[2].rid, reqs[5].rid
    by_env = {id(q.env): q.rid for q in reqs}

    class Flaky(_FakeDomain):
        def __init__(self, env):
            if by_env[id(env)] == bad_build:
                raise RuntimeError("set-up refused")
            super().__init__(env)
            self.rid = by_env[id(env)]

        def step(self, k):
            if self.rid == bad_step and self.steps > 0:
                raise RuntimeError("step refused")
            super().step(k)

    _FakeDomain.live = _FakeDomain.peak = _FakeDomain.live_bytes = _FakeDomain.peak_bytes = 0
    need = max(domain_bytes(load_config(q.env)) for q in reqs)
    rep = Server(budget_bytes=2.2 * need, chunk=25, domain_factory=Flaky, clock=_Clock()).run(reqs, idle_sleep_s=0.0)
    assert sorted(q.rid for q in rep["failed"]) == sorted([bad_build, bad_step])
    assert {q.rid: q.error for q in rep["failed"]} == {bad_build: "RuntimeError: set-up refused",
                                                        bad_step: "RuntimeError: step refused"}
    assert rep["requests"] == 6 and all(q.error is None and q.result["steps"] == q.steps for q in rep["finished"])
    assert _FakeDomain.live == 0 and _FakeDomain.live_bytes == 0


def test_server_rejects_a_request_over_the_budget():
    q = poisson_trace(1, seed=1, cells_range=(1e6, 1e6))[0]
    with pytest.raises(ValueError):
        Server(budget_bytes=1e6, domain_factory=_FakeDomain).run([q])


@pytest.mark.gpu
def test_batch_steps_every_domain():
    import torch

    from lbm_b200.batch import Batch

    envs = ensemble_envs(6, seed=11)
    for e in envs:                     # small versions of the ensemble shapes, whole waves in x
        nx = min(int(e["LBM_LX_M"]), 96)
        e["LBM_LX_M"] = str(nx)
        e["LBM_LY_M"] = str(min(int(e["LBM_LY_M"]), 48))
        e["LBM_LZ_M"] = str(min(int(e["LBM_LZ_M"]), 48))
        e["LBM_BED_WAVELENGTH_M"] = repr(nx / max(1, round(nx / float(e["LBM_BED_WAVELENGTH_M"]))))
        e["LBM_BED_AMP_M"] = repr(min(float(e["LBM_BED_AMP_M"]), 0.07 * float(e["LBM_BED_WAVELENGTH_M"])))
    b = Batch(envs, chunk=10)
    b.step(30)
    b.synchronize()
    for d in b.domains:
        c = d.counters()
        assert c["step"] == 30 and c["status_flags"] == 0
        assert torch.isfinite(d.field("ux")).all()
    b.close()


@pytest.mark.gpu
def test_each_result_is_the_same_alone_and_in_the_mix():
    reqs = poisson_trace(5, rate_hz=100.0, seed=9, cells_range=(3e4, 1.2e5), steps_range=(30, 90))
    mixed = Server(budget_bytes=8e9, chunk=20).run(reqs)
    assert mixed["requests"] == 5 and mixed["peak_active"] >= 2
    by_id = {q.rid: q for q in mixed["finished"]}
    for q in reqs[:3]:
        alone_q = Request(q.rid, 0.0, q.env, q.steps)
        alone = Server(budget_bytes=8e9, chunk=20).run([alone_q])["finished"][0]
        for k in ("rho", "ux", "uy", "uz"):
            a, m = alone.result[k], by_id[q.rid].result[k]
            assert a.shape == m.shape
            assert np.array_equal(a.view(np.uint32), m.view(np.uint32)), (q.rid, k)
