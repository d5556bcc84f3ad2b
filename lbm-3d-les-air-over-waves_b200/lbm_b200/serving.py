"""Continuous-batching request loop for solves on one GPU.

A request is a solve: a configuration (LBM_* options) and a number of
steps.  The server admits requests in arrival order while their device
memory fits the HBM budget, keeps every admitted solve's populations
resident, and advances all active solves together in rounds of `chunk`
steps, each solve on its own CUDA stream so that their kernels overlap on
the device.  Requests that arrive while others run are admitted at the next
round boundary as soon as memory frees up; a finished solve returns its
result (the final velocity and density fields on the host) and releases its
memory.  Latency is completion minus arrival, in wall-clock seconds.

    reqs = poisson_trace(24, rate_hz=20, seed=3)
    report = Server(budget_bytes=150e9).run(reqs)
    report["p50_s"], report["p99_s"], report["mlups"]
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from .batch import domain_bytes
from .config import air_wave_env, load_config, water_gaussian_env


@dataclass
class Request:
    rid: int
    arrival_s: float
    env: dict
    steps: int
    # filled in by the server
    admitted_s: float = -1.0
    done_s: float = -1.0
    result: dict = field(default_factory=dict)

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


def poisson_trace(n: int, rate_hz: float = 20.0, seed: int = 3, cells_range=(1e5, 2e7), steps_range=(500, 5000),
                  storage: str = "f16s") -> list[Request]:
    """Seeded arrival trace: Poisson arrivals, half air-over-wave and half
    water-Gaussian solves, cell counts log-uniform in cells_range, step
    counts uniform in steps_range.  Domain shapes are multiples of 16."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in range(n):
        t += float(rng.exponential(1.0 / rate_hz))
        cells = float(np.exp(rng.uniform(np.log(cells_range[0]), np.log(cells_range[1]))))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        # aspect 4 : 2 : 1.5 -> nx = (cells / 3)^(1/3) * 4 / ... rounded to 16
        base = (cells / 12.0) ** (1.0 / 3.0)
        nx = max(32, int(round(4 * base / 16)) * 16)
        ny = max(16, int(round(2 * base / 16)) * 16)
        nz = max(32, int(round(1.5 * base / 16)) * 16)
        if rng.uniform() < 0.5:
            # whole waves per periodic domain, bed slope at most 0.44
            wavelength = nx / max(1, round(nx / 64.0))
            env = air_wave_env(nx, ny, nz, storage=storage, seed=100 + r, wavelength=wavelength,
                               amp=round(min(4.0, 0.07 * wavelength), 3))
        else:
            depth = float(max(8, nz // 2))
            env = water_gaussian_env(nx, ny, nz, storage=storage, depth=depth, amp=min(8.0, depth / 4),
                                     sigma=float(max(4, nx // 16)), g_lb=1e-5)
        out.append(Request(r, t, env, steps))
    return out


class Server:
    def __init__(self, device="cuda:0", budget_bytes: float = 150e9, chunk: int = 50, domain_factory=None,
                 clock=time.perf_counter):
        self.device = device
        self.budget = float(budget_bytes)
        self.chunk = int(chunk)
        self.clock = clock
        self._factory = domain_factory

    # ------------------------------------------------------------------
    def _make_domain(self, env):
        if self._factory is not None:
            return self._factory(env)
        import torch

        from .domain import Domain

        dom = Domain(env, device=self.device, stream=torch.cuda.Stream(torch.device(self.device)), with_diag=False)
        if dom.cfg.physics_mode == "air":
            dom.set_step_graphs(True)   # rounds of `chunk` steps replay one captured graph per call shape
        return dom

    @staticmethod
    def _result(dom) -> dict:
        if hasattr(dom, "field"):
            return {k: dom.field(k).detach().cpu().numpy() for k in ("rho", "ux", "uy", "uz")}
        return dom.result()

    def run(self, requests, idle_sleep_s: float = 0.0005) -> dict:
        pending = sorted(requests, key=lambda q: (q.arrival_s, q.rid))
        need = {q.rid: domain_bytes(load_config(q.env)) for q in pending}
        for q in pending:
            if need[q.rid] > self.budget:
                raise ValueError(f"request {q.rid} needs {need[q.rid] / 1e9:.1f} GB, over the budget")
        active = []          # [request, domain, remaining steps]
        used = 0.0
        finished = []
        lups = 0
        t0 = self.clock()
        rounds = 0
        peak_active = 0
        setup_s = 0.0
        while pending or active:
            now = self.clock() - t0
            # admission in arrival order, by HBM budget
            while pending and pending[0].arrival_s <= now and used + need[pending[0].rid] <= self.budget:
                q = pending.pop(0)
                ts = self.clock()
                dom = self._make_domain(q.env)
                q.admitted_s = self.clock() - t0
                setup_s += self.clock() - ts
                used += need[q.rid]
                active.append([q, dom, q.steps])
            if not active:
                if pending:
                    wait = pending[0].arrival_s - (self.clock() - t0)
                    if wait > 0:
                        time.sleep(min(wait, 0.01) if idle_sleep_s else 0)
                continue
            peak_active = max(peak_active, len(active))
            # one round: every active solve advances up to `chunk` steps
            for item in active:
                k = min(self.chunk, item[2])
                item[1].step(k)
                item[2] -= k
            for item in active:
                item[1].synchronize()
            rounds += 1
            still = []
            for item in active:
                q, dom, rem = item
                if rem > 0:
                    still.append(item)
                    continue
                q.result = self._result(dom)
                q.done_s = self.clock() - t0
                cfg = dom.cfg
                lups += cfg.Nx * cfg.Ny * cfg.Nz * q.steps
                dom.close()
                used -= need[q.rid]
                finished.append(q)
            active = still
        wall = self.clock() - t0
        lat = np.array([q.latency_s for q in finished]) if finished else np.zeros(1)
        return {
            "requests": len(finished), "wall_s": wall, "mlups": lups / wall / 1e6 if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "rounds": rounds, "peak_active": peak_active, "setup_s": setup_s, "finished": finished,
        }
