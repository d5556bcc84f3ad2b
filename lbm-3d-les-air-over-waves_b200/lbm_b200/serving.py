"""Continuous-batching request loop for solves on one GPU.

A request is a solve: a configuration (LBM_* options) and a number of
steps.  The server admits requests in arrival order while their device
memory fits the HBM budget, keeps every admitted solve's populations
resident, and advances all active solves concurrently, each on its own CUDA
stream with a few calls of `chunk` steps queued, so that their kernels
overlap on the device.  Requests that arrive while others run are admitted
as soon as memory frees up and are set up on a worker thread while the GPU
keeps stepping the others; a finished solve returns its result (the final
velocity and density fields on the host) and releases its memory.  Latency
is completion minus arrival, in wall-clock seconds.

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
    error: str | None = None     # why the solve failed (set-up or a step call raised); None when it finished

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
    """Continuous batching of solves on one GPU.

    Admission runs in arrival order while the requests' device memory fits
    the budget; a solve is built (buffers, initial state) on a worker thread,
    so setting it up overlaps the steps of the solves already on the GPU.
    Every active solve keeps `depth` calls of `chunk` steps queued on its own
    stream; a CUDA event per call tells the host loop when to queue the next
    one, so no step of the loop waits for the whole device.  A finished
    solve's result (density and velocity) is copied to pinned host memory on
    its stream, and the request completes when that copy has landed."""

    def __init__(self, device="cuda:0", budget_bytes: float = 150e9, chunk: int = 50, domain_factory=None,
                 clock=time.perf_counter, depth: int = 2, arith: str | None = None):
        self.device = device
        self.arith = arith        # "exact" / "fast" interior arithmetic of air solves (None: the library default)
        self.budget = float(budget_bytes)
        self.chunk = int(chunk)
        self.depth = max(1, int(depth))
        self.clock = clock
        self._factory = domain_factory

    # ------------------------------------------------------------------
    def _make_domain(self, env):
        if self._factory is not None:
            return self._factory(env)
        import torch

        from .domain import Domain

        dom = Domain(env, device=self.device, stream=torch.cuda.Stream(torch.device(self.device)), with_diag=False)
        if dom.cfg.physics_mode == "air" and self.arith is not None:
            dom.set_arithmetic(self.arith)
        if dom.cfg.physics_mode == "air" or (dom.cfg.free_surface_mode == "height_kinematic"
                                             and dom.cfg.free_surface_tracking_mode != "vof"):
            dom.set_step_graphs(True)   # calls of `chunk` steps replay one captured graph per call shape
        return dom

    def _build(self, env):
        t = time.perf_counter()
        dom = self._make_domain(env)
        return dom, time.perf_counter() - t

    @staticmethod
    def _issue(dom, k):
        """Queue k steps; returns an event that completes with them (None for
        stand-in domains without a stream)."""
        dom.step(k)
        stream = getattr(dom, "stream", None)
        if stream is None:
            return None
        import torch

        ev = torch.cuda.Event()
        ev.record(stream)
        return ev

    @staticmethod
    def _done(ev) -> bool:
        return ev is None or ev.query()

    @staticmethod
    def _start_result(dom):
        """Queue the result's copy to the host: (host arrays, completion event)."""
        if not hasattr(dom, "field"):
            return dom.result(), None
        import torch

        host = {}
        with torch.cuda.stream(dom.stream):
            for k in ("rho", "ux", "uy", "uz"):
                src = dom.field(k)
                dst = torch.empty(src.shape, dtype=src.dtype, pin_memory=True)
                dst.copy_(src, non_blocking=True)
                host[k] = dst
            ev = torch.cuda.Event()
            ev.record(dom.stream)
        return host, ev

    def run(self, requests, idle_sleep_s: float = 0.0005) -> dict:
        from collections import deque
        from concurrent.futures import ThreadPoolExecutor

        pending = deque(sorted(requests, key=lambda q: (q.arrival_s, q.rid)))
        need = {q.rid: domain_bytes(load_config(q.env)) for q in pending}
        for q in pending:
            if need[q.rid] > self.budget:
                raise ValueError(f"request {q.rid} needs {need[q.rid] / 1e9:.1f} GB, over the budget")
        building = deque()   # (request, future) in admission order
        active = []          # {"q", "dom", "rem", "ev": deque of events}
        finishing = []       # (request, domain, host result, event)
        used = 0.0
        finished = []
        lups = 0
        chunks = 0
        peak_active = 0
        setup_s = 0.0
        failed = []
        pool = ThreadPoolExecutor(max_workers=1)
        t0 = self.clock()

        def fail(q, dom, exc):
            nonlocal used
            q.error = f"{type(exc).__name__}: {exc}"
            q.done_s = self.clock() - t0
            if dom is not None:
                try:
                    dom.close()
                except Exception:  # noqa: BLE001 - the solve has already failed
                    pass
            used -= need[q.rid]
            failed.append(q)

        try:
            while pending or building or active or finishing:
                progress = False
                now = self.clock() - t0
                # admission in arrival order, by HBM budget
                while pending and pending[0].arrival_s <= now and used + need[pending[0].rid] <= self.budget:
                    q = pending.popleft()
                    q.admitted_s = self.clock() - t0
                    used += need[q.rid]
                    building.append((q, pool.submit(self._build, q.env)))
                    progress = True
                # solves whose set-up finished join the active set, in admission order; a
                # set-up that raised fails its request alone and releases its memory
                while building and building[0][1].done():
                    q, fut = building.popleft()
                    try:
                        dom, build_s = fut.result()
                    except Exception as exc:  # noqa: BLE001 - reported on the request
                        fail(q, None, exc)
                    else:
                        setup_s += build_s
                        active.append({"q": q, "dom": dom, "rem": q.steps, "ev": deque()})
                    progress = True
                peak_active = max(peak_active, len(active))
                # keep `depth` calls queued per solve
                still = []
                for it in active:
                    while it["ev"] and self._done(it["ev"][0]):
                        it["ev"].popleft()
                    try:
                        while it["rem"] > 0 and len(it["ev"]) < self.depth:
                            k = min(self.chunk, it["rem"])
                            it["ev"].append(self._issue(it["dom"], k))
                            it["rem"] -= k
                            chunks += 1
                            progress = True
                    except Exception as exc:  # noqa: BLE001 - a step call of this solve raised
                        fail(it["q"], it["dom"], exc)
                        progress = True
                        continue
                    if it["rem"] == 0 and not it["ev"]:
                        host, ev = self._start_result(it["dom"])
                        finishing.append((it["q"], it["dom"], host, ev))
                        progress = True
                    else:
                        still.append(it)
                active = still
                # results on the host: the request is complete, its memory is released
                rest = []
                for q, dom, host, ev in finishing:
                    if not self._done(ev):
                        rest.append((q, dom, host, ev))
                        continue
                    q.result = {k: (v.numpy() if hasattr(v, "numpy") else v) for k, v in host.items()} \
                        if isinstance(host, dict) else host
                    q.done_s = self.clock() - t0
                    cfg = dom.cfg
                    lups += cfg.Nx * cfg.Ny * cfg.Nz * q.steps
                    dom.close()
                    used -= need[q.rid]
                    finished.append(q)
                    progress = True
                finishing = rest
                if not progress:
                    if pending and not (building or active or finishing):
                        wait = pending[0].arrival_s - (self.clock() - t0)
                        if wait > 0 and idle_sleep_s:
                            time.sleep(min(wait, 0.01))
                    elif idle_sleep_s:
                        time.sleep(idle_sleep_s)
        finally:
            pool.shutdown(wait=True)
            # leaving early (an exception of the loop itself): release every solve still held
            for q, fut in building:
                if fut.done() and fut.exception() is None:
                    fut.result()[0].close()
            for it in active:
                it["dom"].close()
            for _, dom, _, _ in finishing:
                dom.close()
        wall = self.clock() - t0
        lat = np.array([q.latency_s for q in finished]) if finished else np.zeros(1)
        return {
            "requests": len(finished), "wall_s": wall, "mlups": lups / wall / 1e6 if wall > 0 else 0.0,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "rounds": chunks, "peak_active": peak_active, "setup_s": setup_s, "finished": finished,
            "failed": failed,
        }
