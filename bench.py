"""Throughput of the D3Q19 air-over-moving-wave step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one time step of the whole domain: bed update, pull-stream with
the moving-wall link fractions, Smagorinsky LES and regularized collision.
Workload: air over a moving sinusoidal bed, 512x256x256 cells, FP32
populations (A-B buffers, 5.1 GB, larger than L2), regularized collision,
Smagorinsky Cs = 0.16, tau0 = 0.52, bed z = 8 + 4 sin(2 pi (x - 0.02 t)/64),
seeded synthetic initial state.  Steps run through the public C ABI in
chunks of 100 (the reference's health-report cadence); in the timed region
each chunk is one CUDA step-graph replay (--no-graphs: eager calls).

Printed (rank 0, one JSON line): MLUPS over all ranks (replicas, weak
scaling; device time, max over ranks), the roofline of the dominant kernels
(the interior grids, timed with CUDA events on their stream over the same
K steps run as eager calls right after the timed region), the end-to-end
figure through the API with host buffers, the SM
clocks sampled during the timed region, and the CPU oracle timed on a
bounded sample of the same workload.  On one GPU the same line also
carries the batched and served halves of the metric: "batched" (the
96-domain ensemble in shifted FP16, MLUPS and its ratio to the plain
figure) and "serving" (a seeded Poisson request trace through the
continuous-batching server: p50/p99 latency and aggregate MLUPS);
--plain-only skips them.

--impl reference times the reference algorithm's CPU implementation (the
FP32 C++ restatement in oracle/, OpenMP over all host cores) on a bounded
sample of the same workload; the reference itself needs Taichi, which is
not installed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.join(ROOT, "lbm-3d-les-air-over-waves_b200")
TESTS = os.path.join(ROOT, "tests")
if PKG_ROOT not in sys.path:
    sys.path.insert(0, PKG_ROOT)

NX, NY, NZ = 512, 256, 256
CHUNK = 100                 # steps per API call (health-report cadence of the reference loop)
B_ALG = 152                 # algorithmic bytes per cell update, FP32 populations read + written once (76: 16-bit)
WORKLOAD = "air over moving wave, LES regularized, 512x256x256"
METRIC, UNIT = "MLUPS", "MLUPS"
# bounded CPU samples: periodic sub-blocks of the workload with its full height
# (same bed, same vertical structure), largest first
CPU_SAMPLES = [(128, 64, 256), (64, 64, 256), (64, 32, 256), (64, 16, 256)]
# DRAM bytes per cell update of the interior grids, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum over one launch of each
# interior grid, divided by the cells of the launch).  A profile figure, not
# a live one: the source says which grid, kernels and commit it was taken on.
PROFILE_TRAFFIC = {
    "bytes_per_cell": 170.7,
    "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_tile_edges + k_tile_tma pair at 512x256x256 "
              "(this workload; one pass, --clock-control none), commit fa6d57e; profiles/k_tile_air_interior.md",
}


STORAGE = "f32"             # population storage of the plain run (--plain-storage)
ARITH = "exact"             # arithmetic of the interior kernels (--arith)


def workload_env(nx=None, ny=None, nz=None, seed=12345, storage=None):
    from lbm_b200.config import air_wave_env

    return air_wave_env(nx or NX, ny or NY, nz or NZ, storage=storage or STORAGE, seed=seed)


def base_config():
    return {
        "workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "cells": NX * NY * NZ, "collision": "regularized",
        "les": "smagorinsky Cs=0.16", "tau0": 0.52, "storage": STORAGE, "arithmetic": ARITH, "steps_per_call": CHUNK,
        "l2": (f"inputs larger than L2 ({NX * NY * NZ * B_ALG / 1e9:.2f} GB of populations, A-B)"
               if NX * NY * NZ * B_ALG > 126e6 else "inputs fit in L2 (small profiling case)"),
        "parallelism": "replicas",
    }


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        import tempfile

        fd, self.path = tempfile.mkstemp(prefix="lbm_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        # samples under load: the upper half of the clock readings, the
        # timed region being most of the sampling window
        load = sorted(sm)[len(sm) // 4:] if sm else []
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU oracle
def oracle_sample_rate(budget_s: float, max_steps: int):
    """Time the CPU oracle on a bounded sample; returns (MLUPS, sample text)."""
    if TESTS not in sys.path:
        sys.path.insert(0, TESTS)
    from oracle_runner import OracleSim

    shape = CPU_SAMPLES[0]
    sim = OracleSim(workload_env(*shape, storage="f32"))
    t0 = time.perf_counter()
    sim.step(1)
    t1 = time.perf_counter() - t0
    n = shape[0] * shape[1] * shape[2]
    steps = max(1, min(max_steps, int(budget_s / max(t1, 1e-3))))
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    sim.close()
    rate = n * steps / dt / 1e6
    sample = (f"{shape[0]}x{shape[1]}x{shape[2]} periodic sub-block of the workload (full height, same bed), "
              f"{steps} steps after 1 warm-up step, {dt:.1f} s")
    return rate, sample


def reference_configs(args):
    """The oracle on the stated-size configurations (C1 air, C2 water, C3
    VOF) on all host cores: one untimed step, then steps until a few seconds
    have passed (at most --steps), MLUPS per step extrapolated from them.
    One JSON line."""
    from oracle_runner import OracleSim

    names = args.only.split(",") if args.only else list(CONFIGS)
    out = {}
    for name in names:
        what, storage = CONFIGS[name]
        sim = OracleSim(_config_env(name, storage))
        sim.step(1)
        n = sim.cfg.Nx * sim.cfg.Ny * sim.cfg.Nz
        k, t0 = 0, time.perf_counter()
        while k < max(1, args.steps) and (k == 0 or time.perf_counter() - t0 < 10.0):
            sim.step(1)
            k += 1
        dt = time.perf_counter() - t0
        sim.close()
        out[name] = {"workload": what, "storage": storage, "cells": n, "steps": k, "ms_per_step": dt / k * 1e3,
                     "value": n * k / dt / 1e6, "unit": UNIT,
                     "sample": f"{k} steps after 1 untimed step, extrapolated per step"}
    print(json.dumps({"metric": METRIC, "mode": "configs", "impl": "reference", "n_gpus": 0, "data": "synthetic",
                      "cpu_baseline": {"kind": "port", "cores": host_cores(),
                                       "note": "FP32 C++ restatement of the reference kernels (oracle), OpenMP"},
                      "configs": out}), flush=True)
    return 0


def reference_arm(args):
    """Reference CPU implementation of the path on the host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.mode == "configs":
        if TESTS not in sys.path:
            sys.path.insert(0, TESTS)
        return reference_configs(args)
    if TESTS not in sys.path:
        sys.path.insert(0, TESTS)
    from oracle_runner import OracleSim

    cores = host_cores()
    K, W = args.steps, max(args.warmup, 0)
    budget = 150.0   # seconds for the whole run
    # pick the largest sample whose K + W steps fit the budget, from one probe step
    probe_shape = CPU_SAMPLES[0]
    sim = OracleSim(workload_env(*probe_shape, storage="f32"))
    t0 = time.perf_counter()
    sim.step(1)
    t_probe = time.perf_counter() - t0
    per_cell = t_probe / (probe_shape[0] * probe_shape[1] * probe_shape[2])
    shape = CPU_SAMPLES[-1]
    for s in CPU_SAMPLES:
        if per_cell * s[0] * s[1] * s[2] * (K + W) <= budget:
            shape = s
            break
    if shape != probe_shape:
        sim.close()
        sim = OracleSim(workload_env(*shape, storage="f32"))
    n = shape[0] * shape[1] * shape[2]
    if W:
        sim.step(W)
    t0 = time.perf_counter()
    sim.step(K)
    dt = time.perf_counter() - t0
    sim.close()
    value = n * K / dt / 1e6
    sample = f"{shape[0]}x{shape[1]}x{shape[2]} periodic sub-block of the workload (full height, same bed) per step"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": K, "warmup": W,
        "ms_per_step": dt / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": base_config(), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own solver needs Taichi (absent); timed: the FP32 C++ restatement of its "
                "kernels (oracle), OpenMP over all host cores",
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def run_steps(dom, k):
    done = 0
    while done < k:
        n = min(CHUNK, k - done)
        dom.step(n)
        done += n


def ours(args):
    import ctypes as C

    import numpy as np
    import torch

    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    from lbm_b200.replicas import Replicas

    reps = Replicas("nccl")
    world, rank, local, dev = reps.world, reps.rank, reps.local, reps.device
    barrier, max_over_ranks = reps.barrier, reps.max

    from lbm_b200.domain import Domain

    K, W = args.steps, max(args.warmup, 3)
    env = workload_env(seed=reps.seed(12345))
    dom = Domain(env, device=dev, with_diag=False)
    dom.set_arithmetic(ARITH)
    lib = dom.lib
    s = dom.stream
    ncell = NX * NY * NZ

    # ---- warm-up: pick the interior kernel's planes per block, then W steps
    from lbm_b200.tuning import autotune_tile_chunk

    if args.tile_chunk:
        dom.set_tile_chunk(args.tile_chunk)
        tuned = {"chunk": args.tile_chunk, "ms_per_step": {}}
    else:
        tuned = autotune_tile_chunk(dom)
    run_steps(dom, W)
    dom.synchronize()
    if dom.counters()["status_flags"]:
        raise SystemExit("non-finite state after warm-up")

    # ---- device-resident throughput: step-graph replays (each call of
    # CHUNK steps one graph launch; the shapes of the timed calls are
    # captured in warm-up)
    graphs = not args.no_graphs
    extra_warm = 0
    if graphs:
        # The timed region's calls are replays of captured graphs: step graphs
        # are cached per (steps per call, step parity, current buffer), and
        # two passes of the timed call sequence capture every one of them
        # (parity and buffer flip together, once per step).
        dom.set_step_graphs(True)
        run_steps(dom, K)
        run_steps(dom, K)
        extra_warm = 2 * K
        dom.synchronize()
    l0 = C.c_int64()
    lib.lbm_launch_count(C.byref(l0))
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    run_steps(dom, K)
    e1.record(s)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    l1 = C.c_int64()
    lib.lbm_launch_count(C.byref(l1))
    ms = e0.elapsed_time(e1)
    if dom.counters()["status_flags"]:
        raise SystemExit("non-finite state in the timed region")
    # ---- the dominant kernel's launches timed with events: the same K steps
    # as eager calls (events cannot be read per replay inside a graph)
    dom.set_step_graphs(False)
    dom.set_kernel_timing(True)
    barrier()
    torch.cuda.synchronize(dev)
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(s)
    run_steps(dom, K)
    r1.record(s)
    r1.synchronize()
    eager_ms = r0.elapsed_time(r1)
    k_ms, k_launches, k_cells = dom.kernel_timing()
    dom.set_kernel_timing(False)
    if dom.counters()["status_flags"]:
        raise SystemExit("non-finite state in the timed kernel pass")

    # ---- end to end through the API with host buffers: the reference's main
    # loop (initial state from the host, steps in chunks of 100, the health
    # report's velocity fields read back after every chunk)
    noise_h = torch.from_numpy(np.ascontiguousarray(dom.arrays["init_noise"].cpu().numpy())).pin_memory()
    rho_h = torch.from_numpy(np.ascontiguousarray(dom.arrays["rho_initial"].cpu().numpy())).pin_memory()
    vel_h = [torch.empty(ncell, dtype=torch.float32).pin_memory() for _ in range(3)]
    h2d = noise_h.numel() * 4 + rho_h.numel() * 4
    d2h = 0
    barrier()
    torch.cuda.synchronize(dev)
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(s)
    with torch.cuda.stream(s):
        dom.arrays["init_noise"].copy_(noise_h, non_blocking=True)
        dom.arrays["rho_initial"].copy_(rho_h, non_blocking=True)
    sp = C.c_void_p(s.cuda_stream)
    dom._check(lib.lbm_init_geometry(dom.ctx, sp), "lbm_init_geometry")
    dom._check(lib.lbm_init_fields(dom.ctx, sp), "lbm_init_fields")
    done = 0
    while done < K:
        n = min(CHUNK, K - done)
        dom.step(n)
        done += n
        with torch.cuda.stream(s):
            for h, name in zip(vel_h, ("ux", "uy", "uz")):
                h.copy_(dom.arrays[name].view(-1), non_blocking=True)
        d2h += 3 * ncell * 4
        ctr = dom.counters()     # health report: status and link counters
        if ctr["status_flags"]:
            raise SystemExit("non-finite state in the end-to-end run")
    x1.record(s)
    x1.synchronize()
    barrier()
    e2e_ms = x0.elapsed_time(x1)

    ms, e2e_ms = max_over_ranks([ms, e2e_ms])
    value = world * ncell * K / (ms * 1e-3) / 1e6
    e2e = world * ncell * K / (e2e_ms * 1e-3) / 1e6

    out = None
    if rank == 0:
        peak, peak_kind = measured_hbm_peak()
        roof = None
        if k_launches > 0 and k_ms > 0:
            per_launch_s = k_ms / k_launches * 1e-3
            achieved = B_ALG * k_cells / per_launch_s / 1e9
            tpc = PROFILE_TRAFFIC["bytes_per_cell"]
            roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": tpc * k_cells, "traffic_source": PROFILE_TRAFFIC["source"], "peak_kind": peak_kind,
                    "kernel": "k_tile_edges + k_tile_tma (interior one-pass stream+LES+collide; TMA-staged off the domain edge)", "cells_per_launch": k_cells,
                    "bytes_per_cell": B_ALG, "launch_ms": per_launch_s * 1e3,
                    "step_frac": B_ALG * value * 1e6 / world / (peak * 1e9)}
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            rate, sample = oracle_sample_rate(budget_s=12.0, max_steps=20)
            cpu = {"value": rate, "unit": UNIT, "cores": host_cores(), "kind": "port", "sample": sample}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W + extra_warm,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if STORAGE == "f32" else f"f32 compute, {STORAGE} storage", "data": "synthetic",
            "config": dict(base_config(), tile_chunk=tuned["chunk"],
                           tile_chunk_ms={str(k): round(v, 4) for k, v in tuned["ms_per_step"].items()},
                           step_graphs=graphs, eager_ms_per_step=round(eager_ms / K, 4),
                           warmup_note=(f"{W} eager warm-up steps, then {extra_warm} steps that capture the timed "
                                        f"region's step graphs; before them the autotuner's timing steps "
                                        f"({len(tuned['ms_per_step'])} chunk candidates x 13 steps)"),
                           roofline_timing="interior grids timed with CUDA events over the same K steps run as "
                                           "eager calls right after the timed region"),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K},
            "gpu_launches": int(l1.value - l0.value),
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
        }
    dom.close()
    del dom
    if out is not None and world == 1 and not args.plain_only:
        # the batched and served halves of the metric, same process and GPU
        import torch

        torch.cuda.empty_cache()
        storage = args.storage or "f16s"
        b = run_batched(args.domains, args.batched_steps, 3, storage, graphs=not args.no_graphs)
        b["vs_plain"] = b["value"] / value
        out["batched"] = b
        torch.cuda.empty_cache()
        srv = run_serving(args.requests, args.min_steps, args.max_steps, storage)
        srv["vs_plain"] = srv["value"] / value
        srv["reduction"] = (f"{args.requests} requests with {args.min_steps}-{args.max_steps} steps each, against "
                            f"200 requests with 500-5000 steps in the full trace, so that the run takes minutes")
        out["serving"] = srv
        torch.cuda.empty_cache()
    reps.close()
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


def _device_time(streams, fn):
    """Device time of fn() whose work runs on `streams`: events on the
    current stream bracket the work, joined through per-stream events."""
    import torch

    torch.cuda.synchronize()
    cur = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(cur)
    for st in streams:
        st.wait_event(e0)
    fn()
    for st in streams:
        ev = torch.cuda.Event()
        ev.record(st)
        cur.wait_event(ev)
    e1.record(cur)
    e1.synchronize()
    return e0.elapsed_time(e1)


def run_batched(domains: int, K: int, W: int, storage: str, graphs: bool = True) -> dict:
    """The batched ensemble (seeded air-over-wave domains of uneven size),
    all stepped together: device time of K ensemble steps with one launch
    per phase over all domains (the interior planes as one work queue), and,
    on the same domains, with one stream and step graph per domain."""
    from lbm_b200.batch import Batch, stable_ensemble_envs

    envs = stable_ensemble_envs(domains, seed=7, storage=storage)
    b = Batch(envs, chunk=25, graphs=graphs, queue=True, arith=ARITH)
    W = max(W, 3)
    b.step(W)
    b.synchronize()
    l0 = _launches()
    ms = _device_time(b.streams(), lambda: b.step(K))
    launches = _launches() - l0
    # the same domains, one stream and step graph each
    Wd = max(W, 3 * b.chunk) if graphs else W
    b.step_each(Wd)
    b.synchronize()
    ms_streams = _device_time([d.stream for d in b.domains], lambda: b.step_each(K))
    cells = b.cells
    for d in b.domains:
        if d.counters()["status_flags"]:
            raise SystemExit("non-finite state in the batched run")
    bytes_cell = 76 if storage != "f32" else 152
    out = {
        "value": cells * K / (ms * 1e-3) / 1e6, "unit": UNIT, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "domains": len(envs), "cells": cells, "storage": storage, "bytes_per_cell": bytes_cell,
        "launch": b.mode, "arithmetic": ARITH, "gpu_launches": launches,
        "roofline_step_frac": bytes_cell * cells * K / (ms * 1e-3) / (measured_hbm_peak()[0] * 1e9),
        "per_domain_streams": {"value": cells * K / (ms_streams * 1e-3) / 1e6, "ms_per_step": ms_streams / K,
                               "step_graphs": graphs, "warmup": Wd},
        "workload": f"batched ensemble of {len(envs)} air-over-wave domains (seed 7, stability-screened draws), "
                    f"uneven sizes nx 64-320, ny 32-160, nz 32-128",
    }
    b.close()
    return out


def run_serving(requests: int, min_steps: int, max_steps: int, storage: str) -> dict:
    """The continuous-batching request loop on a seeded Poisson trace."""
    from lbm_b200.serving import Server, poisson_trace

    reqs = poisson_trace(requests, rate_hz=20.0, seed=3, cells_range=(1e5, 2e7),
                         steps_range=(min_steps, max_steps), storage=storage)
    rep = Server(budget_bytes=150e9, chunk=50, arith=ARITH).run(reqs)
    return {
        "value": rep["mlups"], "unit": UNIT, "p50_s": rep["p50_s"], "p99_s": rep["p99_s"], "wall_s": rep["wall_s"],
        "requests": rep["requests"], "failed": len(rep["failed"]), "rounds": rep["rounds"],
        "peak_active": rep["peak_active"], "setup_s": rep["setup_s"], "storage": storage, "arithmetic": ARITH,
        "steps_range": [min_steps, max_steps],
        "workload": f"Poisson(20/s) arrivals, {requests} requests, half air-over-wave, half water Gaussian, cells "
                    f"log-uniform [1e5, 2e7], steps uniform [{min_steps}, {max_steps}], seed 3, HBM budget 150 GB",
    }


def _launches() -> int:
    import ctypes as C

    from lbm_b200 import native

    v = C.c_int64()
    native.load().lbm_launch_count(C.byref(v))
    return int(v.value)


def batched(args):
    storage = args.storage or "f16s"
    r = run_batched(args.domains, args.steps, args.warmup, storage, graphs=not args.no_graphs)
    line = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": r["steps"],
        "warmup": r["warmup"], "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if storage == "f32" else f"f32 compute, {storage} storage",
        "data": "synthetic", "mode": "batched",
        "config": {"workload": r["workload"], "cells": r["cells"], "storage": storage, "launch": r["launch"]},
        "gpu_launches": r["gpu_launches"], "roofline_step_frac": r["roofline_step_frac"],
        "per_domain_streams": r["per_domain_streams"],
    }
    print(json.dumps(line), flush=True)
    return 0


def serving(args):
    storage = args.storage or "f16s"
    r = run_serving(args.requests, args.min_steps, args.max_steps, storage)
    line = {
        "metric": "MLUPS (served trace)", "value": r["value"], "unit": UNIT, "n_gpus": 1,
        "higher_is_better": True, "mode": "serving", "data": "synthetic",
        "p50_s": r["p50_s"], "p99_s": r["p99_s"], "wall_s": r["wall_s"], "requests": r["requests"],
        "failed": r["failed"], "rounds": r["rounds"], "peak_active": r["peak_active"], "setup_s": r["setup_s"],
        "config": {"workload": r["workload"], "storage": storage, "hbm_budget_gb": 150, "round_steps": 50},
    }
    print(json.dumps(line), flush=True)
    return 0


# the stated-size configurations other than the plain roofline run: name -> (env builder, storage)
CONFIGS = {
    "C1": ("air over moving wave 128x64x64, regularized + LES, 1000-step case", "f32"),
    "C2": ("water height path 256x128x96, Gaussian mound, solid x walls", "f32"),
    "C2-f16s": ("water height path 256x128x96, Gaussian mound, solid x walls", "f16s"),
    "C2-bf16s": ("water height path 256x128x96, Gaussian mound, solid x walls", "bf16s"),
    "C3": ("VOF falling block 384x192x192, KBC, collapse and bridge", "f16s"),
}


def _config_env(name: str, storage: str) -> dict:
    from lbm_b200.config import air_wave_env, vof_block_env, water_gaussian_env

    if name == "C1":
        return air_wave_env(128, 64, 64, storage=storage)
    if name.startswith("C2"):
        return water_gaussian_env(256, 128, 96, storage=storage, depth=48.0, amp=8.0, sigma=16.0, g_lb=1e-5,
                                  tau0=0.51)
    return vof_block_env(384, 192, 192, storage=storage)


def configs(args):
    """Device time per step of the stated-size configurations (CUDA events on
    the domain's stream, after warm-up), one JSON line.  Step calls replay
    captured step graphs where the mode allows them (air and the kinematic
    height path; --no-graphs: eager calls); the warm-up captures the timed
    call shape."""
    import torch

    from lbm_b200.domain import Domain

    names = args.only.split(",") if args.only else list(CONFIGS)
    out = {}
    for name in names:
        what, storage = CONFIGS[name]
        d = Domain(_config_env(name, storage), device="cuda:0", with_diag=False)
        d.step(max(3, args.warmup))
        d.synchronize()
        K = args.steps
        graphs = False
        if not args.no_graphs:
            try:
                d.set_step_graphs(True)
                graphs = True
            except RuntimeError:
                graphs = False   # the VOF path runs eager calls
        if graphs:
            for _ in range(3):
                d.step(K)
            d.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(d.stream)
        d.step(K)
        e1.record(d.stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / K
        cells = d.cfg.Nx * d.cfg.Ny * d.cfg.Nz
        out[name] = {"workload": what, "storage": storage, "cells": cells, "steps": K, "ms_per_step": ms,
                     "value": cells / ms / 1e3, "unit": UNIT, "step_graphs": graphs,
                     "status_flags": d.counters()["status_flags"]}
        d.close()
        del d
        torch.cuda.empty_cache()
    print(json.dumps({"metric": METRIC, "mode": "configs", "n_gpus": 1, "data": "synthetic", "configs": out}),
          flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--mode", choices=("plain", "batched", "serving", "configs"), default="plain",
                    help="plain: the 512x256x256 step (default); batched: the 96-domain ensemble; "
                         "serving: the request loop on a Poisson trace; configs: the other stated-size "
                         "configurations (C1 air, C2 water in three storages, C3 VOF)")
    ap.add_argument("--only", type=str, default=None, help="configs mode: comma-separated subset (C1,C2,...)")
    ap.add_argument("--storage", choices=("f32", "f16s", "bf16s"), default=None,
                    help="population storage of the batched and serving modes (default f16s)")
    ap.add_argument("--domains", type=int, default=96, help="batched mode: ensemble size")
    ap.add_argument("--requests", type=int, default=32, help="serving: trace length")
    ap.add_argument("--min-steps", type=int, default=100, help="serving: fewest steps of a request")
    ap.add_argument("--max-steps", type=int, default=1000, help="serving: most steps of a request")
    ap.add_argument("--batched-steps", type=int, default=100, help="plain mode: timed steps of the batched sub-run")
    ap.add_argument("--plain-only", action="store_true",
                    help="plain mode: skip the batched and serving sub-runs")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the timed CPU oracle sample")
    ap.add_argument("--no-graphs", action="store_true",
                    help="time eager step calls instead of CUDA step-graph replays")
    ap.add_argument("--tile-chunk", type=int, default=0,
                    help="planes per block of the interior kernel (default: autotuned in warm-up)")
    ap.add_argument("--plain-storage", choices=("f32", "f16s", "bf16s"), default="f32",
                    help="population storage of the plain run (default f32, the roofline configuration)")
    ap.add_argument("--arith", choices=("exact", "fast"), default="exact",
                    help="arithmetic of the interior kernels: exact (reference order, bit-equal to the oracle) "
                         "or fast (pair-form collision with multiply-add contraction)")
    ap.add_argument("--size", type=str, default=None,
                    help="NXxNYxNZ: another domain size of the same workload (profiling of small cases)")
    args = ap.parse_args()
    global STORAGE, ARITH, B_ALG
    STORAGE, ARITH = args.plain_storage, args.arith
    B_ALG = 152 if STORAGE == "f32" else 76
    if args.size:
        global NX, NY, NZ, WORKLOAD
        NX, NY, NZ = (int(v) for v in args.size.lower().split("x"))
        WORKLOAD = f"air over moving wave, LES regularized, {NX}x{NY}x{NZ}"
    if args.impl == "reference":
        return reference_arm(args)
    if args.mode == "batched":
        return batched(args)
    if args.mode == "serving":
        return serving(args)
    if args.mode == "configs":
        return configs(args)
    return ours(args)


if __name__ == "__main__":
    sys.exit(main())
