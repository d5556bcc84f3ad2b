"""Many independent domains stepped together on one GPU.

    batch = Batch(ensemble_envs(96, seed=7), device="cuda:0")
    batch.step(100)            # every domain advances 100 steps
    batch.synchronize()

Each domain is a full Domain (own buffers, own C-ABI context) on its own
CUDA stream.  A step call issues the domains' launches round-robin in chunks,
so kernels of different domains overlap on the device and small domains
share the SMs.  Results do not depend on the mix: domains share no state.
"""
from __future__ import annotations

import numpy as np

from .config import air_wave_env


def ensemble_envs(n: int = 96, seed: int = 7, storage: str = "f16s") -> list[dict]:
    """The batched air-over-wave ensemble: seeded uneven domain sizes
    (nx in [64,320], ny in [32,160], nz in [32,128], multiples of 16) and
    sweeps over wave amplitude U[1,6], wavelength U[32,128], phase speed
    U[0.005,0.03] and inflow U[0.02,0.08] (lattice units).  The wavelength
    is snapped to nx / (whole number of waves), since the bed is periodic
    in x (otherwise it has a cliff at the seam), and draws whose steepest
    bed slope 2 pi amp / wavelength exceeds 0.5 are drawn again: the
    reference model diverges on such beds (a seam cliff, or slope 0.87,
    blows up within a hundred steps on the CPU oracle as on the GPU)."""
    rng = np.random.default_rng(seed)
    envs = []
    for r in range(n):
        nx = int(rng.integers(4, 21)) * 16
        ny = int(rng.integers(2, 11)) * 16
        nz = int(rng.integers(2, 9)) * 16
        while True:
            amp = float(rng.uniform(1.0, 6.0))
            wavelength = float(rng.uniform(32.0, 128.0))
            wavelength = nx / max(1, round(nx / wavelength))
            if 2.0 * np.pi * amp / wavelength <= 0.5:
                break
        speed = float(rng.uniform(0.005, 0.03))
        inflow = float(rng.uniform(0.02, 0.08))
        level = max(8.0, amp + 4.0)
        env = air_wave_env(nx, ny, nz, storage=storage, seed=1000 + r, amp=round(amp, 3), level=round(level, 3),
                           wavelength=round(wavelength, 3), speed=round(speed, 5), inflow=round(inflow, 4))
        envs.append(env)
    return envs


def stable_ensemble_envs(n: int = 96, seed: int = 7, storage: str = "f16s", device="cuda:0",
                         screen_steps: int = 400, screen_ny: int = 16) -> list[dict]:
    """ensemble_envs with a stability screen: the reference model produces
    negative densities in cells cut almost entirely by the moving bed for
    some draws (the CPU oracle diverges exactly like the GPU), so each draw
    is first run as a y-slice (screen_ny rows, FP32) for screen_steps steps
    and redrawn if it diverges.  Deterministic for a given seed: the draws
    are seeded and the solver is bit-reproducible."""
    import torch

    pool = ensemble_envs(4 * n, seed=seed, storage=storage)
    keep = []
    cursor = 0
    while len(keep) < n and cursor < len(pool):
        cand = pool[cursor:cursor + (n - len(keep))]
        cursor += len(cand)
        slices = []
        for e in cand:
            se = dict(e)
            se["LBM_LY_M"] = str(screen_ny)
            se["LBM_B200_POP_STORAGE"] = "f32"
            slices.append(se)
        b = Batch(slices, device=device, chunk=50)
        b.step(screen_steps)
        b.synchronize()
        for e, d in zip(cand, b.domains):
            if d.counters()["status_flags"] == 0 and bool(torch.isfinite(d.field("ux")).all()):
                keep.append(e)
        b.close()
    if len(keep) < n:
        raise RuntimeError(f"only {len(keep)} stable draws out of {len(pool)}")
    return keep[:n]


def domain_bytes(cfg, with_diag: bool = False) -> int:
    """Device bytes of one domain: caller-owned state plus library scratch."""
    from .state import field_specs

    size = {"f32": 4, "f16": 2, "bf16": 2, "i8": 1, "i32": 4}
    total = 0
    for shape, dt in field_specs(cfg, with_diag).values():
        total += int(np.prod(shape)) * size[dt]
    n, a = cfg.Nx * cfg.Ny * cfg.Nz, cfg.Nx * cfg.Ny
    total += 12 * n + 2 * 42 * 4 * a + 4096     # LES velocity planes, bed slots + column caches, counters
    if getattr(cfg, "free_surface_tracking_mode", "height") == "vof" and getattr(cfg, "water_free_surface_enabled", 0):
        total += 52 * n
    if getattr(cfg, "pop_storage", "f32") != "f32":
        # FP32 stash of the general planes (the bed band and the top row): 76 B per cell
        dx = float(getattr(cfg, "dx", 1.0)) or 1.0
        band = int(np.ceil((float(getattr(cfg, "offset_m", 0.0)) + 2.0 * float(getattr(cfg, "bed_amp_m", 0.0))) / dx)) + 4
        total += 76 * a * min(cfg.Nz, band)
    return total


class Batch:
    """Domains stepped together.

    queue=True (air ensembles): one launch per phase of the step for each
    group of up to 28 domains of one collision model (lbm_batch_*), each
    group on a stream of the library's, joined to the batch's own stream at
    the end of a call: the interior planes of a group's domains form work
    queues of (domain, tile, z chunk) items taken by grids of resident blocks
    (tile copies for the tiles off each domain's edge); the planes next to
    the bed and the top, the bed and the final stream are single grids over
    the group.  Results equal stepping each domain alone, bit for bit.

    arith: "exact" or "fast" interior arithmetic for every domain (default:
    each context's own, from LBM_B200_ARITH).

    queue=False: each domain on its own stream, its calls interleaved so that
    kernels of different domains overlap.  With graphs (the default) each air
    domain's step calls run as CUDA graph replays (lbm_set_step_graphs):
    after the first eager call, one graph per call shape is captured, then a
    call costs two launches instead of about seven per step."""

    def __init__(self, envs, device="cuda:0", chunk: int = 25, graphs: bool = True, queue: bool = False,
                 arith: str | None = None):
        import ctypes as C

        import torch

        from .domain import Domain

        self.device = torch.device(device)
        self.chunk = int(chunk)
        self.domains = [Domain(env, device=self.device, stream=torch.cuda.Stream(self.device), with_diag=False)
                        for env in envs]
        self.graphs = graphs
        if arith is not None:
            for d in self.domains:
                d.set_arithmetic(arith)   # exact or fast interior arithmetic, before any graph capture
        if graphs:
            for d in self.domains:
                if d.cfg.physics_mode == "air":
                    d.set_step_graphs(True)
        self.handle = None
        self.stream = None
        if queue:
            lib = self.domains[0].lib
            self.stream = torch.cuda.Stream(self.device)
            ctxs = (C.c_void_p * len(self.domains))(*[d.ctx.value for d in self.domains])
            h = C.c_void_p()
            status = lib.lbm_batch_create(ctxs, len(self.domains), C.byref(h))
            if status != 0:
                why = [lib.lbm_last_error(d.ctx).decode() for d in self.domains if lib.lbm_last_error(d.ctx)]
                raise RuntimeError(f"lbm_batch_create failed ({status}): {why[0] if why else ''}")
            self.handle = h

    @property
    def mode(self) -> str:
        if self.handle is not None:
            return "one launch per phase over each group of up to 28 domains (interior planes as work queues)"
        return "one stream and one step graph per domain" if self.graphs else "one stream per domain"

    @property
    def cells(self) -> int:
        return sum(d.cfg.Nx * d.cfg.Ny * d.cfg.Nz for d in self.domains)

    def streams(self) -> list:
        """The CUDA streams the ensemble's work runs on."""
        if self.handle is not None:
            return [self.stream]
        return [d.stream for d in self.domains]

    def step(self, n: int):
        import ctypes as C

        if self.handle is not None:
            lib = self.domains[0].lib
            for d in self.domains:          # after work the domains queued on their own streams
                self.stream.wait_stream(d.stream)
            status = lib.lbm_batch_step(self.handle, int(n), C.c_void_p(self.stream.cuda_stream))
            if status != 0:
                raise RuntimeError(f"lbm_batch_step failed ({status}): {lib.lbm_batch_last_error(self.handle).decode()}")
            return
        done = 0
        while done < n:
            k = min(self.chunk, n - done)
            for d in self.domains:
                d.step(k)
            done += k

    def step_each(self, n: int):
        """Advance every domain with its own calls (graphs where enabled),
        even in queue mode."""
        if self.handle is not None:
            self.stream.synchronize()
        done = 0
        while done < n:
            k = min(self.chunk, n - done)
            for d in self.domains:
                d.step(k)
            done += k

    def synchronize(self):
        if self.stream is not None:
            self.stream.synchronize()
        for d in self.domains:
            d.synchronize()

    def close(self):
        if self.handle is not None:
            self.stream.synchronize()
            self.domains[0].lib.lbm_batch_destroy(self.handle)
            self.handle = None
        for d in self.domains:
            d.close()
        self.domains = []
