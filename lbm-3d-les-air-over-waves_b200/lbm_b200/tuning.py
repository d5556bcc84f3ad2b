"""Autotuner for the interior kernel's work unit.

The interior kernel gives each thread block a 16x16 column tile and a chunk
of z planes; each chunk also recomputes the two planes around it for the LES
stencil, so short chunks waste work while long ones leave SMs idle at the
end of the launch.  autotune_tile_chunk times the step for candidate chunk
lengths on a live domain (the timing steps advance the simulation; use it in
warm-up) and keeps the fastest.  Results are cached per domain shape and
configuration for the process.
"""
from __future__ import annotations

CANDIDATES = (8, 12, 16, 24, 32, 48, 64)
_CACHE: dict = {}


def _key(dom) -> tuple:
    c = dom.cfg
    return (c.Nx, c.Ny, c.Nz, c.pop_storage, c.use_LES, c.collision_model, dom.device.index)


def autotune_tile_chunk(dom, candidates=CANDIDATES, steps: int = 6, repeats: int = 2) -> dict:
    """Pick the fastest planes-per-block for this domain and apply it.
    Returns {"chunk": best, "ms_per_step": {candidate: ms}}."""
    import torch

    key = _key(dom)
    if key in _CACHE:
        dom.set_tile_chunk(_CACHE[key]["chunk"])
        return _CACHE[key]
    timings = {}
    for ch in candidates:
        dom.set_tile_chunk(ch)
        dom.step(1)   # one step at the new shape before timing
        best = None
        for _ in range(repeats):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(dom.stream)
            dom.step(steps)
            e1.record(dom.stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            best = ms if best is None else min(best, ms)
        timings[ch] = best
    chunk = min(timings, key=timings.get)
    dom.set_tile_chunk(chunk)
    _CACHE[key] = {"chunk": chunk, "ms_per_step": timings}
    return _CACHE[key]
