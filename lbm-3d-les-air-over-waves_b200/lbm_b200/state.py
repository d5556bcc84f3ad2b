"""Field set of one domain: names, shapes, dtypes, allocation.

The names follow the reference's Taichi fields (CODEX.py:531-620) where one
exists.  Layout: 3-D fields [nz][ny][nx] (x fastest, the reference's
(Nz, Ny, Nx)), populations [19][nz][ny][nx] (structure of arrays),
columns [ny][nx].  Free-surface cell types are int8 (the reference uses
i32; the values are the same FS_GAS/FS_LIQUID/FS_INTERFACE).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .abi import LbmBuffers

# name -> (shape kind, dtype name); dtype "pop" = population storage type
FIELDS = {
    "f0": ("pop", "pop"), "f1": ("pop", "pop"),
    "rho": ("cell", "f32"), "ux": ("cell", "f32"), "uy": ("cell", "f32"), "uz": ("cell", "f32"),
    "omega": ("cell", "f32"),
    "water_h": ("col", "f32"), "water_h_last": ("col", "f32"), "u_wave": ("col", "f32"),
    "v_wave": ("col", "f32"), "w_wave": ("col", "f32"), "fs_h": ("col", "f32"), "fs_h_last": ("col", "f32"),
    "fs_flux_x": ("col", "f32"), "fs_flux_y": ("col", "f32"),
    "piecewise_bed_z": ("x", "f32"), "u_inlet_profile": ("z", "f32"),
    "rho_initial": ("cell", "f32"), "init_noise": ("cell3", "f32"),
    "fs_fill": ("cell", "f32"), "fs_type": ("cell", "i8"), "fs_type_prev": ("cell", "i8"),
    "fs_mass": ("cell", "f32"), "fs_mass_excess": ("cell", "f32"), "fs_excess_dir": ("cell", "i8"),
}
DIAG_FIELDS = {
    "phi": ("cell", "f32"), "obstacle": ("cell", "i32"), "near_obstacle": ("cell", "i32"),
    "lattice_open": ("pop", "i8"), "lattice_open_frac": ("pop", "f32"), "lattice_wall_type": ("pop", "i8"),
    "pressure_reference_head": ("cell", "f32"), "gravity_body_fraction": ("cell", "f32"),
    "vof_exterior_gas": ("cell", "i32"),
}
STORAGE_DTYPES = {"f32": "f32", "f16s": "f16", "bf16s": "bf16"}


def shape_of(kind: str, cfg) -> tuple:
    nz, ny, nx = cfg.Nz, cfg.Ny, cfg.Nx
    return {
        "pop": (19, nz, ny, nx), "cell": (nz, ny, nx), "cell3": (3, nz, ny, nx), "col": (ny, nx),
        "x": (nx,), "z": (nz,),
    }[kind]


def field_specs(cfg, with_diag: bool = True, storage: str | None = None):
    storage = cfg.pop_storage if storage is None else storage
    specs = dict(FIELDS)
    if with_diag:
        specs.update(DIAG_FIELDS)
    out = {}
    for name, (kind, dt) in specs.items():
        if dt == "pop":
            dt = STORAGE_DTYPES[storage]
        out[name] = (shape_of(kind, cfg), dt)
    return out


_NP = {"f32": np.float32, "i8": np.int8, "i32": np.int32}


def allocate_numpy(cfg, with_diag: bool = True) -> dict:
    """Host arrays (the CPU oracle computes in f32 and stores f32 populations)."""
    return {name: np.zeros(shape, dtype=_NP[dt if dt in _NP else "f32"])
            for name, (shape, dt) in field_specs(cfg, with_diag, storage="f32").items()}


def allocate_torch(cfg, device, with_diag: bool = True) -> dict:
    import torch
    tdt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16, "i8": torch.int8,
           "i32": torch.int32}
    return {name: torch.zeros(shape, dtype=tdt[dt], device=device)
            for name, (shape, dt) in field_specs(cfg, with_diag).items()}


def _ptr(arr) -> int | None:
    if arr is None:
        return None
    if isinstance(arr, np.ndarray):
        assert arr.flags["C_CONTIGUOUS"]
        return arr.ctypes.data
    assert arr.is_contiguous()
    return arr.data_ptr()


def make_buffers(arrays: dict) -> LbmBuffers:
    b = LbmBuffers()
    for name, _ in LbmBuffers._fields_:
        setattr(b, name, _ptr(arrays.get(name)))
    return b
