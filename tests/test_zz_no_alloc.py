"""lbm_link_geometry_noalloc: link geometry of a bed shape without allocating.

Some callers of this library must not call cudaMalloc. Examples: a serving
process whose device memory is fully committed to population buffers by its
admission budget, or a host framework that owns all device memory through its
own caching allocator. For them the library exports lbm_link_geometry_noalloc.
It writes the same per-cell link geometry as lbm_export_diagnostics on a
context, but its only scratch is a fixed device array inside the library. These
tests call it through the C ABI and check it against the context path, which
allocates. The file sorts last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import pytest

from lbm_b200 import abi
from lbm_b200.config import air_wave_env, load_config

GEOMETRY = ("phi", "obstacle", "near_obstacle", "lattice_open", "lattice_open_frac", "lattice_wall_type")


def _call(lib, params, bed_ptr, out_ptrs, stream_ptr):
    err = C.create_string_buffer(512)
    status = lib.lbm_link_geometry_noalloc(C.byref(params), bed_ptr, *out_ptrs, stream_ptr, err, len(err))
    return status, err.value.decode()


def test_noalloc_rejects_grids_beyond_its_fixed_array():
    """Oversized grids and unsupported geometry are refused before any device work."""
    from lbm_b200 import native

    lib = native.load()
    nx, ny = 512, 256                       # 131072 columns > LBM_NOALLOC_MAX_COLUMNS
    params = abi.make_params(load_config(air_wave_env(nx, ny, 16)))
    fake = C.c_void_p(256)                  # never dereferenced: the size check fails first
    status, msg = _call(lib, params, fake, [None] * 6, None)
    assert status == abi.LBM_ERR_BAD_ARG
    assert "exceeds the fixed maximum" in msg and "65536" in msg
    env = air_wave_env(32, 16, 16)
    env["LBM_X_BOUNDARY"] = "solid"
    status, msg = _call(lib, abi.make_params(load_config(env)), fake, [None] * 6, None)
    assert status == abi.LBM_ERR_UNSUPPORTED and "periodic x" in msg


@pytest.mark.gpu
def test_noalloc_link_geometry_matches_context_export_twice():
    """Two calls in a row, on two bed states, each equal to lbm_export_diagnostics."""
    import torch

    from lbm_b200.domain import Domain

    env = air_wave_env(64, 32, 24, amp=3.0, level=6.0, wavelength=32.0)
    dom = Domain(env, device="cuda:0", with_diag=True)
    outs = {k: torch.empty_like(dom.field(k)) for k in GEOMETRY}
    stream = C.c_void_p(dom.stream.cuda_stream)
    try:
        for call in range(2):
            if call:
                dom.step(7)                 # the bed moves between the two calls
            dom.export_diagnostics()
            for t in outs.values():         # stale values must all be overwritten
                t.fill_(-3)
            dom.synchronize()
            ptrs = [C.c_void_p(outs[k].data_ptr()) for k in GEOMETRY]
            status, msg = _call(dom.lib, dom.params, C.c_void_p(dom.field("water_h").data_ptr()), ptrs, stream)
            assert status == abi.LBM_OK, msg
            dom.synchronize()
            for k in GEOMETRY:
                ref, got = dom.field(k), outs[k]
                # link geometry is exact: compare bit patterns
                if ref.dtype == torch.float32:
                    ref, got = ref.view(torch.int32), got.view(torch.int32)
                bad = int((ref != got).sum())
                assert bad == 0, f"call {call + 1}: {k} differs in {bad} entries"
            # the bed really changes between the calls (the check is not vacuous)
            if call == 0:
                first_frac = outs["lattice_open_frac"].clone()
        assert not torch.equal(first_frac, outs["lattice_open_frac"])
    finally:
        dom.close()
