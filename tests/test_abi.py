"""The C ABI: both libraries load and export every entry point of
include/lbm_b200.h with the struct layout of the Python binding.  No
compute calls (these run without a GPU)."""
import ctypes as C
import os
import re

import pytest

from lbm_b200 import abi
from oracle_runner import ROOT, oracle_lib

HEADER = os.path.join(ROOT, "include", "lbm_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z0-9_]+\s*\*?\s*(lbm_[a-z0-9_]+)\s*\(", text, re.M)))


def test_header_declares_the_abi():
    names = declared_functions()
    assert set(abi.ABI_SYMBOLS) <= set(names), set(abi.ABI_SYMBOLS) - set(names)


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++17")])
def test_header_compiles_as_plain_c_and_cpp(lang, std):
    """The boundary is a plain C header: it compiles alone, warning-free, as
    C99 (what a cgo / ctypes / JNI binding would include) and as C++."""
    import shutil
    import subprocess

    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("no host compiler")
    p = subprocess.run([cc, "-x", lang, std, "-fsyntax-only", "-Wall", "-Wextra", "-Werror", HEADER],
                       capture_output=True, text=True)
    assert p.returncode == 0, p.stderr


def test_oracle_exports_every_declared_symbol():
    lib = oracle_lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.lbm_backend_name() == b"cpu-oracle"
    abi.check_layout(lib)


def test_cuda_library_exports_every_declared_symbol():
    from lbm_b200 import build

    path = build.build()
    lib = abi.declare(C.CDLL(path))
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.lbm_backend_name() == b"cuda-sm100a"
    assert lib.lbm_abi_version() == abi.LBM_ABI_VERSION
    abi.check_layout(lib)


def test_params_sentinel_rejects_layout_drift():
    lib = oracle_lib()
    p = abi.LbmParams()
    p.abi_version = abi.LBM_ABI_VERSION
    p.nx, p.ny, p.nz = 4, 4, 4
    ctx = C.c_void_p()
    assert lib.lbm_create(C.byref(p), C.byref(ctx)) == -1   # magic_end missing
    p.magic_end = abi.LBM_PARAMS_MAGIC
    assert lib.lbm_create(C.byref(p), C.byref(ctx)) == 0
    assert lib.lbm_destroy(ctx) == 0


def test_unbound_context_reports_error():
    lib = oracle_lib()
    from lbm_b200.config import load_config

    p = abi.make_params(load_config({"LBM_LX_M": "4", "LBM_LY_M": "4", "LBM_LZ_M": "4", "LBM_DX_M": "1"}))
    ctx = C.c_void_p()
    assert lib.lbm_create(C.byref(p), C.byref(ctx)) == 0
    assert lib.lbm_step(ctx, 1, None) == -6
    assert lib.lbm_step(ctx, -1, None) == -1
    lib.lbm_destroy(ctx)
