"""Build the CUDA library in-tree: lbm_b200/_native/liblbm_b200.so.

    python -m lbm_b200.build        (from lbm-3d-les-air-over-waves_b200/)

Flags: sm_100a only; -fmad=false for lbm_api.cu and lbm_device.cu, so that
every f32 expression rounds in source order (the CPU oracle is built with
-ffp-contract=off) and those kernels are bit-comparable with the oracle;
lbm_fast.cu (the fast-arithmetic interior kernels) is compiled with
multiply-add contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
SRC_ROOT = os.path.dirname(PKG)
CSRC = os.path.join(SRC_ROOT, "csrc")
REPO = os.path.dirname(SRC_ROOT)
INCLUDE = os.path.join(REPO, "include")
OUT_DIR = os.path.join(PKG, "_native")
LIB = os.path.join(OUT_DIR, "liblbm_b200.so")
SOURCES = ["lbm_api.cu", "lbm_device.cu", "lbm_fast.cu"]
HEADERS = ["lbm_dev.cuh", "lbm_geom.cuh", "lbm_stages.cuh", "lbm_tile.cuh", "lbm_vof.cuh", "lbm_launch.h",
           "lbm_fast.cuh", "lbm_batch.cuh", "lbm_batch_tile.cuh", "lbm_diag.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xptxas", "-warn-spills",
]
# rounding per translation unit: the reference's order everywhere except the
# fast-arithmetic interior kernels, which contract multiply-adds
SOURCE_FLAGS = {"lbm_api.cu": ["-fmad=false"], "lbm_device.cu": ["-fmad=false"], "lbm_fast.cu": ["-fmad=true"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(INCLUDE, f) for f in ("lbm_b200.h", "lbm_mathfn.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    build_dir = os.path.join(OUT_DIR, "_build")
    os.makedirs(build_dir, exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, *SOURCE_FLAGS[src], *extra, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((src, cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = []
    for src, cmd, proc in procs:
        out, _ = proc.communicate()
        if verbose or proc.returncode:
            sys.stderr.write(out)
        if proc.returncode:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp,
                    "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
