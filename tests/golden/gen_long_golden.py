"""Generate 100-step goldens with the reference solver's own kernels.

Run where a checkout of the reference is available (it is read, never
written; GPU machines do not need it):

    python tests/golden/gen_long_golden.py --reference PATH [--only NAME] [--steps N]

PATH is the reference checkout (default: the LBM_REFERENCE_DIR environment
variable).  For each golden case of gen_golden.py, main() runs N
steps (default 100) exactly as gen_golden.py runs it (taichi_shim for
Taichi, the same seeded initial kick and backscatter draws), and
tests/golden/long/<case>.npz (<case>_<N>.npz for other N) keeps:
  env, noise, seed, nsteps   as in the short goldens
  s<N>_<field>              the state after the last step
  s0_<field>                the initial state, for the cases edited after the
                            reference's init (they start from it)
  health                    the health lines main() printed (every 100 steps,
                            CODEX.py:3930-3954)
"""
from __future__ import annotations

import argparse
import contextlib
import io
import os

import numpy as np

import gen_golden as gg

HERE = os.path.dirname(os.path.abspath(__file__))
LONG_CASES = tuple(gg.CASES)


def run_long(name: str, steps: int) -> dict:
    gg.STEPS[name] = steps
    printed = io.StringIO()
    with contextlib.redirect_stdout(printed):
        out = gg.run_case(name, gg.CASES[name])
    last = f"s{steps}_"
    # an edited case starts from its s0 snapshot (the edit follows the reference's init)
    first = "s0_" if name in gg.INJECT else last
    keep = {k: v for k, v in out.items() if k.startswith(last) or k.startswith(first) or
            k in ("env", "noise", "seed", "nsteps", "injected", "rho_initial")}
    keep["health"] = np.array([ln for ln in printed.getvalue().splitlines() if ln.startswith("Time Step")])
    return keep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("LBM_REFERENCE_DIR", ""),
                    help="reference checkout (default: $LBM_REFERENCE_DIR)")
    ap.add_argument("--only", default=None)
    ap.add_argument("--steps", type=int, default=100)
    args = ap.parse_args()
    gg.REFERENCE = os.path.abspath(args.reference) if args.reference else ""
    if not gg.REFERENCE or not os.path.exists(os.path.join(gg.REFERENCE, gg.SOLVER_FILE)):
        raise SystemExit(f"{gg.SOLVER_FILE} not found: pass --reference PATH or set LBM_REFERENCE_DIR")
    os.makedirs(os.path.join(HERE, "long"), exist_ok=True)
    for name in LONG_CASES:
        if args.only and name != args.only:
            continue
        data = run_long(name, args.steps)
        path = os.path.join(HERE, "long", f"{name}.npz" if args.steps == 100 else f"{name}_{args.steps}.npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path) / 1024:.0f} KiB), health lines: {len(data['health'])}",
              flush=True)


if __name__ == "__main__":
    main()
