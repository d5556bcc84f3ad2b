"""Drop-in solver module backed by the B200 engine.

It has the module surface of LBM_3D_LES_air_over_waves_CODEX.py: the LBM_*
environment options are read at import, and it exposes the same globals,
fields (.to_numpy()), counters ([None]) and main().  The reference's harness
loads it in place of the Taichi solver:

    python run_ab_case.py --module lbm-3d-les-air-over-waves_b200/LBM_3D_LES_air_over_waves_B200.py ...

(the harness's --random-seed path needs Taichi; set LBM_RANDOM_SEED instead).
"""
import os as _os
import sys as _sys

_here = _os.path.dirname(_os.path.abspath(__file__))
if _here not in _sys.path:
    _sys.path.insert(0, _here)

from lbm_b200.facade import install as _install  # noqa: E402

_install(globals())
