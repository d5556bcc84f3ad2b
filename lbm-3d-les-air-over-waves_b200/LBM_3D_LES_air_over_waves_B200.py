"""Drop-in solver module backed by the B200 engine.

It has the module surface of LBM_3D_LES_air_over_waves_CODEX.py: the LBM_*
environment options are read at import, and it exposes the same globals,
fields (.to_numpy()), counters ([None]) and main().  The reference's harness
loads it in place of the Taichi solver:

    python run_ab_case.py --module lbm-3d-les-air-over-waves_b200/LBM_3D_LES_air_over_waves_B200.py ...

(the harness's --random-seed reaches the engine through the harness's
taichi.init wrapper).  Run as a script, it steps the configured case and
writes the harness's metrics CSV, reduced on the device, to
$LBM_OUTPUT_DIR/$LBM_RUN_LABEL_metrics.csv, as the reference's direct run does
(without its frame PNGs).
"""
import os as _os
import sys as _sys

_here = _os.path.dirname(_os.path.abspath(__file__))
if _here not in _sys.path:
    _sys.path.insert(0, _here)

from lbm_b200.facade import configure_direct_visualization as _configure_direct  # noqa: E402
from lbm_b200.facade import install as _install  # noqa: E402

_install(globals())

if __name__ == "__main__":
    _metrics_file = _configure_direct(globals())
    try:
        main()  # noqa: F821 - defined by _install
    finally:
        _metrics_file.close()
