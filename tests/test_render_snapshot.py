"""The render-snapshot writer against the reference's own writer.

tests/golden/render/<case>.npz were written by save_render_snapshot of
run_ab_case.py:140-202 from the seeded inputs of render_inputs()
(gen_render_golden.py beside them).  write_render_snapshot must write the
same file name and the same arrays: names, dtypes, shapes and values."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from gen_render_golden import CASES, STEP, TIME, render_inputs  # noqa: E402

from lbm_b200.facade import write_render_snapshot  # noqa: E402


@pytest.mark.parametrize("case", CASES)
def test_snapshot_matches_the_reference_writer(case, tmp_path):
    path = write_render_snapshot(render_inputs(case), label=case, step=STEP, time_phys=TIME, output_dir=tmp_path)
    assert os.path.basename(path) == f"{case}_render_{STEP:05d}.npz"
    ours = np.load(path)
    ref = np.load(os.path.join(HERE, "golden", "render", f"{case}.npz"))
    assert sorted(ours.files) == sorted(ref.files)
    for name in ref.files:
        a, b = ref[name], ours[name]
        assert a.dtype == b.dtype and a.shape == b.shape, name
        assert np.array_equal(a, b), name
