"""The bounds-checked build (libcardioid_b200_checked.so: every tissue, time,
slot and voxel index the step kernel uses is checked, and one out of range
is recorded as CDB_BOUNDS_FAULT instead of being accessed; the stand-in for
a memory checker where compute-sanitizer is closed) on small and edge-case
tissues: boxes, cables, sheets, a masked tissue, one cell, ragged type
groups, row tiles, all of them in one engine, the ECG sensor, the four staging modes
and the chunked host step, FP64 and mixed.  Each library runs in its own
process (tests/bounds_cases.py); the checked run must report no fault
(cdb_engine_sync) and give the same results as the normal build (bit for
bit, the ECG traces to rounding: their sums end in atomic adds)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECKED = os.path.join(ROOT, "cardioid_b200", "_lib", "libcardioid_b200_checked.so")


@pytest.mark.skipif(not os.path.exists(CHECKED), reason="checked library not built (python -m cardioid_b200.build --checked)")
def test_checked_build_finds_no_index_out_of_range(cdb_lib, tmp_path):
    script = os.path.join(ROOT, "tests", "bounds_cases.py")
    out = {}
    for name, lib in (("normal", None), ("checked", CHECKED)):
        env = dict(os.environ)
        env.pop("CARDIOID_B200_LIB", None)
        if lib:
            env["CARDIOID_B200_LIB"] = lib
        path = str(tmp_path / ("%s.npz" % name))
        r = subprocess.run([sys.executable, script, path], env=env, capture_output=True, text=True, timeout=900)
        assert r.returncode == 0, r.stdout + r.stderr      # a CDB_BOUNDS_FAULT raises in sync
        out[name] = np.load(path)
    assert set(out["normal"].files) == set(out["checked"].files)
    for k in out["normal"].files:
        if k.endswith("_ecg"):
            # ECG sums end in atomic adds, whose order varies run to run
            np.testing.assert_allclose(out["checked"][k], out["normal"][k], rtol=1e-12, atol=1e-15, err_msg=k)
        else:
            np.testing.assert_array_equal(out["checked"][k], out["normal"][k], err_msg=k)
