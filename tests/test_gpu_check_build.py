"""The bounds-checked debug build (libfvr_b200_check.so, -DFVR_CHECK) on
small cases of every instrumented kernel family: every checked access stays
in bounds (all check words zero), and the results equal the normal
library's (5e-6 relative; the guards change no arithmetic).  The normal
library answers FVR_ERR_UNSUPPORTED to fvr_check_words."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parents[1]
LIBDIR = REPO / "diff-fvr_b200" / "fvr"
FVR_ERR_UNSUPPORTED = 3


def _run(lib):
    env = dict(os.environ, FVR_B200_LIB=str(lib))
    r = subprocess.run([sys.executable, str(REPO / "tests" / "check_build_cases.py")], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_check_build_in_bounds_and_equal():
    chk = LIBDIR / "libfvr_b200_check.so"
    if not chk.exists():
        subprocess.run(["make", "-C", str(REPO / "diff-fvr_b200" / "csrc"), "-j8", "check"], check=True)
    normal = _run(LIBDIR / "libfvr_b200.so")
    checked = _run(chk)
    assert normal["check_rc"] == FVR_ERR_UNSUPPORTED
    assert checked["check_rc"] == 0
    assert checked["check_words"] == [0, 0, 0, 0], [hex(w) for w in checked["check_words"]]
    for k, v in normal.items():
        if k.startswith("check"):
            continue
        a, b = np.asarray(v, np.float64), np.asarray(checked[k], np.float64)
        assert a.shape == b.shape, k
        assert np.linalg.norm(a - b) <= 5e-6 * max(np.linalg.norm(a), 1e-30), k
