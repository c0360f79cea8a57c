"""The bounds-checked build (libmpcf_b200_check.so: every computed
shared-memory and global index of the stage kernel checked against its
buffer, MPCF_ERRBIT_BOUNDS on a violation) runs every tile shape, precision
and slab layout of tests/bounds_cases.py without a violation, and its
results equal the ordinary library's bit for bit.  It runs in a child
process, since a process loads one library."""
import os
import subprocess
import sys

import numpy as np
import pytest

import bounds_cases

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CHECK_LIB = os.path.join(os.path.dirname(HERE), "cubism-jr-gpu-mpcf_b200", "lib", "libmpcf_b200_check.so")

CHILD = """
import sys
import numpy as np
sys.path[:0] = [{tests!r}, {pkg!r}]
import mpcf, bounds_cases
np.savez(sys.argv[1], **bounds_cases.run_cases(mpcf))
"""


def test_bounds_checked_build_is_clean_and_identical(mpcf, tmp_path):
    assert os.path.exists(CHECK_LIB), "build the library first (make -C cubism-jr-gpu-mpcf_b200)"
    out = str(tmp_path / "checked.npz")
    env = dict(os.environ, MPCF_B200_LIB=CHECK_LIB)
    code = CHILD.format(tests=HERE, pkg=os.path.join(os.path.dirname(HERE), "cubism-jr-gpu-mpcf_b200"))
    subprocess.run([sys.executable, "-c", code, out], env=env, check=True, timeout=900)
    checked = np.load(out)
    plain = bounds_cases.run_cases(mpcf)
    assert set(checked.files) == set(plain)
    for k in plain:
        if k.startswith("err_"):
            assert int(checked[k][0]) == 0, (k, int(checked[k][0]))
            assert int(plain[k][0]) == 0, (k, int(plain[k][0]))
        else:
            assert np.array_equal(checked[k], plain[k]), k
