"""The bounds-check build of the library on the small extraction cases.

libmeshtrex_b200_check.so (`make -C meshtrex_b200/csrc check`) checks the
shared- and global-memory indices of the extraction kernels and reports the
first one out of range as MTX_ERR_INTERNAL, never by a trap.  The cases run
in a child process that loads that build instead of the normal one
(tests/bounds_check_cases.py): they must finish with no report and with the
oracle's meshes.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_bounds_check_build_runs_the_small_cases_clean():
    lib = os.path.join(ROOT, "meshtrex_b200", "libmeshtrex_b200_check.so")
    assert os.path.exists(lib), "build it with `make -C meshtrex_b200/csrc check`"
    env = dict(os.environ, MESHTREX_B200_LIB=lib)
    r = subprocess.run([sys.executable, os.path.join(HERE, "bounds_check_cases.py")], capture_output=True, text=True,
                       env=env, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "all cases passed" in r.stdout
