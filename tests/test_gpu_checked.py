"""The checked build of the engine (libnbl_b200_checked.so: every cell
slice, candidate, hit-word and output-slot index of the pair passes is tested
on the device and a failure is reported as NBL_ERROR_INTERNAL, never a trap)
runs the golden cases, the workload shapes, every launch shape, row slices,
a batch, the neighbour matrix and the force sink with no check firing and
with the oracle's results.  A child process, because the package picks the
library when it is imported (MATSCIPY_NEIGHBOURS_CHECKED=1)."""
import os
import pathlib
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = pathlib.Path(__file__).resolve().parent
CHECKED_SO = HERE.parent / "matscipy-neighbours_b200" / "matscipy_neighbours" / \
    "libnbl_b200_checked.so"


def test_checked_build_runs_every_pair_pass_path_clean():
    assert CHECKED_SO.exists(), "build it with `python matscipy-neighbours_b200/build.py --checked`"
    env = dict(os.environ, MATSCIPY_NEIGHBOURS_CHECKED="1")
    r = subprocess.run([sys.executable, str(HERE / "_checked_run.py")], env=env,
                       capture_output=True, text=True, timeout=1500)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    last = r.stdout.strip().splitlines()[-1]
    assert last.startswith("checked ok ") and int(last.split()[-1]) > 300, last
