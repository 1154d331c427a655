"""The parity cases of tests/bounds_check_cases.py on the bounds-check build
(needs a B200).

compute-sanitizer is not available on the GPUs these tests run on, so the
library has a bounds-check variant instead (libemergence_b200_bc.so, built
with -DEMG_BOUNDS_CHECK): each global index of the fused sweeps (uniform,
AMR and batched kinds), the uniform ghost fill, the AMR pool loads and the
AMR RK update is compared with its array's extent before the access, and an
out-of-range index skips the access and is reported as EMG_ERR_BOUNDS. The
cases (1-D/2-D/3-D meshes, short periodic and reflecting axes, every flux
mode, both precisions, an AMR run across a regrid, batched lines) must give
the oracle's results with no such report.
"""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_parity_cases_pass_on_the_bounds_check_build():
    lib = os.path.join(ROOT, "emergence_b200", "libemergence_b200_bc.so")
    assert os.path.exists(lib), "the bounds-check build is missing (python -m emergence_b200.build)"
    env = dict(os.environ, EMG_BOUNDS_CHECK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "tests", "bounds_check_cases.py")], env=env,
                       capture_output=True, text=True, timeout=900)
    print(r.stdout[-4000:], r.stderr[-4000:])
    assert r.returncode == 0 and "BOUNDS_CHECK_OK" in r.stdout
