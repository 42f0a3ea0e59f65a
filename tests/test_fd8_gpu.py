"""8th-order finite differences: runs tests/fd8_cases.py in a child process with
BSSN_B200_FD_ORDER=8 (the finite-difference order of the loaded library is fixed per process).
The cases compare libbssn_b200_fd8.so with the reference's generated C at fd_order = 8."""

import os
import pathlib
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_fd8_cases(cuda):
    if not (ROOT / "nrpy_b200" / "libbssn_b200_fd8.so").exists():
        pytest.fail("libbssn_b200_fd8.so not built (python -m nrpy_b200.build --fd-order 8)")
    env = dict(os.environ, BSSN_B200_FD_ORDER="8")
    r = subprocess.run([sys.executable, "-m", "pytest", str(ROOT / "tests" / "fd8_cases.py"), "-q", "-m", "gpu",
                        "-p", "no:cacheprovider"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, r.stdout[-6000:] + r.stderr[-3000:]
    assert " passed" in r.stdout and " skipped" not in r.stdout, r.stdout[-2000:]
