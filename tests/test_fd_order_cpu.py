"""8th-order finite differences on the CPU: the stencil weights, and the fd8 library's ABI.

The weights solved by nrpy_b200/codegen/fdcoeffs.py at order 8 must be the standard 9-point
central weights (first derivative 4/5, -1/5, 4/105, -1/280; second derivative -205/72, 8/5,
-1/5, 8/315, -1/560) and the Kreiss-Oliger operator the 10th difference on 11 points over 2^10,
as nrpy's finite_difference.py builds it (fd_order + 2, sign (-1)^((width+1)/2)). The
libbssn_b200_fd8.so struct layouts must equal the reference project generated at fd_order 8
(NGHOSTS = 5), checked in a child process because the order is fixed per process.
"""

import json
import os
import pathlib
import subprocess
import sys

import pytest
import sympy as sp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_order8_weights():
    from nrpy_b200.codegen import fdcoeffs as fdc

    R = sp.Rational
    try:
        fdc.set_fd_order(8)
        assert fdc.NGHOSTS == 5
        d1 = fdc.first_centred()
        assert {k: d1[k] for k in (1, 2, 3, 4)} == {1: R(4, 5), 2: R(-1, 5), 3: R(4, 105), 4: R(-1, 280)}
        assert all(d1[-k] == -d1[k] for k in (1, 2, 3, 4)) and 0 not in d1
        d2 = fdc.second_centred()
        assert d2 == {0: R(-205, 72), 1: R(8, 5), -1: R(8, 5), 2: R(-1, 5), -2: R(-1, 5), 3: R(8, 315),
                      -3: R(8, 315), 4: R(-1, 560), -4: R(-1, 560)}
        ko = fdc.kreiss_oliger()
        binom = {k: (-1) ** (5 - abs(k)) * sp.binomial(10, 5 - abs(k)) for k in range(-5, 6)}
        assert ko == {k: R(binom[k], 1024) for k in range(-5, 6)}
        up = fdc.upwind(+1)
        assert set(up) == set(range(-3, 6)) and sum(up.values()) == 0
        assert sum(k * w for k, w in up.items()) == 1  # first derivative
        assert fdc.radiation_fd1(0) == {-2: R(1, 12), -1: R(-2, 3), 1: R(2, 3), 2: R(-1, 12)}  # stays 4th order
    finally:
        fdc.set_fd_order(4)
    assert fdc.FD_ORDER == 4 and fdc.NGHOSTS == 3


CHILD = r'''
import ctypes as C, json
from nrpy_b200 import lib as L
lib = L.load()
print(json.dumps({"order": lib.bssn_b200_fd_order(), "nghosts": L.NGHOSTS,
                  "sizeof_bc_struct": C.sizeof(L.BcStruct), "sizeof_griddata": C.sizeof(L.GriddataStruct),
                  "sizeof_commondata": C.sizeof(L.CommondataStruct), "sizeof_params": C.sizeof(L.ParamsStruct),
                  "symbols": all(hasattr(lib, n) for n, _, _ in L.SIGNATURES)}))
'''


def test_fd8_library_abi():
    if not (ROOT / "nrpy_b200" / "libbssn_b200_fd8.so").exists():
        pytest.skip("libbssn_b200_fd8.so not built")
    env = dict(os.environ, BSSN_B200_FD_ORDER="8")
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    got = json.loads(r.stdout.strip().splitlines()[-1])
    assert got["order"] == 8 and got["nghosts"] == 5 and got["symbols"]
    from oracle import ref

    if ref.available("sph3d8"):
        lay = ref.struct_layout("sph3d8")
        for k in ("sizeof_bc_struct", "sizeof_griddata", "sizeof_commondata", "sizeof_params"):
            assert got[k] == lay[k], k


def test_library_of_the_other_order_is_refused():
    if not (ROOT / "nrpy_b200" / "libbssn_b200_fd8.so").exists():
        pytest.skip("libbssn_b200_fd8.so not built")
    env = dict(os.environ, BSSN_B200_FD_ORDER="4", BSSN_B200_LIB=str(ROOT / "nrpy_b200" / "libbssn_b200_fd8.so"))
    r = subprocess.run([sys.executable, "-c", "from nrpy_b200 import lib; lib.load()"], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode != 0 and "built for fd_order 8" in r.stderr
