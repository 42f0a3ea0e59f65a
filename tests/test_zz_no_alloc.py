"""The allocation-free constraint integrals, bssn_b200_constraint_integrals_noalloc.

Some callers cannot allocate device memory: a host framework that routes every
allocation through its own pool or arena, code running while a CUDA graph is captured,
or embedded hosts that forbid allocation after start-up. For them the library offers
this variant of bssn_b200_constraint_integrals whose scratch is a static __device__
array. This test calls it through the C ABI twice in a row and checks both results
against the allocating entry point (different reduction trees, so agreement is to
rounding: relative 1e-12), plus the documented size limit.

Kept in a file of its own, collected last, so a failure here does not hide the others.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from tests.util import load_golden

pytestmark = pytest.mark.gpu


def _grid(name, coord, sym, cuda):
    from nrpy_b200.grid import BSSNGrid

    g = load_golden(name)
    m1, z1, m2, z2 = [float(x) for x in g["bh"]]
    grid = BSSNGrid(coord=coord, Nxx=tuple(int(x) for x in g["Nxx"]), grid_physical_size=float(g["grid_physical_size"]),
                    SINHW=float(g["SINHW"]), BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2,
                    symmetry_axes=sym)
    return grid, torch.from_numpy(np.ascontiguousarray(g["input"])).to(cuda)


@pytest.mark.parametrize("name,coord,sym", [("sinh3d_10x6x6", "SinhSpherical", ""),
                                            ("sphaxi_16x6x2", "Spherical", "2")])
def test_noalloc_matches_allocating_entry_point(cuda, name, coord, sym):
    from nrpy_b200 import lib as L

    lib = L.load()
    grid, inp = _grid(name, coord, sym, cuda)
    diag = grid.constraints_eval(inp)
    torch.cuda.synchronize()
    g = grid.gd[0]
    dptr = C.cast(C.c_void_p(diag.data_ptr()), L.PR)
    stream = grid.stream
    ref = (C.c_double * 4)()
    L.check(lib.bssn_b200_constraint_integrals(C.byref(g.params), g.rfmstruct, dptr, ref, stream))
    ref = np.array(ref[:])
    assert ref[3] > 0 and np.all(np.isfinite(ref))
    for _ in range(2):  # two calls in a row: the shared static scratch must not leak between calls
        out = (C.c_double * 4)()
        L.check(lib.bssn_b200_constraint_integrals_noalloc(C.byref(g.params), g.rfmstruct, dptr, out, stream))
        np.testing.assert_allclose(np.array(out[:]), ref, rtol=1e-12, atol=0)
    grid.close()


def test_noalloc_rejects_oversized_grids(cuda):
    from nrpy_b200 import lib as L

    lib = L.load()
    grid, inp = _grid("sinh3d_10x6x6", "SinhSpherical", "", cuda)
    diag = grid.constraints_eval(inp)
    torch.cuda.synchronize()
    g = grid.gd[0]
    big = L.ParamsStruct()
    C.pointer(big)[0] = g.params
    big.Nxx_plus_2NGHOSTS0 = 4096 + 6
    big.Nxx_plus_2NGHOSTS1 = 4096 + 6
    big.Nxx_plus_2NGHOSTS2 = 3 + 6  # 50.3M interior points, above the 33.5M limit
    out = (C.c_double * 4)()
    rc = lib.bssn_b200_constraint_integrals_noalloc(C.byref(big), g.rfmstruct,
                                                    C.cast(C.c_void_p(diag.data_ptr()), L.PR), out, grid.stream)
    assert rc == -1
    assert b"exceed" in lib.bssn_b200_last_error()
    grid.close()
