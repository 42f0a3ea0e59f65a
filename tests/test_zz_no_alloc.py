"""The allocation-free constraint integrals, bssn_b200_constraint_integrals_noalloc.

Some callers cannot allocate device memory: a host framework that routes every
allocation through its own pool or arena (a cudaMalloc behind its back escapes its
accounting and its memory cap), or an embedded host that forbids allocation after
start-up so that its footprint stays fixed. For them the library offers this variant of
bssn_b200_constraint_integrals whose scratch is a static __device__ array. These tests
call it through the C ABI twice in a row and check both results against the allocating
entry point (different reduction trees, so agreement is to rounding: relative 1e-12).
They cover grids of one partial block and of many (2048 interior points per block, with
point counts that are not a multiple of it), a large grid followed by a small one on the
shared array, and the documented size limit.

Kept in a file of its own, collected last, so a failure here does not hide the others.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from tests.util import load_golden

pytestmark = pytest.mark.gpu

PTS_PER_BLOCK = 2048  # interior points summed by one partial of the static array


def _golden_grid(name, coord, sym, cuda):
    from nrpy_b200.grid import BSSNGrid

    g = load_golden(name)
    m1, z1, m2, z2 = [float(x) for x in g["bh"]]
    grid = BSSNGrid(coord=coord, Nxx=tuple(int(x) for x in g["Nxx"]), grid_physical_size=float(g["grid_physical_size"]),
                    SINHW=float(g["SINHW"]), BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2,
                    symmetry_axes=sym)
    return grid, torch.from_numpy(np.ascontiguousarray(g["input"])).to(cuda)


def _bl_grid(coord, Nxx, seed):
    """A Brill-Lindquist grid a few RK4 steps in, so every constraint has content."""
    from nrpy_b200.grid import BSSNGrid

    rng = np.random.default_rng(seed)
    grid = BSSNGrid(coord=coord, Nxx=Nxx, grid_physical_size=10.0 if coord == "SinhSpherical" else 7.5,
                    SINHW=0.2, BH1_mass=float(rng.uniform(0.3, 0.7)), BH1_posn_z=float(rng.uniform(0.3, 0.8)),
                    BH2_mass=float(rng.uniform(0.3, 0.7)), BH2_posn_z=-float(rng.uniform(0.3, 0.8)))
    for _ in range(3):
        grid.MoL_step_forward_in_time(mode=1)
    return grid, grid.y_n


def _both(grid, inp):
    """(allocating result, [two no-alloc results]) for the diagnostics of `inp`."""
    from nrpy_b200 import lib as L

    lib = L.load()
    diag = grid.constraints_eval(inp)
    torch.cuda.synchronize()
    g = grid.gd[0]
    dptr = C.cast(C.c_void_p(diag.data_ptr()), L.PR)
    ref = (C.c_double * 4)()
    L.check(lib.bssn_b200_constraint_integrals(C.byref(g.params), g.rfmstruct, dptr, ref, grid.stream))
    outs = []
    for _ in range(2):  # two calls in a row: the shared static scratch must not leak between calls
        out = (C.c_double * 4)()
        L.check(lib.bssn_b200_constraint_integrals_noalloc(C.byref(g.params), g.rfmstruct, dptr, out, grid.stream))
        outs.append(np.array(out[:]))
    return np.array(ref[:]), outs


@pytest.mark.parametrize("name,coord,sym", [("sinh3d_10x6x6", "SinhSpherical", ""),
                                            ("sphaxi_16x6x2", "Spherical", "2")])
def test_noalloc_matches_allocating_entry_point(cuda, name, coord, sym):
    grid, inp = _golden_grid(name, coord, sym, cuda)
    ref, outs = _both(grid, inp)
    assert ref[3] > 0 and np.all(np.isfinite(ref))
    for out in outs:
        np.testing.assert_allclose(out, ref, rtol=1e-12, atol=0)
    grid.close()


@pytest.mark.parametrize("coord,Nxx", [("Spherical", (60, 30, 30)), ("SinhSpherical", (64, 32, 32))])
def test_noalloc_many_partials(cuda, coord, Nxx):
    """Grids of many partial blocks: 54,000 points (26.4 blocks, a ragged last block) and
    65,536 points (32 full blocks), summed over several entries of the static array."""
    grid, inp = _bl_grid(coord, Nxx, seed=7 + Nxx[0])
    n = Nxx[0] * Nxx[1] * Nxx[2]
    assert n > 8 * PTS_PER_BLOCK
    ref, outs = _both(grid, inp)
    assert ref[0] > 0 and ref[3] > 0 and np.all(np.isfinite(ref))
    for out in outs:
        np.testing.assert_allclose(out, ref, rtol=1e-12, atol=0)
    grid.close()


def test_noalloc_large_then_small(cuda):
    """A many-block call leaves its partials in the shared array; a following one-block
    call must read only its own entries."""
    big, big_in = _bl_grid("SinhSpherical", (48, 24, 20), seed=11)
    ref_big, outs_big = _both(big, big_in)
    small, small_in = _golden_grid("sinh3d_10x6x6", "SinhSpherical", "", cuda)
    ref_small, outs_small = _both(small, small_in)
    for out in outs_big:
        np.testing.assert_allclose(out, ref_big, rtol=1e-12, atol=0)
    for out in outs_small:
        np.testing.assert_allclose(out, ref_small, rtol=1e-12, atol=0)
    big.close()
    small.close()


def test_noalloc_rejects_oversized_grids(cuda):
    from nrpy_b200 import lib as L

    lib = L.load()
    grid, inp = _golden_grid("sinh3d_10x6x6", "SinhSpherical", "", cuda)
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
