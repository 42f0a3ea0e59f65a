"""GPU parity against the committed golden fixtures (outputs of the reference's own
generated BHaH C, produced by tests/golden/make_golden.py).

Bars: bit-exact for grid coordinates and bcstruct index/parity maps; per-gridfunction
relative L2 <= 1e-12 for one FP64 application of each operator and for one RK4 step.
"""

import numpy as np
import pytest
import torch

from tests.util import as4, interior, load_golden, rel_l2_per_gf

CASES = {
    "sphaxi_16x6x2": dict(coord="Spherical", symmetry_axes="2"),
    "sph3d_10x6x6": dict(coord="Spherical", symmetry_axes=""),
    "sinh3d_10x6x6": dict(coord="SinhSpherical", symmetry_axes=""),
}
TOL = 1e-12

pytestmark = pytest.mark.gpu


def make_grid(name, g, **kw):
    from nrpy_b200.grid import BSSNGrid

    m1, z1, m2, z2 = [float(x) for x in g["bh"]]
    return BSSNGrid(coord=CASES[name]["coord"], Nxx=tuple(int(x) for x in g["Nxx"]),
                    grid_physical_size=float(g["grid_physical_size"]), SINHW=float(g["SINHW"]), BH1_mass=m1,
                    BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2, symmetry_axes=CASES[name]["symmetry_axes"], **kw)


def to_dev(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.fixture(scope="module", params=list(CASES))
def case(request, cuda):
    name = request.param
    g = load_golden(name)
    grid = make_grid(name, g)
    yield name, g, grid
    grid.close()


def test_grid_and_bcstruct_bit_exact(case):
    name, g, grid = case
    assert tuple(grid.N) == tuple(int(x) for x in g["N"])
    xx = grid.xx()
    for d in range(3):
        assert np.array_equal(xx[d], g[f"xx{d}"]), f"xx{d} differs"
    np.testing.assert_allclose(grid.dt, float(g["dt"]), rtol=2e-16, atol=0)
    inner, outer, info = grid.bcstruct()
    assert len(inner) == len(g["inner_dst"])
    dst = np.array([p.dstpt for p in inner])
    src = np.array([p.srcpt for p in inner])
    par = np.array([list(p.parity) for p in inner], dtype=np.int8)
    assert np.array_equal(dst, g["inner_dst"])
    assert np.array_equal(src, g["inner_src"])
    assert np.array_equal(par, g["inner_parity"])
    for gz in range(3):
        for d in range(3):
            ref = g[f"outer_{gz}_{d}"]
            mine = np.array([[o.i0, o.i1, o.i2, o.FACEX0, o.FACEX1, o.FACEX2] for o in outer[(gz, d)]],
                            dtype=np.int16).reshape(-1, 6)
            assert np.array_equal(mine, ref), f"outer list ({gz},{d}) differs"


def test_rfm_precompute(case):
    name, g, grid = case
    rfm = grid.rfm()
    for k in g:
        if k.startswith("rfm_"):
            np.testing.assert_allclose(rfm[k[4:]], g[k], rtol=1e-15, atol=0)


def test_initial_data(case):
    name, g, grid = case
    mine = as4(grid.y_n.cpu().numpy(), grid.N)
    ref = as4(g["initial_data"], grid.N)
    # alpha and cf carry the data; the rest is zero up to rounding in both codes.
    for gf in (6, 10):
        np.testing.assert_allclose(mine[gf], ref[gf], rtol=1e-13, atol=0)
    assert np.max(np.abs(mine - ref)) < 1e-11


def test_ricci(case):
    name, g, grid = case
    inp = to_dev(g["input"], grid.device)
    aux = torch.zeros(6 * grid.ntot, dtype=torch.float64, device=grid.device)
    grid.ricci_eval(inp, aux)
    torch.cuda.synchronize()
    err = rel_l2_per_gf(interior(as4(aux.cpu().numpy(), grid.N)), interior(as4(g["ricci"], grid.N)))
    assert err.max() <= TOL, err


def test_rhs_and_radiation_bcs(case):
    name, g, grid = case
    inp = to_dev(g["input"], grid.device)
    aux = to_dev(g["ricci"], grid.device)
    rhs = torch.zeros(24 * grid.ntot, dtype=torch.float64, device=grid.device)
    grid.rhs_eval(aux, inp, rhs)
    grid.apply_bcs_outerradiation_and_inner(inp, rhs)
    torch.cuda.synchronize()
    mine, ref = as4(rhs.cpu().numpy(), grid.N), as4(g["rhs_bc"], grid.N)
    err_int = rel_l2_per_gf(interior(mine), interior(ref))
    assert err_int.max() <= TOL, err_int
    err_all = rel_l2_per_gf(mine, ref)
    assert err_all.max() <= TOL, err_all


def test_enforce_detgammabar(case):
    name, g, grid = case
    y = to_dev(g["input"], grid.device)
    grid.enforce_detgammabar_equals_detgammahat(y)
    torch.cuda.synchronize()
    mine = as4(y.cpu().numpy(), grid.N)[11:17]
    ref = as4(g["enforce_hDD"], grid.N)
    err = rel_l2_per_gf(mine, ref)
    assert err.max() <= TOL, err


@pytest.mark.parametrize("mode", [0, 1])
def test_one_rk4_step(case, mode):
    name, g, grid = case
    grid.y_n.copy_(to_dev(g["input"], grid.device))
    grid.cd.time, grid.cd.nn = 0.0, 0
    grid.MoL_step_forward_in_time(mode=mode)
    torch.cuda.synchronize()
    err = rel_l2_per_gf(as4(grid.y_n.cpu().numpy(), grid.N), as4(g["step1"], grid.N))
    assert err.max() <= TOL, err
    assert grid.cd.nn == 1 and abs(grid.cd.time - grid.dt) < 1e-15


def test_constraints(case):
    name, g, grid = case
    inp = to_dev(g["input"], grid.device)
    diag = grid.constraints_eval(inp)
    torch.cuda.synchronize()
    mine = interior(as4(diag.cpu().numpy(), grid.N))
    ref = interior(as4(g["constraints"], grid.N))
    err = rel_l2_per_gf(mine, ref)
    assert err.max() <= 1e-10, err
    norms = grid.constraint_norms(inp)
    dV = interior(as4(g["dV"], grid.N))[0]
    ref_int = [(ref[k] ** 2 * dV).sum() for k in range(3)]
    for k, nm in enumerate(["H", "MSQUARED", "LAMBDA_CONSTRAINT"]):
        np.testing.assert_allclose(norms[f"{nm}_L2"] ** 2, ref_int[k], rtol=1e-10)
    np.testing.assert_allclose(norms["volume"], dV.sum(), rtol=1e-12)
