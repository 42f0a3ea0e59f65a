"""8th-order finite differences (libbssn_b200_fd8.so, NGHOSTS = 5) against the reference's own
generated C at fd_order = 8 (oracle variants sph3d8, sinh3d8, sphaxi8, sinhaxi8, sinhcyl8). B200.

Not collected by the main test run: the library's finite-difference order is fixed per
process (BSSN_B200_FD_ORDER, read when nrpy_b200.lib is imported), so test_fd8_gpu.py runs
this file in a child process with BSSN_B200_FD_ORDER=8. Bars as at 4th order: bit-exact
grid and bcstruct, per-gridfunction relative L2 <= 1e-12 for Ricci and the RHS, <= 1e-10
after 20 RK4 steps; initial data alpha and W to 1e-13 relative and every other value to 1e-11;
constraint integrals to 1e-10.
"""

import os

import numpy as np
import pytest
import torch

from oracle import ref as oref
from tests.util import compare_diagnostics_dirs, rel_l2_per_gf

from tests.sinhaxi_cases import test_sinhaxi_20_steps, test_sinhaxi_ricci_rhs  # noqa: F401  (oracle sinhaxi8)
from tests.sinhcyl_cases import (  # noqa: F401  (SinhCylindrical at 8th order: oracle variant sinhcyl8)
    test_sinhcyl_20_steps,
    test_sinhcyl_brill_lindquist_50_steps,
    test_sinhcyl_diagnostics_files,
    test_sinhcyl_dt_matches_reference,
    test_sinhcyl_grid_bcstruct_and_initial_data,
    test_sinhcyl_ricci_rhs_constraints,
)

pytestmark = pytest.mark.gpu
G = 5


def as4(a, N):
    return np.asarray(a).reshape(-1, N[2], N[1], N[0])


def interior(a4):
    return a4[:, G:-G, G:-G, G:-G]


def need(variant):
    if not oref.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")


@pytest.fixture(scope="module", autouse=True)
def fd8_process():
    from nrpy_b200 import lib as L

    assert os.environ.get("BSSN_B200_FD_ORDER") == "8" and L.FD_ORDER == 8 and L.NGHOSTS == G
    assert L.load().bssn_b200_fd_order() == 8


def pair(variant, coord, Nxx, L, bh=(0.45, 0.5, 0.55, -0.6), outer="radiation", sym=""):
    from nrpy_b200.grid import BSSNGrid

    m1, z1, m2, z2 = bh
    rg = oref.RefGrid(variant, Nxx, L, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2,
                      outer_bc_type=outer)
    g = BSSNGrid(coord=coord, Nxx=Nxx, grid_physical_size=L, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2,
                 BH2_posn_z=z2, outer_bc_type=outer, symmetry_axes=sym)
    assert rg.nghosts == G and g.N == rg.N
    return rg, g


CASES = [("sph3d8", "Spherical", (32, 16, 16), 7.5), ("sinh3d8", "SinhSpherical", (48, 16, 16), 10.0)]


@pytest.mark.parametrize("variant,coord,nxx,L", CASES)
def test_grid_bcstruct_and_initial_data(cuda, variant, coord, nxx, L):
    need(variant)
    rg, g = pair(variant, coord, nxx, L)
    for a, b in zip(g.xx(), rg.xx()):
        assert np.array_equal(a, b)
    assert g.dt == rg.dt
    inner, outer, info = g.bcstruct()
    r_inner, r_outer = rg.bcstruct()
    assert len(inner) == len(r_inner)
    assert np.array_equal(np.array([p.dstpt for p in inner]), r_inner["dstpt"])
    assert np.array_equal(np.array([p.srcpt for p in inner]), r_inner["srcpt"])
    assert np.array_equal(np.array([list(p.parity) for p in inner]), r_inner["parity"])
    for (gz, d), arr in r_outer.items():
        mine = outer[(gz, d)]
        assert len(mine) == len(arr)
        assert np.array_equal(np.array([(p.i0, p.i1, p.i2, p.FACEX0, p.FACEX1, p.FACEX2) for p in mine]).reshape(-1, 6),
                              np.stack([arr[k] for k in ("i0", "i1", "i2", "FACEX0", "FACEX1", "FACEX2")], 1))
    torch.cuda.synchronize()
    y_ref = as4(rg.y_n(), g.N)
    y = as4(g.y_n.cpu().numpy(), g.N)
    # alpha and W = cf carry the data (rtol 1e-13); the rest is zero up to rounding in both codes,
    # or lambda^i from finite differences of that rounding (1e-11 absolute), as at 4th order.
    for gf in (6, 10):
        np.testing.assert_allclose(y[gf], y_ref[gf], rtol=1e-13, atol=0)
    diff = np.abs(y - y_ref).reshape(24, -1).max(axis=1)
    assert diff.max() < 1e-11, diff
    rg.close()
    g.close()


@pytest.mark.parametrize("variant,coord,nxx,L", CASES)
def test_ricci_rhs_constraints(cuda, variant, coord, nxx, L):
    need(variant)
    rg, g = pair(variant, coord, nxx, L)
    inp = oref.perturbed_state(rg, seed=5, amp=0.03)
    ricci = rg.ricci(inp)
    rhs = rg.rhs(ricci, inp)
    dev = g.device
    ti = torch.from_numpy(inp).to(dev)
    aux = torch.zeros(6 * g.ntot, dtype=torch.float64, device=dev)
    g.ricci_eval(ti, aux)
    out = torch.zeros(24 * g.ntot, dtype=torch.float64, device=dev)
    g.rhs_eval(aux, ti, out)
    torch.cuda.synchronize()
    e_r = rel_l2_per_gf(interior(as4(aux.cpu().numpy(), g.N)), interior(as4(ricci, g.N)))
    e_rhs = rel_l2_per_gf(interior(as4(out.cpu().numpy(), g.N)), interior(as4(rhs, g.N)))
    assert e_r.max() <= 1e-12, e_r
    assert e_rhs.max() <= 1e-12, e_rhs
    cons = rg.constraints(inp, ricci)
    dV = rg.dV()
    norms = g.constraint_norms(ti)
    for k, nm in enumerate(["H", "MSQUARED", "LAMBDA_CONSTRAINT"]):
        c = cons[k].reshape(g.N[2], g.N[1], g.N[0])[G:-G, G:-G, G:-G]
        ref_int = float((c**2 * dV[G:-G, G:-G, G:-G]).sum())
        assert norms[f"{nm}_L2"] ** 2 == pytest.approx(ref_int, rel=1e-10), nm
    rg.close()
    g.close()


@pytest.mark.parametrize("mode,outer", [(0, "radiation"), (1, "radiation"), (0, "extrapolation")])
def test_20_steps(cuda, mode, outer):
    need("sph3d8")
    rg, g = pair("sph3d8", "Spherical", (32, 16, 16), 7.5, outer=outer)
    inp = oref.perturbed_state(rg, seed=3, amp=0.02)
    rg.set_y_n(inp)
    g.y_n.copy_(torch.from_numpy(inp).to(g.device))
    rg.step(20)
    g.MoL_step_forward_in_time(mode=mode, nsteps=20)
    torch.cuda.synchronize()
    m = g.y_n.cpu().numpy().reshape(24, -1)
    r = rg.y_n().reshape(24, -1)
    err = np.sqrt(((m - r) ** 2).sum(axis=1)) / np.sqrt((r**2).sum(axis=1))
    assert err.max() <= 1e-10, err
    assert g.cd.nn == 20 and g.cd.time == pytest.approx(rg.time, rel=1e-15)
    rg.close()
    g.close()


def test_sinh_steps_graph(cuda):
    """SinhSpherical 48x16x16: 5 RK4 steps replayed from a captured graph."""
    need("sinh3d8")
    rg, g = pair("sinh3d8", "SinhSpherical", (48, 16, 16), 10.0)
    inp = oref.perturbed_state(rg, seed=8, amp=0.02)
    rg.set_y_n(inp)
    g.y_n.copy_(torch.from_numpy(inp).to(g.device))
    rg.step(5)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        g.make_stepper(mode=1, steps_per_graph=5)
        g.run_stepper(1)
    torch.cuda.synchronize()
    m = g.y_n.cpu().numpy().reshape(24, -1)
    r = rg.y_n().reshape(24, -1)
    err = np.sqrt(((m - r) ** 2).sum(axis=1)) / np.sqrt((r**2).sum(axis=1))
    assert err.max() <= 1e-10, err
    g.free_stepper()
    rg.close()
    g.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_axisymmetric_100_steps(cuda, mode):
    """Spherical 72x12x2, symmetry_axes='2' (the small workload at 8th order), 100 RK4 steps
    from the reference's initial data."""
    need("sphaxi8")
    rg, g = pair("sphaxi8", "Spherical", (72, 12, 2), 7.5, bh=(0.5, 0.5, 0.5, -0.5), sym="2")
    g.y_n.copy_(torch.from_numpy(rg.y_n()).to(g.device))
    rg.step(100)
    g.MoL_step_forward_in_time(mode=mode, nsteps=100)
    torch.cuda.synchronize()
    m = g.y_n.cpu().numpy().reshape(24, -1)
    r = rg.y_n().reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    err = num / np.maximum(den, 1e-13 * den.max())  # components that vanish analytically: against a floor
    assert err.max() <= 1e-10, err
    rg.close()
    g.close()


def test_batch_equals_single_grid_path(cuda):
    """Two uneven Spherical grids advanced together by the batched persistent kernels, 4 RK4
    steps, against each grid stepped alone."""
    from nrpy_b200.batch import BatchedEvolutions
    from nrpy_b200.grid import BSSNGrid

    specs = [dict(coord="Spherical", Nxx=(24, 10, 6), grid_physical_size=7.5, BH1_mass=0.45, BH1_posn_z=0.35,
                  BH2_mass=0.6, BH2_posn_z=-0.35),
             dict(coord="Spherical", Nxx=(37, 12, 4), grid_physical_size=7.5, BH1_mass=0.31, BH1_posn_z=0.7,
                  BH2_mass=0.66, BH2_posn_z=-0.7)]
    be = BatchedEvolutions(specs)
    be.build(tile=(32, 4), steps_per_graph=2)
    be.run(2)
    torch.cuda.synchronize()
    for spec, g in zip(specs, be.grids):
        single = BSSNGrid(**spec)
        single.MoL_step_forward_in_time(mode=1, nsteps=4)
        torch.cuda.synchronize()
        a = single.y_n.view(24, -1).cpu().numpy()
        b = g.y_n.view(24, -1).cpu().numpy()
        err = rel_l2_per_gf(b, a, floor=1e-300)
        assert np.nanmax(np.where(np.linalg.norm(a, axis=1) > 0, err, 0)) <= 1e-14, err
        single.close()
    be.close()


def test_diagnostics_files_match_reference(cuda, tmp_path, monkeypatch):
    """The diagnostics() outputs (nearest-point samples, volume integrals) of a perturbed
    8th-order state against the reference's own diagnostics() at fd_order 8."""
    need("sph3d8")
    rg, g = pair("sph3d8", "Spherical", (24, 12, 12), 7.5)
    state = oref.perturbed_state(rg, seed=4)
    rg.set_y_n(state)
    g.y_n.copy_(torch.from_numpy(state).to(g.device))
    for d in ("ref", "ours"):
        (tmp_path / d).mkdir()
    monkeypatch.chdir(tmp_path / "ref")
    rg.diagnostics(0, 0.0, 0.25)
    monkeypatch.chdir(tmp_path / "ours")
    g.diagnostics(0.25, nn=0, time=0.0)
    torch.cuda.synchronize()
    monkeypatch.chdir(tmp_path)
    compare_diagnostics_dirs(tmp_path / "ref", tmp_path / "ours")
    rg.close()
    g.close()


def test_checkpoint_restart_bitwise(cuda, tmp_path, monkeypatch):
    """A run restarted from a checkpoint (5 ghost layers) continues bit-identically."""
    monkeypatch.chdir(tmp_path)
    from nrpy_b200.grid import BSSNGrid

    kw = dict(coord="Spherical", Nxx=(24, 12, 12), grid_physical_size=7.5)
    a = BSSNGrid(**kw)
    a.MoL_step_forward_in_time(nsteps=4)
    b = BSSNGrid(**kw)
    b.MoL_step_forward_in_time(nsteps=2)
    assert b.write_checkpoint(b.cd.time)
    c = BSSNGrid(**kw, initial_data=False)
    assert c.read_checkpoint() is not None
    c.MoL_step_forward_in_time(nsteps=2)
    torch.cuda.synchronize()
    assert torch.equal(a.y_n, c.y_n) and c.cd.nn == 4
    for x in (a, b, c):
        x.close()


def test_adjoint_refused(cuda):
    import ctypes as C

    from nrpy_b200 import lib as L

    lib = L.load()
    out = C.c_void_p()
    rc = lib.bssn_b200_adjoint_create(None, None, 1, 1, None, C.byref(out))
    assert rc == -1 and b"4th-order" in lib.bssn_b200_last_error()
