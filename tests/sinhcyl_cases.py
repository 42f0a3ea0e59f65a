"""SinhCylindrical (symmetry_axes "1", axisymmetric about z, as blackhole_spectroscopy.py runs
it) against the reference's generated C of the same coordinates: oracle variant sinhcyl (4th
order) or sinhcyl8 (8th order), chosen by the finite-difference order of the loaded library.

Collected by tests/test_sinhcyl_gpu.py (4th order, in process) and tests/fd8_cases.py (8th
order, in the child process). Bars as for the Spherical family: bit-exact grid, dt and
bcstruct; initial data alpha and W to 1e-13 relative on the interior and every value to 1e-11;
Ricci and the RHS to 1e-12 per-gridfunction relative L2 (the RHS of trK to 1e-11, see the
test); 20 RK4 steps to 1e-10 (both stage orders, radiation and extrapolation outer BCs); the
constraint integrals to 1e-10; the diagnostics() files with the bars of the spherical families.
"""

import numpy as np
import pytest
import torch

from oracle import ref as oref
from tests.util import compare_diagnostics_dirs, rel_l2_per_gf

pytestmark = pytest.mark.gpu

# rho x phi x z, two phi points as the axisymmetric projects use. AMPLRHO = AMPLZ = 30 puts the
# innermost rho (0.025) where blackhole_spectroscopy's grid (300, 400 x 2 x 1200) has it: the
# (1/rho) d_rho terms near the axis amplify rounding differences of the two codes' expression
# orders by about 1/rho_min^2.
NXX = (40, 2, 64)
L = 30.0


def _ng():
    from nrpy_b200 import lib

    return lib.NGHOSTS, ("sinhcyl" if lib.FD_ORDER == 4 else f"sinhcyl{lib.FD_ORDER}")


def _pair(bh=(0.45, 0.5, 0.55, -0.6), outer="radiation"):
    from nrpy_b200.grid import BSSNGrid

    ng, variant = _ng()
    if not oref.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")
    m1, z1, m2, z2 = bh
    rg = oref.RefGrid(variant, NXX, L, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2,
                      outer_bc_type=outer)
    g = BSSNGrid(coord="SinhCylindrical", Nxx=NXX, grid_physical_size=L, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1,
                 BH2_mass=m2, BH2_posn_z=z2, outer_bc_type=outer, symmetry_axes="1")
    assert rg.nghosts == ng and g.N == rg.N
    return rg, g, ng


def _as4(a, N):
    return np.asarray(a).reshape(-1, N[2], N[1], N[0])


def test_sinhcyl_grid_bcstruct_and_initial_data(cuda):
    rg, g, ng = _pair()
    for a, b in zip(g.xx(), rg.xx()):
        assert np.array_equal(a, b)
    assert g.dt == rg.dt
    from nrpy_b200 import lib

    mine = g.rfm()
    for k, (name, _) in enumerate(lib.RfmStruct._fields_):
        n = g.N[0] if name.startswith("f0") else g.N[2]  # the second rfm function is f3(xx2) here
        np.testing.assert_allclose(mine[name], rg.rfm_field(k, n), rtol=1e-15, atol=0, err_msg=name)
    inner, outer, info = g.bcstruct()
    r_inner, r_outer = rg.bcstruct()
    assert len(inner) == len(r_inner) > 0
    assert np.array_equal(np.array([p.dstpt for p in inner]), r_inner["dstpt"])
    assert np.array_equal(np.array([p.srcpt for p in inner]), r_inner["srcpt"])
    assert np.array_equal(np.array([list(p.parity) for p in inner]), r_inner["parity"])
    n_outer = 0
    for (gz, d), arr in r_outer.items():
        mine_o = outer[(gz, d)]
        assert len(mine_o) == len(arr)
        n_outer += len(arr)
        if len(arr):
            assert np.array_equal(
                np.array([(p.i0, p.i1, p.i2, p.FACEX0, p.FACEX1, p.FACEX2) for p in mine_o]).reshape(-1, 6),
                np.stack([arr[k] for k in ("i0", "i1", "i2", "FACEX0", "FACEX1", "FACEX2")], 1))
    assert n_outer > 0 and all(len(outer[(gz, 1)]) == 0 for gz in range(ng))  # outer faces: rho max, z min/max
    torch.cuda.synchronize()
    y_ref = _as4(rg.y_n(), g.N)
    y = _as4(g.y_n.cpu().numpy(), g.N)
    # alpha and W on the interior to 1e-13 relative. The outer ghost layers are extrapolated
    # (3 f1 - 3 f2 + f3, layer after layer), which multiplies a rounding difference by up to
    # 7 per layer; there, as for every other gridfunction, the bar is 1e-11 absolute.
    sl = (slice(ng, -ng), slice(ng, -ng), slice(ng, -ng))
    for gf in (6, 10):  # alpha, W
        np.testing.assert_allclose(y[gf][sl], y_ref[gf][sl], rtol=1e-13, atol=0)
    diff = np.abs(y - y_ref).reshape(24, -1).max(axis=1)
    assert diff.max() < 1e-11, diff
    rg.close()
    g.close()


def test_sinhcyl_dt_matches_reference(cuda):
    """The CFL timestep equals the reference's bit for bit on grids whose smallest spacing lies
    along z (where the reference's compiled z' sum is a fused multiply-add) and along rho."""
    from nrpy_b200.grid import BSSNGrid

    _, variant = _ng()
    if not oref.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")
    for nxx, L in [((40, 2, 120), 10.0), ((40, 2, 64), 30.0), ((40, 2, 120), 30.0), ((64, 2, 40), 10.0)]:
        rg = oref.RefGrid(variant, nxx, L, SINHW=0.2)
        g = BSSNGrid(coord="SinhCylindrical", Nxx=nxx, grid_physical_size=L, SINHW=0.2, symmetry_axes="1")
        assert g.dt == rg.dt, (nxx, L, g.dt, rg.dt)
        rg.close()
        g.close()


def test_sinhcyl_ricci_rhs_constraints(cuda):
    rg, g, ng = _pair()
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
    sl = (slice(None), slice(ng, -ng), slice(ng, -ng), slice(ng, -ng))
    e_r = rel_l2_per_gf(_as4(aux.cpu().numpy(), g.N)[sl], _as4(ricci, g.N)[sl])
    e_rhs = rel_l2_per_gf(_as4(out.cpu().numpy(), g.N)[sl], _as4(rhs, g.N)[sl])
    assert e_r.max() <= 1e-12, e_r
    # The RHS of trK (-D^2 alpha + ...) differs by ~1e-13 absolute at the first rho points: the
    # second differences of alpha there carry eps * alpha * invdxx0^2 / rho'^2 of rounding, which
    # the two codes' different evaluation orders round differently; trK's RHS is small elsewhere,
    # so its relative L2 is 1.5e-12 (4th order) to 1.8e-12 (8th). Every other RHS is below 1e-12.
    assert e_rhs.max() <= 1e-11, e_rhs
    assert np.delete(e_rhs, 20).max() <= 1e-12, e_rhs
    cons = rg.constraints(inp, ricci)
    dV = rg.dV()
    norms = g.constraint_norms(ti)
    for k, nm in enumerate(["H", "MSQUARED", "LAMBDA_CONSTRAINT"]):
        c = cons[k].reshape(g.N[2], g.N[1], g.N[0])[ng:-ng, ng:-ng, ng:-ng]
        ref_int = float((c**2 * dV[ng:-ng, ng:-ng, ng:-ng]).sum())
        assert norms[f"{nm}_L2"] ** 2 == pytest.approx(ref_int, rel=1e-10), nm
    rg.close()
    g.close()


@pytest.mark.parametrize("mode,outer", [(0, "radiation"), (1, "radiation"), (0, "extrapolation")])
def test_sinhcyl_20_steps(cuda, mode, outer):
    rg, g, ng = _pair(outer=outer)
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


def test_sinhcyl_brill_lindquist_50_steps(cuda):
    """50 fused RK4 steps from the reference's own Brill-Lindquist data (holes on the z axis)."""
    rg, g, ng = _pair(bh=(0.5, 0.6, 0.5, -0.6))
    g.y_n.copy_(torch.from_numpy(rg.y_n()).to(g.device))
    rg.step(50)
    g.MoL_step_forward_in_time(mode=1, nsteps=50)
    torch.cuda.synchronize()
    m = g.y_n.cpu().numpy().reshape(24, -1)
    r = rg.y_n().reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    err = num / np.where(den < 1e-8 * den.max(), den.max(), den)  # vanishing phi components: against the largest
    assert err.max() <= 1e-10, err
    rg.close()
    g.close()


def test_sinhcyl_diagnostics_files(cuda, tmp_path, monkeypatch):
    """diagnostics() of a perturbed state at two output steps against the reference's own:
    the grid-centre point, the y lines at phi = +-pi/2 in the z mid-plane, the z line along the
    axis, the xy plane at mid z, the yz plane at phi = +-pi/2, and the volume integrals with the
    SinhCylindrical volume element."""
    rg, g, ng = _pair()
    state = oref.perturbed_state(rg, seed=4)
    rg.set_y_n(state)
    g.y_n.copy_(torch.from_numpy(state).to(g.device))
    for d in ("ref", "ours"):
        (tmp_path / d).mkdir()
    for nn, t in [(0, 0.0), (7, 0.25)]:
        monkeypatch.chdir(tmp_path / "ref")
        rg.diagnostics(nn, t, 0.25)
        monkeypatch.chdir(tmp_path / "ours")
        g.diagnostics(0.25, nn=nn, time=t)
        torch.cuda.synchronize()
    monkeypatch.chdir(tmp_path)
    names = compare_diagnostics_dirs(tmp_path / "ref", tmp_path / "ours")
    assert any(n.startswith("out1d-z-SinhCylindrical") for n in names)
    assert any("sphere_R_gt_8" in n for n in names)
    rg.close()
    g.close()
