"""GPU parity against the live reference oracle (oracle/_ref: the reference's own generated
BHaH C, compiled by oracle/gen_ref.py) at the workload sizes.

Bars: per-gridfunction relative L2 <= 1e-12 after one FP64 RHS,
<= 1e-10 after 100 FP64 RK4 steps. Starting states are the reference's own initial data
(so that rounding differences of the two initial-data codes do not enter), or the
reference's data plus seeded smooth perturbations of all 24 gridfunctions.
"""

import numpy as np
import pytest
import torch

from oracle import ref as oref
from tests.sinhaxi_cases import test_sinhaxi_20_steps, test_sinhaxi_ricci_rhs  # noqa: F401  (oracle sinhaxi)
from tests.util import as4, interior, rel_l2_per_gf

pytestmark = pytest.mark.gpu


def need(variant):
    if not oref.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")


def pair(variant, coord, Nxx, L, sym, bh=(0.5, 0.5, 0.5, -0.5), outer="radiation"):
    from nrpy_b200.grid import BSSNGrid

    m1, z1, m2, z2 = bh
    rg = oref.RefGrid(variant, Nxx, L, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2,
                      outer_bc_type=outer)
    g = BSSNGrid(coord=coord, Nxx=Nxx, grid_physical_size=L, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2,
                 BH2_posn_z=z2, symmetry_axes=sym, outer_bc_type=outer)
    return rg, g


def evolution_err(mine, ref, rel_floor_frac=1e-13):
    """relL2 per gf. A gridfunction whose reference norm is below rel_floor_frac of the
    largest one (a component that vanishes analytically, e.g. the phi components of
    axisymmetric Brill-Lindquist data) is measured against that floor instead."""
    m = mine.reshape(24, -1)
    r = ref.reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    den = np.maximum(den, rel_floor_frac * den.max())
    return num / den


@pytest.mark.parametrize("mode", [0, 1])
def test_small_config_100_steps(cuda, mode):
    """Spherical 72x12x2, symmetry_axes='2', BL m=0.5 at z=+/-0.5, 100 RK4 steps."""
    need("sphaxi")
    rg, g = pair("sphaxi", "Spherical", (72, 12, 2), 7.5, "2")
    y0 = rg.y_n()
    g.y_n.copy_(torch.from_numpy(y0).to(g.device))
    assert g.dt == pytest.approx(rg.dt, rel=1e-15)
    rg.step(100)
    g.MoL_step_forward_in_time(mode=mode, nsteps=100)
    torch.cuda.synchronize()
    err = evolution_err(g.y_n.cpu().numpy(), rg.y_n())
    assert err.max() <= 1e-10, err
    assert g.cd.nn == 100 and g.cd.time == pytest.approx(rg.time, rel=1e-15)
    rg.close()
    g.close()


def test_large_config_rhs_and_steps(cuda):
    """SinhSpherical 256x64x64 (AMPL=10, SINHW=0.2): one Ricci + RHS on a perturbed state
    (<= 1e-12), then 2 fused RK4 steps from that state (<= 1e-12)."""
    need("sinh3d")
    rg, g = pair("sinh3d", "SinhSpherical", (256, 64, 64), 10.0, "", bh=(0.41, 0.62, 0.58, -0.47))
    inp = oref.perturbed_state(rg, seed=5)
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
    # Two RK4 steps from the perturbed state (every gridfunction nonzero, so the relative
    # measure is meaningful for all 24; from pure Brill-Lindquist data several components
    # vanish analytically and hold only rounding noise in both codes).
    rg.set_y_n(inp)
    g.y_n.copy_(ti)
    rg.step(2)
    g.MoL_step_forward_in_time(mode=1, nsteps=2)
    torch.cuda.synchronize()
    err = evolution_err(g.y_n.cpu().numpy(), rg.y_n())
    assert err.max() <= 1e-12, err
    rg.close()
    g.close()


@pytest.mark.parametrize("outer", ["radiation", "extrapolation"])
def test_sph3d_20_steps(cuda, outer):
    """Spherical full 3-D 32x12x8 (batched/adjoint-workload family), 20 RK4 steps."""
    need("sph3d")
    rg, g = pair("sph3d", "Spherical", (32, 12, 8), 7.5, "", bh=(0.45, 0.5, 0.55, -0.6), outer=outer)
    inp = oref.perturbed_state(rg, seed=3, amp=0.02)
    rg.set_y_n(inp)
    g.y_n.copy_(torch.from_numpy(inp).to(g.device))
    rg.step(20)
    g.MoL_step_forward_in_time(mode=0 if outer == "extrapolation" else 1, nsteps=20)
    torch.cuda.synchronize()
    err = evolution_err(g.y_n.cpu().numpy(), rg.y_n())
    assert err.max() <= 1e-10, err
    rg.close()
    g.close()


def test_constraint_integrals_match_reference_volume_integration(cuda):
    """H, M^2, |Lambda| L2 norms (sum f^2 dV over the interior) on a 3-D grid."""
    need("sph3d")
    rg, g = pair("sph3d", "Spherical", (24, 10, 8), 7.5, "")
    inp = oref.perturbed_state(rg, seed=9, amp=0.03)
    cons = rg.constraints(inp, rg.ricci(inp))
    dV = rg.dV()
    norms = g.constraint_norms(torch.from_numpy(inp).to(g.device))
    G = 3
    for k, nm in enumerate(["H", "MSQUARED", "LAMBDA_CONSTRAINT"]):
        ref_int = float((cons[k].reshape(g.N[2], g.N[1], g.N[0])[G:-G, G:-G, G:-G] ** 2 * dV[G:-G, G:-G, G:-G]).sum())
        assert norms[f"{nm}_L2"] ** 2 == pytest.approx(ref_int, rel=1e-10)
    rg.close()
    g.close()
