"""Axisymmetric SinhSpherical (symmetry_axes "2") against the reference's generated C of the
same coordinates: oracle variant sinhaxi (4th order) or sinhaxi8 (8th order), chosen by the
finite-difference order of the loaded library. Collected by tests/test_parity_oracle_gpu.py
(4th order) and tests/fd8_cases.py (8th order). Bars: Ricci and the RHS to 1e-12 per
gridfunction relative L2 on a perturbed state; 20 RK4 steps to 1e-10 in both stage orders.
"""

import numpy as np
import pytest
import torch

from oracle import ref as oref
from tests.util import rel_l2_per_gf

pytestmark = pytest.mark.gpu

NXX = (64, 16, 2)
L = 10.0


def _pair():
    from nrpy_b200 import lib
    from nrpy_b200.grid import BSSNGrid

    variant = "sinhaxi" if lib.FD_ORDER == 4 else f"sinhaxi{lib.FD_ORDER}"
    if not oref.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")
    bh = dict(BH1_mass=0.45, BH1_posn_z=0.5, BH2_mass=0.55, BH2_posn_z=-0.6)
    rg = oref.RefGrid(variant, NXX, L, SINHW=0.2, **bh)
    g = BSSNGrid(coord="SinhSpherical", Nxx=NXX, grid_physical_size=L, SINHW=0.2, symmetry_axes="2", **bh)
    assert g.N == rg.N
    return rg, g, lib.NGHOSTS


def test_sinhaxi_ricci_rhs(cuda):
    rg, g, ng = _pair()
    inp = oref.perturbed_state(rg, seed=6, amp=0.03)
    ricci = rg.ricci(inp)
    rhs = rg.rhs(ricci, inp)
    ti = torch.from_numpy(inp).to(g.device)
    aux = torch.zeros(6 * g.ntot, dtype=torch.float64, device=g.device)
    g.ricci_eval(ti, aux)
    out = torch.zeros(24 * g.ntot, dtype=torch.float64, device=g.device)
    g.rhs_eval(aux, ti, out)
    torch.cuda.synchronize()
    N = g.N
    sl = (slice(None), slice(ng, -ng), slice(ng, -ng), slice(ng, -ng))
    as4 = lambda a: np.asarray(a).reshape(-1, N[2], N[1], N[0])[sl]  # noqa: E731
    e_r = rel_l2_per_gf(as4(aux.cpu().numpy()), as4(ricci))
    e_rhs = rel_l2_per_gf(as4(out.cpu().numpy()), as4(rhs))
    assert e_r.max() <= 1e-12, e_r
    assert e_rhs.max() <= 1e-12, e_rhs
    rg.close()
    g.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_sinhaxi_20_steps(cuda, mode):
    rg, g, ng = _pair()
    inp = oref.perturbed_state(rg, seed=2, amp=0.02)
    rg.set_y_n(inp)
    g.y_n.copy_(torch.from_numpy(inp).to(g.device))
    rg.step(20)
    g.MoL_step_forward_in_time(mode=mode, nsteps=20)
    torch.cuda.synchronize()
    m = g.y_n.cpu().numpy().reshape(24, -1)
    r = rg.y_n().reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    err = num / np.maximum(den, 1e-13 * den.max())
    assert err.max() <= 1e-10, err
    rg.close()
    g.close()
