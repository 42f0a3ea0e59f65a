"""Mixed precision: Ricci/RHS algebra in FP32 with FP64 stencils, state, RK accumulation,
detgammabar projection and constraint reductions. The stated tolerances: after 20 RK4
steps of a perturbed SinhSpherical state, per-gridfunction relative L2 vs the FP64 path
<= 1e-5 and the Hamiltonian-constraint L2 within 1e-3 relative of the FP64 run's."""

import numpy as np
import pytest
import torch

from tests.util import load_golden

pytestmark = pytest.mark.gpu


def test_mixed_precision_error_vs_fp64(cuda):
    from nrpy_b200.grid import BSSNGrid

    g = load_golden("sinh3d_10x6x6")
    m1, z1, m2, z2 = [float(x) for x in g["bh"]]
    kw = dict(coord="SinhSpherical", Nxx=(24, 12, 12), grid_physical_size=10.0, SINHW=0.2, BH1_mass=m1,
              BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    a, b = BSSNGrid(**kw), BSSNGrid(**kw)
    # a smooth perturbation of every gridfunction (same on both grids)
    rng = np.random.default_rng(3)
    pert = torch.from_numpy(0.01 * rng.standard_normal(a.y_n.numel())).to(a.device)
    for grid in (a, b):
        y = grid.view(grid.y_n)
        p = grid.view(pert.clone())
        p = torch.nn.functional.avg_pool3d(p.unsqueeze(0), 5, stride=1, padding=2).squeeze(0)
        y += p
        grid.apply_bcs_outerextrap_and_inner(grid.y_n)
    torch.cuda.synchronize()
    a.MoL_step_forward_in_time(mode=1, mixed=False, nsteps=20)
    b.MoL_step_forward_in_time(mode=1, mixed=True, nsteps=20)
    torch.cuda.synchronize()
    fa = a.y_n.view(24, -1)
    fb = b.y_n.view(24, -1)
    rel = (torch.linalg.vector_norm(fb - fa, dim=1) / torch.linalg.vector_norm(fa, dim=1)).cpu().numpy()
    assert rel.max() <= 1e-5, rel
    assert rel.max() > 0.0  # the FP32 path is really taken
    ha = a.constraint_norms()["H_L2"]
    hb = b.constraint_norms()["H_L2"]
    assert abs(hb - ha) / ha <= 1e-3, (ha, hb)
    a.close()
    b.close()
