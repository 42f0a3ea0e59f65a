"""The reference's own CUDA build (nrpy --cuda, compiled for sm_100a by oracle/gen_ref.py,
variant sinh3d_cuda) on the B200, as a second oracle and as the GPU baseline that bench.py
times: its MoL_step_forward_in_time agrees with the reference's OpenMP C and with this
library on the same SinhSpherical state (per-gridfunction relative L2 <= 1e-12 after one
RK4 step, <= 1e-10 after 20)."""

import numpy as np
import pytest
import torch

from oracle import ref as oref

pytestmark = pytest.mark.gpu


def evolution_err(mine, ref):
    m = mine.reshape(24, -1)
    r = ref.reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    return num / np.maximum(den, 1e-300)


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-12), (20, 1e-10)])
def test_reference_cuda_step_matches_reference_c_and_library(cuda, nsteps, tol):
    if not (oref.cuda_available("sinh3d_cuda") and oref.available("sinh3d")):
        pytest.skip("oracle/_ref/sinh3d_cuda or sinh3d not built")
    from nrpy_b200.grid import BSSNGrid

    Nxx, L, bh = (48, 16, 16), 10.0, (0.45, 0.55, 0.6, -0.5)
    rg = oref.RefGrid("sinh3d", Nxx, L, SINHW=0.2, BH1_mass=bh[0], BH1_posn_z=bh[1], BH2_mass=bh[2], BH2_posn_z=bh[3])
    rc = oref.RefCudaGrid(Nxx, L, SINHW=0.2, BH1_mass=bh[0], BH1_posn_z=bh[1], BH2_mass=bh[2], BH2_posn_z=bh[3])
    g = BSSNGrid(coord="SinhSpherical", Nxx=Nxx, grid_physical_size=L, SINHW=0.2, BH1_mass=bh[0], BH1_posn_z=bh[1],
                 BH2_mass=bh[2], BH2_posn_z=bh[3])
    assert rc.N == rg.N and rc.dt == pytest.approx(rg.dt, rel=1e-15)
    # The two reference builds' own initial data are not compared: the CUDA build's lambda^i
    # differs from the C build's (printed below); both runs start from one shared state.
    id_err = evolution_err(rc.y_n(), rg.y_n())
    print(f"initial data, reference CUDA vs reference C: per-gf relL2 {np.array2string(id_err, precision=2)}")
    inp = oref.perturbed_state(rg, seed=4, amp=0.02)
    rg.set_y_n(inp)
    rc.set_y_n(inp)
    g.y_n.copy_(torch.from_numpy(inp).to(g.device))
    rg.step(nsteps)
    rc.steps(nsteps)
    g.MoL_step_forward_in_time(mode=1, nsteps=nsteps)
    torch.cuda.synchronize()
    y_c, y_cuda, y_lib = rg.y_n(), rc.y_n(), g.y_n.cpu().numpy()
    e_cuda = evolution_err(y_cuda, y_c)
    e_lib = evolution_err(y_lib, y_cuda)
    assert e_cuda.max() <= tol, e_cuda
    assert e_lib.max() <= tol, e_lib
    rc.close()
    rg.close()
    g.close()
