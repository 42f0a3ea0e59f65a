"""BSSNGrid.step_from_host (uploads and downloads overlapped with the steps, two device
state buffers; steps replayed from captured graphs or launched one by one) gives, for every
host state, exactly what the in-line path gives: copy in, one RK4 step, copy out."""

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_step_from_host_matches_in_line(cuda):
    from nrpy_b200.grid import BSSNGrid

    g = BSSNGrid("SinhSpherical", (32, 8, 8), grid_physical_size=10.0, BH1_mass=0.45, BH1_posn_z=0.4,
                 BH2_mass=0.55, BH2_posn_z=-0.35)
    gen = torch.Generator().manual_seed(3)
    y0 = g.y_n.cpu()
    states = [(y0 * (1.0 + 1e-3 * torch.rand(y0.shape, generator=gen, dtype=torch.float64))).pin_memory()
              for _ in range(5)]
    outs = [torch.empty_like(s).pin_memory() for s in states]
    for mode, graph in ((0, True), (1, True), (1, False), (0, False), (1, True)):
        for o in outs:
            o.fill_(0.0)
        nn = g.cd.nn
        g.step_from_host(states, outs, mode=mode, graph=graph)
        torch.cuda.synchronize()
        assert g.cd.nn == nn + len(states)
        for s, o in zip(states, outs):
            g.y_n.copy_(s)
            g.MoL_step_forward_in_time(mode=mode)
            torch.cuda.synchronize()
            assert torch.equal(g.y_n.cpu(), o)
    g.close()
