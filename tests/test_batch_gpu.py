"""Batched evolutions (one launch per kernel per RK4 stage for the whole batch, replayed as
a CUDA graph) against the single-grid path and against the reference oracle."""

import numpy as np
import pytest
import torch

from tests.util import rel_l2_per_gf

pytestmark = pytest.mark.gpu

SPECS = [
    dict(coord="Spherical", Nxx=(24, 10, 6), grid_physical_size=7.5, BH1_mass=0.45, BH1_posn_z=0.35, BH2_mass=0.6,
         BH2_posn_z=-0.35),
    dict(coord="Spherical", Nxx=(37, 9, 4), grid_physical_size=7.5, BH1_mass=0.31, BH1_posn_z=0.7, BH2_mass=0.66,
         BH2_posn_z=-0.7),
    dict(coord="Spherical", Nxx=(50, 14, 2), grid_physical_size=7.5, BH1_mass=0.55, BH1_posn_z=0.4, BH2_mass=0.5,
         BH2_posn_z=-0.4),
]


@pytest.mark.parametrize("tile", [(32, 4), (64, 2), (0, 0)])
def test_batch_equals_single_grid_path(cuda, tile):
    from nrpy_b200.batch import BatchedEvolutions
    from nrpy_b200.grid import BSSNGrid

    be = BatchedEvolutions(SPECS)
    be.build(tile=tile, steps_per_graph=2)
    be.run(3)  # 6 RK4 steps
    torch.cuda.synchronize()
    for spec, g in zip(SPECS, be.grids):
        single = BSSNGrid(**spec)
        single.MoL_step_forward_in_time(mode=1, nsteps=6)
        torch.cuda.synchronize()
        a = single.y_n.view(24, -1).cpu().numpy()
        b = g.y_n.view(24, -1).cpu().numpy()
        err = rel_l2_per_gf(b, a, floor=1e-300)
        assert np.nanmax(np.where(np.linalg.norm(a, axis=1) > 0, err, 0)) <= 1e-14, err
        assert g.cd.nn == 6 and g.cd.time == pytest.approx(single.cd.time, rel=1e-15)
        single.close()
    be.close()


def test_batch_matches_reference_oracle(cuda):
    from oracle import ref as oref

    from nrpy_b200.batch import BatchedEvolutions

    if not oref.available("sph3d"):
        pytest.skip("oracle/_ref not built")
    be = BatchedEvolutions(SPECS[:2])
    refs = []
    for spec, g in zip(SPECS[:2], be.grids):
        rg = oref.RefGrid("sph3d", spec["Nxx"], spec["grid_physical_size"], BH1_mass=spec["BH1_mass"],
                          BH1_posn_z=spec["BH1_posn_z"], BH2_mass=spec["BH2_mass"], BH2_posn_z=spec["BH2_posn_z"])
        inp = oref.perturbed_state(rg, seed=21, amp=0.02)
        rg.set_y_n(inp)
        g.y_n.copy_(torch.from_numpy(inp).to(g.device))
        rg.step(10)
        refs.append(rg)
    be.build(tile=(32, 4), steps_per_graph=5)
    be.run(2)
    torch.cuda.synchronize()
    for rg, g in zip(refs, be.grids):
        err = rel_l2_per_gf(g.y_n.view(24, -1).cpu().numpy(), rg.y_n().reshape(24, -1))
        assert err.max() <= 1e-10, err
        rg.close()
    be.close()


def test_autotuner_picks_a_measured_configuration(cuda):
    from nrpy_b200.batch import BatchedEvolutions

    be = BatchedEvolutions(SPECS)
    y0 = [g.y_n.clone() for g in be.grids]
    res = be.autotune(steps=1, tiles=[(32, 4), (64, 2)])
    assert len(res["table"]) == 2 and res["ms_per_step"] == min(r["ms_per_step"] for r in res["table"])
    for g, y in zip(be.grids, y0):
        assert torch.equal(g.y_n, y)  # states restored
    be.close()


def test_batch_of_more_evolutions_than_one_launch_holds(cuda):
    """125 small evolutions: more than the 120 descriptors one launch of a group kernel carries,
    so every stage runs two launches per group kernel. Evolutions on both sides of the split
    must equal the single-grid path after 4 RK4 steps."""
    from nrpy_b200.batch import BatchedEvolutions
    from nrpy_b200.grid import BSSNGrid

    rng = np.random.default_rng(11)
    specs = [dict(coord="Spherical", Nxx=(int(rng.integers(8, 20)), int(rng.integers(4, 9)), 2 * int(rng.integers(1, 3))),
                  grid_physical_size=7.5, BH1_mass=float(rng.uniform(0.3, 0.7)), BH1_posn_z=0.4,
                  BH2_mass=float(rng.uniform(0.3, 0.7)), BH2_posn_z=-0.4) for _ in range(125)]
    be = BatchedEvolutions(specs)
    be.build(tile=(0, 0), steps_per_graph=2)
    be.run(2)
    torch.cuda.synchronize()
    for k in (0, 119, 120, 124):
        single = BSSNGrid(**specs[k])
        single.MoL_step_forward_in_time(mode=1, nsteps=4)
        torch.cuda.synchronize()
        a = single.y_n.view(24, -1).cpu().numpy()
        b = be.grids[k].y_n.view(24, -1).cpu().numpy()
        err = rel_l2_per_gf(b, a, floor=1e-300)
        assert np.nanmax(np.where(np.linalg.norm(a, axis=1) > 0, err, 0)) <= 1e-14, (k, err)
        single.close()
    be.close()
