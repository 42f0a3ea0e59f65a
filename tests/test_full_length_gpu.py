"""Full-length parity of the stated workloads against the reference's own generated C.

* SinhSpherical 256x64x64 (AMPL 10, SINHW 0.2, seeded Brill-Lindquist masses ~U[0.3,0.7]
  at z = +/-U[0.3,0.8], seed 2024 as in bench.py): 200 FP64 RK4 steps against the oracle
  (variant sinh3d). The Hamiltonian-constraint L2 (sum over the interior of H^2 dV, the
  reference's diagnostics_volume_integration measure) every 20 steps within 1e-10 relative
  of the oracle's; the per-gridfunction relative L2 measured against the spread between the
  reference's own C and CUDA builds on the same run (see the test).
* The same 200 steps with the Ricci/RHS algebra in FP32 (state, RK accumulation,
  detgammabar projection and reductions in FP64), against the same oracle run: H-constraint
  L2 within 1e-8 relative at every 20 steps, and per-gridfunction relative L2 <= 2e-3.
* The batched workload: all 64 evolutions (Spherical, Nxx from [48..128]x[8..32]x[2..16],
  seed 7) advanced 100 RK4 steps as one batch, each against its own sequential run of the
  oracle (variant sph3d, its AVX2 build) from the same initial state: per-gridfunction
  relative L2 <= 1e-10.

Gridfunctions that vanish analytically (the phi components, for holes on the z axis) are
measured against the largest gridfunction's norm (evolution_err). The oracle runs on the
host cores; these tests take about a minute each on a 16-core host.
"""

import numpy as np
import pytest
import torch

from oracle import ref as oref

pytestmark = pytest.mark.gpu

G = 3


def need(variant):
    if not oref.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")


def bl_params(seed):
    rng = np.random.default_rng(seed)
    m1, m2 = rng.uniform(0.3, 0.7, 2)
    z1, z2 = rng.uniform(0.3, 0.8), -rng.uniform(0.3, 0.8)
    return float(m1), float(z1), float(m2), float(z2)


VANISHING = 1e-8  # a gridfunction whose oracle norm is below this fraction of the largest one


def evolution_err(mine, ref, vanishing=VANISHING):
    """Per-gridfunction relative L2 ||mine - ref|| / ||ref||. Brill-Lindquist data with both
    holes on the z axis has analytically vanishing phi components (h_02, h_12, a_02, a_12,
    lambda^2, vet^2, bet^2): on a full 3-D grid they hold only rounding noise, which the two
    codes grow differently. A gridfunction whose oracle norm is below `vanishing` of the
    largest is therefore measured against the largest norm: its difference must be as small,
    relative to the solution, as that of every other gridfunction."""
    m = mine.reshape(24, -1)
    r = ref.reshape(24, -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    return num / np.where(den < vanishing * den.max(), den.max(), den)


def ref_h_l2_squared(rg, y, dV):
    """sum over the interior of H^2 dV from the reference's own Ricci_eval + constraints_eval."""
    cons = rg.constraints(y, rg.ricci(y))
    H = cons[0].reshape(rg.N[2], rg.N[1], rg.N[0])[G:-G, G:-G, G:-G]
    return float((H**2 * dV).sum())


def interior_dV(rg):
    """The reference's volume element sqrt(det gammahat) dxx0 dxx1 dxx2 on the interior,
    from its own rfm arrays (|f0' f0^2 f1| dxx0 dxx1 dxx2), spot-checked against its dV()."""
    N0, N1, N2 = rg.N
    f0 = rg.rfm_field(0, N0)
    f0_D0 = rg.rfm_field(1, N0)
    f1 = rg.rfm_field(4, N1)
    x0, x1, x2 = rg.xx()
    dvol = abs((x0[1] - x0[0]) * (x1[1] - x1[0]) * (x2[1] - x2[0]))
    dV = np.abs(f0_D0[None, None, :] * f0[None, None, :] ** 2 * f1[None, :, None]) * dvol
    dV = np.broadcast_to(dV, (N2, N1, N0))[G:-G, G:-G, G:-G]
    rng = np.random.default_rng(0)
    for _ in range(8):
        i0, i1, i2 = (int(rng.integers(G, n - G)) for n in (N0, N1, N2))
        assert dV[i2 - G, i1 - G, i0 - G] == pytest.approx(rg.lib.ref_dV(rg.h, i0, i1, i2), rel=1e-12)
    return np.ascontiguousarray(dV)


def test_sinh256_200_steps_fp64_and_mixed_against_reference(cuda):
    need("sinh3d")
    if not oref.cuda_available("sinh3d_cuda"):
        pytest.skip("oracle/_ref/sinh3d_cuda not built")
    from nrpy_b200.grid import BSSNGrid

    m1, z1, m2, z2 = bl_params(2024)
    Nxx = (256, 64, 64)
    rg = oref.RefGrid("sinh3d", Nxx, 10.0, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    rc = oref.RefCudaGrid(Nxx, 10.0, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    kw = dict(coord="SinhSpherical", Nxx=Nxx, grid_physical_size=10.0, SINHW=0.2, BH1_mass=m1, BH1_posn_z=z1,
              BH2_mass=m2, BH2_posn_z=z2)
    g64 = BSSNGrid(**kw)
    g32 = BSSNGrid(**kw, initial_data=False)
    y0 = rg.y_n()
    rc.set_y_n(y0)
    g64.y_n.copy_(torch.from_numpy(y0).to(cuda))
    g32.y_n.copy_(g64.y_n)
    assert g64.dt == pytest.approx(rg.dt, rel=1e-15)
    dV = interior_dV(rg)
    h64, h32, href, ratio = [], [], [], {}
    for blk in range(10):
        rg.step(20)
        rc.steps(20)
        g64.MoL_step_forward_in_time(mode=1, nsteps=20)
        g32.MoL_step_forward_in_time(mode=1, mixed=True, nsteps=20)
        h64.append(g64.constraint_norms()["H_L2"] ** 2)
        h32.append(g32.constraint_norms()["H_L2"] ** 2)
        yref = rg.y_n()
        href.append(ref_h_l2_squared(rg, yref, dV))
        spread = evolution_err(rc.y_n(), yref).max()  # the reference's own CUDA build vs its C build
        mine = evolution_err(g64.y_n.cpu().numpy(), yref).max()
        ratio[20 * (blk + 1)] = (mine, spread)
        print(f"step {20 * (blk + 1)}: FP64 vs reference C {mine:.2e}; reference CUDA vs reference C {spread:.2e}")
    torch.cuda.synchronize()
    err64 = evolution_err(g64.y_n.cpu().numpy(), yref)
    err32 = evolution_err(g32.y_n.cpu().numpy(), yref)
    h64, h32, href = np.sqrt(h64), np.sqrt(h32), np.sqrt(href)
    print(f"FP64: max per-gf relL2 {err64.max():.3e}; H-L2 max rel diff {np.max(np.abs(h64 / href - 1)):.3e}")
    print(f"mixed: max per-gf relL2 {err32.max():.3e}; H-L2 max rel diff {np.max(np.abs(h32 / href - 1)):.3e}")
    print("FP64 per-gf:", np.array2string(err64, precision=2))
    print("mixed per-gf:", np.array2string(err32, precision=2))
    print("H-L2 (oracle) every 20 steps:", href.tolist())
    assert g64.cd.nn == 200 and g64.cd.time == pytest.approx(rg.time, rel=1e-15)
    # The Hamiltonian constraint, every 20 steps, to 1e-10 of the reference's.
    np.testing.assert_allclose(h64, href, rtol=1e-10, atol=0)
    # Per-gridfunction state. On this workload rounding differences grow: the reference's own
    # two builds (C and CUDA, the same generated algebra) drift apart to 2-4e-8 within 60 steps,
    # so the 1e-10 bar of the small workload is out of reach of any second build here. The bar is
    # that spread: within 10x of it after 100 steps, and within 100x after 200 (a change of
    # upwind side at a point where a shift component crosses zero is a discrete jump of
    # truncation size, and two codes with different rounding take it at different steps).
    mine100, spread100 = ratio[100]
    assert mine100 <= max(1e-10, 10 * spread100), (mine100, spread100)
    mine200, spread200 = ratio[200]
    assert mine200 <= max(1e-10, 100 * spread200), (mine200, spread200)
    # Mixed precision (FP32 algebra): H-L2 within 1e-8 of the reference's, state within 2e-3.
    np.testing.assert_allclose(h32, href, rtol=1e-8, atol=0)
    assert err32.max() <= 2e-3, err32
    rc.close()
    rg.close()
    g64.close()
    g32.close()


def test_batch_64_evolutions_100_steps_against_reference(cuda):
    need("sph3d")
    from nrpy_b200.batch import BatchedEvolutions, batching_workload

    specs = batching_workload(seed=7, n=64)
    be = BatchedEvolutions(specs)
    y0 = [g.y_n.cpu().numpy() for g in be.grids]
    be.build(tile=(0, 0), steps_per_graph=20)  # a tile shape per grid
    be.run(5)  # 100 RK4 steps
    torch.cuda.synchronize()
    worst, compared, nonfinite = 0.0, 0, []
    for k, (spec, g) in enumerate(zip(specs, be.grids)):
        # The AVX2 build of the oracle: with AVX-512 the reference's vector loops run past the
        # end of a row into the next row's first interior point when Nxx0 = 1 (mod 8) (10 of
        # these 64 grids), a write that races with the thread computing that row.
        rg = oref.RefGrid("sph3d", spec["Nxx"], spec["grid_physical_size"], BH1_mass=spec["BH1_mass"],
                          BH1_posn_z=spec["BH1_posn_z"], BH2_mass=spec["BH2_mass"], BH2_posn_z=spec["BH2_posn_z"],
                          isa="avx2")
        assert g.dt == pytest.approx(rg.dt, rel=1e-15), k
        ym = g.y_n.cpu().numpy()
        rg.set_y_n(y0[k])
        rg.step(100)
        yr = rg.y_n()
        assert g.cd.nn == 100 and g.cd.time == pytest.approx(rg.time, rel=1e-15)
        rg.close()
        if not np.isfinite(yr).all():
            nonfinite.append((k, spec["Nxx"], bool(np.isfinite(ym).all())))
            continue
        err = evolution_err(ym, yr)
        worst = max(worst, float(err.max()))
        compared += 1
        assert err.max() <= 1e-10, (k, spec["Nxx"], err)
    print(f"{compared} of 64 evolutions x 100 steps: worst per-gf relL2 vs reference {worst:.3e}; "
          f"reference not finite (index, Nxx, ours finite): {nonfinite}")
    assert compared == 64
    be.close()
