"""Device diagnostics against the generated project's own diagnostics() (B200 + oracle).

Both write the nearest-point files (out0d at the point next to the origin, out1d along the
lines nearest the y and z axes, out2d on the planes nearest xy and yz) and the volume
integrals (out3d-integrals, recipes whole_domain and sphere_R_gt_8) for the same state at two
output steps. The file names and every comment line must be identical; numbers agree to
1e-12 relative for coordinates, 1e-9 of each column's largest magnitude for the sampled
H and M^2, and 1e-10 relative for the integrals.
"""

import pytest

from tests.util import compare_diagnostics_dirs

pytestmark = pytest.mark.gpu

CASES = [("sph3d", "Spherical", (24, 8, 8), 7.5), ("sinh3d", "SinhSpherical", (24, 8, 8), 10.0)]


@pytest.mark.parametrize("variant,coord,nxx,gps", CASES)
def test_diagnostics_files_match_reference(cuda, tmp_path, monkeypatch, variant, coord, nxx, gps):
    import torch

    from nrpy_b200.grid import BSSNGrid
    from oracle import ref

    if not ref.available(variant):
        pytest.skip("oracle/_ref not built")
    bh = dict(BH1_mass=0.45, BH1_posn_z=0.4, BH2_mass=0.55, BH2_posn_z=-0.35)
    rg = ref.RefGrid(variant, nxx, gps, SINHW=0.2, **bh)
    state = ref.perturbed_state(rg, seed=4)
    rg.set_y_n(state)
    g = BSSNGrid(coord, nxx, grid_physical_size=gps, SINHW=0.2, **bh)
    g.y_n.copy_(torch.from_numpy(state))
    every = 0.25
    for k, (nn, t) in enumerate([(0, 0.0), (7, 0.25)]):
        (tmp_path / "ref").mkdir(exist_ok=True)
        (tmp_path / "ours").mkdir(exist_ok=True)
        monkeypatch.chdir(tmp_path / "ref")
        rg.diagnostics(nn, t, every)
        monkeypatch.chdir(tmp_path / "ours")
        g.diagnostics(every, nn=nn, time=t)
        torch.cuda.synchronize()
    rg.close()
    monkeypatch.chdir(tmp_path)
    names = compare_diagnostics_dirs(tmp_path / "ref", tmp_path / "ours")
    assert any(n.startswith("out0d") for n in names) and any(n.startswith("out3d") for n in names)
