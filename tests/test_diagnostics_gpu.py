"""Device diagnostics against the generated project's own diagnostics() (B200 + oracle).

Both write the nearest-point files (out0d at the point next to the origin, out1d along the
lines nearest the y and z axes, out2d on the planes nearest xy and yz) and the volume
integrals (out3d-integrals, recipes whole_domain and sphere_R_gt_8) for the same state at two
output steps. The file names and every comment line must be identical; numbers agree to
1e-12 relative for coordinates, 1e-9 of each column's largest magnitude for the sampled
H and M^2, and 1e-10 relative for the integrals.
"""

import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("sph3d", "Spherical", (24, 8, 8), 7.5), ("sinh3d", "SinhSpherical", (24, 8, 8), 10.0)]


def read(path: pathlib.Path):
    comments, rows = [], []
    for line in path.read_text().splitlines():
        (comments if line.startswith("#") else rows).append(line)
    return comments, np.array([[float(x) for x in r.split()] for r in rows])


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
    names_ref = sorted(p.name for p in (tmp_path / "ref").iterdir())
    names_ours = sorted(p.name for p in (tmp_path / "ours").iterdir())
    assert names_ours == names_ref
    assert any(n.startswith("out0d") for n in names_ref) and any(n.startswith("out3d") for n in names_ref)
    for name in names_ref:
        c_ref, d_ref = read(tmp_path / "ref" / name)
        c_ours, d_ours = read(tmp_path / "ours" / name)
        assert c_ours == c_ref, name
        assert d_ours.shape == d_ref.shape, name
        if name.startswith("out3d"):
            np.testing.assert_allclose(d_ours, d_ref, rtol=1e-10, atol=0, err_msg=name)
            continue
        ncoord = 1 if name.startswith(("out0d", "out1d")) else 2
        np.testing.assert_allclose(d_ours[:, :ncoord], d_ref[:, :ncoord], rtol=1e-12, atol=1e-12, err_msg=name)
        vals_ref, vals_ours = d_ref[:, ncoord:], d_ours[:, ncoord:]
        scale = np.abs(vals_ref).max(axis=0)
        assert np.all(np.abs(vals_ours - vals_ref) <= 1e-9 * scale + 1e-300), name
