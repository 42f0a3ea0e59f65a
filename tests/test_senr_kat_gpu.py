"""The library's bcstruct (built by libbssn_b200's bcstruct_set_up) against the reference's
inner-boundary known-answer files (SENR output, 4x4x4 grid, 3 ghost layers; see
tests/golden/make_senr_kat.py): the source point and the ten parity signs of every point.
SinhCylindrical is checked against the Cylindrical file (same eigen coordinates; sinh is odd)."""

import numpy as np
import pytest

from tests.util import GOLDEN, senr_kat_values

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("coord,kat,sym", [("Spherical", "Spherical", ""), ("SinhSpherical", "Spherical", ""),
                                           ("SinhCylindrical", "Cylindrical", "1")])
def test_library_bcstruct_matches_senr_kat(cuda, coord, kat, sym):
    from nrpy_b200 import lib
    from nrpy_b200.grid import BSSNGrid

    if lib.NGHOSTS != 3:
        pytest.skip("the known-answer files have 3 ghost layers (4th-order build)")
    with np.load(GOLDEN / "senr_kat.npz") as z:
        ijk, values = z[f"{kat}_ijk"], z[f"{kat}_values"]
    g = BSSNGrid(coord=coord, Nxx=(4, 4, 4), grid_physical_size=2.0, SINHW=0.2, BH1_mass=0.5, BH1_posn_z=0.3,
                 BH2_mass=0.5, BH2_posn_z=-0.3, symmetry_axes=sym)
    assert g.N == (10, 10, 10)
    inner, _, _ = g.bcstruct()
    got = senr_kat_values([(q.dstpt, q.srcpt, list(q.parity)) for q in inner], ijk)
    np.testing.assert_array_equal(got, values)
    g.close()
