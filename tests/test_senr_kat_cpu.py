"""The reference's inner-boundary known-answer test (SENR output on a 4x4x4 grid with 3 ghost
layers, tests/golden/senr_kat.npz) against the numpy restatement of bcstruct_set_up
(oracle/bssn_port.py): every point's source and the parity of each of the ten gridfunction
types. SinhCylindrical is checked against the Cylindrical file: both use the Cylindrical
eigen coordinates, and sinh is odd, so the index maps and parities are the same."""

import numpy as np
import pytest

from oracle import bssn_port as port
from tests.util import GOLDEN, senr_kat_values


@pytest.mark.parametrize("coord,kat", [("Spherical", "Spherical"), ("SinhCylindrical", "Cylindrical")])
def test_port_bcstruct_matches_senr_kat(coord, kat):
    with np.load(GOLDEN / "senr_kat.npz") as z:
        ijk, values = z[f"{kat}_ijk"], z[f"{kat}_values"]
    p = port.grid_params(coord, (4, 4, 4), 2.0)
    assert p["N"] == (10, 10, 10)
    inner, _ = port.bcstruct(p)
    assert len(inner) > 0
    np.testing.assert_array_equal(senr_kat_values(inner, ijk), values)
