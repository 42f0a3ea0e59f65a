"""SinhCylindrical (axisymmetric about z) at 4th order against the reference's generated C:
the cases of tests/sinhcyl_cases.py, collected here with the 4th-order library (the 8th-order
library runs them from tests/fd8_cases.py)."""

import pytest

from tests.sinhcyl_cases import (  # noqa: F401  (collected by pytest)
    test_sinhcyl_20_steps,
    test_sinhcyl_brill_lindquist_50_steps,
    test_sinhcyl_diagnostics_files,
    test_sinhcyl_dt_matches_reference,
    test_sinhcyl_grid_bcstruct_and_initial_data,
    test_sinhcyl_ricci_rhs_constraints,
)

pytestmark = pytest.mark.gpu
