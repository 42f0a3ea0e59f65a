"""Write tests/golden/fd_coeffs.json: the reference's finite-difference coefficient tables.

Runs nrpy.finite_difference.compute_fdcoeffs_fdstencl (nrpy/finite_difference.py:202-330)
for the 4th-order operators on the hot path. Needs the reference importable, e.g.
  PYTHONPATH=oracle/_ref/shim:$NRPY_REFERENCE python tests/golden/make_fd_coeffs.py
($NRPY_REFERENCE: the nrpy checkout)
(oracle/gen_ref.py writes the import shims under oracle/_ref/shim).
"""

import json
import pathlib

import nrpy.finite_difference as fin  # noqa: E402  (the reference)

OUT = pathlib.Path(__file__).resolve().parent / "fd_coeffs.json"
tab = {}
for d in range(3):
    for op in (f"dD{d}", f"dupD{d}", f"ddnD{d}", f"dKOD{d}", f"dDD{d}{d}"):
        coeffs, stencil = fin.compute_fdcoeffs_fdstencl(op, 4)
        tab[op] = {"coeffs": [float(c) for c in coeffs], "stencil": [list(s) for s in stencil]}
OUT.write_text(json.dumps(tab, indent=1))
print("wrote", OUT)
