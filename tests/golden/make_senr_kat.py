"""Write tests/golden/senr_kat.npz from the reference's inner-boundary known-answer files.

The reference ships two outputs of the SENR code (nrpy/infrastructures/BHaH/
CurviBoundaryConditions/SENRout4x4x4-{Spherical,Cylindrical}_NGHOSTS4oFD.txt, made with the
patch SENR.patch-83cf8f5f... beside them): on a 4x4x4 grid with 3 ghost layers (10x10x10
points), ten gridfunctions (vet^1..3, a_11, a_12, a_13, a_22, a_23, a_33, cf) were filled with
IDX4(gf, i, j, k) = i + 10 j + 100 k + 1000 gf, the inner boundary conditions were applied,
and every point's ten values were printed as integers "i j k | v_0 ... v_9". A ghost point
then holds +-(1000 gf + its source point's index), so each line gives the source point and
the parity of each gridfunction type.

Stored per coordinate system: ijk (1000, 3) and values (1000, 10), the lines as printed.
Run: python tests/golden/make_senr_kat.py   (reads $NRPY_REFERENCE, else ../reference)
"""

import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REF = pathlib.Path(os.environ.get("NRPY_REFERENCE", HERE.parents[1].parent / "reference"))
DIR = REF / "nrpy" / "infrastructures" / "BHaH" / "CurviBoundaryConditions"

out = {}
for coord in ("Spherical", "Cylindrical"):
    ijk, vals = [], []
    for line in (DIR / f"SENRout4x4x4-{coord}_NGHOSTS4oFD.txt").read_text().splitlines():
        left, right = line.split("|")
        ijk.append([int(x) for x in left.split()])
        vals.append([int(x) for x in right.split()])
    out[f"{coord}_ijk"] = np.array(ijk, dtype=np.int16)
    out[f"{coord}_values"] = np.array(vals, dtype=np.int32)
np.savez_compressed(HERE / "senr_kat.npz", **out)
print("wrote", HERE / "senr_kat.npz", {k: v.shape for k, v in out.items()})
