"""Generate the pointwise BSSN device functions (nrpy_b200/csrc/gen/*.cuh).

Code-generation time only: needs the nrpy package (the reference's equation modules) on
PYTHONPATH. The emitted headers are committed, so building the CUDA library does not
need nrpy. Each (CoordSystem, symmetry) variant is generated in its own process because
nrpy caches equation objects per CoordSystem and reads ``symmetry_axes`` globally.

Usage: python -m nrpy_b200.codegen.generate [--reference PATH] [--variants ...]
"""

import argparse
import os
import pathlib
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parents[2]
OUTDIR = ROOT / "nrpy_b200" / "csrc" / "gen"
VARIANTS = {
    # tag: (CoordSystem, symmetry_axes)
    "sph_axi": ("Spherical", "2"),
    "sph_3d": ("Spherical", ""),
    "sinh_axi": ("SinhSpherical", "2"),
    "sinh_3d": ("SinhSpherical", ""),
}


def generate_variant(tag: str) -> None:
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen.emit_cuda import emit_point_function

    coord, sym = VARIANTS[tag]
    be.setup_nrpy(sym)
    t0 = time.time()
    rhs, betaU = be.rhs_exprs(coord)
    ricci = be.ricci_exprs(coord)
    cons = be.constraint_exprs(coord)
    enf = be.enforce_exprs(coord)
    parts = []
    stats = {}
    code, st = emit_point_function(
        f"ricci_point_{tag}",
        [(f"out[{i}]", ricci[k]) for i, k in enumerate(be.RBAR_ORDER)],
        symmetry_axes=sym,
        comment=f"Rbar_ij, {coord} (symmetry_axes='{sym}'): Ricci_eval.py:27-167",
    )
    parts.append(code)
    stats["ricci"] = st
    code, st = emit_point_function(
        f"rhs_point_{tag}",
        [(f"out[{i}]", rhs[g]) for i, g in enumerate(be.GF_ORDER)],
        upwind_vec=betaU,
        symmetry_axes=sym,
        comment=f"BSSN RHS + KO (CAKO), {coord} (symmetry_axes='{sym}'): rhs_eval.py:122-220",
    )
    parts.append(code)
    stats["rhs"] = st
    code, st = emit_point_function(
        f"constraints_point_{tag}",
        [(f"out[{i}]", cons[k]) for i, k in enumerate(["H", "MSQUARED", "LAMBDA_CONSTRAINT"])],
        symmetry_axes=sym,
        comment=f"H, M^2, |Lambda constraint|, {coord}: constraints_eval.py:364-492",
    )
    parts.append(code)
    stats["constraints"] = st
    code, st = emit_point_function(
        f"enforce_point_{tag}",
        [(f"out[{i}]", enf[k]) for i, k in enumerate(["hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22"])],
        symmetry_axes=sym,
        comment=f"det(gammabar)=det(gammahat) projection of hDD, {coord}: "
        "enforce_detgammabar_equals_detgammahat.py:85-110",
    )
    parts.append(code)
    stats["enforce"] = st
    lam = be.lambda_id_exprs(coord)
    code, st = emit_point_function(
        f"lambda_point_{tag}",
        [(f"out[{i}]", lam[f"lambdaU{i}"]) for i in range(3)],
        symmetry_axes=sym,
        comment=f"initial-data lambda^i from centred FD of hDD, {coord}: "
        "ADM_Initial_Data_Reader__BSSN_Converter.py:462-580",
    )
    parts.append(code)
    stats["lambda"] = st
    hdr = (
        "// Generated by nrpy_b200/codegen/generate.py from NRPy's BSSN equation modules.\n"
        f"// Variant {tag}: CoordSystem={coord}, symmetry_axes='{sym}', 4th-order FD, KO (CAKO).\n"
        f"// Stencil loads / derivative evaluations per point: {stats}\n"
        "#pragma once\n\n"
    )
    OUTDIR.mkdir(parents=True, exist_ok=True)
    (OUTDIR / f"bssn_{tag}.cuh").write_text(hdr + "\n".join(parts))
    print(f"{tag}: {stats} ({time.time() - t0:.1f}s)")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--variants", default=",".join(VARIANTS))
    ap.add_argument("--one", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.one:
        generate_variant(args.one)
        return
    shim = ROOT / "oracle" / "_ref" / "shim"
    env = dict(os.environ)
    env["PYTHONPATH"] = f"{ROOT}:{shim}:{args.reference}"
    procs = [
        subprocess.Popen([sys.executable, "-m", "nrpy_b200.codegen.generate", "--one", tag], env=env, cwd=ROOT)
        for tag in args.variants.split(",")
    ]
    rc = [p.wait() for p in procs]
    if any(rc):
        raise SystemExit(f"generation failed: {rc}")


if __name__ == "__main__":
    main()
