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


# Output groups: each group is one kernel (its own CSE); groups trade recomputed shared
# subexpressions for fewer live values per thread. Values beyond REG_CAPACITY live doubles
# go to per-thread shared-memory slots.
RICCI_GROUPS = [["RbarDD00", "RbarDD01"], ["RbarDD02", "RbarDD11"], ["RbarDD12", "RbarDD22"]]
RHS_GROUPS = [
    ["aDD00", "aDD01", "aDD02", "aDD11", "aDD12", "aDD22"],
    ["alpha", "cf", "hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22", "trK", "vetU0", "vetU1", "vetU2"],
    ["betU0", "betU1", "betU2", "lambdaU0", "lambdaU1", "lambdaU2"],
]
REG_CAPACITY = 90


def _group_struct(kind: str, tag: str, g: int, fname: str, gfs, slots: int) -> str:
    cases = " ".join(f"case {k}: return {x};" for k, x in enumerate(gfs))
    return (
        f"template <> struct {kind}_{tag}<{g}> {{\n"
        f"  static constexpr int N = {len(gfs)};\n"
        f"  static constexpr int SLOTS = {slots};\n"
        f"  __host__ __device__ static constexpr int GF(int k) {{\n"
        f"    switch (k) {{ {cases} }}\n    return -1;\n  }}\n"
        f"  template <typename T, typename TF, typename Ctx>\n"
        f"  __device__ __forceinline__ static void eval(const Ctx &ctx, T *out, volatile T *sm) {{\n"
        f"    {fname}<T, TF>(ctx, out, sm);\n  }}\n}};\n"
    )


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
    structs = [f"template <int G> struct RicciGroup_{tag};\n", f"template <int G> struct RhsGroup_{tag};\n"]
    for g, names in enumerate(RICCI_GROUPS):
        fname = f"ricci_point_{tag}_g{g}"
        code, st = emit_point_function(
            fname, [(f"out[{i}]", ricci[k]) for i, k in enumerate(names)], symmetry_axes=sym,
            comment=f"Rbar_ij {names}, {coord} (symmetry_axes='{sym}'): Ricci_eval.py:27-167",
            reg_capacity=REG_CAPACITY,
        )
        parts.append(code)
        stats[f"ricci_g{g}"] = st
        structs.append(_group_struct("RicciGroup", tag, g, fname, [be.RBAR_ORDER.index(k) for k in names],
                                     st["smem_slots"]))
    for g, names in enumerate(RHS_GROUPS):
        fname = f"rhs_point_{tag}_g{g}"
        code, st = emit_point_function(
            fname, [(f"out[{i}]", rhs[k]) for i, k in enumerate(names)], upwind_vec=betaU, symmetry_axes=sym,
            comment=f"BSSN RHS + KO (CAKO) of {names}, {coord} (symmetry_axes='{sym}'): rhs_eval.py:122-220",
            reg_capacity=REG_CAPACITY,
        )
        parts.append(code)
        stats[f"rhs_g{g}"] = st
        structs.append(_group_struct("RhsGroup", tag, g, fname, [be.GF_ORDER.index(k) for k in names],
                                     st["smem_slots"]))
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
        f"// Per point: {stats}\n"
        "#pragma once\n\n"
    )
    OUTDIR.mkdir(parents=True, exist_ok=True)
    (OUTDIR / f"bssn_{tag}.cuh").write_text(hdr + "\n".join(parts) + "\n" + "\n".join(structs))
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
