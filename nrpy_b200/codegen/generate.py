"""Generate the pointwise BSSN device functions (nrpy_b200/csrc/gen/*.cuh).

Code-generation time only: needs the nrpy package (the reference's equation modules) on
PYTHONPATH. The emitted headers are committed, so building the CUDA library does not
need nrpy. Each (CoordSystem, symmetry) variant is generated in its own process because
nrpy caches equation objects per CoordSystem and reads ``symmetry_axes`` globally.

Usage: python -m nrpy_b200.codegen.generate [--reference PATH] [--variants ...] [--fd-order N --adjoint ""]
"""

import argparse
import os
import pathlib
import subprocess
import sys
import time

ROOT = pathlib.Path(__file__).resolve().parents[2]
OUTDIR = pathlib.Path(os.environ.get("BSSN_GEN_OUTDIR", str(ROOT / "nrpy_b200" / "csrc" / "gen")))
VARIANTS = {
    # tag: (CoordSystem, symmetry_axes)
    "sph_axi": ("Spherical", "2"),
    "sph_3d": ("Spherical", ""),
    "sinh_axi": ("SinhSpherical", "2"),
    "sinh_3d": ("SinhSpherical", ""),
    # SinhCylindrical with symmetry_axes="1" (axisymmetry about z), as blackhole_spectroscopy.py sets it up
    "sinhcyl_axi": ("SinhCylindrical", "1"),
}


# Output groups: each group is one kernel (its own CSE); groups trade recomputed shared
# subexpressions for fewer live values per thread. Values beyond each group's register budget
# go to per-thread shared-memory slots. The split was chosen by timing every candidate
# group kernel of SinhSpherical 256x64x32 on a B200 (Ricci: 1x6, 2x3, 3x2 and 6x1 outputs;
# RHS: the gauge/metric/extrinsic-curvature outputs together or in two or three parts).
RICCI_GROUPS = [["RbarDD00", "RbarDD01", "RbarDD02"], ["RbarDD11", "RbarDD12", "RbarDD22"]]
RHS_GROUPS = [
    ["aDD00", "aDD01", "aDD02", "aDD11", "aDD12", "aDD22", "alpha", "cf", "hDD00", "hDD01", "hDD02", "hDD11",
     "hDD12", "hDD22", "trK", "vetU0", "vetU1", "vetU2"],
    ["betU0", "betU1", "betU2", "lambdaU0", "lambdaU1", "lambdaU2"],
]
# The reverse-mode functions keep their own (smaller) groups.
ADJ_RICCI_GROUPS = [["RbarDD00", "RbarDD01"], ["RbarDD02", "RbarDD11"], ["RbarDD12", "RbarDD22"]]
ADJ_RHS_GROUPS = [
    ["aDD00", "aDD01", "aDD02", "aDD11", "aDD12", "aDD22"],
    ["alpha", "cf", "hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22", "trK", "vetU0", "vetU1", "vetU2"],
    ["betU0", "betU1", "betU2", "lambdaU0", "lambdaU1", "lambdaU2"],
]
# Per group: (remat_first, deriv_remat, statement order) of the value allocator --
# whether register eviction prefers recomputable values (stencil loads, rfm, parameters),
# whether finite differences are recomputed from their stencils instead of kept in a slot,
# and the statement order ("dfs": one output at a time; "sched": greedy live-range
# schedule; "sched_dfs": the dfs order rescheduled greedily). Chosen by timing every group
# kernel of SinhSpherical 256x64x32 on a B200 under each allocation, order and block size
# (nrpy_b200/codegen/tune_groups.py); lower register budgets with forced occupancy were
# slower in every group (local-memory spills).
RICCI_ALLOC = [(True, True, "sched_dfs"), (True, False, "sched_dfs")]
RHS_ALLOC = [(True, False, "dfs"), (True, False, "sched")]
# Per group register budget (values kept in registers), from the same timing sweep: the
# Ricci groups gain from keeping more values in registers (fewer slots leave more L1 for
# stencil loads) even with a few local-memory spills.
RICCI_CAPS = [160, 150]
RHS_CAPS = [72, 80]
# The FP32 (mixed-precision) instantiations get their own allocation where a budget of their
# own was faster: an FP32 value takes one register instead of two. Timed on SinhSpherical
# 256x64x32 with the FP32 algebra (tune_groups generate-caps --dtype float, budgets 72 to 250):
# Ricci group 0 87.6 -> 71.8 us and group 1 81.6 -> 65.8 us with every value in registers
# (budget 250); RHS group 1 171 -> 160 us at budget 200; RHS group 0 was fastest at 72.
RICCI_CAPS_F32 = [250, 250]
RHS_CAPS_F32 = [72, 200]
# Statements between an L1 prefetch of a stencil row and its first load, per group (0: no
# prefetch), in the FP64 and the FP32 evaluation. Timed on the bench workload (SinhSpherical
# 256x64x64, mixed precision): RHS group 0 in FP32 at distances 25-100 gave 154.9-175.0 M
# pt-updates/s against 156.7 M without, best at 52-55 (174.3-175.0 M); a prefetch in RHS
# group 1 or in the Ricci groups gave nothing or lost.
# At 8th order the same FP32 prefetch lost (mixed 67.5 -> 65.6 M at 256x64x64), so the
# distances apply to 4th order; other orders get none unless --prefetch-f32/-f64 says so.
RICCI_PREFETCH = [0, 0]
RHS_PREFETCH = [0, 0]
RICCI_PREFETCH_F32 = [0, 0]
RHS_PREFETCH_F32 = [55, 0]
PREFETCH_FD_ORDER = 4
# Prefetch statement of the FP64 groups: PREFETCH_ROW (L1) or PREFETCH_ROW_L2.
PREFETCH_MACRO = "PREFETCH_ROW"
# Value types for which a group's slot array is plain instead of volatile (volatile: every slot
# access stays where the allocator put it; plain: the compiler may schedule the accesses), per
# group, from a timing sweep: plain slots help the RHS groups in FP32 and cost in FP64.
RICCI_PLAIN_SLOTS = [(), ()]
RHS_PLAIN_SLOTS = [("float",), ("float",)]
# Threads per block of a group kernel: 128, or 64 when two 128-thread blocks of its
# shared-memory slots would not fit in the 227 KB of one SM.
SMEM_PER_SM = 227 * 1024


def threads_for(slots: int) -> int:
    return 128 if 2 * slots * 8 * 128 <= SMEM_PER_SM else 64
# Reverse-mode (adjoint) functions: generated for these variants only; fewer values in
# registers because the VJP kernels run 64 threads per block with shared-memory slots.
ADJOINT_VARIANTS = ["sph_3d"]
# VJP kernels run 64 threads per block; recompute-first eviction and rematerialized finite
# differences shrink the slot arrays of the largest group from 250 to 199 values (2 blocks
# per SM instead of 1): the 200-step backward of the 128x32x32 workload went from 3.42 s to
# 2.84 s on a B200 (a 90-value budget gave 2.84 s with more spills). Under the "sched_dfs"
# order, budgets of 64/90/120/150/180/210/240 values ran the backward in 2.65/2.61/2.56/
# 2.51/2.55/2.54/2.83 s; at 150 the largest group (rhs_g2) keeps 99 slots instead of 193.
ADJ_REG_CAPACITY = 150
# The greedy reschedule of the dfs order ("sched_dfs") ran the backward in 2.64 s ("dfs": 2.75 s,
# "sched": 3.33 s).
ADJ_REMAT = dict(remat_first=True, deriv_remat=True, order="sched_dfs")


def _group_struct(kind: str, tag: str, g: int, fname: str, gfs, slots: int, plain_slots=(),
                  fname_f32: str = "", slots_f32: int = -1) -> str:
    """The group's descriptor struct. With fname_f32, FP32 evaluations (T = float) call that
    function, which has an allocation of its own with slots_f32 slots."""
    cases = " ".join(f"case {k}: return {x};" for k, x in enumerate(gfs))
    # The kernels hand a group a volatile slot pointer, or a plain one to ask for plain slots;
    # for the value types listed in plain_slots the group drops the qualifier itself (the
    # dynamic shared memory is not a volatile object).
    plain = " || ".join(["!std::is_volatile<S>::value"] + [f"std::is_same<T, {t}>::value" for t in plain_slots])
    if not fname_f32:
        fname_f32, slots_f32 = fname, slots
    nt = threads_for(slots)
    assert 2 * slots_f32 * 4 * nt <= SMEM_PER_SM, "FP32 slots must fit the FP64 block size"

    def call(sm: str) -> str:
        return (f"if constexpr (std::is_same<T, float>::value) {fname_f32}<T, TF, NTB>(ctx, out, {sm});\n"
                f"      else {fname}<T, TF, NTB>(ctx, out, {sm});")
    return (
        f"template <> struct {kind}_{tag}<{g}> {{\n"
        f"  static constexpr int N = {len(gfs)};\n"
        f"  static constexpr int SLOTS = {slots};          // per-thread slots of the FP64 evaluation\n"
        f"  static constexpr int SLOTS_F32 = {slots_f32};  // and of the FP32 evaluation\n"
        f"  static constexpr int NT = {nt};  // threads per block of the single-grid kernels\n"
        f"  __host__ __device__ static constexpr int GF(int k) {{\n"
        f"    switch (k) {{ {cases} }}\n    return -1;\n  }}\n"
        f"  template <typename T, typename TF, int NTB, typename Ctx, typename S>\n"
        f"  __device__ __forceinline__ static void eval(const Ctx &ctx, T *out, S *sm) {{\n"
        f"    if constexpr ({plain}) {{\n"
        f"      {call('const_cast<T *>(sm)')}\n"
        f"    }} else {{\n"
        f"      {call('sm')}\n"
        f"    }}\n  }}\n}};\n"
    )


def header_name(tag: str, fd_order: int) -> str:
    """Generated header of a variant: bssn_<tag>.cuh (4th order) or bssn_<tag>_fd<order>.cuh."""
    return f"bssn_{tag}.cuh" if fd_order == 4 else f"bssn_{tag}_fd{fd_order}.cuh"


def generate_variant(tag: str, fd_order: int = 4) -> None:
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen import fdcoeffs as fdc
    from nrpy_b200.codegen.emit_cuda import emit_point_function

    coord, sym = VARIANTS[tag]
    if fd_order != PREFETCH_FD_ORDER:
        for lst in (RICCI_PREFETCH, RHS_PREFETCH, RICCI_PREFETCH_F32, RHS_PREFETCH_F32):
            lst[:] = [0] * len(lst)
    fdc.set_fd_order(fd_order)
    be.setup_nrpy(sym, fd_order)
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
        remat_first, deriv_remat, order = RICCI_ALLOC[g]
        cap = RICCI_CAPS[g]
        code, st = emit_point_function(
            fname, [(f"out[{i}]", ricci[k]) for i, k in enumerate(names)], symmetry_axes=sym,
            comment=f"Rbar_ij {names}, {coord} (symmetry_axes='{sym}'): Ricci_eval.py:27-167",
            reg_capacity=cap, remat_first=remat_first, deriv_remat=deriv_remat, order=order,
            prefetch_rows=RICCI_PREFETCH[g], prefetch_macro=PREFETCH_MACRO,
        )
        parts.append(code)
        stats[f"ricci_g{g}"] = st
        f32 = {}
        if RICCI_CAPS_F32[g] != cap or RICCI_PREFETCH_F32[g] != RICCI_PREFETCH[g]:
            code, st32 = emit_point_function(
                fname + "_f32", [(f"out[{i}]", ricci[k]) for i, k in enumerate(names)], symmetry_axes=sym,
                comment=f"Rbar_ij {names}, {coord}: the FP32 evaluation's allocation",
                reg_capacity=RICCI_CAPS_F32[g], remat_first=remat_first, deriv_remat=deriv_remat, order=order,
                prefetch_rows=RICCI_PREFETCH_F32[g],
            )
            parts.append(code)
            stats[f"ricci_g{g}_f32"] = st32
            f32 = dict(fname_f32=fname + "_f32", slots_f32=st32["smem_slots"])
        structs.append(_group_struct("RicciGroup", tag, g, fname, [be.RBAR_ORDER.index(k) for k in names],
                                     st["smem_slots"], RICCI_PLAIN_SLOTS[g], **f32))
    for g, names in enumerate(RHS_GROUPS):
        fname = f"rhs_point_{tag}_g{g}"
        remat_first, deriv_remat, order = RHS_ALLOC[g]
        cap = RHS_CAPS[g]
        code, st = emit_point_function(
            fname, [(f"out[{i}]", rhs[k]) for i, k in enumerate(names)], upwind_vec=betaU, symmetry_axes=sym,
            comment=f"BSSN RHS + KO (CAKO) of {names}, {coord} (symmetry_axes='{sym}'): rhs_eval.py:122-220",
            reg_capacity=cap, remat_first=remat_first, deriv_remat=deriv_remat, order=order,
            prefetch_rows=RHS_PREFETCH[g], prefetch_macro=PREFETCH_MACRO,
        )
        parts.append(code)
        stats[f"rhs_g{g}"] = st
        f32 = {}
        if RHS_CAPS_F32[g] != cap or RHS_PREFETCH_F32[g] != RHS_PREFETCH[g]:
            code, st32 = emit_point_function(
                fname + "_f32", [(f"out[{i}]", rhs[k]) for i, k in enumerate(names)], upwind_vec=betaU,
                symmetry_axes=sym, comment=f"BSSN RHS + KO (CAKO) of {names}, {coord}: the FP32 evaluation's allocation",
                reg_capacity=RHS_CAPS_F32[g], remat_first=remat_first, deriv_remat=deriv_remat, order=order,
                prefetch_rows=RHS_PREFETCH_F32[g],
            )
            parts.append(code)
            stats[f"rhs_g{g}_f32"] = st32
            f32 = dict(fname_f32=fname + "_f32", slots_f32=st32["smem_slots"])
        structs.append(_group_struct("RhsGroup", tag, g, fname, [be.GF_ORDER.index(k) for k in names],
                                     st["smem_slots"], RHS_PLAIN_SLOTS[g], **f32))
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
    structs.append(f"constexpr int ricci_group_count_{tag} = {len(RICCI_GROUPS)};\n"
                   f"constexpr int rhs_group_count_{tag} = {len(RHS_GROUPS)};\n")
    hdr = (
        "// Generated by nrpy_b200/codegen/generate.py from NRPy's BSSN equation modules.\n"
        f"// Variant {tag}: CoordSystem={coord}, symmetry_axes='{sym}', {fd_order}th-order FD, KO (CAKO).\n"
        f"// Register budgets Ricci {RICCI_CAPS}, RHS {RHS_CAPS} values (FP32 evaluation: Ricci {RICCI_CAPS_F32}, "
        f"RHS {RHS_CAPS_F32}); L1 row prefetch distance Ricci {RICCI_PREFETCH}, RHS {RHS_PREFETCH} (FP32: "
        f"Ricci {RICCI_PREFETCH_F32}, RHS {RHS_PREFETCH_F32}); "
        f"allocation (remat_first, deriv_remat, "
        f"order): Ricci {RICCI_ALLOC}, RHS {RHS_ALLOC}; plain slots Ricci {RICCI_PLAIN_SLOTS}, RHS {RHS_PLAIN_SLOTS}.\n"
        f"// Per point: {stats}\n"
        "#pragma once\n\n"
    )
    OUTDIR.mkdir(parents=True, exist_ok=True)
    (OUTDIR / header_name(tag, fd_order)).write_text(hdr + "\n".join(parts) + "\n" + "\n".join(structs))
    print(f"{tag} (fd_order {fd_order}): {stats} ({time.time() - t0:.1f}s)")


def _c_rational(r) -> str:
    import sympy as sp

    r = sp.Rational(r)
    return f"{int(r.p)}.0" if r.q == 1 else f"{int(r.p)}.0 / {int(r.q)}.0"


def _vjp_struct(kind: str, tag: str, g: int, fname: str, seeds, slots: int) -> str:
    cases = " ".join(f"case {k}: return {x};" for k, x in enumerate(seeds))
    return (
        f"template <> struct {kind}_{tag}<{g}> {{\n"
        f"  static constexpr int N = {len(seeds)};\n"
        f"  static constexpr int SLOTS = {slots};\n"
        f"  __host__ __device__ static constexpr int SEED(int k) {{\n"
        f"    switch (k) {{ {cases} }}\n    return -1;\n  }}\n"
        f"  template <typename T, typename TF, typename Ctx>\n"
        f"  __device__ __forceinline__ static void eval(const Ctx &ctx, volatile T *sm) {{\n"
        f"    {fname}<T, TF>(ctx, sm);\n  }}\n}};\n"
    )


def generate_adjoint(tag: str) -> None:
    """Reverse-mode point functions of one variant (nrpy_b200/csrc/gen/bssn_adj_<tag>.cuh).

    * a leaf table: one row per gridfunction value and per finite-difference derivative
      that Ricci, the RHS or H reads (gf, kind, directions), which the stencil-transpose
      kernel walks;
    * stencil weights at offsets -3..3 (centred first/second derivative, upwind, KO) and
      the shifted radiation first-derivative stencils;
    * VJP functions of the Ricci and RHS output groups, of H and of the detgammabar
      projection; and the upwind-selector bits of a point.
    """
    import sympy as sp

    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen import fdcoeffs as fdc
    from nrpy_b200.codegen.emit_cuda import PointKernel
    from nrpy_b200.codegen.reverse import emit_vjp_function, leaf_table

    coord, sym = VARIANTS[tag]
    be.setup_nrpy(sym)
    t0 = time.time()
    rhs, betaU = be.rhs_exprs(coord)
    ricci = be.ricci_exprs(coord)
    cons = be.constraint_exprs(coord)
    enf = be.enforce_exprs(coord)
    names = set()
    for e in list(rhs.values()) + list(ricci.values()) + [cons["H"]]:
        names |= {x.name for x in sp.sympify(e).free_symbols}
    rows = leaf_table(sorted(names))
    row_of = {r[0]: i for i, r in enumerate(rows)}
    parts = [f"constexpr int adj_nrows_{tag} = {len(rows)};\n",
             "// leaf rows: {gridfunction, kind (0 value, 1 dD, 2 dDD, 3 dupD, 4 dKOD), dir1, dir2}\n",
             f"constexpr signed char adj_rows_{tag}[{len(rows)}][4] = {{\n"]
    parts += [f"    {{{gf}, {kind}, {d1}, {d2}}},  // {name}\n" for name, gf, kind, d1, d2 in rows]
    parts.append("};\n")

    def wrow(w):
        return "{" + ", ".join(_c_rational(w.get(s, 0)) for s in range(-3, 4)) + "}"

    up = fdc.upwind(+1)
    parts.append("// stencil weights at offsets -3..3 (before the invdxx factors)\n")
    parts.append(f"constexpr double adj_wD_{tag}[7] = {wrow(fdc.first_centred())};\n")
    parts.append(f"constexpr double adj_wDD_{tag}[7] = {wrow(fdc.second_centred())};\n")
    parts.append(f"constexpr double adj_wUP_{tag}[7] = {wrow(up)};\n")
    parts.append(f"constexpr double adj_wKO_{tag}[7] = {wrow(fdc.kreiss_oliger())};\n")
    fd1 = ", ".join("{" + ", ".join(_c_rational(fdc.radiation_fd1(o).get(s, 0)) for s in range(-4, 5)) + "}"
                    for o in range(-2, 3))
    parts.append(f"// radiation first derivative, stencil shift -2..2, offsets -4..4\n"
                 f"constexpr double adj_wFD1_{tag}[5][9] = {{{fd1}}};\n\n")
    stats = {}
    structs = [f"template <int G> struct RicciVjp_{tag};\n", f"template <int G> struct RhsVjp_{tag};\n"]
    for g, gnames in enumerate(ADJ_RICCI_GROUPS):
        fname = f"ricci_vjp_{tag}_g{g}"
        code, st = emit_vjp_function(fname, [ricci[k] for k in gnames], row_of, symmetry_axes=sym,
                                     comment=f"VJP of Rbar_ij {gnames} (Ricci_eval.py:27-167)",
                                     reg_capacity=ADJ_REG_CAPACITY, **ADJ_REMAT)
        parts.append(code)
        stats[f"ricci_g{g}"] = st
        structs.append(_vjp_struct("RicciVjp", tag, g, fname, [be.RBAR_ORDER.index(k) for k in gnames],
                                   st["smem_slots"]))
    for g, gnames in enumerate(ADJ_RHS_GROUPS):
        fname = f"rhs_vjp_{tag}_g{g}"
        code, st = emit_vjp_function(fname, [rhs[k] for k in gnames], row_of, upwind_vec=betaU,
                                     symmetry_axes=sym, comment=f"VJP of the RHS of {gnames} (rhs_eval.py:122-220)",
                                     reg_capacity=ADJ_REG_CAPACITY, **ADJ_REMAT)
        parts.append(code)
        stats[f"rhs_g{g}"] = st
        structs.append(_vjp_struct("RhsVjp", tag, g, fname, [be.GF_ORDER.index(k) for k in gnames],
                                   st["smem_slots"]))
    code, st = emit_vjp_function(f"h_vjp_{tag}", [cons["H"]], row_of, symmetry_axes=sym,
                                 comment="VJP of the Hamiltonian constraint H (constraints_eval.py:364-492)",
                                 reg_capacity=ADJ_REG_CAPACITY, **ADJ_REMAT)
    parts.append(code)
    stats["H"] = st
    hnames = ["hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22"]
    code, st = emit_vjp_function(f"enforce_vjp_{tag}", [enf[k] for k in hnames], row_of, symmetry_axes=sym,
                                 comment="VJP of the detgammabar projection "
                                 "(enforce_detgammabar_equals_detgammahat.py:85-110)",
                                 reg_capacity=ADJ_REG_CAPACITY, **ADJ_REMAT)
    parts.append(code)
    stats["enforce"] = st
    pk = PointKernel(sym)
    pk.upwind_vec = betaU
    pk._ensure_upwind()
    body = "\n".join("  " + ln for ln in pk.lines)
    parts.append(
        "// Upwind selectors of a point (bit i: betaU[i] = vetU[i]*ReU[i] > 0), the same expressions\n"
        "// the RHS functions evaluate.\n"
        f"template <typename T, typename TF, typename Ctx>\n"
        f"__device__ __forceinline__ int upwind_bits_{tag}(const Ctx &ctx) {{\n{body}\n"
        "  return (Upwind0 ? 1 : 0) | (Upwind1 ? 2 : 0) | (Upwind2 ? 4 : 0);\n}\n"
    )
    hdr = (
        "// Generated by nrpy_b200/codegen/generate.py (reverse mode, nrpy_b200/codegen/reverse.py).\n"
        f"// Variant {tag}: CoordSystem={coord}, symmetry_axes='{sym}'.\n"
        f"// Per point: {stats}\n"
        "#pragma once\n\n"
    )
    OUTDIR.mkdir(parents=True, exist_ok=True)
    (OUTDIR / f"bssn_adj_{tag}.cuh").write_text(hdr + "".join(parts) + "\n" + "\n".join(structs))
    print(f"adjoint {tag}: {len(rows)} leaf rows, {stats} ({time.time() - t0:.1f}s)")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("NRPY_REFERENCE", str(ROOT.parent / "reference")),
                    help="the nrpy checkout (default: $NRPY_REFERENCE, else ../reference beside this repository)")
    ap.add_argument("--variants", default=",".join(VARIANTS))
    ap.add_argument("--adjoint", default=",".join(ADJOINT_VARIANTS))
    ap.add_argument("--fd-order", type=int, default=4,
                    help="interior FD order of the forward variants (the adjoint is 4th order only)")
    ap.add_argument("--prefetch-f32", default=None,
                    help="tuning: L1 row-prefetch distances of the FP32 groups, 'ricci0,ricci1,rhs0,rhs1'")
    ap.add_argument("--prefetch-f64", default=None, help="tuning: the same for the FP64 groups")
    ap.add_argument("--prefetch-f64-l2", action="store_true", help="tuning: FP64 row prefetches into L2")
    ap.add_argument("--caps-f64", default=None, help="tuning: FP64 register budgets 'ricci0,ricci1,rhs0,rhs1'")
    ap.add_argument("--caps-f32", default=None, help="tuning: the same for the FP32 groups")
    ap.add_argument("--one", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--one-adjoint", default=None, help=argparse.SUPPRESS)
    args = ap.parse_args()
    global PREFETCH_FD_ORDER
    if args.prefetch_f32 or args.prefetch_f64:
        PREFETCH_FD_ORDER = args.fd_order  # explicit distances hold for the order being generated
        for lst in (RICCI_PREFETCH, RHS_PREFETCH, RICCI_PREFETCH_F32, RHS_PREFETCH_F32):
            lst[:] = [0] * len(lst)
    if args.prefetch_f32:
        d = [int(x) for x in args.prefetch_f32.split(",")]
        RICCI_PREFETCH_F32[:] = d[:2]
        RHS_PREFETCH_F32[:] = d[2:4]
    if args.caps_f64:
        d = [int(x) for x in args.caps_f64.split(",")]
        RICCI_CAPS[:] = d[:2]
        RHS_CAPS[:] = d[2:4]
    if args.caps_f32:
        d = [int(x) for x in args.caps_f32.split(",")]
        RICCI_CAPS_F32[:] = d[:2]
        RHS_CAPS_F32[:] = d[2:4]
    global PREFETCH_MACRO
    if args.prefetch_f64_l2:
        PREFETCH_MACRO = "PREFETCH_ROW_L2"
    if args.prefetch_f64:
        d = [int(x) for x in args.prefetch_f64.split(",")]
        RICCI_PREFETCH[:] = d[:2]
        RHS_PREFETCH[:] = d[2:4]
    if args.one:
        generate_variant(args.one, args.fd_order)
        return
    if args.one_adjoint:
        generate_adjoint(args.one_adjoint)
        return
    shim = ROOT / "oracle" / "_ref" / "shim"
    env = dict(os.environ)
    env["PYTHONPATH"] = f"{ROOT}:{shim}:{args.reference}"
    procs = [
        subprocess.Popen([sys.executable, "-m", "nrpy_b200.codegen.generate", "--one", tag, "--fd-order",
                          str(args.fd_order)] + (["--prefetch-f32", args.prefetch_f32] if args.prefetch_f32 else [])
                         + (["--prefetch-f64", args.prefetch_f64] if args.prefetch_f64 else [])
                         + (["--prefetch-f64-l2"] if args.prefetch_f64_l2 else [])
                         + (["--caps-f64", args.caps_f64] if args.caps_f64 else [])
                         + (["--caps-f32", args.caps_f32] if args.caps_f32 else []),
                         env=env, cwd=ROOT)
        for tag in args.variants.split(",") if tag
    ]
    if args.fd_order != 4 and args.adjoint:
        raise SystemExit("the adjoint variants are 4th order only: pass --adjoint ''")
    procs += [
        subprocess.Popen([sys.executable, "-m", "nrpy_b200.codegen.generate", "--one-adjoint", tag], env=env,
                         cwd=ROOT)
        for tag in args.adjoint.split(",") if tag
    ]
    rc = [p.wait() for p in procs]
    if any(rc):
        raise SystemExit(f"generation failed: {rc}")


if __name__ == "__main__":
    main()
