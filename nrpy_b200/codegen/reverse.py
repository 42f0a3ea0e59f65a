"""Reverse-mode (adjoint) point functions, derived from the forward point algebra.

Code-generation time only. For a list of forward outputs o_j(leaves) the emitted function
computes, at one grid point, the vector-Jacobian product

    leaf_bar[l] = sum_j  obar_j * d o_j / d leaf_l

for every *active* leaf: gridfunction values, finite-difference derivatives and Rbar_ij.
rfm-precompute values and scalar parameters are constants. The derivation is plain
reverse accumulation over the CSE'd straight-line forward program:

1. ``sympy.cse`` splits the outputs into statements t_k = e_k(t_<k, leaves);
2. statements that do not depend on an active leaf are marked passive;
3. walking the active statements backwards, each operand x of e_k receives the
   contribution (d e_k / d x) * tbar_k; tbar_k is complete (and emitted) when the walk
   reaches t_k's definition, because every user of t_k comes later in the forward order.

The emitted body is the forward statements, then the adjoint statements, then one
``OUT(row) = ...`` per active leaf. ``OUT`` is defined by the including translation unit
(an accumulating reference into the leaf-adjoint rows); seeds are read through
``ADJIN(j)``. Values beyond the register budget go to per-thread slots ``SMEM(k)``
(allocated by ``emit_cuda.allocate_values``) that the including code maps to memory.

The finite-difference leaves are linear in the stencil values; their transposes (stencil
gathers) are separate kernels, driven by the leaf table ``leaf_table``.
"""

from collections import defaultdict
from typing import Callable, Dict, List, Sequence, Tuple

import sympy as sp

from .bssn_exprs import GF_ORDER, RBAR_ORDER
from .emit_cuda import GF_INDEX, RBAR_INDEX, PointKernel, allocate_values, dfs_order, parse_deriv, schedule_lines

KIND_CODE = {"C": 0, "D": 1, "DD": 2, "upD": 3, "KOD": 4}


def is_active_leaf(name: str) -> bool:
    return name in GF_INDEX or name in RBAR_INDEX or parse_deriv(name) is not None


class _Abs(sp.Function):
    """|x| with d|x|/dx = sign(x) (nrpyAbs of the forward algebra)."""

    def fdiff(self, argindex=1):
        return _Sign(self.args[0])


class _Sign(sp.Function):
    def fdiff(self, argindex=1):
        return sp.S.Zero


def _replace_abs(e: sp.Expr) -> sp.Expr:
    return e.replace(lambda x: isinstance(x, sp.Function) and x.func.__name__ in ("nrpyAbs", "Abs"),
                     lambda x: _Abs(x.args[0]))


def reverse_program(outputs: Sequence[sp.Expr], active_leaf: Callable[[str], bool] = is_active_leaf):
    """Return (statements, leaf_adjoints): statements = forward then adjoint (name, expr),
    leaf_adjoints = {leaf name: expr} (only leaves with a nonzero adjoint)."""
    exprs = [_replace_abs(sp.sympify(e)) for e in outputs]
    syms = (sp.Symbol(f"_cse{i}") for i in range(10**7))
    repl, reduced = sp.cse(exprs, symbols=syms, order="none")
    fwd = [(s.name, e) for s, e in repl]
    active = set()
    for name, e in fwd:
        if any(x.name in active or active_leaf(x.name) for x in e.free_symbols):
            active.add(name)

    contribs: Dict[str, List[sp.Expr]] = defaultdict(list)

    def propagate(e: sp.Expr, bar: sp.Expr) -> None:
        for x in sorted(e.free_symbols, key=lambda s: s.name):
            if x.name in active or active_leaf(x.name):
                d = sp.diff(e, x)
                if d != 0:
                    contribs[x.name].append(d * bar)

    for j, e in enumerate(reduced):
        propagate(e, sp.Symbol(f"AO{j}"))
    rev = []
    for name, e in reversed(fwd):
        if name not in active or not contribs.get(name):
            continue
        bar = sp.Symbol(f"_a{name}")
        rev.append((bar.name, sp.Add(*contribs.pop(name))))
        propagate(e, bar)
    leaf_adj = {k: sp.Add(*v) for k, v in contribs.items() if active_leaf(k)}
    return fwd + rev, leaf_adj


def leaf_table(names: Sequence[str]) -> List[Tuple[str, int, int, int, int]]:
    """Rows of the leaf-adjoint buffer: (name, gf index, kind code, dir1, dir2).

    Rows 0..23 are the gridfunction values (kind C); then the derivative leaves in
    gridfunction-major, sorted order. Rbar_ij adjoints live in their own buffer."""
    rows = [(g, GF_INDEX[g], KIND_CODE["C"], -1, -1) for g in GF_ORDER]
    ders = []
    for n in names:
        pd = parse_deriv(n)
        if pd is None:
            continue
        gf, kind, dirs = pd
        d1 = dirs[0]
        d2 = dirs[1] if len(dirs) > 1 else -1
        ders.append((n, GF_INDEX[gf], KIND_CODE[kind], d1, d2))
    ders = sorted(set(ders), key=lambda r: (r[1], r[2], r[3], r[4]))
    return rows + ders


def emit_vjp_function(fname: str, outputs: Sequence[sp.Expr], row_of: Dict[str, int], upwind_vec=None,
                      symmetry_axes: str = "", comment: str = "", reg_capacity: int = 64, remat_first: bool = False,
                      deriv_remat: bool = False, order: str = "dfs"):
    """Emit the VJP of `outputs` as `fname(ctx, sm)` plus `fname_SMEM_SLOTS`.

    Gridfunction and derivative leaf adjoints go to OUT(row_of[name]); Rbar_ij adjoints
    go to OUTR(k)."""
    stmts, leaf_adj = reverse_program(outputs)
    pk = PointKernel(symmetry_axes)
    outs = []
    for name in sorted(leaf_adj, key=lambda n: (n not in RBAR_INDEX, row_of.get(n, -1), n)):
        lhs = f"OUTR({RBAR_INDEX[name]})" if name in RBAR_INDEX else f"OUT({row_of[name]})"
        outs.append((lhs, leaf_adj[name]))
    pk.build_program(stmts, outs, upwind_vec)
    ordered = {"dfs": lambda: dfs_order(pk.lines), "sched": lambda: pk.lines,
               "sched_dfs": lambda: schedule_lines(dfs_order(pk.lines))}[order]()
    lines, nslots = allocate_values(ordered, reg_capacity, remat_first, deriv_remat)
    body = "\n".join("  " + ln for ln in lines)
    head = f"// {comment}\n" if comment else ""
    code = (
        f"{head}constexpr int {fname}_SMEM_SLOTS = {nslots};\n"
        f"template <typename T, typename TF, typename Ctx>\n"
        f"__device__ __forceinline__ void {fname}(const Ctx &ctx, volatile T *sm) {{\n"
        f"  (void)sm;\n{body}\n}}\n"
    )
    stats = dict(pk.stats)
    stats.update(smem_slots=nslots, statements=len(lines), leaf_outputs=len(outs))
    return code, stats


__all__ = ["reverse_program", "leaf_table", "emit_vjp_function", "is_active_leaf", "KIND_CODE", "RBAR_ORDER"]
