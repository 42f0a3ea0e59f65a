"""Emit CUDA device code for one pointwise BSSN kernel from SymPy expressions.

Own code generator (not NRPy's c_codegen): it takes the expression lists assembled in
``bssn_exprs`` and writes a templated ``__device__`` function that evaluates them at one
grid point. Structure of the emitted body:

1. Common subexpressions come from ``sympy.cse``.
2. Every leaf symbol (gridfunction value, finite-difference derivative, rfm precompute
   value, parameter) is defined lazily, right before the first statement that reads it,
   to keep register live ranges short.
3. Finite differences read stencil points through the ``LD(gf, d0, d1, d2)`` macro that
   the including translation unit defines (global loads or shared-memory tiles), so the
   same algebra serves several kernel layouts.

Derivative symbol grammar (the names NRPy's equation modules use, c_codegen.py:752-1140):
``<gf>_d<kind><indices>`` with kind in {D, DD, upD, KOD}; the first ``rank(gf)`` digits
are the gridfunction's component indices and the rest are derivative directions.
Upwinded derivatives select, per direction, the stencil shifted toward the upwind side
(``UPWIND_ALG(v) = v > 0``, nrpy/helpers/cuda_intrinsics.h:43) using the control vector
betaU[i] = vetU[i] * ReU[i].
"""

import re
from typing import Dict, List, Optional, Sequence, Set, Tuple

import sympy as sp
from sympy.printing.c import C99CodePrinter

from . import fdcoeffs as fdc
from .bssn_exprs import GF_ORDER, RBAR_ORDER

GF_INDEX = {g: i for i, g in enumerate(GF_ORDER)}
RBAR_INDEX = {g: i for i, g in enumerate(RBAR_ORDER)}
BASE_RANK = {"aDD": 2, "hDD": 2, "vetU": 1, "betU": 1, "lambdaU": 1, "alpha": 0, "cf": 0, "trK": 0}
DERIV_RE = re.compile(r"^(aDD|hDD|vetU|betU|lambdaU|alpha|cf|trK)_d(upD|KOD|DD|D)(\d+)$")
RFM_FIELDS = {
    "f0_of_xx0": ("rfm_f0", 0),
    "f0_of_xx0__D0": ("rfm_f0_D0", 0),
    "f0_of_xx0__DD00": ("rfm_f0_DD00", 0),
    "f0_of_xx0__DDD000": ("rfm_f0_DDD000", 0),
    "f1_of_xx1": ("rfm_f1", 1),
    "f1_of_xx1__D1": ("rfm_f1_D1", 1),
    "f1_of_xx1__DD11": ("rfm_f1_DD11", 1),
    # Cylindrical family: the second function of the reference metric depends on xx2 and
    # takes the same three rfm_struct slots (SinhCylindrical's rfm_struct lists f3_of_xx2*
    # where the Spherical family lists f1_of_xx1*).
    "f3_of_xx2": ("rfm_f1", 2),
    "f3_of_xx2__D2": ("rfm_f1_D1", 2),
    "f3_of_xx2__DD22": ("rfm_f1_DD11", 2),
}
SCALAR_PARAMS = {"eta", "KreissOliger_strength_gauge", "KreissOliger_strength_nongauge"}


def parse_deriv(name: str) -> Optional[Tuple[str, str, Tuple[int, ...]]]:
    m = DERIV_RE.match(name)
    if not m:
        return None
    base, kind, digits = m.groups()
    rank = BASE_RANK[base]
    comp = digits[:rank]
    dirs = tuple(int(c) for c in digits[rank:])
    want = 2 if kind == "DD" else 1
    if len(dirs) != want:
        raise ValueError(f"cannot parse derivative symbol {name}")
    return base + comp, kind, dirs


def off_name(o: int) -> str:
    return "0" if o == 0 else (f"p{o}" if o > 0 else f"m{-o}")


class _Printer(C99CodePrinter):
    """C++ printer: algebra type ``T``, integer powers as products, no libm pow()."""

    def __init__(self, names: Dict[str, str]):
        super().__init__({"math_macros": {}})
        self._names = names

    def _print_Symbol(self, expr):
        n = expr.name
        return self._names.get(n, n)

    def _print_Rational(self, expr):
        p, q = int(expr.p), int(expr.q)
        if q == 1:
            return f"T({p}.0)"
        return f"T({p}.0/{q}.0)"

    def _print_Integer(self, expr):
        return f"T({int(expr)}.0)"

    def _print_Float(self, expr):
        return f"T({repr(float(expr))})"

    def _print_Pow(self, expr):
        b, e = expr.base, expr.exp
        bs = self.parenthesize(b, 100)
        if e.is_Integer:
            n = int(e)
            if n == 0:
                return "T(1.0)"
            mag = abs(n)
            prod = "*".join([bs] * mag) if mag <= 4 else f"ipow({self._print(b)}, {mag})"
            if mag > 1:
                prod = f"({prod})"
            return prod if n > 0 else f"(T(1.0)/{prod})"
        if e == sp.Rational(1, 2):
            return f"sqrt({self._print(b)})"
        if e == sp.Rational(-1, 2):
            return f"(T(1.0)/sqrt({self._print(b)}))"
        if e == sp.Rational(1, 3):
            return f"cbrt({self._print(b)})"
        if e == sp.Rational(-1, 3):
            return f"(T(1.0)/cbrt({self._print(b)}))"
        if e == sp.Rational(2, 3):
            return f"(cbrt({self._print(b)})*cbrt({self._print(b)}))"
        if e.is_Rational and int(e.q) in (2, 3):
            root = f"{'sqrt' if int(e.q) == 2 else 'cbrt'}({self._print(b)})"
            mag = abs(int(e.p))
            prod = "*".join([root] * mag) if mag <= 4 else f"ipow({root}, {mag})"
            return f"({prod})" if e > 0 else f"(T(1.0)/({prod}))"
        raise NotImplementedError(f"power {expr}")

    def _print_Function(self, expr):
        fname = expr.func.__name__
        if fname in ("nrpyAbs", "_Abs"):
            return f"fabs({self._print(expr.args[0])})"
        if fname == "_Sign":
            return f"copysign(T(1.0), {self._print(expr.args[0])})"
        return super()._print_Function(expr)

    def _print_Abs(self, expr):
        return f"fabs({self._print(expr.args[0])})"


class PointKernel:
    """Collects leaf definitions and CSE'd statements for one pointwise function."""

    def __init__(self, symmetry_axes: str = "", leaf_index: Optional[Dict[str, int]] = None):
        self.sym_axes = {int(c) for c in symmetry_axes}
        # With a leaf index, finite-difference leaves are read from a precomputed leaf array
        # (LDLEAF(k)) instead of being evaluated from stencil loads.
        self.leaf_index = leaf_index
        self.lines: List[str] = []
        self.defined: Set[str] = set()
        self.loaded: Set[Tuple[str, Tuple[int, int, int]]] = set()
        self.names: Dict[str, str] = {}
        self.upwind_vec: Optional[List[sp.Expr]] = None
        self.printer = _Printer(self.names)
        self.stats = {"loads": 0, "derivs": 0}

    # ---- leaves -----------------------------------------------------------------
    def _load(self, gf: str, off: Tuple[int, int, int]) -> str:
        var = f"v_{gf}_{off_name(off[0])}_{off_name(off[1])}_{off_name(off[2])}"
        if (gf, off) not in self.loaded:
            self.loaded.add((gf, off))
            self.stats["loads"] += 1
            self.lines.append(f"const double {var} = LD({GF_INDEX[gf]}, {off[0]}, {off[1]}, {off[2]});")
        return var

    def _pt(self, gf: str, d: int, o: int, d2: int = -1, o2: int = 0) -> str:
        off = [0, 0, 0]
        off[d] += o
        if d2 >= 0:
            off[d2] += o2
        return self._load(gf, tuple(off))

    def _define_leaf(self, name: str) -> None:
        if name in self.defined:
            return
        self.defined.add(name)
        if name in GF_INDEX:
            v = self._load(name, (0, 0, 0))
            self.lines.append(f"const T {name} = T({v});")
            return
        if name in RBAR_INDEX:
            self.lines.append(f"const T {name} = T(LDAUX({RBAR_INDEX[name]}));")
            return
        if name in RFM_FIELDS:
            arr, d = RFM_FIELDS[name]
            self.lines.append(f"const T {name} = T(RFM({arr}, {d}));")
            return
        if name in SCALAR_PARAMS:
            self.lines.append(f"const T {name} = T(PARAM({name}));")
            return
        m = re.fullmatch(r"AO(\d+)", name)
        if m:  # adjoint seed of forward output m (reverse-mode functions)
            self.lines.append(f"const T {name} = T(ADJIN({m.group(1)}));")
            return
        pd = parse_deriv(name)
        if pd is None:
            raise KeyError(f"unknown symbol {name}")
        gf, kind, dirs = pd
        self.stats["derivs"] += 1
        if self.leaf_index is not None:
            self.lines.append(f"const T {name} = T(LDLEAF({self.leaf_index[name]}));")
            return
        self.lines.append(self._deriv_code(name, gf, kind, dirs))

    def _deriv_code(self, name: str, gf: str, kind: str, dirs: Tuple[int, ...]) -> str:
        """Finite-difference statement, evaluated in the stencil type TF, stored as T."""

        def c(r) -> str:  # rational constant in TF
            p, q = int(sp.Rational(r).p), int(sp.Rational(r).q)
            return f"TF({p}.0/{q}.0)" if q != 1 else f"TF({p}.0)"

        def v(var: str) -> str:
            return f"TF({var})"

        if kind == "D":
            (d,) = dirs
            w = fdc.first_centred()
            terms = [f"{c(w[o])}*({v(self._pt(gf, d, o))} - {v(self._pt(gf, d, -o))})" for o in sorted(k for k in w if k > 0)]
            return f"const T {name} = T(TF(invdxx{d}) * ({' + '.join(terms)}));"
        if kind == "DD":
            d1, d2 = dirs
            if d1 == d2:
                w = fdc.second_centred()
                terms = [f"{c(w[0])}*{v(self._pt(gf, d1, 0))}"]
                for o in sorted(k for k in w if k > 0):
                    terms.append(f"{c(w[o])}*({v(self._pt(gf, d1, o))} + {v(self._pt(gf, d1, -o))})")
                return f"const T {name} = T(TF(invdxx{d1})*TF(invdxx{d1}) * ({' + '.join(terms)}));"
            w = fdc.first_centred()
            pos = sorted(k for k in w if k > 0)

            def inner(a: int) -> str:
                return " + ".join(
                    f"{c(w[b])}*({v(self._pt(gf, d1, a, d2, b))} - {v(self._pt(gf, d1, a, d2, -b))})" for b in pos
                )

            outer = " + ".join(f"{c(w[a])}*(({inner(a)}) - ({inner(-a)}))" for a in pos)
            return f"const T {name} = T(TF(invdxx{d1})*TF(invdxx{d2}) * ({outer}));"
        if kind == "upD":
            (d,) = dirs
            up = fdc.upwind(+1)
            # downwind weights satisfy dn[s] = -up[-s]: select the sample, not the weight.
            terms = []
            for t in sorted(up):
                fu = self._pt(gf, d, t)
                fd = self._pt(gf, d, -t)
                terms.append(f"{c(up[t])}*(Upwind{d} ? {v(fu)} : -{v(fd)})")
            return f"const T {name} = T(TF(invdxx{d}) * ({' + '.join(terms)}));"
        if kind == "KOD":
            (d,) = dirs
            w = fdc.kreiss_oliger()
            terms = [f"{c(w[0])}*{v(self._pt(gf, d, 0))}"]
            for o in sorted(k for k in w if k > 0):
                terms.append(f"{c(w[o])}*({v(self._pt(gf, d, o))} + {v(self._pt(gf, d, -o))})")
            return f"const T {name} = T(TF(invdxx{d}) * ({' + '.join(terms)}));"
        raise ValueError(kind)

    def _ensure(self, expr: sp.Expr) -> None:
        for s in sorted(expr.free_symbols, key=lambda x: x.name):
            if s.name.startswith("_"):
                continue
            if parse_deriv(s.name) and parse_deriv(s.name)[1] == "upD" and self.leaf_index is None:
                self._ensure_upwind()
            self._define_leaf(s.name)

    def _ensure_upwind(self) -> None:
        if "Upwind0" in self.defined:
            return
        self.defined.add("Upwind0")
        assert self.upwind_vec is not None
        for i, e in enumerate(self.upwind_vec):
            self._ensure(e)
            self.lines.append(f"const bool Upwind{i} = ({self.printer._print(e)}) > T(0.0);")

    # ---- driver -------------------------------------------------------------------
    def _chain(self, name: str, expr: sp.Expr, order_of) -> List[Tuple[str, sp.Expr]]:
        """Split a long sum into a chain of partial sums, terms ordered by when their
        operands become available, so that each term's operands can die early."""
        if not expr.is_Add or len(expr.args) <= 3:
            return [(name, expr)]
        terms = sorted(expr.args, key=lambda t: max([order_of(x) for x in t.free_symbols] + [-1]))
        out: List[Tuple[str, sp.Expr]] = []
        acc = sp.Add(terms[0], terms[1], evaluate=False)
        for j, t in enumerate(terms[2:]):
            nm = f"{name}_p{j}"
            out.append((nm, acc))
            acc = sp.Add(sp.Symbol(nm), t, evaluate=False)
        out.append((name, acc))
        return out

    def build(self, outputs: Sequence[Tuple[str, sp.Expr]], upwind_vec=None) -> str:
        self.upwind_vec = upwind_vec
        exprs = [sp.sympify(e) for _, e in outputs]
        syms = (sp.Symbol(f"_cse{i}") for i in range(10**7))
        repl, reduced = sp.cse(exprs, symbols=syms, order="none")
        pos = {s.name: i for i, (s, _) in enumerate(repl)}

        def order_of(x):
            return pos.get(x.name, -1)

        stmts: List[Tuple[str, sp.Expr, bool]] = []  # (name, expr, is_output)
        for sym, e in repl:
            stmts += [(n, x, False) for n, x in self._chain(sym.name, e, order_of)]
        for k, ((lhs, _), e) in enumerate(zip(outputs, reduced)):
            chain = self._chain(f"_out{k}", e, order_of)
            stmts += [(n, x, False) for n, x in chain[:-1]]
            stmts.append((lhs, chain[-1][1], True))
        # Leaf definitions are created lazily in first-use order (their "natural" slots).
        nodes: List[Tuple[str, str]] = []  # (defined name or "", code line)
        for name, e, is_out in stmts:
            self._ensure(e)
            self.lines.append(f"{name} = {self.printer._print(e)};" if is_out
                              else f"const T {name} = {self.printer._print(e)};")
        self.lines = schedule_lines(self.lines)
        return "\n".join("  " + ln for ln in self.lines)

    def build_program(self, stmts: Sequence[Tuple[str, sp.Expr]], outputs: Sequence[Tuple[str, sp.Expr]],
                      upwind_vec=None) -> None:
        """Emit an already-CSE'd straight-line program (name, expr) and then the outputs
        (lhs code, expr); long sums are split into partial-sum chains as in build()."""
        self.upwind_vec = upwind_vec
        pos = {name: i for i, (name, _) in enumerate(stmts)}

        def order_of(x):
            return pos.get(x.name, -1)

        flat: List[Tuple[str, sp.Expr, bool]] = []
        for name, e in stmts:
            flat += [(n, x, False) for n, x in self._chain(name, e, order_of)]
        for k, (lhs, e) in enumerate(outputs):
            chain = self._chain(f"_res{k}", e, order_of)
            flat += [(n, x, False) for n, x in chain[:-1]]
            flat.append((lhs, chain[-1][1], True))
        for name, e, is_out in flat:
            self._ensure(e)
            self.lines.append(f"{name} = {self.printer._print(e)};" if is_out
                              else f"const T {name} = {self.printer._print(e)};")
        self.lines = schedule_lines(self.lines)


_DEF_RE = re.compile(r"\s*const (?:T|double|bool) (\w+) =")
_TOK_RE = re.compile(r"[A-Za-z_]\w*")


def schedule_lines(lines: List[str]) -> List[str]:
    """Reorder straight-line statements to keep few values live (greedy list scheduling).

    Among statements whose operands are all available, pick the one that ends the most
    live ranges net of the value it creates; ties keep the original order.
    """
    defs: Dict[str, int] = {}
    for i, ln in enumerate(lines):
        m = _DEF_RE.match(ln)
        if m:
            defs[m.group(1)] = i
    deps: List[List[int]] = []
    users: List[List[int]] = [[] for _ in lines]
    for i, ln in enumerate(lines):
        body = ln.split("=", 1)[1]
        ds = sorted({defs[t] for t in _TOK_RE.findall(body) if t in defs and defs[t] != i})
        deps.append(ds)
        for d in ds:
            users[d].append(i)
    remaining = [len(u) for u in users]
    npend = [len(d) for d in deps]
    is_def = [1 if _DEF_RE.match(ln) else 0 for ln in lines]
    ready = {i for i in range(len(lines)) if npend[i] == 0}
    order: List[int] = []
    while ready:
        best, bscore = -1, None
        for s in ready:
            kill = 0
            for d in deps[s]:
                if remaining[d] == 1:
                    kill += 1
            score = (kill - is_def[s], -s)
            if bscore is None or score > bscore:
                bscore, best = score, s
        ready.remove(best)
        order.append(best)
        for d in deps[best]:
            remaining[d] -= 1
        for u in users[best]:
            npend[u] -= 1
            if npend[u] == 0:
                ready.add(u)
    if len(order) != len(lines):
        raise RuntimeError("statement dependency cycle")
    return [lines[i] for i in order]


def dfs_order(lines: List[str]) -> List[str]:
    """Topological order that completes one output at a time (post-order DFS from each
    output in turn), so values shared by later outputs are the only long-lived ones."""
    defs: Dict[str, int] = {}
    for i, ln in enumerate(lines):
        m = _DEF_RE.match(ln)
        if m:
            defs[m.group(1)] = i
    deps = []
    for i, ln in enumerate(lines):
        body = ln.split("=", 1)[1]
        deps.append([defs[t] for t in dict.fromkeys(_TOK_RE.findall(body)) if t in defs and defs[t] != i])
    done = [False] * len(lines)
    order: List[int] = []

    def visit(root: int) -> None:
        stack = [(root, 0)]
        while stack:
            node, k = stack.pop()
            if done[node]:
                continue
            if k < len(deps[node]):
                stack.append((node, k + 1))
                d = deps[node][k]
                if not done[d]:
                    stack.append((d, 0))
            else:
                done[node] = True
                order.append(node)

    for i, ln in enumerate(lines):
        if not _DEF_RE.match(ln):
            visit(i)
    for i in range(len(lines)):
        if not done[i]:
            visit(i)
    return [lines[i] for i in order]


def _parse(lines: List[str]):
    """(defined name or None, type or None, rhs text, is_output) per statement."""
    out = []
    for ln in lines:
        m = re.match(r"\s*const (T|double|bool) (\w+) = (.*);\s*$", ln)
        if m:
            out.append((m.group(2), m.group(1), m.group(3), False))
        else:
            lhs, rhs = ln.split("=", 1)
            out.append((lhs.strip(), None, rhs.strip().rstrip(";"), True))
    return out


def _is_remat(ty: str, rhs: str, remat: Dict[str, str], deriv_remat: bool = False) -> bool:
    if ty == "double" and rhs.startswith("LD("):
        return True
    if ty == "T" and (rhs.startswith("T(RFM(") or rhs.startswith("T(PARAM(") or rhs.startswith("T(LDAUX(")
                      or rhs.startswith("T(LDLEAF(")):
        return True
    if deriv_remat and ty == "T" and rhs.startswith("T(TF(invdxx"):
        return True  # finite difference: recomputed from its stencil loads at each use
    m = re.fullmatch(r"T\((v_\w+)\)", rhs)
    return bool(m and m.group(1) in remat)


def allocate_values(lines: List[str], reg_capacity: int, remat_first: bool = False,
                    deriv_remat: bool = False) -> Tuple[List[str], int]:
    """Keep at most `reg_capacity` values in registers at any statement.

    Linear scan over live intervals (Poletto-Sarkar): when too many values are live, one
    leaves the register set -- the one whose interval ends last, or with `remat_first` the
    furthest-ending value that can be recomputed from memory (stencil loads, rfm arrays,
    parameters, and with `deriv_remat` finite differences) if any is live. Recomputable
    values are re-read (re-evaluated) at each use; all others are stored once to a
    per-thread shared-memory slot, SMEM(k), and read from it at each use (the slot array is
    volatile, so the compiler cannot keep the value in a register).
    Returns the rewritten statements and the number of shared-memory slots.
    """
    st = _parse(lines)
    n = len(st)
    idx = {name: i for i, (name, ty, _, is_out) in enumerate(st) if not is_out}
    last = {}
    for i, (_, _, rhs, _) in enumerate(st):
        for t in _TOK_RE.findall(rhs):
            if t in idx:
                last[t] = i
    remat: Dict[str, str] = {}  # name -> expression in loads / rfm / parameters only

    def expand(rhs: str) -> str:
        return _TOK_RE.sub(lambda m: f"({remat[m.group(0)]})" if m.group(0) in remat else m.group(0), rhs)

    for name, ty, rhs, is_out in st:
        if not is_out and _is_remat(ty, rhs, remat, deriv_remat):
            remat[name] = expand(rhs)
    # intervals of values that need storage (bools stay in registers: predicates)
    iv = [(idx[v], last.get(v, idx[v]), v) for v in idx if st[idx[v]][1] != "bool"]
    iv.sort()
    active: List[Tuple[int, str]] = []  # (end, name) of values in registers
    spilled: Dict[str, bool] = {}
    import bisect

    for start, end, v in iv:
        active = [(e, a) for e, a in active if e > start]  # intervals ending at start are done
        bisect.insort(active, (end, v))
        if len(active) > reg_capacity:
            victim = None
            if remat_first:
                for k in range(len(active) - 1, -1, -1):
                    if active[k][1] in remat:
                        victim = active.pop(k)[1]
                        break
            if victim is None:
                victim = active.pop()[1]  # furthest end
            spilled[victim] = True
    # shared-memory slots for spilled, non-rematerializable values (interval colouring)
    slot_of: Dict[str, int] = {}
    free: List[int] = []
    busy: List[Tuple[int, int]] = []  # (end, slot)
    nslots = 0
    for start, end, v in iv:
        if v not in spilled or v in remat:
            continue
        keep = []
        for e, k in busy:
            if e < start:
                free.append(k)
            else:
                keep.append((e, k))
        busy = keep
        if free:
            free.sort()
            k = free.pop(0)
        else:
            k = nslots
            nslots += 1
        slot_of[v] = k
        busy.append((end, k))

    def rewrite(rhs: str) -> str:
        def sub(m):
            t = m.group(0)
            if t in spilled:
                if t in remat:
                    return f"({remat[t]})"
                return f"SMEM({slot_of[t]})"
            return t

        return _TOK_RE.sub(sub, rhs)

    out: List[str] = []
    for name, ty, rhs, is_out in st:
        r = rewrite(rhs)
        if is_out:
            out.append(f"{name} = {r};")
        elif name in spilled and name in remat:
            continue  # re-read at each use
        elif name in slot_of:
            out.append(f"SMEM({slot_of[name]}) = {r};")
        else:
            out.append(f"const {ty} {name} = {r};")
    return out, nslots


def emit_point_function(
    fname: str,
    outputs: Sequence[Tuple[str, sp.Expr]],
    upwind_vec=None,
    symmetry_axes: str = "",
    comment: str = "",
    reg_capacity: int = 0,
    remat_first: bool = False,
    deriv_remat: bool = False,
    order: str = "dfs",
    leaf_index: Optional[Dict[str, int]] = None,
    prefetch_rows: int = 0,
    prefetch_macro: str = "PREFETCH_ROW",
) -> Tuple[str, Dict[str, int]]:
    """Emit `fname` and the constant `fname_SMEM_SLOTS`. With prefetch_rows = D > 0, each
    stencil row (gridfunction, i1 offset, i2 offset) is prefetched into L1
    (PREFETCH_ROW(gf, b, c), provided by the caller's context) D statements before the
    statement that first loads from it. With reg_capacity > 0 the values
    beyond that many live doubles go to shared-memory slots (SMEM(k), provided by the
    caller through the `sm` argument: slot k of this thread; the template parameter NT is
    the slot stride, i.e. the threads of a block). The slot pointer type S is the caller's:
    `volatile T` keeps every slot access a shared-memory access at its place in the program,
    plain `T` lets the compiler move and merge them (each thread only touches its own slots)."""
    pk = PointKernel(symmetry_axes, leaf_index)
    pk.build(outputs, upwind_vec)
    if reg_capacity > 0:
        # Statement order: "dfs" completes one output at a time (dfs_order); "sched" keeps the
        # greedy live-range schedule; "sched_dfs" reschedules the dfs order greedily.
        ordered = {"dfs": lambda: dfs_order(pk.lines), "sched": lambda: pk.lines,
                   "sched_dfs": lambda: schedule_lines(dfs_order(pk.lines))}[order]()
        lines, nslots = allocate_values(ordered, reg_capacity, remat_first, deriv_remat)
    else:
        lines, nslots = pk.lines, 0
    if prefetch_rows > 0:
        lines = insert_row_prefetches(lines, prefetch_rows, prefetch_macro)
    body = "\n".join("  " + ln for ln in lines)
    head = f"// {comment}\n" if comment else ""
    code = (
        f"{head}constexpr int {fname}_SMEM_SLOTS = {nslots};\n"
        f"template <typename T, typename TF, int NT = 128, typename Ctx, typename S>\n"
        f"__device__ __forceinline__ void {fname}(const Ctx &ctx, T *__restrict__ out, S *sm) {{\n"
        f"  (void)sm;\n{body}\n}}\n"
    )
    stats = dict(pk.stats)
    stats["smem_slots"] = nslots
    return code, stats


_LD_RE = re.compile(r"LD\((\d+), *(-?\d+), *(-?\d+), *(-?\d+)\)")


def insert_row_prefetches(lines: Sequence[str], distance: int, macro: str = "PREFETCH_ROW") -> List[str]:
    """Insert PREFETCH_ROW(gf, b, c) `distance` statements before the first statement that
    loads from stencil row (gf, b, c); rows first loaded within the first `distance`
    statements are prefetched at the top, in the order of their first loads."""
    first = {}
    for k, ln in enumerate(lines):
        for m in _LD_RE.finditer(ln):
            key = (int(m.group(1)), int(m.group(3)), int(m.group(4)))
            first.setdefault(key, k)
    at = {}
    for key, k in first.items():
        at.setdefault(max(0, k - distance), []).append(key)
    out = []
    for k, ln in enumerate(lines):
        for gf, b, c in at.get(k, []):
            out.append(f"{macro}({gf}, {b}, {c});")
        out.append(ln)
    return out


def leaf_names(exprs: Sequence[sp.Expr]) -> List[str]:
    """Finite-difference leaves of a set of expressions, grouped by gridfunction (sorted)."""
    names = set()
    for e in exprs:
        for x in sp.sympify(e).free_symbols:
            if parse_deriv(x.name):
                names.add(x.name)
    return sorted(names, key=lambda n: (parse_deriv(n)[0], n))


def emit_leaf_function(fname: str, names: Sequence[str], upwind_vec=None, symmetry_axes: str = "",
                       comment: str = "") -> Tuple[str, Dict[str, int]]:
    """Emit `fname`, which evaluates the finite-difference leaves `names` at one point from
    stencil loads (the same statements the point functions use) and stores leaf k through
    LEAFOUT(k, value). The upwinded leaves use the point's shift vector (upwind_vec)."""
    pk = PointKernel(symmetry_axes)
    pk.upwind_vec = upwind_vec
    for k, name in enumerate(names):
        if parse_deriv(name)[1] == "upD":
            pk._ensure_upwind()
        pk._define_leaf(name)
        pk.lines.append(f"LEAFOUT({k}, {name});")
    body = "\n".join("  " + ln for ln in pk.lines)
    head = f"// {comment}\n" if comment else ""
    code = (
        f"{head}constexpr int {fname}_NUM_LEAVES = {len(names)};\n"
        f"template <typename T, typename TF, typename Ctx>\n"
        f"__device__ __forceinline__ void {fname}(const Ctx &ctx) {{\n{body}\n}}\n"
    )
    return code, dict(pk.stats)
