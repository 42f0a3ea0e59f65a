"""Finite-difference weights of the BHaH stencils (4th order by default), derived from Taylor series.

The operator set and stencil placement follow nrpy/finite_difference.py:202-330:

Offsets below are for the default 4th order; ``set_fd_order`` selects another even order
(radius order/2, KO derivative of order order+2 on order+3 points).

* ``dD``   first derivative, centred, offsets -2..2;
* ``dDD``  second derivative, centred (unmixed) or the product of two centred first
  derivatives (mixed, 4x4 points);
* ``dupD`` / ``ddnD`` first derivative on a stencil shifted by +1 / -1 (offsets -1..3 /
  -3..1), selected per point by the sign of the upwind vector;
* ``dKOD`` Kreiss-Oliger dissipation: the 6th derivative on offsets -3..3, times
  (-1)^((w+1)/2) / 2^6 with w = 7 points, i.e. (1/64) * [1,-6,15,-20,15,-6,1].

Every operator is scaled by ``invdxx`` once per derivative index (the KO operator once).
The weights are solved here independently from the moment conditions
sum_k w_k s_k^m / m! = delta_{m,d}, m = 0..n-1, in exact rationals.
"""

from functools import lru_cache
from typing import Dict, Tuple

import sympy as sp

FD_ORDER = 4
NGHOSTS = 3
# The outer radiation condition keeps its own 4th-order one-sided derivatives whatever the
# interior order (radiation_BC_fd_order = 4 in the generated projects).
RADIATION_BC_FD_ORDER = 4


def set_fd_order(order: int) -> None:
    """Interior finite-difference order (even); NGHOSTS = order/2 + 1 (one more for the
    upwinded stencils and KO dissipation)."""
    global FD_ORDER, NGHOSTS
    if order < 2 or order % 2:
        raise ValueError(f"fd_order {order}: an even order >= 2")
    FD_ORDER, NGHOSTS = order, order // 2 + 1


@lru_cache(maxsize=None)
def weights(offsets: Tuple[int, ...], deriv: int) -> Tuple[sp.Rational, ...]:
    n = len(offsets)
    M = sp.Matrix(n, n, lambda m, k: sp.Rational(offsets[k]) ** m / sp.factorial(m))
    rhs = sp.Matrix([1 if m == deriv else 0 for m in range(n)])
    w = M.LUsolve(rhs)
    return tuple(sp.nsimplify(x) for x in w)


def centred_offsets(radius: int) -> Tuple[int, ...]:
    return tuple(range(-radius, radius + 1))


def first_centred() -> Dict[int, sp.Rational]:
    w = weights(centred_offsets(FD_ORDER // 2), 1)
    return {s: c for s, c in zip(centred_offsets(FD_ORDER // 2), w) if c != 0}


def second_centred() -> Dict[int, sp.Rational]:
    w = weights(centred_offsets(FD_ORDER // 2), 2)
    return {s: c for s, c in zip(centred_offsets(FD_ORDER // 2), w) if c != 0}


def upwind(shift: int) -> Dict[int, sp.Rational]:
    offs = tuple(s + shift for s in centred_offsets(FD_ORDER // 2))
    w = weights(offs, 1)
    return {s: c for s, c in zip(offs, w) if c != 0}


def kreiss_oliger() -> Dict[int, sp.Rational]:
    order = FD_ORDER + 2
    width = order + 1
    offs = centred_offsets(order // 2)
    w = weights(offs, order)
    sign = (-1) ** sp.Rational(width + 1, 2)
    return {s: c * sign / 2**order for s, c in zip(offs, w) if c != 0}


def radiation_fd1(offset: int) -> Dict[int, sp.Rational]:
    """First derivative on a 5-point stencil shifted by ``offset`` (radiation BCs).

    Mirrors FD1_arbitrary_upwind_x*_dirn of
    nrpy/infrastructures/BHaH/CurviBoundaryConditions/apply_bcs_outerradiation_and_inner.py:122-278
    for radiation_BC_fd_order = 4 (offset in -2..2).
    """
    offs = tuple(s + offset for s in centred_offsets(RADIATION_BC_FD_ORDER // 2))
    w = weights(offs, 1)
    return {s: c for s, c in zip(offs, w) if c != 0}
