"""CPU restatement (numpy / plain Python) of the reference algorithms on the hot path that
are not pointwise BSSN algebra. Test infrastructure only: used by tests/ as a second,
independent checker beside the reference's own generated C (oracle/_ref) and the golden
fixtures; never imported by the product.

Each function cites the reference generator it restates (paths relative to nrpy/).
The pointwise BSSN algebra itself (Ricci, RHS, constraints, detgammabar projection) is
checked against the reference's generated C directly (oracle/ref.py) and the committed
golden fixtures generated from it.
"""

import math
from typing import Dict, List, Tuple

import numpy as np

NGHOSTS = 3
PI = 3.14159265358979323846264338327950288
# BHaH_defines.h (generated): parity type, outer wave speed and asymptotic value per evolved gf
EVOL_GF_PARITY = [4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 0, 4, 5, 6, 7, 8, 9, 1, 2, 3, 0, 1, 2, 3]
WAVESPEED = [1.0] * 24
WAVESPEED[6] = 1.41421356237310
F_INFINITY = [0.0] * 24
F_INFINITY[6] = 1.0
F_INFINITY[10] = 1.0


# ------------------------------------------------------------------------ grid
def grid_params(coord: str, Nxx, grid_physical_size: float, sinhw: float = 0.2) -> Dict:
    """numerical_grids_and_timestep.py:31-190 (cell-centred grid, default xxmin/xxmax)."""
    p = {"coord": coord, "Nxx": tuple(Nxx), "SINHW": sinhw}
    if coord == "SinhSpherical":
        p["AMPL"] = grid_physical_size
        xmin, xmax = [0.0, 0.0, -PI], [1.0, PI, PI]
    elif coord == "Spherical":
        p["RMAX"] = grid_physical_size
        xmin, xmax = [0.0, 0.0, -PI], [grid_physical_size, PI, PI]
    elif coord == "SinhCylindrical":
        p["AMPLRHO"] = p["AMPLZ"] = grid_physical_size
        xmin, xmax = [0.0, -PI, -1.0], [1.0, PI, 1.0]
    else:
        raise ValueError(coord)
    p["N"] = tuple(n + 2 * NGHOSTS for n in Nxx)
    p["dxx"] = [(xmax[d] - xmin[d]) / Nxx[d] for d in range(3)]
    p["invdxx"] = [Nxx[d] / (xmax[d] - xmin[d]) for d in range(3)]
    p["xx"] = [np.array([xmin[d] + ((j - NGHOSTS) + 0.5) * p["dxx"][d] for j in range(p["N"][d])]) for d in range(3)]
    return p


def r_of_xx0(p: Dict, xx0):
    """reference_metric.py:1195-1330: r = xx0 (Spherical), AMPL sinh(xx0/w)/sinh(1/w) (SinhSpherical)."""
    if p["coord"] == "Spherical":
        return np.asarray(xx0, dtype=float)
    w, A = p["SINHW"], p["AMPL"]
    return A * (np.exp(xx0 / w) - np.exp(-xx0 / w)) / (np.exp(1.0 / w) - np.exp(-1.0 / w))


def dr_dxx0(p: Dict, xx0):
    if p["coord"] == "Spherical":
        return np.ones_like(np.asarray(xx0, dtype=float))
    w, A = p["SINHW"], p["AMPL"]
    return A * (np.exp(xx0 / w) / w + np.exp(-xx0 / w) / w) / (np.exp(1.0 / w) - np.exp(-1.0 / w))


def cfl_dt(p: Dict, cfl: float = 0.5) -> float:
    """cfl_limited_timestep (numerical_grids_and_timestep.py:498-560): dt = CFL min over ALL points of
    min(|dr/dxx0| dxx0, |r| dxx1, |r sin(xx1)| dxx2)."""
    x0, x1 = p["xx"][0], p["xx"][1]
    r = r_of_xx0(p, x0)[None, :]
    ds0 = np.abs(p["dxx"][0] * dr_dxx0(p, x0))[None, :] * np.ones((len(x1), 1))
    ds1 = np.abs(p["dxx"][1] * r) * np.ones((len(x1), 1))
    ds2 = np.abs(p["dxx"][2] * r * np.sin(x1)[:, None])
    return cfl * float(min(ds0.min(), ds1.min(), ds2.min()))


# ------------------------------------------------------------------------ bcstruct
def _eigen_map(p: Dict, i0: int, i1: int, i2: int) -> Tuple[Tuple[int, int, int], Tuple[float, float, float]]:
    """EigenCoord_set_x0x1x2_inbounds__i0i1i2_inbounds_single_pt (bcstruct_set_up.py:195-440):
    (x0,x1,x2) -> Cartesian in the eigen-coordinate (Spherical, or Cylindrical for the
    cylindrical family: the xx values are taken as the eigen coordinates themselves) ->
    (x0,x1,x2)' -> nearest index."""
    xx = p["xx"]
    x0, x1, x2 = xx[0][i0], xx[1][i1], xx[2][i2]
    if p["coord"] == "SinhCylindrical":
        X, Y, Z = x0 * math.cos(x1), x0 * math.sin(x1), x2
        xin = (math.sqrt(X * X + Y * Y), math.atan2(Y, X), Z)
    else:
        t = x0 * math.sin(x1)
        X, Y, Z = t * math.cos(x2), t * math.sin(x2), x0 * math.cos(x1)
        r = math.sqrt(X * X + Y * Y + Z * Z)
        xin = (r, math.acos(Z / r), math.atan2(Y, X))
    idx = []
    for d in range(3):
        dx = p["dxx"][d]
        xmin = xx[d][0] - ((0 - NGHOSTS) + 0.5) * dx
        idx.append(int((xin[d] - xmin - 0.5 * dx + NGHOSTS * dx) / dx + 0.5))
    return tuple(idx), tuple(xx[d][idx[d]] for d in range(3))


def _parity(x1: float, x2: float, xin, coord: str = "Spherical") -> List[int]:
    """set_parity_for_inner_boundary_single_pt (bcstruct_set_up.py:38-190): unit-vector dot products
    of the point and its source, in the eigen basis (Spherical; Cylindrical: rho-hat and phi-hat
    turn with the phi difference, z-hat does not)."""
    if coord == "SinhCylindrical":
        t = math.sin(x1) * math.sin(xin[1]) + math.cos(x1) * math.cos(xin[1])
        vals = [1.0, t, t, 1.0, t * t, t * t, t, t * t, t, 1.0]
        for v in vals:
            if abs(v) < 1 - 1e-8 or abs(v) > 1 + 1e-8:
                raise ValueError(f"parity {v} not +/-1")
        return [-1 if v < 0 else 1 for v in vals]
    y1, y2 = xin[1], xin[2]
    a = math.cos(x1) * math.cos(y1)
    b = math.sin(x1) * math.sin(y1)
    c = math.sin(x2) * math.sin(y2)
    d = math.cos(x2) * math.cos(y2)
    p1 = a + b * c + b * d
    p2 = a * c + a * d + b
    p3 = c + d
    vals = [1.0, p1, p2, p3, p1 * p1, p1 * p2, p1 * p3, p2 * p2, p2 * p3, p3 * p3]
    for v in vals:
        if abs(v) < 1 - 1e-8 or abs(v) > 1 + 1e-8:
            raise ValueError(f"parity {v} not +/-1")
    return [-1 if v < 0 else 1 for v in vals]


def bcstruct(p: Dict):
    """bcstruct_set_up (bcstruct_set_up.py:442-792): inner points in i2-i1-i0 order with their source
    point and 10 parity signs; pure outer points per (ghost layer, face direction), inside out."""
    N0, N1, N2 = p["N"]
    inner = []
    for i2 in range(N2):
        for i1 in range(N1):
            for i0 in range(N0):
                if NGHOSTS <= i0 < N0 - NGHOSTS and NGHOSTS <= i1 < N1 - NGHOSTS and NGHOSTS <= i2 < N2 - NGHOSTS:
                    continue
                (j0, j1, j2), xin = _eigen_map(p, i0, i1, i2)
                if (j0, j1, j2) == (i0, i1, i2):
                    continue
                inner.append((i0 + N0 * (i1 + N1 * i2), j0 + N0 * (j1 + N1 * j2),
                              _parity(p["xx"][1][i1], p["xx"][2][i2], xin, p["coord"])))
    imin = [NGHOSTS] * 3
    imax = [N0 - NGHOSTS, N1 - NGHOSTS, N2 - NGHOSTS]
    bounds = []
    for _gz in range(NGHOSTS):
        faces = []
        faces.append((imin[0] - 1, imin[0], imin[1], imax[1], imin[2], imax[2]))
        imin[0] -= 1
        faces.append((imax[0], imax[0] + 1, imin[1], imax[1], imin[2], imax[2]))
        imax[0] += 1
        faces.append((imin[0], imax[0], imin[1] - 1, imin[1], imin[2], imax[2]))
        imin[1] -= 1
        faces.append((imin[0], imax[0], imax[1], imax[1] + 1, imin[2], imax[2]))
        imax[1] += 1
        faces.append((imin[0], imax[0], imin[1], imax[1], imin[2] - 1, imin[2]))
        imin[2] -= 1
        faces.append((imin[0], imax[0], imin[1], imax[1], imax[2], imax[2] + 1))
        imax[2] += 1
        bounds.append(faces)
    outer = {}
    for gz in range(NGHOSTS):
        for dirn in range(3):
            pts = []
            for face in (2 * dirn, 2 * dirn + 1):
                f = ((face == 0) - (face == 1), (face == 2) - (face == 3), (face == 4) - (face == 5))
                b = bounds[gz][face]
                for i2 in range(b[4], b[5]):
                    for i1 in range(b[2], b[3]):
                        for i0 in range(b[0], b[1]):
                            if _eigen_map(p, i0, i1, i2)[0] == (i0, i1, i2):
                                pts.append((i0, i1, i2) + f)
            outer[(gz, dirn)] = np.array(pts, dtype=np.int16).reshape(-1, 6)
    return inner, outer


# ------------------------------------------------------------------------ boundary conditions
def apply_inner(gfs: np.ndarray, inner, ntot: int, ngfs: int = 24) -> None:
    """apply_bcs_inner_only.py:26-199: gf[dst] = parity * gf[src]."""
    g = gfs.reshape(ngfs, ntot)
    for dst, src, par in inner:
        for k in range(ngfs):
            g[k, dst] = g[k, src] * par[EVOL_GF_PARITY[k]]


def apply_extrap(gfs: np.ndarray, outer, N, ngfs: int = 24) -> None:
    """apply_bcs_outerextrap_and_inner.py:28-157: f0 = 3 f1 - 3 f2 + f3 along the inward normal."""
    g = gfs.reshape(ngfs, N[2], N[1], N[0])
    for gz in range(NGHOSTS):
        for dirn in range(3):
            for i0, i1, i2, f0, f1, f2 in outer[(gz, dirn)]:
                for k in range(ngfs):
                    v = [g[k, i2 + m * f2, i1 + m * f1, i0 + m * f0] for m in range(4)]
                    g[k, i2, i1, i0] = 3.0 * v[1] - 3.0 * v[2] + 1.0 * v[3]


_FD1 = {  # FD1_arbitrary_upwind_x0_dirn (apply_bcs_outerradiation_and_inner.py:122-278), 4th order
    0: {-2: 1 / 12, -1: -2 / 3, 1: 2 / 3, 2: -1 / 12},
    1: {-1: -1 / 4, 0: -5 / 6, 1: 3 / 2, 2: -1 / 2, 3: 1 / 12},
    -1: {-3: -1 / 12, -2: 1 / 2, -1: -3 / 2, 0: 5 / 6, 1: 1 / 4},
    2: {0: -25 / 12, 1: 4.0, 2: -3.0, 3: 4 / 3, 4: -1 / 4},
    -2: {-4: 1 / 4, -3: -4 / 3, -2: 3.0, -1: -4.0, 0: 25 / 12},
}


def apply_radiation(p: Dict, gfs: np.ndarray, rhs: np.ndarray, outer) -> None:
    """apply_bcs_outerradiation_and_inner.py:366-460: at pure outer points
    rhs = -c (d_r f + (f - f_inf)/r) + k / r^3 with k = r_int^3 (rhs_int - outgoing_int)."""
    N = p["N"]
    f = gfs.reshape(24, N[2], N[1], N[0])
    r_ = rhs.reshape(24, N[2], N[1], N[0])
    x0 = p["xx"][0]

    def dfdr(k, i0, i1, i2, face):
        off = face
        if i0 < 2:
            off = 2 - i0
        elif i0 > N[0] - 3:
            off = (N[0] - 3) - i0
        d = sum(w * f[k, i2, i1, i0 + s] for s, w in _FD1[off].items()) * p["invdxx"][0]
        return float(d) / float(dr_dxx0(p, x0[i0]))

    for gz in range(NGHOSTS):
        for dirn in range(3):
            for i0, i1, i2, f0, f1, f2 in outer[(gz, dirn)]:
                if dirn != 0:
                    raise ValueError("outer points off the x0 face")
                j0, j1, j2 = i0 + f0, i1 + f1, i2 + f2
                r = float(r_of_xx0(p, x0[i0]))
                ri = float(r_of_xx0(p, x0[j0]))
                for k in range(24):
                    c, fi = WAVESPEED[k], F_INFINITY[k]
                    out_int = -c * (dfdr(k, j0, j1, j2, f0) + (f[k, j2, j1, j0] - fi) / ri)
                    kk = ri ** 3 * (r_[k, j2, j1, j0] - out_int)
                    r_[k, i2, i1, i0] = -c * (dfdr(k, i0, i1, i2, f0) + (f[k, i2, i1, i0] - fi) / r) + kk / r ** 3


# ------------------------------------------------------------------------ RK4, diagnostics, initial data
def rk4_step(y: np.ndarray, rhs_fn, dt: float) -> np.ndarray:
    """Classic RK4 in the low-storage form of MoL_step_forward_in_time.py:322-485 (k_odd/k_even,
    running total), with rhs_fn(state) -> d state/dt."""
    k = rhs_fn(y)
    run = dt / 6 * k
    s = y + dt / 2 * k
    k = rhs_fn(s)
    run = dt / 3 * k + run
    s = y + dt / 2 * k
    k = rhs_fn(s)
    run = dt / 3 * k + run
    s = y + dt * k
    k = rhs_fn(s)
    return dt / 6 * k + y + run


def volume_integrals(p: Dict, diag3: np.ndarray) -> np.ndarray:
    """diagnostics_volume_integration_helpers.h:400-470: sum over the interior of f^2 dV (f = H, M^2,
    |Lambda|) and sum dV, dV = sqrt(det gammahat) |dxx0 dxx1 dxx2|."""
    N = p["N"]
    G = NGHOSTS
    x0 = p["xx"][0][G:-G]
    x1 = p["xx"][1][G:-G]
    r = r_of_xx0(p, x0)
    sq = np.abs(dr_dxx0(p, x0)[None, None, :] * (r * r)[None, None, :] * np.sin(x1)[None, :, None])
    dV = sq * abs(p["dxx"][0] * p["dxx"][1] * p["dxx"][2]) * np.ones((N[2] - 2 * G, 1, 1))
    d = diag3.reshape(3, N[2], N[1], N[0])[:, G:-G, G:-G, G:-G]
    return np.array([(d[k] ** 2 * dV).sum() for k in range(3)] + [dV.sum()])


def brill_lindquist_alpha_cf(p: Dict, m1: float, z1: float, m2: float, z2: float):
    """InitialData_Cartesian.py:111-141 with the ADM->BSSN converter: alpha = cf = psi^-2,
    psi = 1 + m1/(2|x-x1|) + m2/(2|x-x2|)."""
    x0, x1, x2 = p["xx"]
    r = r_of_xx0(p, x0)[None, None, :]
    X = r * np.sin(x1)[None, :, None] * np.cos(x2)[:, None, None]
    Y = r * np.sin(x1)[None, :, None] * np.sin(x2)[:, None, None]
    Z = r * np.cos(x1)[None, :, None] * np.ones((len(x2), 1, 1))
    psi = 1 + 0.5 * m1 / np.sqrt(X**2 + Y**2 + (Z - z1) ** 2) + 0.5 * m2 / np.sqrt(X**2 + Y**2 + (Z - z2) ** 2)
    return psi**-2, psi**-2
