"""Gradients of an evolved-state functional with respect to Brill-Lindquist parameters.

The functional (one Spherical grid, no symmetry axes, radiation outer BCs):

    J(theta) = sum over interior points of H^2  +  alpha(NGHOSTS, N1/2, N2/2)

evaluated after ``nsteps`` FP64 RK4 steps from Brill-Lindquist initial data with
theta = (BH1_mass, BH1_posn_z, BH2_mass, BH2_posn_z). The lapse term is taken at the grid
point the reference's diagnostics call the grid centre (i0 = NGHOSTS, i1 = N1/2,
i2 = N2/2, diagnostics_nearest_grid_center.py:56-68); a cell-centred grid has no point at
r = 0.

``BLGradient`` drives libbssn_b200's hand-written discrete adjoint: the forward keeps the
state every ``checkpoint_every`` steps; the backward recomputes each segment from its
checkpoint and runs the reverse of each RK4 step (stage-by-stage step, generated VJPs of
the Ricci / RHS / H / projection algebra, stencil transposes, boundary-condition
transposes) down to the initial data, where the Brill-Lindquist derivatives of
alpha = W = psi^-2 give dJ/dtheta. ``BLFunctional`` wraps it as a torch.autograd.Function.
"""

import ctypes as C
from typing import Dict, Optional, Sequence, Tuple

import numpy as np
import torch

from . import lib as L
from .grid import BSSNGrid, _ptr

THETA_NAMES = ("BH1_mass", "BH1_posn_z", "BH2_mass", "BH2_posn_z")


class BLGradient:
    """One grid plus the adjoint's tape; forward() / backward() as in reverse-mode AD."""

    def __init__(self, Nxx: Sequence[int] = (128, 32, 32), grid_physical_size: float = 7.5, nsteps: int = 200,
                 checkpoint_every: int = 20, CFL_FACTOR: float = 0.5, eta: float = 1.0,
                 theta: Sequence[float] = (0.5, 0.5, 0.5, -0.5), device: Optional[torch.device] = None):
        m1, z1, m2, z2 = [float(x) for x in theta]
        self.grid = BSSNGrid("Spherical", tuple(Nxx), grid_physical_size=grid_physical_size, BH1_mass=m1,
                             BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2, CFL_FACTOR=CFL_FACTOR, eta=eta,
                             outer_bc_type="radiation", symmetry_axes="", initial_data=False, device=device)
        self.lib = self.grid.lib
        self.nsteps, self.checkpoint_every = nsteps, checkpoint_every
        h = C.c_void_p()
        L.check(self.lib.bssn_b200_adjoint_create(C.byref(self.grid.cd), self.grid.gd, nsteps, checkpoint_every,
                                                  self.grid.stream, C.byref(h)))
        self._h = h
        self.theta = tuple(float(x) for x in theta)

    # ---------------------------------------------------------------- set-up
    def set_theta(self, theta: Sequence[float]) -> None:
        """Brill-Lindquist initial data for theta = (m1, z1, m2, z2) into y_n; time reset to 0."""
        cd = self.grid.cd
        cd.BH1_mass, cd.BH1_posn_z, cd.BH2_mass, cd.BH2_posn_z = [float(x) for x in theta]
        cd.time = cd.t_0 = 0.0
        cd.nn = cd.nn_0 = 0
        torch.cuda.synchronize(self.grid.device)
        self.lib.initial_data(C.byref(cd), self.grid.gd)
        self.theta = tuple(float(x) for x in theta)

    # ---------------------------------------------------------------- reverse mode
    def forward(self, theta: Optional[Sequence[float]] = None) -> Dict[str, float]:
        """J after nsteps steps from the initial data of theta (default: the current theta)."""
        self.set_theta(self.theta if theta is None else theta)
        out = (C.c_double * 3)()
        L.check(self.lib.bssn_b200_adjoint_forward(self._h, out))
        return {"J": out[0], "sum_H2": out[1], "alpha_center": out[2]}

    def backward(self, Jbar: float = 1.0, ybar0: Optional[torch.Tensor] = None) -> np.ndarray:
        """Jbar * dJ/dtheta (order BH1_mass, BH1_posn_z, BH2_mass, BH2_posn_z) for the last forward."""
        g = (C.c_double * 4)()
        L.check(self.lib.bssn_b200_adjoint_backward(self._h, float(Jbar),
                                                    _ptr(ybar0) if ybar0 is not None else None, g))
        return np.array(g[:], dtype=np.float64)

    def value_and_grad(self, theta: Sequence[float]) -> Tuple[float, np.ndarray]:
        J = self.forward(theta)["J"]
        return J, self.backward(1.0)

    # ---------------------------------------------------------------- pieces (tests)
    def functional(self, y: torch.Tensor) -> Dict[str, float]:
        out = (C.c_double * 3)()
        L.check(self.lib.bssn_b200_adjoint_functional(self._h, _ptr(y), out))
        return {"J": out[0], "sum_H2": out[1], "alpha_center": out[2]}

    def functional_vjp(self, y: torch.Tensor, Jbar: float = 1.0) -> torch.Tensor:
        ybar = torch.empty_like(y)
        L.check(self.lib.bssn_b200_adjoint_functional_vjp(self._h, _ptr(y), float(Jbar), _ptr(ybar)))
        return ybar

    def step_vjp(self, y_n: torch.Tensor, ybar_next: torch.Tensor) -> torch.Tensor:
        """(dF/dy)^T ybar_next for one stage-by-stage RK4 step F at y_n (overwrites y_n_gfs)."""
        ybar = ybar_next.clone()
        L.check(self.lib.bssn_b200_adjoint_step_vjp(self._h, _ptr(y_n), _ptr(ybar)))
        return ybar

    def id_vjp(self, ybar0: torch.Tensor) -> np.ndarray:
        g = (C.c_double * 4)()
        L.check(self.lib.bssn_b200_adjoint_id_vjp(self._h, _ptr(ybar0), g))
        return np.array(g[:], dtype=np.float64)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None:
            self.lib.bssn_b200_adjoint_destroy(self._h)
            self._h = None
        self.grid.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BLFunctional(torch.autograd.Function):
    """J(theta) with theta = (m1, z1, m2, z2) as a float64 tensor; backward by the adjoint."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, problem: BLGradient) -> torch.Tensor:
        vals = problem.forward(theta.detach().cpu().double().tolist())
        ctx.problem = problem
        return torch.tensor(vals["J"], dtype=torch.float64, device=theta.device)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        g = ctx.problem.backward(float(gJ))
        return torch.tensor(g, dtype=torch.float64, device=gJ.device), None


def bl_functional(theta: torch.Tensor, problem: BLGradient) -> torch.Tensor:
    return BLFunctional.apply(theta, problem)


def differentiation_workload(seed: int = 2024) -> Dict:
    """Spherical 128x32x32, grid_physical_size 7.5, 200 RK4 steps, checkpoints every 20;
    theta drawn from default_rng(seed): m_i ~ U[0.3,0.7], z1 = +U[0.3,0.8], z2 = -U[0.3,0.8]."""
    rng = np.random.default_rng(seed)
    m1, m2 = rng.uniform(0.3, 0.7, 2)
    z1, z2 = rng.uniform(0.3, 0.8), -rng.uniform(0.3, 0.8)
    return dict(Nxx=(128, 32, 32), grid_physical_size=7.5, nsteps=200, checkpoint_every=20,
                theta=(float(m1), float(z1), float(m2), float(z2)), seed=seed)


__all__ = ["BLGradient", "BLFunctional", "bl_functional", "differentiation_workload", "THETA_NAMES"]
