"""The hand-written discrete adjoint against finite differences (B200).

* each link of the chain separately, by dot-product tests against central differences of
  the forward on the same inputs: the initial-data transpose (Brill-Lindquist psi^-2 through
  the extrapolation and parity BCs), the functional J(y) = sum H^2 + alpha(centre), and one
  stage-by-stage RK4 step (Ricci, RHS, radiation and parity BCs, RK update, detgammabar
  projection) at a smoothly perturbed state where every RHS term is active;
* the whole gradient dJ/d(m1, z1, m2, z2) through a short evolution with checkpoints
  against central differences (h = 1e-6) of the forward, to 1e-6 relative.
The full-size case (Spherical 128x32x32, 200 steps) is in test_adjoint_full_gpu.py.
"""

import numpy as np
import pytest
import torch

from tests.util import smooth_fields

pytestmark = pytest.mark.gpu

THETA = (0.45, 0.4, 0.55, -0.35)
NXX = (16, 8, 8)


@pytest.fixture(scope="module")
def problem(cuda):
    from nrpy_b200.adjoint import BLGradient

    p = BLGradient(Nxx=NXX, grid_physical_size=7.5, nsteps=10, checkpoint_every=4, theta=THETA)
    yield p
    p.close()


def perturbed(problem, seed=3, amp=0.05):
    """Initial data of THETA plus smooth perturbations of all 24 gridfunctions."""
    g = problem.grid
    problem.set_theta(THETA)
    pert = smooth_fields(g.xx(), seed, amp)
    y = g.view(g.y_n.clone()).cpu().numpy()
    for gf in range(24):
        if gf in (6, 10):
            y[gf] *= 1.0 + pert[gf]
        else:
            y[gf] += pert[gf]
    return torch.from_numpy(y.reshape(-1)).to(g.device)


def central(f, x, u, eps):
    return (f(x + eps * u) - f(x - eps * u)) / (2 * eps)


def test_id_transpose(problem):
    g = problem.grid
    w = torch.randn(g.y_n.numel(), dtype=torch.float64, device=g.device, generator=torch.Generator(g.device).manual_seed(1))

    def J0(theta):
        problem.set_theta(theta)
        torch.cuda.synchronize()
        return float(torch.dot(w, g.y_n))

    problem.set_theta(THETA)
    grad = problem.id_vjp(w)
    h = 1e-6
    for k in range(4):
        tp, tm = list(THETA), list(THETA)
        tp[k] += h
        tm[k] -= h
        fd = (J0(tp) - J0(tm)) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-7 * max(abs(fd), 1e-300), (k, grad[k], fd)


def test_functional_transpose(problem):
    g = problem.grid
    y = perturbed(problem)
    u = torch.from_numpy(smooth_fields(g.xx(), 11, 1.0).reshape(-1)).to(g.device)
    ybar = problem.functional_vjp(y, 1.0)
    lhs = float(torch.dot(ybar, u))
    rhs = central(lambda z: problem.functional(z)["J"], y, u, 1e-6)
    assert abs(lhs - rhs) <= 1e-6 * abs(rhs), (lhs, rhs)


def test_step_transpose(problem):
    """<v, dF u> (central differences of the stage-by-stage step) == <dF^T v, u>."""
    g = problem.grid
    y = perturbed(problem, seed=5)
    u = torch.from_numpy(smooth_fields(g.xx(), 12, 1.0).reshape(-1)).to(g.device)
    v = torch.randn(y.numel(), dtype=torch.float64, device=g.device, generator=torch.Generator(g.device).manual_seed(2))

    def F(z):
        g.y_n.copy_(z)
        g.MoL_step_forward_in_time(mode=0)
        torch.cuda.synchronize()
        return g.y_n.clone()

    dFu = central(F, y, u, 1e-6)
    lhs = float(torch.dot(v, dFu))
    rhs = float(torch.dot(problem.step_vjp(y, v), u))
    assert abs(lhs - rhs) <= 1e-6 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_gradient_vs_central_differences(problem):
    J, grad = problem.value_and_grad(THETA)
    assert np.isfinite(J) and np.all(np.isfinite(grad))
    h = 1e-6
    for k in range(4):
        tp, tm = list(THETA), list(THETA)
        tp[k] += h
        tm[k] -= h
        fd = (problem.forward(tp)["J"] - problem.forward(tm)["J"]) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * abs(fd), (k, grad[k], fd)


def test_autograd_function(problem):
    from nrpy_b200.adjoint import bl_functional

    theta = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    J = bl_functional(theta, problem)
    J.backward()
    _, grad = problem.value_and_grad(THETA)
    np.testing.assert_allclose(theta.grad.numpy(), grad, rtol=1e-12)
