"""Adjoint gradient of the full-size differentiation workload (B200).

Spherical 128x32x32 (grid_physical_size 7.5), 200 FP64 RK4 steps, checkpoints every 20,
J = sum over the interior of H^2 + alpha at the grid centre point, theta = (m1, z1, m2, z2)
from default_rng(2024). The adjoint gradient must match, to 1e-6 relative per component,
* central differences (h = 1e-6) of this library's forward, and
* central differences (h = 1e-6) of the reference's own generated C forward (the oracle:
  its initial data, 200 RK4 steps and constraint evaluation), when oracle/_ref is built.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = 1e-6


@pytest.fixture(scope="module")
def workload(cuda):
    from nrpy_b200.adjoint import BLGradient, differentiation_workload

    w = differentiation_workload()
    p = BLGradient(Nxx=w["Nxx"], grid_physical_size=w["grid_physical_size"], nsteps=w["nsteps"],
                   checkpoint_every=w["checkpoint_every"], theta=w["theta"])
    J, grad = p.value_and_grad(w["theta"])
    yield w, p, J, grad
    p.close()


def fd_gradient(f, theta):
    out = []
    for k in range(4):
        tp, tm = list(theta), list(theta)
        tp[k] += H
        tm[k] -= H
        out.append((f(tp) - f(tm)) / (2 * H))
    return np.array(out)


def test_adjoint_vs_own_forward(workload):
    w, p, J, grad = workload
    fd = fd_gradient(lambda t: p.forward(t)["J"], w["theta"])
    print("\nJ", J, "adjoint", grad, "own FD", fd, "rel", np.abs(grad - fd) / np.abs(fd))
    np.testing.assert_allclose(grad, fd, rtol=1e-6, atol=0)


def reference_J(theta, w):
    from oracle import ref

    m1, z1, m2, z2 = theta
    rg = ref.RefGrid("sph3d", w["Nxx"], w["grid_physical_size"], BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2,
                     BH2_posn_z=z2)
    rg.step(w["nsteps"])
    y = rg.y_n()
    Hc = rg.constraints(y, rg.ricci(y))[0].reshape(rg.N[2], rg.N[1], rg.N[0])
    G = 3
    alpha = y.reshape(24, rg.N[2], rg.N[1], rg.N[0])[6, rg.N[2] // 2, rg.N[1] // 2, G]
    rg.close()
    return float((Hc[G:-G, G:-G, G:-G] ** 2).sum() + alpha)


def test_adjoint_vs_reference_forward(workload):
    from oracle import ref

    if not ref.available("sph3d"):
        pytest.skip("oracle/_ref not built")
    w, p, J, grad = workload
    J_ref = reference_J(w["theta"], w)
    fd = fd_gradient(lambda t: reference_J(t, w), w["theta"])
    print("\nJ", J, "J_ref", J_ref, "adjoint", grad, "reference FD", fd, "rel", np.abs(grad - fd) / np.abs(fd))
    assert abs(J_ref - J) <= 1e-7 * abs(J)
    np.testing.assert_allclose(grad, fd, rtol=1e-6, atol=0)
