"""CPU tests: pin the oracle before trusting it.

* the numpy restatement (oracle/bssn_port.py) against the golden fixtures made from the
  reference's own generated C: grid, timestep, bcstruct maps (bit-exact), inner /
  extrapolation / radiation BCs, volume integrals, Brill-Lindquist lapse and conformal
  factor;
* the reference oracle itself (oracle/_ref, when built) against the committed fixtures,
  bit-exactly, so that the fixtures and the live oracle are the same reference;
* the codegen's finite-difference weights against the reference's coefficient tables
  (tests/golden/fd_coeffs.json, written from nrpy by tests/golden/make_fd_coeffs.py).
"""

import json

import numpy as np
import pytest

from oracle import bssn_port as port
from tests.util import GOLDEN, as4, interior, load_golden

CASES = {
    "sphaxi_16x6x2": ("Spherical", "sphaxi"),
    "sph3d_10x6x6": ("Spherical", "sph3d"),
    "sinh3d_10x6x6": ("SinhSpherical", "sinh3d"),
}


def params(name):
    g = load_golden(name)
    coord = CASES[name][0]
    return g, port.grid_params(coord, tuple(int(x) for x in g["Nxx"]), float(g["grid_physical_size"]),
                               float(g["SINHW"]))


@pytest.mark.parametrize("name", list(CASES))
def test_port_grid_and_dt(name):
    g, p = params(name)
    assert tuple(p["N"]) == tuple(int(x) for x in g["N"])
    for d in range(3):
        np.testing.assert_allclose(p["xx"][d], g[f"xx{d}"], rtol=0, atol=4e-16 * max(1.0, abs(g[f"xx{d}"]).max()))
    np.testing.assert_allclose(port.cfl_dt(p), float(g["dt"]), rtol=1e-14)


@pytest.mark.parametrize("name", list(CASES))
def test_port_bcstruct_bit_exact(name):
    g, p = params(name)
    # Use the reference's own xx so that only the algorithm is compared.
    p["xx"] = [g["xx0"], g["xx1"], g["xx2"]]
    inner, outer = port.bcstruct(p)
    assert [i[0] for i in inner] == list(g["inner_dst"])
    assert [i[1] for i in inner] == list(g["inner_src"])
    assert np.array_equal(np.array([i[2] for i in inner], dtype=np.int8), g["inner_parity"])
    for gz in range(3):
        for d in range(3):
            assert np.array_equal(outer[(gz, d)], g[f"outer_{gz}_{d}"])


@pytest.mark.parametrize("name", list(CASES))
def test_port_radiation_and_inner_bcs(name):
    g, p = params(name)
    p["xx"] = [g["xx0"], g["xx1"], g["xx2"]]
    inner, outer = port.bcstruct(p)
    N = p["N"]
    ntot = N[0] * N[1] * N[2]
    rhs = as4(g["rhs_bc"], N).copy()
    mask = np.zeros_like(rhs, dtype=bool)
    mask[:, 3:-3, 3:-3, 3:-3] = True
    rhs[~mask] = 0.0  # keep only the interior RHS, rebuild every ghost value
    rhs = np.ascontiguousarray(rhs.reshape(-1))
    port.apply_radiation(p, g["input"].copy(), rhs, outer)
    port.apply_inner(rhs, inner, ntot)
    ref = g["rhs_bc"]
    np.testing.assert_allclose(rhs, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", list(CASES))
def test_port_extrapolation_bcs(name):
    g, p = params(name)
    p["xx"] = [g["xx0"], g["xx1"], g["xx2"]]
    inner, outer = port.bcstruct(p)
    N = p["N"]
    ntot = N[0] * N[1] * N[2]
    y = g["input"].copy()  # input was made with the reference's extrapolation + inner BCs
    y4 = as4(y, N)
    keep = y4[:, 3:-3, 3:-3, 3:-3].copy()
    y4[:] = 0.0
    y4[:, 3:-3, 3:-3, 3:-3] = keep
    port.apply_extrap(y, outer, N)
    port.apply_inner(y, inner, ntot)
    np.testing.assert_allclose(y, g["input"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("name", list(CASES))
def test_port_volume_integrals(name):
    g, p = params(name)
    p["xx"] = [g["xx0"], g["xx1"], g["xx2"]]
    vals = port.volume_integrals(p, g["constraints"])
    dV = interior(as4(g["dV"], p["N"]))[0]
    cons = interior(as4(g["constraints"], p["N"]))
    ref = [(cons[k] ** 2 * dV).sum() for k in range(3)] + [dV.sum()]
    np.testing.assert_allclose(vals, ref, rtol=1e-12)


@pytest.mark.parametrize("name", list(CASES))
def test_port_brill_lindquist(name):
    g, p = params(name)
    p["xx"] = [g["xx0"], g["xx1"], g["xx2"]]
    m1, z1, m2, z2 = [float(x) for x in g["bh"]]
    alpha, cf = port.brill_lindquist_alpha_cf(p, m1, z1, m2, z2)
    y = as4(g["initial_data"], p["N"])
    # ghost values come from BCs in the reference; compare the interior
    np.testing.assert_allclose(alpha[3:-3, 3:-3, 3:-3], y[6][3:-3, 3:-3, 3:-3], rtol=1e-13)
    np.testing.assert_allclose(cf[3:-3, 3:-3, 3:-3], y[10][3:-3, 3:-3, 3:-3], rtol=1e-13)


def test_port_rk4_exact_on_linear_ode():
    """The low-storage RK4 of the port reproduces exp(dt*lambda) to 4th order."""
    lam = -1.7
    y = np.array([1.0])
    dt = 0.05
    y1 = port.rk4_step(y, lambda s: lam * s, dt)
    z = lam * dt
    assert abs(y1[0] - (1 + z + z**2 / 2 + z**3 / 6 + z**4 / 24)) < 1e-15


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_reproduces_fixtures(name):
    """The live reference oracle (if built here) regenerates the committed fixture bit-exactly."""
    from oracle import ref

    variant = CASES[name][1]
    if not ref.available(variant):
        pytest.skip("oracle/_ref not built")
    g = load_golden(name)
    m1, z1, m2, z2 = [float(x) for x in g["bh"]]
    rg = ref.RefGrid(variant, tuple(int(x) for x in g["Nxx"]), float(g["grid_physical_size"]),
                     SINHW=float(g["SINHW"]), BH1_mass=m1, BH1_posn_z=z1, BH2_mass=m2, BH2_posn_z=z2)
    assert np.array_equal(rg.y_n(), g["initial_data"])
    inp = ref.perturbed_state(rg, seed=int(g["seed"]))
    assert np.array_equal(inp, g["input"])
    ricci = rg.ricci(inp)
    # The reference's SIMD loop runs past the last interior point of a row when Nxx0 is not a
    # multiple of the vector width and leaves run-dependent values in the next row's ghost
    # cells; only the interior is defined.
    assert np.array_equal(interior(as4(ricci, rg.N)), interior(as4(g["ricci"], rg.N)))
    ricci = g["ricci"].copy()
    rhs = rg.rhs(ricci, inp)
    rg.bc_radiation(inp.copy(), rhs)
    assert np.array_equal(rhs, g["rhs_bc"])
    rg.close()


def test_fd_weights_match_reference_tables():
    """Codegen FD weights == nrpy.finite_difference.compute_fdcoeffs_fdstencl (fixture)."""
    from nrpy_b200.codegen import fdcoeffs as f

    tab = json.loads((GOLDEN / "fd_coeffs.json").read_text())

    def as_dict(entry):
        return {tuple(k): v for k, v in zip(entry["stencil"], entry["coeffs"])}

    def mine(weights, d):
        out = {}
        for s, w in weights.items():
            st = [0, 0, 0]
            st[d] = s
            out[tuple(st)] = float(w)
        return out

    for d in range(3):
        for name, w in [(f"dD{d}", f.first_centred()), (f"dupD{d}", f.upwind(+1)), (f"ddnD{d}", f.upwind(-1)),
                        (f"dKOD{d}", f.kreiss_oliger()), (f"dDD{d}{d}", f.second_centred())]:
            ref = as_dict(tab[name])
            got = mine(w, d)
            assert set(ref) == set(got), name
            for k in ref:
                assert abs(ref[k] - got[k]) < 1e-15, (name, k)
