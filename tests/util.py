"""Shared helpers for the parity tests."""

import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
NG = 3


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


def as4(a: np.ndarray, N) -> np.ndarray:
    a = np.asarray(a)
    return a.reshape(-1, N[2], N[1], N[0])


def interior(a4: np.ndarray) -> np.ndarray:
    return a4[:, NG:-NG, NG:-NG, NG:-NG]


def rel_l2_per_gf(mine: np.ndarray, ref: np.ndarray, floor: float = 1e-300) -> np.ndarray:
    """Per-gridfunction ||mine - ref||_2 / ||ref||_2 over the given points."""
    m = mine.reshape(mine.shape[0], -1)
    r = ref.reshape(ref.shape[0], -1)
    num = np.sqrt(((m - r) ** 2).sum(axis=1))
    den = np.sqrt((r**2).sum(axis=1))
    return num / np.maximum(den, floor)


def smooth_fields(xx, seed: int, amp: float = 0.05, ngfs: int = 24) -> np.ndarray:
    """Seeded smooth fields sin(k0 pi x0/max x0 + p0) cos(k1 x1 + p1) cos(k2 x2 + p2), one per
    gridfunction, with amplitudes amp*U[0.5,1]; shape (ngfs, N2, N1, N0)."""
    rng = np.random.default_rng(seed)
    x0, x1, x2 = xx
    X0, X1, X2 = x0[None, None, :], x1[None, :, None], x2[:, None, None]
    x0max = max(abs(x0).max(), 1e-300)
    out = np.empty((ngfs, len(x2), len(x1), len(x0)))
    for gf in range(ngfs):
        k0, k1, k2 = rng.uniform(0.5, 2.0, 3)
        p0, p1, p2 = rng.uniform(0, 2 * np.pi, 3)
        a = amp * rng.uniform(0.5, 1.0)
        out[gf] = a * np.sin(k0 * np.pi * X0 / x0max + p0) * np.cos(k1 * X1 + p1) * np.cos(k2 * X2 + p2)
    return out


def read_diagnostics_file(path: pathlib.Path):
    """Comment lines and the numeric rows of one diagnostics output file."""
    comments, rows = [], []
    for line in path.read_text().splitlines():
        (comments if line.startswith("#") else rows).append(line)
    return comments, np.array([[float(x) for x in r.split()] for r in rows])


def compare_diagnostics_dirs(ref_dir: pathlib.Path, ours_dir: pathlib.Path) -> list:
    """The diagnostics() files of two runs: the same names and identical comment lines;
    coordinates to 1e-12, sampled values to 1e-9 of each column's largest magnitude, volume
    integrals (out3d) to 1e-10 relative. Returns the compared names."""
    names = sorted(p.name for p in ref_dir.iterdir())
    assert names and sorted(p.name for p in ours_dir.iterdir()) == names
    for name in names:
        c_ref, d_ref = read_diagnostics_file(ref_dir / name)
        c_ours, d_ours = read_diagnostics_file(ours_dir / name)
        assert c_ours == c_ref, name
        assert d_ours.shape == d_ref.shape, name
        if name.startswith("out3d"):
            np.testing.assert_allclose(d_ours, d_ref, rtol=1e-10, atol=0, err_msg=name)
            continue
        nc = 1 if name.startswith(("out0d", "out1d")) else 2
        np.testing.assert_allclose(d_ours[:, :nc], d_ref[:, :nc], rtol=1e-12, atol=1e-12, err_msg=name)
        scale = np.abs(d_ref[:, nc:]).max(axis=0)
        assert np.all(np.abs(d_ours[:, nc:] - d_ref[:, nc:]) <= 1e-9 * scale + 1e-300), name
    return names


# The SENR inner-boundary known-answer files (tests/golden/senr_kat.npz, made by
# tests/golden/make_senr_kat.py) list ten gridfunctions in SENR's order: vet^1..3, a_11, a_12,
# a_13, a_22, a_23, a_33, cf. Their parity types in the reference's numbering (0 scalar, 1-3
# vector components, 4-9 the symmetric rank-2 components 00, 01, 02, 11, 12, 22):
SENR_PARITY_TYPE = [1, 2, 3, 4, 5, 6, 7, 8, 9, 0]


def senr_kat_values(inner, ijk: np.ndarray, n: int = 10) -> np.ndarray:
    """The KAT's printed values predicted from an inner-boundary list of (dstpt, srcpt, parity[10])
    on an n^3 grid: gridfunction g at point p holds 1000 g + index(p), and after the inner BCs a
    ghost point holds parity[type(g)] * (1000 g + index(source))."""
    src = {int(d): (int(s), [int(x) for x in par]) for d, s, par in inner}
    out = np.empty((len(ijk), 10), dtype=np.int64)
    for row, (i, j, k) in enumerate(ijk):
        p = int(i) + n * (int(j) + n * int(k))
        s, par = src.get(p, (p, [1] * 10))
        for g in range(10):
            out[row, g] = par[SENR_PARITY_TYPE[g]] * (1000 * g + s)
    return out
