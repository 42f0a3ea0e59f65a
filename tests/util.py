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
