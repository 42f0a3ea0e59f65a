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
