"""Synthetic inputs: the modified Shepp-Logan ellipsoid table and seeded random ellipsoids.

The table is read from ``data/modified_shepp_logan.txt`` (extracted from TomoGPI's
Data3D_0256/phantom3d.m by ``data/make_shepp_logan_table.py``). Ellipsoid rows use the
phantom3d.m convention: A, a, b, c, x0, y0, z0 on the [-1, 1]^3 grid, Euler angles
phi, theta, psi in degrees.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

_TABLE = Path(__file__).resolve().parent / "data" / "modified_shepp_logan.txt"


def modified_shepp_logan() -> np.ndarray:
    return np.loadtxt(_TABLE, comments="#", dtype=np.float64).reshape(-1, 10)


def random_ellipsoids(seed: int, count: int, n: int) -> np.ndarray:
    """``count`` seeded ellipsoids for an n^3 volume: centres uniform in the inscribed
    cylinder (the field of view), semi-axes uniform in [0.05, 0.3]*n voxels, intensities
    uniform in (-0.2, 0.2), Euler angles uniform in [0, 360) degrees."""
    rng = np.random.default_rng(seed)
    half = (n - 1) / 2.0
    out = np.zeros((count, 10), np.float64)
    for i in range(count):
        r = np.sqrt(rng.uniform(0.0, 1.0))
        t = rng.uniform(0.0, 2.0 * np.pi)
        out[i, 0] = rng.uniform(-0.2, 0.2)
        out[i, 1:4] = rng.uniform(0.05, 0.3, size=3) * n / half
        out[i, 4] = r * np.cos(t)
        out[i, 5] = r * np.sin(t)
        out[i, 6] = rng.uniform(-1.0, 1.0)
        out[i, 7:10] = rng.uniform(0.0, 360.0, size=3)
    return out


def config_phantom(seed: int, n: int, extra: int = 5) -> np.ndarray:
    """Shepp-Logan plus ``extra`` random ellipsoids (the iterative benchmark's phantom)."""
    return np.concatenate([modified_shepp_logan(), random_ellipsoids(seed, extra, n)], axis=0)
