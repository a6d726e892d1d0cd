"""Per-cell shape measures shared by the long-horizon fixtures and tests.

perimeter: sum over the grid of |grad phi_n| dx, with the central differences
0.5 (phi[i+1] - phi[i-1]) on the periodic grid.  rho_mass: sum of rho_n dx^2.
Both are float64 sums of the stored fields, identical for every path that
stores the same state.
"""
from __future__ import annotations

import numpy as np


def perimeter(phi, dx: float) -> np.ndarray:
    phi = np.asarray(phi, np.float64)
    gi = 0.5 * (np.roll(phi, -1, axis=1) - np.roll(phi, 1, axis=1))
    gj = 0.5 * (np.roll(phi, -1, axis=2) - np.roll(phi, 1, axis=2))
    return np.sqrt(gi * gi + gj * gj).sum(axis=(1, 2)) * dx


def rho_mass(rho, dx: float) -> np.ndarray:
    return np.asarray(rho, np.float64).sum(axis=(1, 2)) * dx * dx


def rel(a, b, mask=None) -> float:
    """max |a - b| / max |b| (over `mask` when given)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    if not b.size:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-300))


def rel_each(a, b) -> float:
    """max over entries of |a - b| / |b|."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))
