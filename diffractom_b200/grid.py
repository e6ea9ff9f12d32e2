"""Orientation grids: K rotation matrices (crystal -> sample) with a Gaussian kernel width sigma each.

The operator reads a grid through leaf_arrays() -> ((K, 3, 3) rotation matrices, (K,) sigmas), the interface of
diffractom's MatrixGrid (utils/grid.py:610-647). Grid.from_random_fundamental_zone follows diffractom's published
construction (utils/grid.py:295-378): uniformly random rotations, each replaced by the symmetry-equivalent
R g (g in the Laue group) closest to the identity (largest trace). diffractom's Grid (a tree of nodes) is accepted by
the operator as well (active_leaf_nodes / nodes).
"""
from __future__ import annotations

import numpy as np

from .material import rotation_group


def random_rotations(n: int, rng: np.random.Generator) -> np.ndarray:
    """(n, 3, 3) rotations uniform on SO(3): normalised 4-D Gaussian quaternions."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1)], 1)


def reduce_to_fundamental_zone(R: np.ndarray, symmetry: str) -> np.ndarray:
    """Every rotation R replaced by the R g of largest trace over the Laue group of `symmetry`."""
    G = rotation_group(symmetry)
    prod = np.einsum("nij,gjk->ngik", R, G)
    best = np.argmax(np.einsum("ngii->ng", prod), axis=1)
    return prod[np.arange(len(R)), best]


class MatrixGrid:
    """A single-level grid held as arrays."""

    def __init__(self, R_mats, sigma):
        R_mats = np.asarray(R_mats, dtype=np.float64)
        if R_mats.ndim != 3 or R_mats.shape[1:] != (3, 3):
            raise ValueError("R_mats must have shape (N, 3, 3)")
        self.matrices = R_mats
        self.sigmas = np.broadcast_to(np.asarray(sigma, dtype=np.float64), (len(R_mats),)).copy()
        self.sigma_levels = [float(self.sigmas[0])] if len(R_mats) else []

    def __len__(self):
        return len(self.matrices)

    def leaf_arrays(self):
        return self.matrices, self.sigmas

    def active_leaf_nodes(self):
        return range(len(self.matrices))


class Grid(MatrixGrid):
    """MatrixGrid with diffractom's constructors."""

    @classmethod
    def from_rotation_matrices(cls, R_mats, sigma):
        return cls(R_mats, sigma)

    @classmethod
    def from_random_fundamental_zone(cls, n_orientations: int, symmetry: str, sigma: float, seed=None):
        rng = np.random.default_rng(seed)
        return cls(reduce_to_fundamental_zone(random_rotations(int(n_orientations), rng), symmetry), sigma)


def grid_arrays(grid):
    """((K, 3, 3) float64 rotations, (K,) float32 sigmas) of this package's grids or of diffractom's Grid."""
    if hasattr(grid, "leaf_arrays"):
        mats, sig = grid.leaf_arrays()
        return np.asarray(mats, np.float64), np.asarray(sig, np.float32)
    nodes = [grid.nodes[i] for i in grid.active_leaf_nodes()]
    return (np.stack([n.R.as_matrix() for n in nodes]).astype(np.float64),
            np.array([n.sigma for n in nodes], np.float32))


def grid_sigma_min(grid) -> float:
    """Smallest kernel width (radians, float64 as the grid holds it): sets the automatic quadrature rule."""
    if hasattr(grid, "leaf_arrays"):
        return float(np.min(grid.leaf_arrays()[1]))
    return float(min(grid.nodes[i].sigma for i in grid.active_leaf_nodes()))
