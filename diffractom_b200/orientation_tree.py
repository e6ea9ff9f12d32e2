"""Nested cells of an orientation basis for the hierarchical total variation of SPDHGPoisson(tv_tree=)
(optimization/orientation_tree.py of diffractom), and the node-pixel index arrays the solver's tree kernels use.

The penalty. The basis is cut into nested cells of radii r_0 > r_1 > ... > r_(L-1) degrees (a greedy cover per parent
cell, crystal symmetry respected). A cell's sum s_n(j) adds the coefficients of its orientations in voxel j, and

    R(x) = tv * sum over cells n and voxels j of e_n |grad s_n(j)|,

with e_n the length of the tree edge above the cell: r_(L-1) / 2 for the leaves (single orientations), (r_(l-1) - r_l)
/ 2 for a cell of level l >= 1, and top_edge (default 0: no term) above level 0. Moving a unit of mass across a voxel
edge between two orientations whose smallest common cell has level l then costs about r_l: a tree-Wasserstein
distance between neighbouring voxels' orientation distributions. One radius (r,) is the plain total variation with
weight tv r / 2."""
from __future__ import annotations

import numpy as np


def _chord(angle_deg):
    """The Euclidean distance of two unit quaternions whose rotations differ by angle_deg."""
    return 2.0 * np.sin(np.radians(angle_deg) / 4.0)


def _both_signs(p):
    """q and -q are one rotation: the point set with both signs."""
    return np.concatenate([p, -p])


def _cover(q, eq, members, radius):
    """Cell labels 0..m-1 of the orientations `members` and m (orientation_tree.py:_cover): walking the members in
    order, every member not yet within `radius` of a centre (through any symmetric copy) becomes a centre; then every
    member joins its nearest centre. q: (K, 4) unit quaternions, eq: (K, S, 4) the quaternions of U S."""
    from scipy.spatial import cKDTree
    S = eq.shape[1]
    copies = _both_signs(eq[members].reshape(-1, 4))
    whose = np.tile(np.repeat(np.arange(len(members)), S), 2)
    near = cKDTree(copies)
    covered = np.zeros(len(members), bool)
    centres = []
    chord = _chord(radius)
    for i, m in enumerate(members):
        if not covered[i]:
            centres.append(i)
            covered[whose[near.query_ball_point(q[m], chord)]] = True
    centres = np.asarray(centres, np.int64)
    ccopies = _both_signs(eq[members[centres]].reshape(-1, 4))
    cwhose = np.tile(np.repeat(np.arange(len(centres)), S), 2)
    _, nearest = cKDTree(ccopies).query(q[members])
    return cwhose[nearest], len(centres)


class OrientationTree:
    """rotations: (K, 3, 3) crystal-to-sample matrices of the basis, in the operator's grid order; symmetry: (S, 3, 3)
    rotations with U S equivalent to U (None: none); radii_deg: the cell radii, coarsest first, strictly decreasing;
    top_edge: the edge length (degrees) above the cells of level 0 (orientation_tree.py:OrientationTree).

    nodes: per level the (K,) cell of every orientation (cells of a level numbered within their parents' order);
    n_nodes: cells per level; edges: per level the edge above its cells; leaf_edge: the edge above the leaves."""

    def __init__(self, rotations, symmetry, radii_deg, top_edge=0.0):
        from scipy.spatial.transform import Rotation
        R = np.asarray(rotations, np.float64)
        if R.ndim != 3 or R.shape[1:] != (3, 3):
            raise ValueError("rotations must have shape (K, 3, 3)")
        radii = [float(r) for r in radii_deg]
        if not radii or min(radii) <= 0 or any(a <= b for a, b in zip(radii, radii[1:])):
            raise ValueError("radii_deg must be positive and strictly decreasing (coarsest first)")
        S = np.eye(3)[None] if symmetry is None else np.asarray(symmetry, np.float64)
        K = len(R)
        q = Rotation.from_matrix(R).as_quat()
        eq = Rotation.from_matrix(np.einsum("kij,sjl->ksil", R, S).reshape(-1, 3, 3)).as_quat().reshape(K, len(S), 4)
        self.K, self.radii = K, radii
        self.nodes, self.n_nodes = [], []
        parent = np.zeros(K, np.int64)
        for r in radii:
            cell = np.empty(K, np.int64)
            count = 0
            for p in np.unique(parent):
                members = np.flatnonzero(parent == p)
                lab, m = _cover(q, eq, members, r)
                cell[members] = lab + count
                count += m
            self.nodes.append(cell)
            self.n_nodes.append(count)
            parent = cell
        self.edges = [float(top_edge)] + [(a - b) / 2.0 for a, b in zip(radii, radii[1:])]
        self.leaf_edge = radii[-1] / 2.0

    def levels(self):
        """(cell array, edge) of the levels with a penalty (edge > 0), coarsest first; the leaves are not among them."""
        return [(n, e) for n, e in zip(self.nodes, self.edges) if e > 0]


def tree_level_arrays(k, iy, ix, pi, Ny, Nx, n_coef, T, tree):
    """Per penalised level of `tree`, the host arrays of its node-pixels on a local basis (spdhg_poisson.py:946-978):
    the node-pixels are the (cell, iy, ix) triples holding at least one coefficient, in ascending (cell, iy, ix)
    order; ptr / idx (CSR, int32): the flat coefficients of every node-pixel in the support's pair order; map (int32,
    n_coef): a coefficient's node-pixel, -1: none; right / down / left / up (int32): the neighbouring node-pixel of the
    same cell, -1: none; A (float32): the float64 sum of the coefficients' primal steps T, the node-pixel's step in
    the dual update. k, iy, ix, pi: the local operator's (orientation, row, column, flat index) pairs."""
    k, iy, ix, pi = (np.asarray(a, np.int64) for a in (k, iy, ix, pi))
    T = np.asarray(T, np.float64)
    out = []
    for cell, edge in tree.levels():
        key = (np.asarray(cell, np.int64)[k] * Ny + iy) * Nx + ix
        u, inv = np.unique(key, return_inverse=True)
        nn = len(u)
        order = np.argsort(inv, kind="stable")
        ptr = np.concatenate([[0], np.cumsum(np.bincount(inv, minlength=nn))])
        mp = np.full(int(n_coef), -1, np.int32)
        mp[pi] = inv
        ux, uy = u % Nx, (u // Nx) % Ny

        def neighbour(target, inside):
            j = np.minimum(np.searchsorted(u, target), nn - 1)
            return np.where(inside & (u[j] == target), j, -1).astype(np.int32)

        out.append(dict(n=nn, edge=float(edge), ptr=ptr.astype(np.int32), idx=pi[order].astype(np.int32), map=mp,
                        right=neighbour(u + 1, ux < Nx - 1), down=neighbour(u + Nx, uy < Ny - 1),
                        left=neighbour(u - 1, ux > 0), up=neighbour(u - Nx, uy > 0),
                        A=np.bincount(inv, weights=T[pi], minlength=nn).astype(np.float32)))
    return out
