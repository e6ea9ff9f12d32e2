"""Crystal lattice, symmetry and reflections: the host inputs of the forward operator.

What the operator reads from a material (diffractom's Material keeps the same attributes, so either can be passed):

  point_group_matrices  (G, 9) float32, the proper rotations of the crystal's Laue group in the Cartesian crystal frame
  h_vecs, h_vecs_normed (N, 3) reciprocal-lattice vectors of the reflections (2 pi convention) and their directions
  reflections           structured array with 'hkl', 'multiplicity', 'd_spacing', 'two_theta', 'intensity'
  intensities()         the 'intensity' column (NaN: unknown; there is no atomic basis here)

The Cartesian crystal frame is Busing & Levy's (a* along x, b* in the xy-plane, c along z), the frame of diffractom's
Material (crystallography/material.py:72-105), so orientation matrices mean the same in both. The rotation groups are
generated here from two generators each by closure (the same groups as the tables of
diffractom/crystallography/point_groups.py); equivalent reflections are grouped with the integer (hkl-space) form of
the same groups plus Friedel pairs (material.py:160-172). Matrix entries are stored as float32, as the reference
stores them (material.py:1294-1302), which fixes the last bits of the pole axes derived from them.
"""
from __future__ import annotations

from typing import Sequence

import numpy as np

REFLECTION_DTYPE = np.dtype([("hkl", "i4", (3,)), ("multiplicity", "i4"), ("d_spacing", "f8"),
                             ("two_theta", "f8"), ("intensity", "f8")])
HC_KEV_A = 12.39842   # h c in keV Angstrom (energy <-> wavelength of the material's two-theta column)


def _axis_rotation(axis, angle_deg):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    t = np.deg2rad(angle_deg)
    K = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + np.sin(t) * K + (1 - np.cos(t)) * (K @ K)


_EXACT = np.array([0.0, 0.5, 1.0, np.sqrt(3.0) / 2.0])


def _snap(m):
    """Entries within 1e-9 of 0, +-1/2, +-sqrt(3)/2, +-1 set to those values (products of generators drift)."""
    out = m.copy()
    a = np.abs(out)
    for v in _EXACT:
        hit = np.abs(a - v) < 1e-9
        out[hit] = np.sign(out[hit]) * v
    return out + 0.0          # no negative zeros (they would make equal matrices look different)


def _closure(generators, exact_int=False):
    """All products of the generators (a finite group): a list of matrices, identity first."""
    eye = np.eye(3, dtype=np.int64 if exact_int else np.float64)
    group = [eye]
    keys = {eye.tobytes() if exact_int else np.round(eye, 8).tobytes()}
    frontier = [eye]
    while frontier:
        nxt = []
        for g in frontier:
            for h in generators:
                m = h @ g
                m = m if exact_int else _snap(m)
                key = m.tobytes() if exact_int else np.round(m, 8).tobytes()
                if key not in keys:
                    keys.add(key)
                    group.append(m)
                    nxt.append(m)
        frontier = nxt
    return group


# generators of the proper rotation groups (Cartesian crystal frame) and of their hkl-space forms
_CARTESIAN_GENERATORS = {
    "triclinic": [],
    "monoclinic": [((0, 0, 1), 180)],
    "orthorhombic": [((1, 0, 0), 180), ((0, 1, 0), 180)],
    "tetragonal": [((0, 0, 1), 90), ((1, 0, 0), 180)],
    "trigonal": [((0, 0, 1), 120), ((0, 1, 0), 180)],
    "hexagonal": [((0, 0, 1), 60), ((1, 0, 0), 180)],
    "cubic": [((0, 0, 1), 90), ((1, 1, 1), 120)],
}
_HKL_GENERATORS = {
    "triclinic": [],
    "monoclinic": [[[-1, 0, 0], [0, -1, 0], [0, 0, 1]]],
    "orthorhombic": [[[1, 0, 0], [0, -1, 0], [0, 0, -1]], [[-1, 0, 0], [0, 1, 0], [0, 0, -1]]],
    "tetragonal": [[[0, -1, 0], [1, 0, 0], [0, 0, 1]], [[1, 0, 0], [0, -1, 0], [0, 0, -1]]],
    "trigonal": [[[0, 1, 0], [-1, -1, 0], [0, 0, 1]], [[0, 1, 0], [1, 0, 0], [0, 0, -1]]],
    "hexagonal": [[[1, 1, 0], [-1, 0, 0], [0, 0, 1]], [[1, 0, 0], [-1, -1, 0], [0, 0, -1]]],
    "cubic": [[[0, -1, 0], [1, 0, 0], [0, 0, 1]], [[0, 1, 0], [0, 0, 1], [1, 0, 0]]],
}
_ORDER = {"triclinic": 1, "monoclinic": 2, "orthorhombic": 4, "tetragonal": 8, "trigonal": 6, "hexagonal": 12,
          "cubic": 24}


def rotation_group(system: str) -> np.ndarray:
    """(G, 3, 3) float64 proper rotations of a crystal system's Laue group (Cartesian crystal frame)."""
    gens = [_axis_rotation(ax, ang) for ax, ang in _CARTESIAN_GENERATORS[system]]
    g = _closure(gens)
    assert len(g) == _ORDER[system], (system, len(g))
    return np.stack(g)


def hkl_group(system: str) -> list[np.ndarray]:
    gens = [np.asarray(m, np.int64) for m in _HKL_GENERATORS[system]]
    g = _closure(gens, exact_int=True)
    assert len(g) == _ORDER[system], (system, len(g))
    return g


def lattice_matrix(a, b, c, alpha, beta, gamma) -> np.ndarray:
    """Direct lattice matrix, columns = lattice vectors (Angstrom), Busing-Levy frame: a* along x, c along z."""
    if alpha == 90.0 and beta == 90.0 and gamma == 90.0:
        return np.diag([float(a), float(b), float(c)])
    ca, cb, cg = (np.cos(np.deg2rad(t)) for t in (alpha, beta, gamma))
    G = np.array([[a * a, a * b * cg, a * c * cb], [a * b * cg, b * b, b * c * ca], [a * c * cb, b * c * ca, c * c]])
    Gi = np.linalg.inv(G)                                   # reciprocal metric
    ast, bst, cst = np.sqrt(np.diag(Gi))
    cos_bs, cos_gs = Gi[0, 2] / (ast * cst), Gi[0, 1] / (ast * bst)
    Bm = np.array([[ast, bst * cos_gs, cst * cos_bs],
                   [0.0, bst * np.sqrt(1 - cos_gs ** 2), -cst * np.sqrt(1 - cos_bs ** 2) * ca],
                   [0.0, 0.0, 1.0 / c]])                    # columns a*, b*, c* without 2 pi
    return np.linalg.inv(Bm).T


def infer_crystal_system(a, b, c, alpha, beta, gamma, tol=5e-2) -> str:
    eq = lambda x, y: abs(x - y) < tol
    right = eq(alpha, 90) and eq(beta, 90) and eq(gamma, 90)
    if eq(a, b) and eq(b, c) and right:
        return "cubic"
    if eq(a, b) and eq(alpha, 90) and eq(beta, 90) and eq(gamma, 120):
        return "hexagonal"
    if eq(a, b) and right:
        return "tetragonal"
    if eq(a, b) and eq(b, c) and eq(alpha, beta) and eq(beta, gamma) and not eq(alpha, 90):
        return "trigonal"
    if right:
        return "orthorhombic"
    if eq(alpha, 90) and eq(gamma, 90):
        return "monoclinic"
    return "triclinic"


class Material:
    """Lattice, Laue group and reflection families of a phase, without an atomic basis (intensities unknown)."""

    def __init__(self, name: str = ""):
        self.name = name
        self.crystal_system = None
        self.lattice_params = None
        self.A = self.B = None
        self.reflections = None
        self.hkl = self.h_vecs = self.h_vecs_normed = None
        self.point_group_matrices = None
        self.num_sym_ops = None

    @classmethod
    def from_lattice_parameters(cls, *, a: float, b: float | None = None, c: float | None = None,
                                alpha: float = 90.0, beta: float = 90.0, gamma: float = 90.0,
                                symmetry_group: str | None = None, crystal_system: str | None = None,
                                wavelength_A: float | None = None, energy_keV: float | None = None,
                                energy_kev: float | None = None, hkl_list: Sequence | None = None,
                                min_two_theta: float | None = None, max_two_theta: float | None = None,
                                q_min: float | None = None, q_max: float | None = None,
                                name: str = "custom_lattice") -> "Material":
        """Keyword arguments as diffractom's Material.from_lattice_parameters (material.py:639-759): cell lengths
        (Angstrom) and angles (degrees), the crystal system (inferred from the metric if not given), a wavelength or
        energy (two-theta of the reflections), and an explicit hkl list or a q / two-theta range (radians)."""
        m = cls(name)
        b = a if b is None else b
        c = a if c is None else c
        m.lattice_params = dict(a=float(a), b=float(b), c=float(c), alpha=float(alpha), beta=float(beta),
                                gamma=float(gamma))
        sysname = (crystal_system or symmetry_group)
        m.crystal_system = sysname.lower() if sysname else infer_crystal_system(a, b, c, alpha, beta, gamma)
        if m.crystal_system not in _ORDER:
            raise ValueError(f"no point group for crystal system {m.crystal_system!r}")
        m.A = lattice_matrix(a, b, c, alpha, beta, gamma)
        m.B = 2.0 * np.pi * np.linalg.inv(m.A).T
        lam = None
        if wavelength_A is not None:
            lam = float(wavelength_A)
        elif energy_keV is not None or energy_kev is not None:
            lam = HC_KEV_A / float(energy_keV if energy_keV is not None else energy_kev)
        if hkl_list is None:
            if q_min is None or q_max is None:
                if lam is None or max_two_theta is None:
                    raise ValueError("provide hkl_list, q_min and q_max, or a wavelength and max_two_theta")
                q_min = 4 * np.pi / lam * np.sin(0.5 * float(min_two_theta or 0.0))
                q_max = 4 * np.pi / lam * np.sin(0.5 * float(max_two_theta))
        m._compute_reflections(lam, hkl_list, q_min, q_max)
        return m

    def _compute_reflections(self, lam, hkl_list, q_min, q_max):
        ops = hkl_group(self.crystal_system)
        if hkl_list is not None:
            raw = [tuple(int(v) for v in h) for h in np.asarray(hkl_list).reshape(-1, 3)]
        else:
            n = [int(np.ceil(q_max / L)) + 1 for L in np.linalg.norm(self.B, axis=0)]
            grid = np.stack(np.meshgrid(*[np.arange(-k, k + 1) for k in n], indexing="ij"), -1).reshape(-1, 3)
            grid = grid[np.any(grid != 0, axis=1)]
            q = np.linalg.norm(self.B @ grid.T, axis=0)
            raw = [tuple(int(v) for v in h) for h in grid[(q >= q_min) & (q <= q_max)]]
        families, mult, seen = [], [], set()
        for h in raw:
            if h in seen:
                continue
            eq = set()
            for R in ops:
                w = tuple(int(v) for v in R @ np.asarray(h))
                eq.add(w)
                eq.add(tuple(-v for v in w))
            seen |= eq
            families.append(min(eq))
            mult.append(len(eq))
        hkl = np.array(families, np.int32).reshape(-1, 3)
        mult = np.array(mult, np.int32)
        q = np.linalg.norm(self.B @ hkl.T, axis=0)
        d = 2 * np.pi / q
        if lam is not None:
            st = q * lam / (4 * np.pi)
            keep = st <= 1.0
            tth = np.where(keep, 2 * np.arcsin(np.clip(st, 0, 1)), 0.0)
        else:
            keep = np.ones(len(hkl), bool)
            tth = np.zeros(len(hkl))
        order = np.argsort(tth[keep] if lam is not None else -d[keep], kind="stable")
        sel = np.nonzero(keep)[0][order]
        refl = np.empty(len(sel), REFLECTION_DTYPE)
        refl["hkl"], refl["multiplicity"], refl["d_spacing"] = hkl[sel], mult[sel], d[sel]
        refl["two_theta"], refl["intensity"] = tth[sel], np.nan
        self.reflections = refl
        self.hkl = refl["hkl"].copy()
        self.h_vecs = (self.B @ self.hkl.astype(np.float64).T).T
        self.h_vecs_normed = self.h_vecs / (np.linalg.norm(self.h_vecs, axis=1, keepdims=True) + 1e-12)
        mats = rotation_group(self.crystal_system)
        self.point_group_matrices = mats.reshape(-1, 9).astype(np.float32)
        self.num_sym_ops = len(mats)

    def intensities(self) -> np.ndarray:
        return self.reflections["intensity"]

    def __len__(self):
        return 0 if self.reflections is None else len(self.reflections)


def group_reflections_into_rings(material, rtol=1e-6):
    """Reflections with the same two-theta (relative tolerance rtol) form one ring; rings by increasing two-theta
    (diffractom/crystallography/intensity.py:156-169)."""
    tt = np.asarray(material.reflections["two_theta"], dtype=np.float64)
    rings = []
    for i in np.argsort(tt, kind="stable"):
        if rings and np.isclose(tt[i], tt[rings[-1][0]], rtol=rtol, atol=0.0):
            rings[-1].append(int(i))
        else:
            rings.append([int(i)])
    return rings
