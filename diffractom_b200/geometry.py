"""Host-side geometry of the single-phase forward operator (float64 on the host, float32 on the device).

Everything here is computed once per operator. The float32 arrays uploaded to the GPU are built with the same
NumPy expressions and dtypes as diffractom's operator builds them (cited per function), so that they agree with the
reference bit for bit; tests/test_geometry.py checks that against the golden fixtures.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.spatial.transform import Rotation

ENERGY_KEV_A = 12.398   # the operator's cfg["energy"] (keV) -> wavelength (Angstrom)


def two_theta_of_rings(h_first_f32: np.ndarray, energy_kev: float) -> np.ndarray:
    """Two-theta of every ring from the float32 reciprocal vector of its first reflection
    (SinglePhaseForwardOperator.detector_coordinates, SPFO:553-556)."""
    lam = ENERGY_KEV_A / energy_kev
    return (2.0 * np.arcsin(np.linalg.norm(h_first_f32, axis=1) / (4.0 * np.pi) * lam)).astype(np.float32)


def probed_directions(two_theta_f32, omega_nodes, eta_nodes, n_omega, n_eta, cfg) -> np.ndarray:
    """coords (R, S, C, S_eta, P, 3) float32: v = R(omega)^T u(eta, theta_p), u = cos(theta) (cos(eta) d0 +
    sin(eta) d90) - sin(theta) p0, R(omega) the rotation by omega about k0 (SPFO:549-622)."""
    S = len(omega_nodes) // n_omega
    Se = len(eta_nodes) // n_eta
    eta2 = np.asarray(eta_nodes, np.float64).reshape(n_eta, Se)
    d0 = np.array(cfg["detector_direction_origin"])
    d90 = np.array(cfg["detector_direction_positive_90"])
    p0 = np.array(cfg["p_direction_0"])
    k0 = np.asarray(cfg["k_direction_0"])
    rot = Rotation.from_rotvec(np.asarray(omega_nodes, np.float64)[:, None] * k0).as_matrix()
    base = np.cos(eta2)[..., None] * d0[None, None, :] + np.sin(eta2)[..., None] * d90[None, None, :]
    per_ring = []
    for tt in two_theta_f32:                       # np.float32 scalars: cos / sin in float32, as the reference
        half = tt / 2.0
        dirs = base * np.cos(half) - np.sin(half) * p0
        per_ring.append(np.einsum("oij,esi->oesj", rot, dirs).reshape(n_omega, S, n_eta, Se, 3))
    return np.asarray(np.stack(per_ring, axis=-2), dtype=np.float32, order="C")


def axis_directions(omega_nodes, eta_nodes, n_omega, n_eta, cfg):
    """The probed directions of reflection_two_theta, stored once for all channels (SPFO:581-591): u (R, S, C, S_eta,
    3) float32 = R(omega)^T (cos(eta) d0 + sin(eta) d90) and w (R * S, 3) float32 = R(omega)^T p0; a pole axis with
    Bragg angle theta probes v = cos(theta) u - sin(theta) w."""
    S = len(omega_nodes) // n_omega
    Se = len(eta_nodes) // n_eta
    eta2 = np.asarray(eta_nodes, np.float64).reshape(n_eta, Se)
    d0 = np.array(cfg["detector_direction_origin"])
    d90 = np.array(cfg["detector_direction_positive_90"])
    p0 = np.array(cfg["p_direction_0"])
    k0 = np.asarray(cfg["k_direction_0"])
    rot = Rotation.from_rotvec(np.asarray(omega_nodes, np.float64)[:, None] * k0).as_matrix()
    base = np.cos(eta2)[..., None] * d0[None, None, :] + np.sin(eta2)[..., None] * d90[None, None, :]
    u = np.asarray(np.einsum("oij,esi->oesj", rot, base).reshape(n_omega, S, n_eta, Se, 3), np.float32, order="C")
    w = np.asarray(np.einsum("oij,i->oj", rot, p0), np.float32, order="C")
    return u, w


def image_direction(lab_xy, omega):
    """A lab-frame in-plane direction at rotation omega in image coordinates (col, row): turned into the sample frame
    (R(omega)^T about the rotation axis z), then (x, y) -> (-x, y), normalised (differentiable/absorption.py:107-114)."""
    c, s = np.cos(omega), np.sin(omega)
    x, y = lab_xy[..., 0], lab_xy[..., 1]
    xs, ys = c * x + s * y, -s * x + c * y
    d = np.stack([-xs, ys], -1)
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


@dataclass
class PoleAxes:
    axes: np.ndarray        # (A, 3) float64 unit axes (crystal frame), rings one after the other
    counts: np.ndarray      # (A,) float32 images per axis (family-share weighted)
    start: np.ndarray       # (P + 1,) int32 first axis of every ring
    family_weights: list
    two_theta: np.ndarray = None   # (A,) float64: the Bragg angle of every axis (its reflections' share-weighted mean)


def pole_axes(material, ring_reflections, ring_overlap, shares=None, refl_two_theta=None) -> PoleAxes:
    """The distinct symmetry images S_g h of every ring's reflections, up to sign, with their (share-weighted)
    counts (SPFO:742-825). shares: per ring the family shares before normalisation (default multiplicity x overlap:
    the normalized operator). Images are rounded to 6 decimals before they are merged, and the axes are the merged
    rounded vectors normalised, as in the reference. refl_two_theta (per reflection, float64): also the Bragg angle
    of every axis, the share-weighted mean of its images' (the plain mean where the shares are 0; SPFO:795-806)."""
    h = np.asarray(material.h_vecs_normed, dtype=np.float64)
    sym = np.asarray(material.point_group_matrices, dtype=np.float64).reshape(-1, 3, 3)
    mult = np.asarray(material.reflections["multiplicity"], dtype=np.float64)
    axes, counts, start, fw, tths = [], [], [0], [], []
    for ip, (refl, overlap) in enumerate(zip(ring_reflections, ring_overlap)):
        refl = np.asarray(refl)
        share = (mult[refl] if shares is None else np.asarray(shares[ip], np.float64)) * overlap
        if overlap.sum() <= 0 or not np.all(np.isfinite(share)) or share.sum() <= 0:
            share = mult[refl] * (overlap if overlap.sum() > 0 else 1.0)
        share = share / share.sum()
        fw.append(share)
        imgs = np.concatenate([sym @ h[f] for f in refl])
        wts = np.concatenate([np.full(len(sym), w) for w in share])
        img_tth = None if refl_two_theta is None else np.repeat(np.asarray(refl_two_theta, np.float64)[refl], len(sym))
        lead = np.argmax(np.abs(imgs) > 1e-6, axis=1)
        imgs = imgs * np.sign(imgs[np.arange(len(imgs)), lead])[:, None]
        uniq, inv = np.unique(np.round(imgs, 6), axis=0, return_inverse=True)
        cnt = np.bincount(inv.ravel(), weights=wts, minlength=len(uniq))
        counts.append(cnt)
        if img_tth is not None:
            nimg = np.bincount(inv.ravel(), minlength=len(uniq))
            tth = np.bincount(inv.ravel(), weights=img_tth, minlength=len(uniq)) / nimg
            has = cnt > 0
            tth[has] = np.bincount(inv.ravel(), weights=wts * img_tth, minlength=len(uniq))[has] / cnt[has]
            tths.append(tth)
        axes.append(uniq / np.linalg.norm(uniq, axis=1, keepdims=True))
        start.append(start[-1] + len(uniq))
    return PoleAxes(np.concatenate(axes), np.concatenate(counts).astype(np.float32), np.asarray(start, np.int32), fw,
                    np.concatenate(tths) if tths else None)


def rotate_axes(rot: np.ndarray, axes: np.ndarray, block: int = 4096) -> np.ndarray:
    """poles[k, a] = U_k axis_a, float32 (K, A, 3); in blocks of orientations (each element computed alike)."""
    out = np.empty((len(rot), len(axes), 3), np.float32)
    for lo in range(0, len(rot), block):
        out[lo:lo + block] = np.einsum("kij,aj->kai", rot[lo:lo + block], axes)
    return out


def kernel_factors(sigma_f32: np.ndarray):
    """1 / sigma^2 and the Gaussian's normalisation 1 / (8 pi sigma^2), float32 arithmetic as SPFO:822-824."""
    sigma = np.asarray(sigma_f32, np.float32)
    return (1.0 / (sigma * sigma)).astype(np.float32), (1.0 / (8.0 * np.pi * sigma * sigma)).astype(np.float32)


@dataclass
class RadonGeometry:
    geo: np.ndarray      # (R, 4) float32: X, Y, T0, angle weight
    scale: np.float32    # forward factor delta_x^2 / delta_s
    n_taps: int          # detector bins a pixel can touch (trapezoid)


def radon_geometry(angles, n_x, n_y, n_det, image_width, detector_width, detector_shift, angle_weights,
                   kernel="trapezoid") -> RadonGeometry:
    """Parallel-beam geometry of diffractom's ParallelRadon (parallel_radon.py:92-124): detector coordinate of
    pixel (x, y) at angle theta, t = X x + Y y + T0 bins, X = cos(theta - pi/2) / rho, Y = sin(theta - pi/2) / rho,
    rho = delta_s / delta_x, T0 centring the image on the detector and applying the shift (per angle allowed)."""
    angles = np.asarray(angles, np.float64)
    R = len(angles)
    w = np.broadcast_to(np.asarray(angle_weights, np.float64), (R,)).copy()
    delta_x = image_width / float(max(n_x, n_y))
    delta_s = float(detector_width) / n_det
    rho = delta_s / delta_x
    X = np.cos(angles - 0.5 * np.pi) / rho
    Y = np.sin(angles - 0.5 * np.pi) / rho
    T0 = (n_det - 1) / 2.0 - X * (n_x - 1) / 2.0 - Y * (n_y - 1) / 2.0 - np.asarray(detector_shift) / delta_s
    a_max = float(np.maximum(np.abs(X), np.abs(Y)).max())
    if kernel not in ("hat", "trapezoid"):
        raise ValueError(f"kernel must be 'hat' or 'trapezoid', not {kernel!r}")
    if kernel == "hat" and a_max > 1.0 + 1e-6:
        raise ValueError("kernel='hat' needs pixels no larger than the detector bins (delta_x <= delta_s); "
                         "use kernel='trapezoid'")
    n_taps = max(2, int(np.ceil(1.0 + a_max - 1e-6)))
    geo = np.stack([X, Y, T0, w], axis=1).astype(np.float32)
    return RadonGeometry(np.ascontiguousarray(geo), np.float32(delta_x * delta_x / delta_s), n_taps)


def fov_support_mask(n_x, n_y, n_det, angles=None, image_width=None, detector_width=None, detector_shift=0.0):
    """(Ny, Nx) bool: pixel centres that project onto the detector at every angle (utils/support.py:5-51);
    angles None: the disk r <= detector_width / 2 - |shift|."""
    image_width = float(n_x if image_width is None else image_width)
    detector_width = float(n_det if detector_width is None else detector_width)
    dx = image_width / max(n_x, n_y)
    x = (np.arange(n_x) - (n_x - 1) / 2.0)[None, :] * dx
    y = (np.arange(n_y) - (n_y - 1) / 2.0)[:, None] * dx
    half = detector_width / 2.0
    if angles is None:
        return x ** 2 + y ** 2 <= (half - abs(float(detector_shift))) ** 2
    mask = np.ones((n_y, n_x), dtype=bool)
    for a in np.asarray(angles, np.float64):
        t = np.cos(a - 0.5 * np.pi) * x + np.sin(a - 0.5 * np.pi) * y - detector_shift
        mask &= np.abs(t) <= half + 1e-9 * detector_width
    return mask


class OperatorGeometry:
    """All host-side set-up of a SinglePhaseForwardOperator (SPFO:376-494), computable without a GPU:
    rings, angles and quadrature nodes, probed directions, orientations, pole axes and rotated poles, kernel
    factors, ring intensities and the projector geometry. Attribute names are the reference operator's."""

    def __init__(self, cfg, material, grid, *, normalized=False, quadrature="auto", quadrature_tol=0.05,
                 pf_cutoff_sigma=4.0, radon_kernel="trapezoid", rings=None, ring_two_theta=None,
                 ring_intensities=None, reflection_two_theta=False):
        from .grid import grid_arrays, grid_sigma_min
        from .material import group_reflections_into_rings
        from .quadrature import pf_cut_value, setup_quadrature
        self.cfg = dict(cfg)
        self.normalized = bool(normalized)
        self.pf_cutoff_sigma = pf_cutoff_sigma
        self.N_eta = int(cfg["N_eta"])
        if rings is None:
            self.ring_reflections = group_reflections_into_rings(material)
            self.ring_overlap = [np.ones(len(r)) for r in self.ring_reflections]
        else:
            self.ring_reflections = [np.asarray(ix, dtype=np.int64) for ix, _ in rings]
            self.ring_overlap = [np.asarray(w, dtype=np.float64) for _, w in rings]
            if any(len(ix) == 0 or len(ix) != len(w) or np.any(w < 0) for ix, w in
                   zip(self.ring_reflections, self.ring_overlap)):
                raise ValueError("rings: every channel needs >= 1 reflection index and one weight >= 0 per index")
        self.N_peaks = len(self.ring_reflections)
        self.N_seg = self.N_peaks * self.N_eta
        self.Nx, self.Ny = int(cfg["Nx"]), int(cfg["Ny"])
        self.My, self.N_Omega = int(cfg["My"]), int(cfg["N_Omega"])
        self.cor_offset = cfg["cor_offset"]
        vs = cfg.get("voxel_size")
        self.voxel_size = None if vs is None else float(vs)
        self.image_width = float(self.Nx) if vs is None else float(vs) * max(self.Nx, self.Ny)
        self.angle_range = np.array(cfg["angle_range"]) / 180 * np.pi
        delta = (self.angle_range[1] - self.angle_range[0]) / self.N_Omega
        self.angles = np.linspace(self.angle_range[0], self.angle_range[1], self.N_Omega, endpoint=False) + delta / 2
        self.eta_angle_range = np.array(cfg.get("eta_angle_range", [0, 360])) / 180 * np.pi
        ed = (self.eta_angle_range[1] - self.eta_angle_range[0]) / self.N_eta
        self.eta_angles = np.linspace(self.eta_angle_range[0], self.eta_angle_range[1], self.N_eta,
                                      endpoint=False) + ed / 2
        q = setup_quadrature(self.angle_range, self.N_Omega, self.eta_angle_range, self.N_eta, cfg, quadrature,
                             quadrature_tol, grid_sigma_min(grid), pf_cutoff_sigma)
        self.quadrature, self.quadrature_bound, self.quadrature_tol = q.rule, q.bound, float(quadrature_tol)
        self.N_Omega_subdivisions, self.N_eta_subdivisions = q.rule.n_omega, q.rule.n_eta
        self.angles_subdivided, self.eta_angles_subdivided = q.omega_nodes, q.eta_nodes
        self.quad_weights_cpu = q.weights
        self.pf_cut = pf_cut_value(pf_cutoff_sigma)
        first = [r[0] for r in self.ring_reflections]
        self.h_cpu = np.asarray(material.h_vecs, dtype=np.float32)[first].copy(order="C")
        self.two_theta_peaks = two_theta_of_rings(self.h_cpu, float(cfg["energy"]))
        if ring_two_theta is not None:
            self.two_theta_peaks = np.asarray(ring_two_theta, dtype=np.float32).copy()
        elif rings is not None:
            # a window: the overlap-weighted mean two-theta of its reflections, float32 as for one ring (SPFO:560-566)
            lam = ENERGY_KEV_A / float(cfg["energy"])
            hh = np.asarray(material.h_vecs, dtype=np.float32)
            tth = (2.0 * np.arcsin(np.linalg.norm(hh, axis=1) / (4.0 * np.pi) * lam)).astype(np.float32)
            self.two_theta_peaks = np.array([np.average(tth[ix], weights=w) if w.sum() > 0 else tth[ix[0]]
                                             for ix, w in zip(self.ring_reflections, self.ring_overlap)],
                                            dtype=np.float32)
        if self.normalized:
            self.intens_cpu = np.ones(self.N_peaks, np.float32)
        else:
            if ring_intensities is None:
                raise ValueError("normalized=False needs the ring intensities (ring_intensities=...), which come "
                                 "from structure factors; or use normalized=True")
            ri = np.asarray(ring_intensities, np.float64).reshape(self.N_peaks)
            if not np.all(np.isfinite(ri)) or np.any(ri <= 0):
                raise ValueError("ring_intensities must be finite and positive")
            self.intens_cpu = ri.astype(np.float32)
        self.reflection_two_theta = bool(reflection_two_theta)
        if self.reflection_two_theta:
            self.coords_cpu, self.w_cpu = axis_directions(self.angles_subdivided, self.eta_angles_subdivided,
                                                          self.N_Omega, self.N_eta, cfg)
        else:
            self.coords_cpu = probed_directions(self.two_theta_peaks, self.angles_subdivided,
                                                self.eta_angles_subdivided, self.N_Omega, self.N_eta, cfg)
            self.w_cpu = None
        self.grid_rot_cpu, self.sigma_cpu = grid_arrays(grid)
        self.K = len(self.sigma_cpu)
        lam = ENERGY_KEV_A / float(cfg["energy"])
        refl_tth = 2.0 * np.arcsin(np.linalg.norm(np.asarray(material.h_vecs, np.float64), axis=1) / (4.0 * np.pi)
                                   * lam)
        pa = pole_axes(material, self.ring_reflections, self.ring_overlap,
                       refl_two_theta=refl_tth if self.reflection_two_theta else None)
        self.pole_axes_cpu, self.axis_count_cpu, self.axis_start_cpu = pa.axes, pa.counts, pa.start
        self.axis_two_theta_built = pa.two_theta
        self._two_theta_built = np.asarray(self.two_theta_peaks, np.float64).copy()
        self.axis_two_theta_cpu, self.axis_sin_cpu, self.axis_cos_cpu = self.axis_theta()
        self.ring_family_weights = pa.family_weights
        self.N_axes = len(pa.axes)
        self.poles_cpu = rotate_axes(self.grid_rot_cpu, pa.axes)
        self.inv_sigma2_cpu, self.norm_factor_cpu = kernel_factors(self.sigma_cpu)
        # backprojection weights pi / N_Omega: the adjoint is the transpose for any angle range (SPFO:457-466)
        self._bp_scale = 1.0 if self.voxel_size is None else self.voxel_size ** 2
        self.angle_weight = np.pi / self.N_Omega * self._bp_scale
        self.radon_kernel = radon_kernel
        self.radon_geo = radon_geometry(self.angles, self.Nx, self.Ny, self.My, self.image_width, self.My,
                                        self.detector_shifts(), self.angle_weight, radon_kernel)

    def axis_theta(self):
        """reflection_two_theta: the Bragg angle of every pole axis, its reflections' own, moved by its channel's
        change of two_theta since the operator was built, with sin and cos of theta as float32 (SPFO:829-842);
        (None, None, None) otherwise."""
        if not self.reflection_two_theta:
            return None, None, None
        tth = np.asarray(self.axis_two_theta_built, np.float64).copy()
        shift = np.asarray(self.two_theta_peaks, np.float64) - self._two_theta_built
        for p, d in enumerate(shift):
            tth[self.axis_start_cpu[p]:self.axis_start_cpu[p + 1]] += d
        th = 0.5 * tth
        return tth, np.sin(th).astype(np.float32), np.cos(th).astype(np.float32)

    def detector_shifts(self):
        """Detector shift of every projection angle: cor_offset minus per-angle shifts (SPFO:1616-1620)."""
        shift = getattr(self, "angle_shift", None)
        return np.full(int(self.N_Omega), float(self.cor_offset)) - (0.0 if shift is None else np.asarray(shift))

    def support_mask(self):
        """(Ny, Nx) bool mask of the pixels inside the field of view at every projection angle (SPFO:544-547)."""
        return fov_support_mask(self.Nx, self.Ny, self.My, angles=self.angles, image_width=self.image_width,
                                detector_width=self.My, detector_shift=self.cor_offset)


def interleaved_subsets(R: int, M: int):
    """M interleaved angle subsets: angle i in subset i % M (SPFO:1568-1572)."""
    if not 1 <= M <= R:
        raise ValueError(f"the number of subsets must be between 1 and N_Omega = {R}")
    return [np.arange(m, R, M) for m in range(M)]
