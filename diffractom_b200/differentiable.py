"""Derivatives of the forward model with respect to its continuous parameters, and the parameter updates.

Drop-ins for diffractom's differentiable/gradients.py (PFGradient, ProjGradient) and differentiable/update.py
(rotate_orientations, set_pf_parameters, set_proj_parameters, set_geometry). The model and the parameters are those
of diffractom's float64 ReferenceModel (differentiable/reference.py:1-30):

    d[a, s, j]  = sum_k PF[a, k, j] S_k[a, s],     PF[a, k, j] = I_p N(sigma_k) sum_nodes w sum_h m_h g(n_kh . v)
    rot (K, 3)  left increment U_k <- exp([rot_k]x) U_k (derivative at 0);  sigma (K,) kernel widths
    two_theta (P,), eta_offset (eta <- eta + offset), axis_tilt (2,) (k0 <- exp([t1 e1 + t2 e2]x) k0)
    shift (R,) detector shift of every projection (bins), cor (centre of rotation, cor_offset units)

PFGradient evaluates the derivative of every PF non-zero on the device (dfx_pf_param_vjp) against
G = sum_y res S, the batch's projections read from the operator's batch sinogram; the probed directions' derivatives
with respect to the eta offset, the axis tilt and the Bragg angles are made on the host in float64 (as the
reference's ReferenceModel.probed_derivatives) and uploaded as float32. ProjGradient projects every batch through
the derivative ray table (K' weights) and sums it against Z = PF^T res per angle (dfx_angle_dot).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
from scipy.spatial.transform import Rotation

from .arrays import as_host, check_device, is_device, stream_scope
from .geometry import axis_directions, kernel_factors, probed_directions, radon_geometry, rotate_axes

PF_GROUPS = ("rot", "sigma", "eta_offset", "axis_tilt", "two_theta")

__all__ = ["PF_GROUPS", "PFGradient", "ProjGradient", "perp_basis", "probed_derivatives", "rotate_orientations",
           "set_pf_parameters", "set_proj_parameters", "set_geometry"]


def perp_basis(k):
    """Two unit directions e1, e2 perpendicular to the rotation axis k, the axes of the tilt parameters
    (reference.py:33-39): e1 = k x a / |k x a| with a = x unless k is nearly along x (then y), e2 = k x e1."""
    k = np.asarray(k, np.float64)
    k = k / np.linalg.norm(k)
    a = np.array([1.0, 0.0, 0.0]) if abs(k[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(k, a)
    e1 /= np.linalg.norm(e1)
    return e1, np.cross(k, e1)


def probed_derivatives(op, groups=("eta_offset", "axis_tilt", "two_theta")):
    """The derivatives of the probed directions v = R(omega)^T u(eta, theta_p) of the operator's quadrature nodes,
    each (R, S, C, S_eta, P, 3) float64 like the operator's coords (reference.py:105-145): "eta_offset",
    ("axis_tilt", 0), ("axis_tilt", 1) (d v / d t_i = e_i x v - R^T (e_i x u)) and "two_theta" (ring p's slice:
    d v / d (2 theta_p))."""
    R, C, P = int(op.N_Omega), int(op.N_eta), int(op.N_peaks)
    S, Se = int(op.N_Omega_subdivisions), int(op.N_eta_subdivisions)
    cfg = op.cfg
    vec = lambda key: np.asarray(cfg[key], np.float64)
    k0, p0, d0, d90 = vec("k_direction_0"), vec("p_direction_0"), vec("detector_direction_origin"), \
        vec("detector_direction_positive_90")
    om = np.asarray(op.angles_subdivided, np.float64).reshape(R * S)
    eta = np.asarray(op.eta_angles_subdivided, np.float64).reshape(C * Se)
    rot = Rotation.from_rotvec(om[:, None] * k0).as_matrix()                      # (R S, 3, 3)
    e = np.cos(eta)[:, None] * d0 + np.sin(eta)[:, None] * d90                    # (C Se, 3)
    de = -np.sin(eta)[:, None] * d0 + np.cos(eta)[:, None] * d90
    th = 0.5 * np.asarray(op.two_theta_peaks, np.float64)
    ct, st = np.cos(th)[None, :, None], np.sin(th)[None, :, None]                 # (1, P, 1)
    u = ct * e[:, None, :] - st * p0                                              # (C Se, P, 3)
    shape = (R, S, C, Se, P, 3)
    turn = lambda w: np.einsum("oij,qpi->oqpj", rot, w).reshape(shape)           # R(omega)^T w per node
    out = {}
    if "eta_offset" in groups:
        out["eta_offset"] = turn(ct * de[:, None, :])
    if "two_theta" in groups:
        out["two_theta"] = turn(0.5 * (-st * e[:, None, :] - ct * p0))
    if "axis_tilt" in groups:
        v = turn(u)
        for i, ei in enumerate(perp_basis(k0)):
            out[("axis_tilt", i)] = np.cross(ei, v) - turn(np.cross(ei, u))
    return out


def probed_parts_derivatives(op, groups=("eta_offset", "axis_tilt")):
    """reflection_two_theta: the derivatives of u (R, S, C, S_eta, 3) and w (R * S, 3), v = cos(theta) u - sin(theta) w,
    float64 (reference.py:151-167): "eta_offset" (du), ("axis_tilt", i) (du), ("axis_tilt_w", i) (dw)."""
    R, C = int(op.N_Omega), int(op.N_eta)
    S, Se = int(op.N_Omega_subdivisions), int(op.N_eta_subdivisions)
    vec = lambda key: np.asarray(op.cfg[key], np.float64)
    k0, p0, d0, d90 = vec("k_direction_0"), vec("p_direction_0"), vec("detector_direction_origin"), \
        vec("detector_direction_positive_90")
    om = np.asarray(op.angles_subdivided, np.float64).reshape(R * S)
    eta = np.asarray(op.eta_angles_subdivided, np.float64).reshape(C * Se)
    rot = Rotation.from_rotvec(om[:, None] * k0).as_matrix()
    e = np.cos(eta)[:, None] * d0 + np.sin(eta)[:, None] * d90
    turn = lambda a: np.einsum("oij,qi->oqj", rot, a).reshape(R, S, C, Se, 3)
    out = {}
    if "eta_offset" in groups:
        out["eta_offset"] = turn(-np.sin(eta)[:, None] * d0 + np.cos(eta)[:, None] * d90)
    if "axis_tilt" in groups:
        u = turn(e)
        w = np.einsum("oij,i->oj", rot, p0)
        for i, ei in enumerate(perp_basis(k0)):
            out[("axis_tilt", i)] = np.cross(ei, u) - turn(np.cross(ei[None, :], e))
            out[("axis_tilt_w", i)] = np.cross(ei, w) - np.einsum("oij,i->oj", rot, np.cross(ei, p0))
    return out


def _f32_dev(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float32), device=dev)


def _coeffs_in(op, c, name="c"):
    if is_device(c):
        return check_device(c, op.coeff_shape, name)
    return torch.as_tensor(as_host(c, op.coeff_shape, name), device=op.device)


def _data_in(op, r, name):
    if is_device(r):
        return check_device(r, op.data_shape, name)
    return torch.as_tensor(as_host(r, op.data_shape, name), device=op.device)


def _project_batch(op, c, ib):
    """The projections of batch ib's coefficients into the operator's batch sinogram (R, My, Kstride): gathered (the
    (K, Ny, Nx) layout) or scattered from the patches (local basis) into the batch image, then projected."""
    b = op.batches[ib]
    k0, kb = b["k_start"], b["K_batch"]
    if getattr(op, "coefficient_layout", "dense") == "local":
        op._fill(op._img_k, 0.0)
        lb = op.local_batches[ib]
        if lb is not None:
            op._scatter(lb, c, op._img_k)
    else:
        op._call("dfx_gather_channels", c.data_ptr(), op._img_k.data_ptr(), op.npix, k0, kb, op.Kstride, op._s())
    return kb


class PFGradient:
    """grad = PFGradient(op)(c, r): the gradients of <r, A(c)> with respect to the PF parameters at the operator's
    current parameters (gradients.py:19-204). op: pf_mode "sparse" or "generated" (the derivative is evaluated on the
    non-zeros of its PF matrix), the (K, Ny, Nx) or the local coefficient layout. hessian: also "hess" (K, 4, 4),
    the Gauss-Newton blocks J_k^T diag(curv) J_k of the rotation and width of every orientation. local_size is
    accepted (the kernel's block is fixed)."""

    def __init__(self, op, hessian=False, local_size=64):
        if op.pf_mode not in ("sparse", "generated"):
            raise NotImplementedError(f"PFGradient needs pf_mode 'sparse' or 'generated' (this operator: "
                                      f"{op.pf_mode!r})")
        layout = getattr(op, "coefficient_layout", "dense")
        if layout not in ("dense", "local"):
            raise NotImplementedError("PFGradient needs the (K, Ny, Nx) or the local coefficient layout")
        if int(op.N_peaks) > 16:
            raise NotImplementedError("PFGradient supports at most 16 rings")
        self.op = op
        self.hessian = bool(hessian)
        self.local_size = int(local_size)
        self.P = int(op.N_peaks)
        self.nq = int(op._lib.dfx_pf_param_nq(self.P, int(self.hessian)))
        nh = 10 if self.hessian else 0
        self.q_eta, self.q_tilt, self.q_tth = 4 + nh, 5 + nh, 7 + nh
        self.dv = {}
        self._alloc()

    def _alloc(self):
        op = self.op
        self.kmax, self.version = op.K_batch_max, op._pf_version
        self.rows = torch.empty(op.N_Omega * op.K_batch_max * self.nq, dtype=torch.float64, device=op.device)
        self.per_k = torch.empty(op.K * self.nq, dtype=torch.float64, device=op.device)

    def refresh(self):
        """Forget the probed directions' derivatives (after the operator's geometry changed)."""
        self.dv = {}

    def _dv(self, groups):
        if getattr(self.op, "reflection_two_theta", False):
            return self._dv_axis(groups)
        need = [g for g in ("eta_offset", "axis_tilt", "two_theta") if g in groups and g not in self.dv]
        if need:
            d = probed_derivatives(self.op, need)
            dev = self.op.device
            if "eta_offset" in d:
                self.dv["eta_offset"] = _f32_dev(d["eta_offset"], dev)
            if "two_theta" in d:
                self.dv["two_theta"] = _f32_dev(d["two_theta"], dev)
            if ("axis_tilt", 0) in d:
                self.dv["axis_tilt"] = (_f32_dev(d[("axis_tilt", 0)], dev), _f32_dev(d[("axis_tilt", 1)], dev))
        ptr = lambda t: None if t is None else t.data_ptr()
        tilt = self.dv.get("axis_tilt", (None, None))
        return (ptr(self.dv.get("eta_offset") if "eta_offset" in groups else None),
                ptr(tilt[0] if "axis_tilt" in groups else None), ptr(tilt[1] if "axis_tilt" in groups else None),
                ptr(self.dv.get("two_theta") if "two_theta" in groups else None), None, None)

    def _dv_axis(self, groups):
        """reflection_two_theta: du / d eta, du and dw / d tilt (the Bragg angle's derivative is formed on the
        device)."""
        need = [g for g in ("eta_offset", "axis_tilt") if g in groups and g not in self.dv]
        if need:
            d = probed_parts_derivatives(self.op, need)
            dev = self.op.device
            if "eta_offset" in d:
                self.dv["eta_offset"] = _f32_dev(d["eta_offset"], dev)
            if ("axis_tilt", 0) in d:
                self.dv["axis_tilt"] = tuple(_f32_dev(d[key], dev) for key in
                                             (("axis_tilt", 0), ("axis_tilt", 1), ("axis_tilt_w", 0), ("axis_tilt_w", 1)))
        ptr = lambda t: None if t is None else t.data_ptr()
        tilt = self.dv.get("axis_tilt", (None,) * 4) if "axis_tilt" in groups else (None,) * 4
        return (ptr(self.dv.get("eta_offset") if "eta_offset" in groups else None), ptr(tilt[0]), ptr(tilt[1]), None,
                ptr(tilt[2]), ptr(tilt[3]))

    def __call__(self, c, r, groups=PF_GROUPS, curv=None):
        """c: coefficients (the operator's coeff_shape), r: dL/d data (N_Omega, My, N_seg) (NumPy arrays are
        uploaded); curv: the loss's curvature per data point for the Gauss-Newton blocks (hessian=True; default 1).
        Returns "rot" (K, 3), "sigma" (K,), "eta_offset", "axis_tilt" (2,), "two_theta" (P,) as requested, and
        "hess" (K, 4, 4) with hessian=True (gradients.py:112-174)."""
        op = self.op
        with stream_scope(op):
            if op.K_batch_max != self.kmax or op._pf_version != self.version:   # a rebuilt operator
                self.refresh()
                self._alloc()
            c = _coeffs_in(op, c)
            r = _data_in(op, r, "r")
            cv = None
            if self.hessian:
                cv = torch.ones(op.data_shape, dtype=torch.float32, device=op.device) if curv is None \
                    else _data_in(op, curv, "curv")
            dv_eta, dv_t1, dv_t2, dv_tth, dw_t1, dw_t2 = self._dv(groups)
            flags = (1 if "eta_offset" in groups else 0) | (2 if "axis_tilt" in groups else 0) | \
                (4 if "two_theta" in groups else 0)
            R, My, nq, s = op.N_Omega, op.My, self.nq, op._s()
            local = getattr(op, "coefficient_layout", "dense") == "local"
            for ib, b in enumerate(op.batches):
                k0, kb = b["k_start"], b["K_batch"]
                if local:
                    if op.local_batches[ib] is None:       # no coefficients: zero gradients
                        self.per_k[k0 * nq:(k0 + kb) * nq].zero_()
                        continue
                    op._project_local(c, ib)
                else:
                    _project_batch(op, c, ib)
                    op._radon_fwd(op._img_k.data_ptr(), op.coeffs_sino_C.data_ptr(), None, R, kb)
                rp, col, _, _ = op._pf_batch(ib, False)
                op._call("dfx_pf_param_vjp", ctypes.byref(op._pfg), rp.data_ptr(), col.data_ptr(), r.data_ptr(),
                         None if cv is None else cv.data_ptr(), op.coeffs_sino_C.data_ptr(), My, op.Kstride, k0, kb,
                         flags, dv_eta, dv_t1, dv_t2, dv_tth, dw_t1, dw_t2, int(self.hessian), self.rows.data_ptr(),
                         s)
                op._call("dfx_pf_rows_sum", self.rows.data_ptr(), R, kb, nq,
                         self.per_k.data_ptr() + 8 * k0 * nq, s)
            per_k = self.per_k.view(op.K, nq).cpu().numpy()
        out = {}
        if "rot" in groups:
            out["rot"] = per_k[:, 0:3].copy()
        if "sigma" in groups:
            out["sigma"] = per_k[:, 3].copy()
        if "eta_offset" in groups:
            out["eta_offset"] = float(per_k[:, self.q_eta].sum())
        if "axis_tilt" in groups:
            out["axis_tilt"] = per_k[:, self.q_tilt:self.q_tilt + 2].sum(axis=0)
        if "two_theta" in groups:
            out["two_theta"] = per_k[:, self.q_tth:self.q_tth + self.P].sum(axis=0)
        if self.hessian:
            iu = np.triu_indices(4)
            H = np.zeros((op.K, 4, 4))
            H[:, iu[0], iu[1]] = per_k[:, 4:14]
            H[:, iu[1], iu[0]] = per_k[:, 4:14]
            out["hess"] = H
        return out


class ProjGradient:
    """grad = ProjGradient(op)(c, r): the gradients of <r, A(c)> with respect to a detector shift of every projection
    ("shift" (N_Omega,), bins: t_a(x) <- t_a(x) + shift_a) and the centre of rotation ("cor", cor_offset units)
    (gradients.py:207-258). Native projector, pf_mode "sparse" or "generated"; local_size is accepted."""

    def __init__(self, op, local_size=256):
        if op.projector != "native":
            raise NotImplementedError("ProjGradient needs the native projector")
        if op.pf_mode not in ("sparse", "generated"):
            raise NotImplementedError("ProjGradient needs pf_mode 'sparse' or 'generated'")
        self.op = op
        self.version = None
        self.dS = None

    def _tables(self):
        """The derivative ray table (the projector's taps with K' weights) and the dS buffer, per geometry."""
        op = self.op
        if self.version == op._pf_version and self.dS is not None and self.dS.shape[2] == op.Kstride:
            return
        self.dent = torch.empty_like(op._ray_ent)
        op._call("dfx_radon_dtable_fill", op.geo_gpu.data_ptr(), op.N_Omega, op.Nx, op.Ny, op.My, op._kernel_id,
                 op._ray_rp.data_ptr(), self.dent.data_ptr(), op._s())
        self.dS = torch.empty((op.N_Omega, op.My, op.Kstride), dtype=torch.float32, device=op.device)
        self.version = op._pf_version

    def __call__(self, c, r):
        op = self.op
        with stream_scope(op):
            self._tables()
            c = _coeffs_in(op, c)
            r = _data_in(op, r, "r")
            R, My, s = op.N_Omega, op.My, op._s()
            part = torch.empty((len(op.batches), R), dtype=torch.float32, device=op.device)
            for ib, b in enumerate(op.batches):
                kb = b["K_batch"]
                rp, col, val, compact = op._pf_batch(ib, False)
                op._pf_adjoint_product(r.data_ptr(), rp, col, val, op.coeffs_sino_C.data_ptr(), None, R, kb, 1.0,
                                       compact, s)
                _project_batch(op, c, ib)
                op._call("dfx_radon_forward_table", op._img_k.data_ptr(), self.dS.data_ptr(), op._ray_rp.data_ptr(),
                         self.dent.data_ptr(), None, R, My, op.Kstride, kb, float(op.radon_geo.scale), s)
                op._call("dfx_angle_dot", op.coeffs_sino_C.data_ptr(), self.dS.data_ptr(), R, My, op.Kstride, kb,
                         part[ib].data_ptr(), s)
            out = part.cpu().numpy().astype(np.float64).sum(axis=0)
        return {"shift": out, "cor": -float(out.sum())}      # t = ... - cor / delta_s, delta_s = 1 bin


# ---------------------------------------------------------------------------------------------- parameter updates
def rotate_orientations(rotations, increments):
    """U_k <- exp([increment_k]x) U_k, the left increment the gradients refer to (update.py:10-12)."""
    return Rotation.from_rotvec(np.asarray(increments, np.float64)).as_matrix() @ np.asarray(rotations, np.float64)


def _set(op, **attrs):
    """Set attributes on the operator and on its host geometry (the operator keeps copies of the geometry's, and
    the geometry's methods, e.g. detector_shifts and support_mask, read its own)."""
    for k, v in attrs.items():
        setattr(op, k, v)
        setattr(op.geometry, k, v)


def _initial_geometry(op):
    """The geometry the operator was built with, recorded on the first call (update.py:60-70)."""
    if getattr(op, "_geo_initial", None) is None:
        op._geo_initial = {"k0": np.asarray(op.cfg["k_direction_0"], np.float64).copy(),
                           "eta": tuple(np.array(a, dtype=np.float64) for a in
                                        (op.eta_angle_range, op.eta_angles, op.eta_angles_subdivided)),
                           "two_theta": np.asarray(op.two_theta_peaks, np.float64).copy(),
                           "cor": float(op.cor_offset)}
    return op._geo_initial


def _tilted_cfg(op, k0, axis_tilt):
    e1, e2 = perp_basis(k0)
    q = Rotation.from_rotvec(axis_tilt[0] * e1 + axis_tilt[1] * e2).as_matrix()
    cfg = dict(op.cfg)                          # the caller's dict stays as it was
    cfg["k_direction_0"] = list(q @ np.asarray(k0, np.float64))
    _set(op, cfg=cfg)


def set_pf_parameters(op, rotations=None, sigma=None, two_theta=None, eta_offset=0.0, axis_tilt=None):
    """New PF parameters for the operator, relative to its current ones, and a rebuild of what depends on them: poles
    and widths, probed directions, the sparse PF matrix as it was set up (update.py:15-57). rotations (K, 3, 3),
    sigma (K,) radians, two_theta (P,) radians, eta_offset (added to the azimuths), axis_tilt (2,) (the current axis
    turned about its two perpendicular directions). The quadrature rule is kept; the batches may change with the
    fill (coefficient arrays keep their shape)."""
    _initial_geometry(op)
    pf_changed = geo_changed = False
    if rotations is not None:
        _set(op, grid_rot_cpu=np.asarray(rotations, np.float64).reshape(op.K, 3, 3).copy())
        pf_changed = True
    if sigma is not None:
        _set(op, sigma_cpu=np.asarray(sigma, np.float32).reshape(op.K).copy())
        pf_changed = True
    if two_theta is not None:
        _set(op, two_theta_peaks=np.asarray(two_theta, np.float32).reshape(op.N_peaks).copy())
        geo_changed = True
    if eta_offset:
        d = float(eta_offset)
        _set(op, eta_angle_range=np.asarray(op.eta_angle_range, np.float64) + d,
             eta_angles=np.asarray(op.eta_angles) + d, eta_angles_subdivided=np.asarray(op.eta_angles_subdivided) + d)
        geo_changed = True
    if axis_tilt is not None and np.any(np.asarray(axis_tilt) != 0):
        _tilted_cfg(op, op.cfg["k_direction_0"], axis_tilt)
        geo_changed = True
    if pf_changed or geo_changed:
        _rebuild(op, pf_changed, geo_changed)
    return op


def set_geometry(op, eta_offset=None, axis_tilt=None, two_theta=None, cor=None, shift=None):
    """The operator's geometry set ABSOLUTELY, relative to the geometry it was built with (update.py:73-101):
    eta_offset added to the initial azimuths; axis_tilt (2,) turns the initial axis; two_theta (P,) Bragg angles;
    cor, shift (N_Omega,) as set_proj_parameters. None keeps a parameter as it is."""
    g0 = _initial_geometry(op)
    geo_changed = False
    if eta_offset is not None:
        d = float(eta_offset)
        rng, ang, sub = (a + d for a in g0["eta"])
        _set(op, eta_angle_range=rng, eta_angles=ang, eta_angles_subdivided=sub)
        geo_changed = True
    if axis_tilt is not None:
        _tilted_cfg(op, g0["k0"], axis_tilt)
        geo_changed = True
    if two_theta is not None:
        _set(op, two_theta_peaks=np.asarray(two_theta, np.float32).reshape(op.N_peaks).copy())
        geo_changed = True
    if geo_changed:
        _rebuild(op, False, True)
    if cor is not None or shift is not None:
        set_proj_parameters(op, cor=cor, shift=shift)
    return op


def _rebuild(op, pf_changed, geo_changed):
    """Rebuild what depends on the PF parameters (update.py:104-131): poles and widths, probed directions, the PF
    kernels' parameter block, the sparse PF matrix (and the dense BF16 copy), the local basis's batch tables."""
    with stream_scope(op):
        dev = op.device
        if pf_changed:
            poles = rotate_axes(op.grid_rot_cpu, op.pole_axes_cpu)
            inv_s2, norm = kernel_factors(op.sigma_cpu)
            _set(op, poles_cpu=poles, inv_sigma2_cpu=inv_s2, norm_factor_cpu=norm)
            op.poles_gpu = _f32_dev(poles, dev)
            op.inv_sigma2_gpu = _f32_dev(inv_s2, dev)
            op.norm_factor_gpu = _f32_dev(norm, dev)
        if geo_changed:
            if getattr(op, "reflection_two_theta", False):
                # u and w do not depend on the Bragg angles; the axes' angles follow their channels' two_theta
                u, w = axis_directions(op.angles_subdivided, op.eta_angles_subdivided, op.N_Omega, op.N_eta, op.cfg)
                _set(op, coords_cpu=u, w_cpu=w)
                tth, sn, cs = op.geometry.axis_theta()
                _set(op, axis_two_theta_cpu=tth, axis_sin_cpu=sn, axis_cos_cpu=cs)
                op.coords_gpu = _f32_dev(u, dev)
                op._upload_axis_theta()
            else:
                coords = probed_directions(op.two_theta_peaks, op.angles_subdivided, op.eta_angles_subdivided,
                                           op.N_Omega, op.N_eta, op.cfg)
                _set(op, coords_cpu=coords)
                op.coords_gpu = _f32_dev(coords, dev)
        op._make_pfg()
        op.release_streamer()
        op.release_omega_subsets()
        op.sparse_batches = None
        op.build_sparse_pf(**op._pf_build)
        if op.precision == "bf16":
            op.pf_bf16 = None
            op.build_dense_bf16_pf()
        if getattr(op, "coefficient_layout", "dense") == "local":
            op._setup_local()
        op._pf_version += 1


def set_proj_parameters(op, cor=None, shift=None):
    """A new centre of rotation (cor_offset units) and / or a detector shift of every projection (shift (N_Omega,),
    bins, added to the detector coordinate) for the operator (native projector), and a rebuild of its projector
    geometry and ray tables; the PF matrix is not affected (update.py:134-155)."""
    if op.projector != "native":
        raise NotImplementedError("set_proj_parameters needs the native projector")
    _initial_geometry(op)
    with stream_scope(op):
        if cor is not None:
            _set(op, cor_offset=float(cor))
        if shift is not None:
            _set(op, angle_shift=np.asarray(shift, np.float64).reshape(int(op.N_Omega)).copy())
        rg = radon_geometry(op.angles, op.Nx, op.Ny, op.My, op.image_width, op.My, op.detector_shifts(),
                            op.angle_weight, op.radon_kernel)
        _set(op, radon_geo=rg)
        op.geo_gpu = torch.as_tensor(rg.geo, device=op.device)
        op._ray_rp, op._ray_ent, op.ray_taps = op._build_ray_table()
        op._ray_grp = op._build_group_table()
        op._tcf_tab = None
        op._ray_supp = {}
        op.release_streamer()
        op.release_omega_subsets()
        if getattr(op, "coefficient_layout", "dense") == "local":
            op._setup_local()
        op._pf_version += 1
    return op
