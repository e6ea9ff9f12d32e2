"""CPU oracle of the parameter gradients of the forward model: TEST INFRASTRUCTURE ONLY.

A float64 NumPy restatement, for small cases, of diffractom's ReferenceModel derivatives
(differentiable/reference.py): the probed directions' derivatives (probed_derivatives, reference.py:128-145), the
vector-Jacobian products with respect to the PF parameters (vjp / _pf_grads, reference.py:248-314) and the
projector's detector shifts (reference.py:214-239, 262-267), and the Gauss-Newton blocks of the rotation and width
of every orientation (the quantity of differentiable/pf_grad.cl:8-10). Inputs are the arrays the golden fixtures
record (tests/golden/make_golden.py). Used by tests/ only, as the checker; pinned against the reference's own
values in the fixtures (tests/test_gradients.py).
"""
from __future__ import annotations

import numpy as np
from scipy.spatial.transform import Rotation


def perp_basis(k):
    """reference.py:33-39."""
    k = np.asarray(k, np.float64)
    k = k / np.linalg.norm(k)
    a = np.array([1.0, 0.0, 0.0]) if abs(k[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(k, a)
    e1 = e1 / np.linalg.norm(e1)
    return e1, np.cross(k, e1)


def probed_parts(cfg, om_nodes, eta_nodes, two_theta):
    """Rotations R(omega) (R, S, 3, 3), u (C, Se, P, 3), du/d eta, du/d 2theta_p (reference.py:105-119)."""
    vec = lambda key: np.asarray(cfg[key], np.float64)
    k0, p0, d0, d90 = (vec(k) for k in ("k_direction_0", "p_direction_0", "detector_direction_origin",
                                         "detector_direction_positive_90"))
    om = np.asarray(om_nodes, np.float64)
    eta = np.asarray(eta_nodes, np.float64)
    rot = Rotation.from_rotvec(om.reshape(-1, 1) * k0).as_matrix().reshape(om.shape + (3, 3))
    e = np.cos(eta)[..., None] * d0 + np.sin(eta)[..., None] * d90
    de = -np.sin(eta)[..., None] * d0 + np.cos(eta)[..., None] * d90
    th = 0.5 * np.asarray(two_theta, np.float64)
    ct, st = np.cos(th)[None, None, :, None], np.sin(th)[None, None, :, None]
    u = ct * e[:, :, None, :] - st * p0
    return rot, u, ct * de[:, :, None, :], 0.5 * (-st * e[:, :, None, :] - ct * p0), k0


def probed(rot, u):
    return np.einsum("rsij,cepi->rscepj", rot, u)


def probed_derivatives(cfg, om_nodes, eta_nodes, two_theta):
    """dict eta_offset, tilt0, tilt1, two_theta, each (R, S, C, Se, P, 3) (reference.py:128-145)."""
    rot, u, du_eta, du_tth, k0 = probed_parts(cfg, om_nodes, eta_nodes, two_theta)
    v = probed(rot, u)
    out = {"eta_offset": probed(rot, du_eta), "two_theta": probed(rot, du_tth)}
    for i, e in enumerate(perp_basis(k0)):
        out[f"tilt{i}"] = np.cross(e, v) - probed(rot, np.cross(e[None, None, None, :], u))
    return out


def _g(d, s, cut):
    """g, dg/d(n.v), dg/ds (reference.py:180-187)."""
    ad = np.abs(d)
    x1, x2 = (1.0 - ad) * s, (1.0 + ad) * s
    e1, e2 = np.exp(-x1), np.exp(-x2)
    if cut is not None:
        e1, e2 = np.where(x1 < cut, e1, 0.0), np.where(x2 < cut, e2, 0.0)
    return e1 + e2, np.sign(d) * s * (e1 - e2), -(1.0 - ad) * e1 - (1.0 + ad) * e2


def model_geometry(cfg, shift=None):
    """(X, Y, T0 - cor / delta_s + shift) per angle and the forward scale, in float64 as the reference model
    (reference.py:84-94): image width Nx, one detector bin per unit."""
    R, nx, ny, ns = int(cfg["N_Omega"]), int(cfg["Nx"]), int(cfg["Ny"]), int(cfg["My"])
    rng = np.array(cfg["angle_range"], np.float64) / 180 * np.pi
    ang = np.linspace(rng[0], rng[1], R, endpoint=False) + (rng[1] - rng[0]) / R / 2
    delta_x = nx / max(nx, ny)
    rho = 1.0 / delta_x
    X, Y = np.cos(ang - 0.5 * np.pi) / rho, np.sin(ang - 0.5 * np.pi) / rho
    T0 = (ns - 1) / 2.0 - X * (nx - 1) / 2.0 - Y * (ny - 1) / 2.0 - float(cfg["cor_offset"])
    if shift is not None:
        T0 = T0 + np.asarray(shift, np.float64)
    return np.stack([X, Y, T0], 1), delta_x ** 2


def projection_matrices(geo, nx, ny, ns, scale, kernel):
    """P and dP/dt (R, ns, nx ny) of the projector geometry geo (R, >= 3) (X, Y, T0) (reference.py:214-239)."""
    geo = np.asarray(geo, np.float64)
    yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    px, py = xx.ravel().astype(np.float64), yy.ravel().astype(np.float64)
    R = len(geo)
    Pm = np.zeros((R, ns, nx * ny))
    dPm = np.zeros((R, ns, nx * ny))
    for a in range(R):
        X, Y, T0 = geo[a, :3]
        A = max(abs(X), abs(Y))
        t = X * px + Y * py + T0
        for s in range(ns):
            d = t - s
            if kernel == "hat":
                k = np.maximum(1.0 - np.abs(d), 0.0)
                dk = np.where(np.abs(d) < 1.0, -np.sign(d), 0.0)
            else:
                hw, top = 0.5 * (1.0 + A), min(1.0, A)
                q = hw - np.abs(d)
                k = np.clip(q, 0.0, top) / A
                dk = np.where((q > 0.0) & (q < top), -np.sign(d) / A, 0.0)
            Pm[a, s] = scale * k
            dPm[a, s] = scale * dk
    return Pm, dPm


class GradientModel:
    """The parameter gradients of <r, d(c)> at the fixture's parameters (rot = 0, the recorded widths and angles)."""

    def __init__(self, f, f32_geometry=False):
        """f: a golden fixture. f32_geometry: the probed directions and poles the operator computes with (the
        fixture's float32 coords and poles, in float64 arithmetic) instead of the model's float64 ones: the
        gradients of the operator's own float32 PF geometry."""
        import json
        cfg = f["cfg"]
        self.cfg = cfg if isinstance(cfg, dict) else json.loads(str(cfg))
        self.rot0 = np.asarray(f["rot"], np.float64)
        self.sigma = np.asarray(f["sigma"], np.float64)
        self.axes = np.asarray(f["axes"], np.float64)
        self.counts = np.asarray(f["counts"], np.float64)
        self.start = np.asarray(f["start"])
        self.intens = np.asarray(f["intens"], np.float64)
        self.two_theta = np.asarray(f["two_theta"], np.float64)
        self.K = len(self.sigma)
        self.R, self.My, self.C = int(self.cfg["N_Omega"]), int(self.cfg["My"]), int(self.cfg["N_eta"])
        self.P = len(self.two_theta)
        self.Nx, self.Ny = int(self.cfg["Nx"]), int(self.cfg["Ny"])
        om = np.asarray(f["angles_sub"], np.float64)
        eta = np.asarray(f["eta_sub"], np.float64)
        self.S, self.Se = len(om) // self.R, len(eta) // self.C
        self.om = om.reshape(self.R, self.S)
        self.eta = eta.reshape(self.C, self.Se)
        qw = np.asarray(f["quad_w"], np.float64)
        self.qw = np.full((self.S, self.Se), 1.0 / (self.S * self.Se)) if qw.size == 0 else qw.reshape(self.S, self.Se)
        self.cut = 4.0 ** 2 / 2                     # pf_cutoff_sigma 4 of the fixtures' operators
        self.geo, self.scale = model_geometry(self.cfg)
        self.f32 = None
        if f32_geometry:
            self.f32 = (np.asarray(f["coords"], np.float64).reshape(self.R, self.S, self.C, self.Se, self.P, 3),
                        np.asarray(f["poles"], np.float64))
        self.kernel = str(f["kernel"])

    def poles(self):
        if self.f32 is not None:
            return self.f32[1]
        return np.einsum("kij,aj->kai", self.rot0, self.axes)

    def pf_terms(self):
        """R(omega), u, du/d eta, du/d 2theta and the probed directions v (R, S, C, Se, P, 3)."""
        rot, u, du_eta, du_tth, k0 = probed_parts(self.cfg, self.om, self.eta, self.two_theta)
        return rot, u, du_eta, du_tth, (probed(rot, u) if self.f32 is None else self.f32[0])

    def pf(self, sigma=None):
        """PF (R, K, C, P) at the fixture's orientations and the widths sigma (default the recorded ones)
        (reference.py:189-211)."""
        _, _, _, _, v = self.pf_terms()
        n = self.poles()
        sig = self.sigma if sigma is None else np.asarray(sigma, np.float64)
        s = 1.0 / sig ** 2
        norm = 1.0 / (8.0 * np.pi * sig ** 2)
        out = np.zeros((self.R, self.K, self.C, self.P))
        for p in range(self.P):
            a0, a1 = self.start[p], self.start[p + 1]
            d = np.einsum("rscex,kax->rsceka", v[..., p, :], n[:, a0:a1])
            g, _, _ = _g(d, s[:, None], self.cut)
            node = np.einsum("rsceka,a,se->rkc", g, self.counts[a0:a1], self.qw)
            out[..., p] = self.intens[p] * norm[None, :, None] * node
        return out

    def projections(self, c):
        Pm, dPm = projection_matrices(self.geo, self.Nx, self.Ny, self.My, self.scale, self.kernel)
        S = np.einsum("asp,kp->ask", Pm, np.asarray(c, np.float64).reshape(self.K, -1))
        return Pm, dPm, S

    def pf_grads(self, c, r, curv=None):
        """rot (K, 3), sigma (K,), eta_offset, axis_tilt (2,), two_theta (P,), hess (K, 4, 4) (reference.py:273-314;
        hess: sum_{a, j} Hs q q^T with Hs = sum_y curv S^2, q = d PF[a, k, j] / d (rot, sigma))."""
        R, K, C, P, My = self.R, self.K, self.C, self.P, self.My
        r = np.asarray(r, np.float64).reshape(R, My, C * P)
        _, _, S = self.projections(c)
        G = np.einsum("asj,ask->akj", r, S).reshape(R, K, C, P)
        cv = np.ones_like(r) if curv is None else np.asarray(curv, np.float64).reshape(R, My, C * P)
        Hs = np.einsum("asj,ask->akj", cv, S * S).reshape(R, K, C, P)
        dv = probed_derivatives(self.cfg, self.om, self.eta, self.two_theta)
        _, _, _, _, v = self.pf_terms()
        n = self.poles()
        sig = self.sigma
        s = 1.0 / sig ** 2
        norm = 1.0 / (8.0 * np.pi * sig ** 2)
        out = {"rot": np.zeros((K, 3)), "sigma": np.zeros(K), "two_theta": np.zeros(P), "eta_offset": 0.0,
               "axis_tilt": np.zeros(2)}
        Q = np.zeros((R, K, C, P, 4))                                    # d PF / d (rot, sigma) per entry
        for p in range(P):
            a0, a1 = self.start[p], self.start[p + 1]
            vp, npp = v[..., p, :], n[:, a0:a1]
            d = np.einsum("rscex,kax->rsceka", vp, npp)
            g, dgd, dgs = _g(d, s[:, None], self.cut)
            wc = self.counts[a0:a1]
            f = self.intens[p] * norm                                     # (K,)
            # per node and axis: w_node m_h g'(d); the entry's derivative sums them
            Wn = self.qw[None, :, None, :, None, None] * wc * dgd          # (R, S, C, Se, K, A)
            cr = np.cross(npp[None, None, None, None], vp[:, :, :, :, None, None, :])
            drot = np.einsum("rsceka,rscekax->rckx", Wn, cr) * f[None, None, :, None]
            node = np.einsum("rsceka,a,se->rck", g, wc, self.qw)
            dnode = np.einsum("rsceka,a,se->rck", dgs, wc, self.qw)
            dsig = f[None, None, :] * (-2.0 / sig * node - 2.0 / sig ** 3 * dnode)
            Q[:, :, :, p, :3] = drot.transpose(0, 2, 1, 3)
            Q[:, :, :, p, 3] = dsig.transpose(0, 2, 1)
            Gp = G[..., p]                                                # (R, K, C)
            out["rot"] += np.einsum("rkc,rckx->kx", Gp, drot)
            out["sigma"] += np.einsum("rkc,rck->k", Gp, dsig)
            for key, dvk in dv.items():
                dd = np.einsum("rscex,kax->rsceka", dvk[..., p, :], npp)
                val = np.einsum("rsceka,rsceka,rkc,k->", Wn, dd, Gp, f)
                if key == "two_theta":
                    out["two_theta"][p] += val
                elif key == "eta_offset":
                    out["eta_offset"] += val
                else:
                    out["axis_tilt"][int(key[-1])] += val
        out["hess"] = np.einsum("rkcp,rkcpu,rkcpv->kuv", Hs, Q, Q)
        return out

    def shift_grads(self, c, r, pf):
        """shift (R,), cor (reference.py:262-267): sum over k, s, p of dP c times Z = PF^T r."""
        R, K, My = self.R, self.K, self.My
        r = np.asarray(r, np.float64).reshape(R, My, -1)
        _, dPm, _ = self.projections(c)
        Z = np.einsum("akj,asj->ask", np.asarray(pf, np.float64).reshape(R, K, -1), r)
        gs = np.einsum("asp,kp,ask->a", dPm, np.asarray(c, np.float64).reshape(K, -1), Z)
        return {"shift": gs, "cor": -gs.sum()}
