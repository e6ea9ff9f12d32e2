"""OrientationRefiner: Gauss-Newton refinement of the basis orientations and their kernel widths, alternated with
coefficient fits (diffractom's differentiable/refine.py).

A step at the current coefficients x and Poisson deviance f (PoissonTerm, on the fitted angles):
1. r = df/dpred and the Fisher curvature c of the prediction (dfx_poisson_term); PFGradient gives the gradient of f
   with respect to every orientation's rotation (a left increment) and width, and the 4 x 4 Gauss-Newton block
   J_k^T diag(c) J_k of every orientation (the coupling between orientations ignored).
2. A damped Newton step per orientation, (H_k + damping diag(H_k))^-1 grad_k, the rotation limited to max_rot_deg (a
   trust region), the width change to max_dsigma x sigma and the width to [sigma_min_deg, sigma_max_deg].
3. A backtracking search over the step lengths alphas at fixed x: the first that lowers f is kept, else the old
   parameters come back.
Then the caller refits the coefficients (solve(x), e.g. a new SPDHGPoisson run). The operator needs pf_mode "sparse"
or "generated", the dense or the local coefficient layout.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from .arrays import as_host, is_device
from .differentiable import PFGradient, rotate_orientations, set_pf_parameters
from .poisson_term import PoissonTerm

__all__ = ["OrientationRefiner"]


class OrientationRefiner:
    """Gauss-Newton steps on the orientations and widths of op's basis (module docstring; refine.py:33-133)."""

    def __init__(self, op, b, weights=None, gain=None, background=None, fit_rows=None, eps_counts=1e-3,
                 max_rot_deg=0.2, max_dsigma=0.3, sigma_min_deg=0.05, sigma_max_deg=5.0, damping=1e-3,
                 alphas=(1.0, 0.5, 0.25, 0.1), refine_sigma=True, curv_floor_counts=0.25):
        self.op = op
        self.pt = PoissonTerm(op.queue, op.data_shape, b if is_device(b) else
                              torch.as_tensor(as_host(b, op.data_shape, "b"), device=op.device),
                              weights, gain, background, fit_rows, eps_counts)
        self.grad = PFGradient(op, hessian=True)
        self.max_rot = np.radians(float(max_rot_deg))
        self.max_dsigma = float(max_dsigma)
        self.sig_lo, self.sig_hi = np.radians(float(sigma_min_deg)), np.radians(float(sigma_max_deg))
        self.damping = float(damping)
        self.alphas = tuple(float(a) for a in alphas)
        self.refine_sigma = bool(refine_sigma)
        self.curv_floor = float(curv_floor_counts)
        self.pred = torch.empty(tuple(op.data_shape), dtype=torch.float32, device=op.device)
        self.history = []

    def _dev(self, x):
        if is_device(x):
            return x
        return torch.as_tensor(as_host(x, self.op.coeff_shape, "x"), device=self.op.device)

    def loss(self, x):
        """The deviance of A x on the fitted angles (x NumPy or CUDA)."""
        self.op.direct_cl(self._dev(x), self.pred)
        return self.pt.deviance(self.pred)

    def newton_steps(self, x):
        """(K, 4) steps (rotation increment, width change; radians) at x before the limits, and f(x)."""
        xd = self._dev(x)
        self.op.direct_cl(xd, self.pred)
        f0 = self.pt.deviance(self.pred)
        r = torch.empty_like(self.pred)
        c = torch.empty_like(self.pred)
        self.pt.grad_curv(self.pred, r, c, self.curv_floor)
        g = self.grad(xd, r, groups=("rot", "sigma"), curv=c)
        grad = np.concatenate([g["rot"], g["sigma"][:, None]], axis=1)
        H = np.asarray(g["hess"], np.float64)
        n = 4 if self.refine_sigma else 3
        Hn, gn = H[:, :n, :n], grad[:, :n]
        tr = np.trace(Hn, axis1=1, axis2=2)
        ok = tr > 0
        st = np.zeros((len(grad), 4))
        if ok.any():
            eye = np.eye(n)[None]
            Hd = Hn[ok] + self.damping * np.einsum("kii->ki", Hn[ok])[:, :, None] * eye + 1e-12 * tr[ok, None, None] * eye
            st[ok, :n] = -np.linalg.solve(Hd, gn[ok][..., None])[..., 0]
        return st, f0

    def step(self, x):
        """One Gauss-Newton step at fixed coefficients x (unchanged). Returns alpha (0: rejected), f0 and f, the
        median and largest rotation (deg) and the median width (deg) after the step."""
        t0 = time.perf_counter()
        op = self.op
        xd = self._dev(x)
        st, f0 = self.newton_steps(xd)
        sig0 = np.asarray(op.sigma_cpu, np.float64).copy()
        U0 = np.asarray(op.grid_rot_cpu, np.float64).copy()
        st[:, 3] = np.clip(st[:, 3], -self.max_dsigma * sig0, self.max_dsigma * sig0)
        rn = np.linalg.norm(st[:, :3], axis=1)
        st[:, :3] *= np.minimum(1.0, self.max_rot / np.maximum(rn, 1e-30))[:, None]
        acc, f = 0.0, f0
        for a in self.alphas:
            set_pf_parameters(op, rotations=rotate_orientations(U0, a * st[:, :3]),
                              sigma=np.clip(sig0 + a * st[:, 3], self.sig_lo, self.sig_hi))
            fa = self.loss(xd)
            if fa < f0:
                acc, f = a, fa
                break
        if acc == 0.0:
            set_pf_parameters(op, rotations=U0, sigma=sig0)
        moved = np.degrees(acc * np.linalg.norm(st[:, :3], axis=1))
        return {"alpha": acc, "f0": f0, "f": f, "rot_deg_median": float(np.median(moved)),
                "rot_deg_max": float(moved.max()) if moved.size else 0.0,
                "sigma_deg_median": float(np.degrees(np.median(op.sigma_cpu))), "time": time.perf_counter() - t0}

    def run(self, x, solve, n_steps, verbose=False):
        """n_steps of [Gauss-Newton step, then x = solve(x)]; returns x. self.history holds every step's dict and
        "f_fit" (the deviance after the refit)."""
        for t in range(int(n_steps)):
            info = self.step(x)
            x = solve(x)
            info["f_fit"] = self.loss(x)
            info["step"] = t + 1
            self.history.append(info)
            if verbose:
                print(f"GN step {t + 1}: alpha {info['alpha']}, deviance {info['f0']:.6g} -> {info['f']:.6g} "
                      f"(refit {info['f_fit']:.6g}), rotation median {info['rot_deg_median']:.3f} deg, "
                      f"width median {info['sigma_deg_median']:.3f} deg", flush=True)
        return x
