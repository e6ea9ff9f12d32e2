"""OrientationRefiner: refinement of the basis orientations and kernel widths of an operator by damped Gauss-Newton
steps, alternated with coefficient refits (the role of diffractom's differentiable/refine.py, refine.py:33-133).

The refinement works orientation by orientation. With the coefficients x held fixed, the Poisson deviance f of the
prediction A x on the fitted angles (PoissonTerm) depends on each orientation's rotation (a left increment, 3
parameters) and width (1). PFGradient supplies, per orientation k, the gradient g_k of f and the Gauss-Newton matrix
H_k = J_k^T diag(c) J_k, c being the Fisher curvature of the prediction; the coupling between orientations is left
out, so a step is K independent 4 x 4 (or 3 x 3, widths fixed) solves:

    proposal   d_k = -(H_k + damping diag(H_k) + 1e-12 tr(H_k) I)^-1 g_k        (orientations with tr(H_k) > 0)
    limits     |rotation part| <= max_rot_deg (scaled down as a whole), |width part| <= max_dsigma sigma_k
    search     the first step length alpha in `alphas` whose parameters lower f is kept (widths clipped to
               [sigma_min_deg, sigma_max_deg]); if none does, the operator gets its old parameters back

The operator is rebuilt for every trial (set_pf_parameters), so after step() it holds the accepted parameters.
run() alternates step() with the caller's refit solve(x). The operator needs pf_mode "sparse" or "generated", with
the dense or the local coefficient layout.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from .arrays import as_host, is_device
from .differentiable import PFGradient, rotate_orientations, set_pf_parameters
from .poisson_term import PoissonTerm

__all__ = ["OrientationRefiner"]


@dataclass
class _Trial:
    """The parameters a step starts from and the (limited) per-orientation step: rotation increments (K, 3) and
    width changes (K,), radians."""
    rot0: np.ndarray
    sigma0: np.ndarray
    d_rot: np.ndarray
    d_sigma: np.ndarray

    def at(self, alpha, lo, hi):
        return (rotate_orientations(self.rot0, alpha * self.d_rot),
                np.clip(self.sigma0 + alpha * self.d_sigma, lo, hi))


def _damped_solve(grad, gn, damping):
    """Per-orientation steps -(H + damping diag(H) + ridge)^-1 g for the blocks with a positive trace (0 elsewhere):
    grad (K, n), gn (K, n, n) float64."""
    k, n = grad.shape
    out = np.zeros((k, n))
    trace = np.einsum("kii->k", gn)
    live = np.flatnonzero(trace > 0)
    if live.size:
        A = gn[live].copy()
        diag = np.arange(n)
        A[:, diag, diag] *= 1.0 + damping
        A[:, diag, diag] += 1e-12 * trace[live, None]
        out[live] = -np.linalg.solve(A, grad[live, :, None])[:, :, 0]
    return out


class OrientationRefiner:
    """Damped Gauss-Newton refinement of op's orientations and widths (module docstring).

    b, weights, gain, background: the data and its terms as the Poisson solvers take them; fit_rows: the fitted
    angles (bool (N_Omega,) or indices; None: all), so that held-out angles do not steer the refinement;
    refine_sigma=False keeps the widths and moves the rotations only; curv_floor_counts: the floor of the prediction
    in the Fisher curvature (in counts of the gain)."""

    def __init__(self, op, b, weights=None, gain=None, background=None, fit_rows=None, eps_counts=1e-3,
                 max_rot_deg=0.2, max_dsigma=0.3, sigma_min_deg=0.05, sigma_max_deg=5.0, damping=1e-3,
                 alphas=(1.0, 0.5, 0.25, 0.1), refine_sigma=True, curv_floor_counts=0.25):
        self.op = op
        b_dev = b if is_device(b) else torch.as_tensor(as_host(b, op.data_shape, "b"), device=op.device)
        self.pt = PoissonTerm(op.queue, op.data_shape, b_dev, weights, gain, background, fit_rows, eps_counts)
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

    # ---------------------------------------------------------------- pieces
    def _on_device(self, x):
        return x if is_device(x) else torch.as_tensor(as_host(x, self.op.coeff_shape, "x"), device=self.op.device)

    def loss(self, x):
        """The deviance of A x on the fitted angles (x NumPy or CUDA)."""
        self.op.direct_cl(self._on_device(x), self.pred)
        return self.pt.deviance(self.pred)

    def newton_steps(self, x):
        """The unlimited per-orientation steps (K, 4): rotation increment (3) and width change, radians; and f(x)."""
        xd = self._on_device(x)
        f0 = self.loss(xd)
        r, c = torch.empty_like(self.pred), torch.empty_like(self.pred)
        self.pt.grad_curv(self.pred, r, c, self.curv_floor)
        blocks = self.grad(xd, r, groups=("rot", "sigma"), curv=c)
        n = 4 if self.refine_sigma else 3
        grad = np.column_stack([blocks["rot"], blocks["sigma"]]).astype(np.float64)
        gn = np.asarray(blocks["hess"], np.float64)
        steps = np.zeros((grad.shape[0], 4))
        steps[:, :n] = _damped_solve(grad[:, :n], gn[:, :n, :n], self.damping)
        return steps, f0

    def _limited(self, steps):
        """The trial of the current parameters with the step limits applied."""
        op = self.op
        sigma0 = np.array(op.sigma_cpu, np.float64)
        d_rot = steps[:, :3]
        norm = np.linalg.norm(d_rot, axis=1)
        shrink = np.where(norm > self.max_rot, self.max_rot / np.maximum(norm, 1e-30), 1.0)
        bound = self.max_dsigma * sigma0
        return _Trial(rot0=np.array(op.grid_rot_cpu, np.float64), sigma0=sigma0, d_rot=d_rot * shrink[:, None],
                      d_sigma=np.clip(steps[:, 3], -bound, bound))

    def _search(self, trial, x, f0):
        """(accepted alpha or 0, deviance there); the operator ends with the accepted (or the old) parameters."""
        for alpha in self.alphas:
            rot, sig = trial.at(alpha, self.sig_lo, self.sig_hi)
            set_pf_parameters(self.op, rotations=rot, sigma=sig)
            f = self.loss(x)
            if f < f0:
                return alpha, f
        set_pf_parameters(self.op, rotations=trial.rot0, sigma=trial.sigma0)
        return 0.0, f0

    # ---------------------------------------------------------------- steps
    def step(self, x):
        """One Gauss-Newton step at the fixed coefficients x (not changed). Returns a dict: alpha (the accepted step
        length, 0: rejected), f0 and f (deviance before and after), rot_deg_median / rot_deg_max (the rotations
        applied, deg), sigma_deg_median (after the step) and time (s)."""
        t0 = time.perf_counter()
        xd = self._on_device(x)
        steps, f0 = self.newton_steps(xd)
        trial = self._limited(steps)
        alpha, f = self._search(trial, xd, f0)
        turned = np.degrees(alpha * np.linalg.norm(trial.d_rot, axis=1))
        return {"alpha": alpha, "f0": f0, "f": f,
                "rot_deg_median": float(np.median(turned)) if turned.size else 0.0,
                "rot_deg_max": float(turned.max()) if turned.size else 0.0,
                "sigma_deg_median": float(np.degrees(np.median(self.op.sigma_cpu))),
                "time": time.perf_counter() - t0}

    def run(self, x, solve, n_steps, verbose=False):
        """n_steps rounds of step(x) followed by x = solve(x) (the caller's refit, e.g. a new SPDHGPoisson run);
        returns the last x. self.history gets each round's step() dict plus "f_fit" (the deviance after the refit)
        and "step" (1-based)."""
        for i in range(1, int(n_steps) + 1):
            rec = self.step(x)
            x = solve(x)
            rec.update(f_fit=self.loss(x), step=i)
            self.history.append(rec)
            if verbose:
                print(f"refinement {i}: step length {rec['alpha']}, deviance {rec['f0']:.6g} -> {rec['f']:.6g}, "
                      f"after the refit {rec['f_fit']:.6g}; median rotation {rec['rot_deg_median']:.3f} deg, "
                      f"median width {rec['sigma_deg_median']:.3f} deg", flush=True)
        return x
