"""Shared pieces of the Poisson solvers: periodic weight / gain / background arrays, the support mask, FP64
reductions through the C ABI, and device-array plumbing.

Periodic arrays (diffractom/optimization/fista_poisson.py:287-308): one value per segment (N_seg), per
(translation, segment) (My * N_seg) or per data point; element i of the data uses a[i % period]; None: the constant
1 (weights, gain) or 0 (background).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .arrays import check_device, is_device


def periodic(a, dshape, name, device):
    """(device tensor or None, period)."""
    if a is None:
        return None, 0
    n_seg, n_ys, n_all = dshape[-1], dshape[-2] * dshape[-1], int(np.prod(dshape))
    if is_device(a):
        if a.dtype != torch.float32 or not a.is_contiguous() or a.numel() not in (n_seg, n_ys, n_all):
            raise ValueError(f"{name} must be contiguous float32 with N_seg = {n_seg}, My * N_seg = {n_ys} or "
                             f"{n_all} elements; got shape {tuple(a.shape)}, {a.dtype}")
        return a.reshape(-1), int(a.numel())
    h = np.ascontiguousarray(a, dtype=np.float32)
    if h.size == 1:
        h = np.full(n_seg, float(h.ravel()[0]), np.float32)
    if h.size not in (n_seg, n_ys, n_all):
        raise ValueError(f"{name} must have N_seg = {n_seg} elements (one per segment), My * N_seg = {n_ys} or the "
                         f"data shape {tuple(dshape)}; got shape {h.shape}")
    return torch.as_tensor(h.ravel(), device=device), int(h.size)


def support_mask_to_device(operator, support, device):
    """The support option ("fov", None/False, or an (Ny, Nx) bool array) as a uint8 (Ny * Nx) tensor or None
    (diffractom/optimization/prox.py:75-99)."""
    if support is None or support is False:
        return None
    if getattr(operator, "coefficient_layout", "dense") != "dense":
        # a local-basis operator: its support (field of view included) is part of the operator
        if isinstance(support, str) and support == "fov":
            return None
        raise ValueError("a support mask cannot be applied to this operator's coefficients; restrict the "
                         "operator's LocalSupport instead (LocalSupport.restrict)")
    if isinstance(support, str):
        if support != "fov":
            raise ValueError(f"support must be 'fov', None or an (Ny, Nx) array, not {support!r}")
        mask = operator.support_mask()
    else:
        mask = np.asarray(support)
    if mask.shape != (operator.Ny, operator.Nx):
        raise ValueError(f"support mask shape {mask.shape} != (Ny, Nx) = {(operator.Ny, operator.Nx)}")
    return torch.as_tensor(np.ascontiguousarray(mask, dtype=np.uint8).ravel(), device=device)


class Reducer:
    """FP64 sums through the C ABI with a reusable scratch and result buffer on the device."""

    def __init__(self, op):
        self.op = op
        self.out = torch.zeros(4, dtype=torch.float64, device=op.device)

    def _scr(self, n):
        nb = self.op._lib.dfx_reduce_scratch_bytes(int(n))
        return self.op.scratch(nb), nb

    def deviance(self, mu, b, w, pw, g, pg, bg, pbg, eps, write_grad=False, mode=0, floor_counts=1.0):
        scr, nb = self._scr(mu.numel())
        _lib.call("dfx_poisson_value_grad", mu.data_ptr(), b.data_ptr(), _p(w), pw, _p(g), pg, _p(bg), pbg,
                  float(eps), int(write_grad), int(mode), float(floor_counts), mu.numel(), self.out.data_ptr(),
                  scr.data_ptr(), nb, self.op._s())
        return float(self.out[0].item())

    def deviance_into(self, out, mu, b, w, pw, g, pg, bg, pbg, eps):
        """deviance() written to the float64 device tensor out[0] on the operator's stream (no host read); out has
        room for the kernel's 4 values."""
        scr, nb = self._scr(mu.numel())
        _lib.call("dfx_poisson_value_grad", mu.data_ptr(), b.data_ptr(), _p(w), pw, _p(g), pg, _p(bg), pbg,
                  float(eps), 0, 0, 1.0, mu.numel(), out.data_ptr(), scr.data_ptr(), nb, self.op._s())

    def mean_counted(self, a, w, pw):
        scr, nb = self._scr(a.numel())
        _lib.call("dfx_mean_counted", a.data_ptr(), _p(w), pw, a.numel(), self.out.data_ptr(), scr.data_ptr(), nb,
                  self.op._s())
        s, n = self.out[:2].tolist()
        return s, n

    def ls_residual(self, ax, b, w, pw, clip, delta):
        """ax <- w (ax - b) (clipped to [-delta, delta] if clip) in place; returns the sum of squares before the
        clip (float64)."""
        scr, nb = self._scr(ax.numel())
        _lib.call("dfx_ls_residual", ax.data_ptr(), b.data_ptr(), _p(w), pw, int(clip), float(delta), ax.numel(),
                  self.out.data_ptr(), scr.data_ptr(), nb, self.op._s())
        return float(self.out[0].item())

    def dot(self, x, y=None):
        scr, nb = self._scr(x.numel())
        _lib.call("dfx_dot_f64", x.data_ptr(), _p(y), x.numel(), self.out.data_ptr(), scr.data_ptr(), nb,
                  self.op._s())
        return float(self.out[0].item())


def _p(t):
    return None if t is None else t.data_ptr()


def as_device_data(b, dshape, device):
    if is_device(b):
        return check_device(b, dshape, "b")
    h = np.ascontiguousarray(b, dtype=np.float32)
    if h.shape != tuple(dshape):
        raise ValueError(f"b must have shape {tuple(dshape)}, not {h.shape}")
    from .streaming import host_copier
    out = torch.empty(tuple(dshape), dtype=torch.float32, device=device)
    host_copier().to_device(h, out)
    return out
