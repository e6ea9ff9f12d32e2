"""PoissonTerm: the Poisson data term of a prediction pred = A x on the device (diffractom's
optimization/poisson_term.py), for the refiners and solvers that work with a prediction:

    f = sum_i fit_i w_i / g_i [ mu_i - b_i + b_i log(b_i / mu_i) ],   mu_i = max(pred_i, 0) + bg_i + eps_counts g_i

fit_i: the angle of point i is fitted. w, g, bg per segment, per (translation, segment) or data-shaped (the solvers'
conventions; None: w = g = 1, bg = 0). The deviance is a float64 sum (dfx_poisson_value_grad); the gradient and
Fisher curvature, the EM ratio and w / g are one elementwise kernel (dfx_poisson_term). The fitted angles enter as
weights: with fit_rows, w is expanded to the data shape and zero on the other angles.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .arrays import as_host, check_device, is_device
from .solvers import periodic


class PoissonTerm:
    def __init__(self, queue, data_shape, b, weights=None, gain=None, background=None, fit_rows=None,
                 eps_counts=1e-3):
        """queue: the CUDA stream to work on (None: the current stream); b: counts (CUDA tensor or NumPy);
        fit_rows: bool (N_Omega,) or indices of the fitted angles (None: all) (poisson_term.py:27-48)."""
        self.dshape = dshape = tuple(int(d) for d in data_shape)
        dev = b.device if is_device(b) else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.queue = queue
        self.b = check_device(b, dshape, "b") if is_device(b) else torch.as_tensor(as_host(b, dshape, "b"), device=dev)
        fit = np.ones(dshape[0], bool)
        if fit_rows is not None:
            rr = np.asarray(fit_rows)
            fit[:] = False
            fit[np.flatnonzero(rr) if rr.dtype == bool else rr.astype(np.int64)] = True
        self.fit_host = fit
        n = int(np.prod(dshape))
        if fit.all():
            self.w, self.pw = periodic(weights, dshape, "weights", dev)
        else:
            w = np.ones(1, np.float32) if weights is None else \
                (weights.cpu().numpy() if is_device(weights) else np.asarray(weights, np.float32))
            wf = np.resize(np.asarray(w, np.float32).ravel(), n).reshape(dshape[0], -1)
            wf[~fit] = 0.0
            self.w, self.pw = torch.as_tensor(wf.ravel(), device=dev), n
        self.g, self.pg = periodic(gain, dshape, "gain", dev)
        self.bg, self.pbg = periodic(background, dshape, "background", dev)
        if self.pg and float(self.g.min().item()) <= 0:
            raise ValueError("the gain must be positive everywhere")
        self.eps = float(np.float32(eps_counts))
        self.n = n
        self._out = torch.zeros(4, dtype=torch.float64, device=dev)
        self._scr = torch.empty(0, dtype=torch.uint8, device=dev)

    def _s(self):
        st = self.queue if self.queue is not None else torch.cuda.current_stream(self.device)
        return ctypes.c_void_p(st.cuda_stream)

    @staticmethod
    def _p(t):
        return None if t is None else t.data_ptr()

    def deviance(self, pred):
        """The deviance of the prediction (data-shaped CUDA tensor) on the fitted angles (float64)."""
        check_device(pred, self.dshape, "pred")
        lib = _lib.lib()
        nb = lib.dfx_reduce_scratch_bytes(self.n)
        if self._scr.numel() < nb:
            self._scr = torch.empty(nb, dtype=torch.uint8, device=self.device)
        _lib.call("dfx_poisson_value_grad", pred.data_ptr(), self.b.data_ptr(), self._p(self.w), self.pw,
                  self._p(self.g), self.pg, self._p(self.bg), self.pbg, self.eps, 0, 0, 1.0, self.n,
                  self._out.data_ptr(), self._scr.data_ptr(), nb, self._s())
        return float(self._out[0].item())

    def n_points(self):
        """The number of counted data points (fitted angle, weight != 0)."""
        if self.w is None:
            return int(self.fit_host.sum()) * (self.n // self.dshape[0])
        w = np.resize(self.w.cpu().numpy(), self.n).reshape(self.dshape[0], -1)[self.fit_host]
        return int(np.count_nonzero(w))

    def _term(self, pred, mode, r, c=None, floor=0.25):
        check_device(r, self.dshape, "out")
        if c is not None:
            check_device(c, self.dshape, "c")
        if pred is not None:
            check_device(pred, self.dshape, "pred")
        _lib.call("dfx_poisson_term", self._p(pred), self.b.data_ptr(), self._p(self.w), self.pw, self._p(self.g),
                  self.pg, self._p(self.bg), self.pbg, self.eps, float(floor), int(mode), r.data_ptr(), self._p(c),
                  self.n, self._s())

    def grad_curv(self, pred, r, c, floor_counts=0.25):
        """r = d f / d pred = w/g (1 - b/mu) and c = w / (g max(mu, floor_counts g)) (the Fisher information, mu at
        least floor_counts photons) on the fitted angles, 0 elsewhere (poisson_term.py:100-104)."""
        self._term(pred, 0, r, c, floor_counts)

    def em_ratio(self, pred, out):
        """out = w b / (g mu) on the fitted angles (0 elsewhere)."""
        self._term(pred, 1, out)

    def weight_over_gain(self, out):
        """out = w / g on the fitted angles (0 elsewhere)."""
        self._term(None, 2, out)
