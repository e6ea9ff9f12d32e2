"""FISTAPoisson: FISTA in the separable-quadratic-surrogate metric with backtracking for the Poisson deviance, on a B200.

Drop-in for diffractom's FISTAPoisson (optimization/fista_poisson.py:311-...) for device-resident arrays: the same
model f(x) = sum_i w_i / g_i [mu_i' - b_i + b_i log(b_i / mu_i')], mu' = max(A x, 0) + bg + eps g, the same metric
D = 1 / A^T(c A 1_S) (c the Poisson curvature at the prediction), the weighted-least-squares start, the descent-lemma
test with a metric refresh at the extrapolated point and step halving, function-value restarts, the refresh
schedule, the prediction of the extrapolated point formed from the last two predictions, and the same state dict.
All element-wise work and the float64 sums run in this package's CUDA kernels; the scalars of the control flow are
read back per iteration, as in the reference.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .arrays import as_host, check_device, is_device, on_op_stream
from .streaming import host_copier
from .solvers import Reducer, as_device_data, periodic, support_mask_to_device

DEFAULT_REFRESH = (5, 10, 20, 40, 80, 160, 320, 640, 1280, 2560, 5120)


def _p(t):
    return None if t is None else t.data_ptr()


class FISTAPoisson:
    """min_x sum_i w_i / g_i [mu_i' - b_i + b_i log(b_i / mu_i')] + lam sum(x), x >= 0 in the support (module
    docstring)."""

    def __init__(self, operator, prox_kind="nonneg", lam=0.0, support="fov", eps_counts=1e-3, floor_counts=1.0,
                 refresh=DEFAULT_REFRESH, refresh_on_failure=True, max_backtracks=60, start="wls", n_start=20):
        if prox_kind not in ("nonneg", "nonneg_l1"):
            raise ValueError("FISTAPoisson supports prox_kind 'nonneg' and 'nonneg_l1' (element-wise proximal "
                             "operators in the diagonal metric)")
        if start not in ("wls", "uniform", "x0"):
            raise ValueError("start must be 'wls', 'uniform' or 'x0'")
        self.op = operator
        self.ctx, self.queue = operator.ctx, operator.queue
        self.prox_kind = prox_kind
        self.lam = float(lam) if prox_kind == "nonneg_l1" else 0.0
        self.eps_counts = float(eps_counts)
        self.floor_counts = float(floor_counts)
        self.refresh = tuple(int(r) for r in refresh)
        self.max_backtracks = int(max_backtracks)
        self.refresh_on_failure = bool(refresh_on_failure)
        self.start = start
        self.n_start = int(n_start)
        self._mode = 0
        self.adjoint_scale = 1.0
        self.support_gpu = support_mask_to_device(operator, support, operator.device)
        self.state = None

    # ---- helpers
    def _supp(self):
        return (None, 0) if self.support_gpu is None else (self.support_gpu.data_ptr(), self.op.npix)

    def _scr(self, n):
        nb = self.op._lib.dfx_reduce_scratch_bytes(int(n))
        return self.op.scratch(nb), nb

    def _sums(self, name, *args, n, k):
        scr, nb = self._scr(n)
        _lib.call(name, *args, self.red.out.data_ptr(), scr.data_ptr(), nb, self.op._s())
        return self.red.out[:k].tolist()

    def _data_term(self, mu, write_grad):
        return self.red.deviance(mu, self.b, self.w, self.pw, self.g, self.pg, self.bg, self.pbg, self.eps_counts,
                                 write_grad=write_grad, mode=self._mode, floor_counts=self.floor_counts)

    def _copy(self, src, dst):
        _lib.call("dfx_copy_f32", src.data_ptr(), dst.data_ptr(), src.numel(), self.op._s())

    def _ones_forward(self, scratch, x_tmp):
        sp, npx = self._supp()
        _lib.call("dfx_support_ones", x_tmp.data_ptr(), sp, npx, x_tmp.numel(), self.op._s())
        self.op.direct_cl(x_tmp, scratch)

    def _metric(self, mu, scratch, x_tmp, D):
        """D = 1 / A^T(c A 1_S), c the curvature at mu (fista_poisson.py:393-412); scratch and x_tmp overwritten."""
        sp, npx = self._supp()
        self._ones_forward(scratch, x_tmp)
        u_r = self._sums("dfx_times_curvature", scratch.data_ptr(), mu.data_ptr(), self.b.data_ptr(), _p(self.w),
                         self.pw, _p(self.g), self.pg, _p(self.bg), self.pbg, self.floor_counts, self._mode,
                         scratch.numel(), n=scratch.numel(), k=1)[0]
        self.op.adjoint_cl(scratch, x_tmp)
        at_u = self._sums("dfx_support_sum", x_tmp.data_ptr(), sp, npx, x_tmp.numel(), n=x_tmp.numel(), k=1)[0]
        if u_r > 0 and at_u > 0:
            self.adjoint_scale = at_u / u_r
        _lib.call("dfx_invert_metric", D.data_ptr(), x_tmp.data_ptr(), sp, npx, D.numel(), self.op._s())

    # ---- run
    @on_op_stream
    def run(self, x0, b, niter, weights=None, gain=None, background=None, verbose=0, diagnostics_interval=10,
            state=None, callback=None):
        """As diffractom's FISTAPoisson.run (fista_poisson.py:414-...) for a CUDA x0 (updated in place) or a NumPy
        x0 (uploaded; the result is copied back into it)."""
        t_start = time.perf_counter()
        op = self.op
        dev = op.device
        s = op._s()
        cshape, dshape = tuple(op.coeff_shape), tuple(op.data_shape)
        host_x0 = None
        if is_device(x0):
            x = check_device(x0, cshape, "x0")
        else:
            host_x0 = as_host(x0, cshape, "x0", writeable=True)
            x = torch.empty(cshape, dtype=torch.float32, device=dev)
            host_copier().to_device(host_x0, x)
        self.b = as_device_data(b, dshape, dev)
        self.w, self.pw = periodic(weights, dshape, "weights", dev)
        self.g, self.pg = periodic(gain, dshape, "gain", dev)
        self.bg, self.pbg = periodic(background, dshape, "background", dev)
        if self.pg and float(self.g.min().item()) <= 0:
            raise ValueError("the gain must be positive everywhere")
        self.red = Reducer(op)
        new = lambda shape: torch.empty(shape, dtype=torch.float32, device=dev)
        xn, grad, D = new(cshape), new(cshape), new(cshape)
        Ax, Axn, Ay = new(dshape), new(dshape), new(dshape)
        sp, npx = self._supp()
        nx, nd = x.numel(), Ax.numel()
        _lib.call("dfx_project_support", x.data_ptr(), sp, npx, nx, s)
        zero_start = state is None and float(x.max().item()) == 0.0
        wls_until = 0
        if self.start == "wls" and self.n_start > 0:
            if zero_start:
                wls_until = self.n_start
            elif state is not None and state.get("wls_until", 0) > int(state["it"]):
                wls_until = int(state["wls_until"])
        self._mode = 1 if wls_until else 0
        if zero_start and self.start == "uniform":
            self._ones_forward(Axn, xn)
            sb, sa = self._sums("dfx_weighted_sums", Axn.data_ptr(), self.b.data_ptr(), _p(self.w), self.pw, nd,
                                n=nd, k=2)
            if sa > 0 and sb > 0:
                self._copy(xn, x)
                _lib.call("dfx_scale_f32", x.data_ptr(), float(np.float32(sb / sa)), nx, s)

        it0, t_mom, theta = 0, 1.0, 1.0
        if state is not None:
            it0, t_mom, theta = int(state["it"]), float(state["t"]), float(state["theta"])
            y = torch.as_tensor(as_host(state["y"], cshape, "state['y']"), device=dev)
        else:
            y = new(cshape)
            self._copy(x, y)
        op.direct_cl(x, Ax)
        if state is not None:
            op.direct_cl(y, Ay)
        else:
            self._copy(Ax, Ay)
        self._metric(Ax, Axn, xn, D)
        t_metric = time.perf_counter() - t_start
        f_x = self._data_term(Ax, False)
        F_x = f_x + self.lam * (self.red.dot(x) if self.lam else 0.0)
        self.iter_stats = []
        n_bt_total, n_restart, n_metric = 0, 0, 0
        for k in range(niter):
            it = it0 + k + 1
            f_y = self._data_term(Ay, True)          # Ay now holds df/dmu at y
            op.adjoint_cl(Ay, grad)
            theta = min(1.0, 2.0 * theta)
            n_bt = 0
            local = False
            while True:
                _lib.call("dfx_metric_step", xn.data_ptr(), y.data_ptr(), grad.data_ptr(), D.data_ptr(),
                          float(np.float32(theta)), float(np.float32(self.lam)), nx, s)
                op.direct_cl(xn, Axn)
                f_n = self._data_term(Axn, False)
                lin_adj, q1, xsum = self._sums("dfx_step_sums", xn.data_ptr(), y.data_ptr(), grad.data_ptr(),
                                               D.data_ptr(), nx, n=nx, k=3)
                lin = lin_adj / self.adjoint_scale
                quad = q1 / (theta * self.adjoint_scale)
                if f_n <= f_y + lin + 0.5 * quad + 1e-6 * abs(f_y) or quad == 0.0:
                    break
                n_bt += 1
                if not local and self.refresh_on_failure:
                    op.direct_cl(y, Axn)
                    self._metric(Axn, Ay, xn, D)
                    local, theta = True, 1.0
                    n_metric += 1
                    continue
                theta *= 0.5
                if n_bt > self.max_backtracks:
                    raise RuntimeError(f"FISTAPoisson: no sufficient decrease after {n_bt} step reductions (iteration "
                                       f"{it}, mode {self._mode}: f(y) {f_y:.10e}, f(x_new) {f_n:.10e}, derivative "
                                       f"{lin:.4e}, quadratic term {quad:.4e}, theta {theta:.3g})")
            n_bt_total += n_bt
            F_n = f_n + self.lam * xsum
            restarted = F_n > F_x
            if restarted:
                t_mom = 1.0
                n_restart += 1
            t_new = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t_mom * t_mom))
            beta = float(np.float32((t_mom - 1.0) / t_new))
            t_mom = t_new
            _lib.call("dfx_extrapolate", y.data_ptr(), xn.data_ptr(), x.data_ptr(), beta, nx, s)
            _lib.call("dfx_extrapolate", Ay.data_ptr(), Axn.data_ptr(), Ax.data_ptr(), beta, nd, s)
            self._copy(xn, x)
            Ax, Axn = Axn, Ax
            f_x, F_x = f_n, F_n
            switch = self._mode == 1 and it >= wls_until
            if switch:
                self._mode = 0
                f_x = self._data_term(Ax, False)
                F_x = f_x + self.lam * xsum
            refreshed = (it in self.refresh or switch) and k + 1 < niter and self._mode == 0
            if refreshed:
                self._metric(Ax, Axn, xn, D)
                t_mom, theta = 1.0, 1.0
                self._copy(x, y)
                self._copy(Ax, Ay)
            elif it % 50 == 0:
                op.direct_cl(y, Ay)
            stats = {"iter": it, "f": f_n, "obj": F_n, "phase": "wls" if it <= wls_until else "poisson",
                     "theta": theta, "backtracks": n_bt, "local_metric": local, "restart": bool(restarted),
                     "metric_refresh": bool(refreshed), "time": time.perf_counter() - t_start}
            self.iter_stats.append(stats)
            stop = bool(callback(it, x, stats)) if callback is not None else False
            if verbose and (k == 0 or (k + 1) % diagnostics_interval == 0 or k + 1 == niter or stop):
                print(f"[iter {it:5d}] f={f_n:.8e} obj={F_n:.8e} theta={theta:.3g} backtracks={n_bt_total} "
                      f"metric updates={n_metric} restarts={n_restart} {time.perf_counter() - t_start:.1f} s",
                      flush=True)
            if stop:
                break
        done = len(self.iter_stats)
        y_host = np.empty(tuple(y.shape), np.float32)
        host_copier().to_host(y, y_host)
        self.state = {"it": it0 + done, "t": t_mom, "theta": theta, "y": y_host, "wls_until": wls_until}
        self.final_stats = {"niter": done, "final_f": f_x, "final_obj": F_x, "backtracks": n_bt_total,
                            "metric_updates_on_failure": n_metric, "adjoint_scale": self.adjoint_scale,
                            "restarts": n_restart, "metric_setup_s": t_metric, "time": time.perf_counter() - t_start}
        self.b = self.w = self.g = self.bg = None
        if host_x0 is not None:
            host_copier().to_host(x, host_x0)
            return host_x0
        return x
