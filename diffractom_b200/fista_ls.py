"""FISTAL2 and FISTAHuber: FISTA for 0.5 ||A x - b||^2 (+ an element-wise prox) and its Huber variant, on a B200.

Drop-ins for diffractom's FISTAL2 (optimization/fista_l2.py) and FISTAHuber (optimization/fista_huber.py) with the
fused update (fused_update.py): the same arguments, iteration, step size tau = 1/L, momentum
t' = (1 + sqrt(1 + 4 t^2)) / 2, beta = (t - 1) / t', diagnostics and stats. One iteration:

    Ax = A y                    (for iterations after the first: projected batch by batch in the previous pass)
    r = w (Ax - b), f = 0.5 sum r^2, r <- clip(r, -delta, delta)          (Huber; FISTAL2: no weights, no clip)
    per orientation batch: g = A^T r (batch);  v = prox(y - tau g), 0 outside the support;
                           y = v + beta (v - x);  x = v;  then A y (batch) into the next iteration's Ax

x and y live in the operator's channel-fastest batch layout (no gather / scatter per iteration), on the device for
a CUDA x0, or in pinned host memory streamed through two device slots for a NumPy x0 (as the reference streams
them). The forward projections read the ray table restricted to the support (y is zero outside it). Sums are
float64 and reproducible (fixed-order partials). prox_kind 'nonneg_tv' (the TV prox couples the pixels of an image)
is not provided.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .arrays import as_host, check_device, is_device, on_op_stream
from .solvers import Reducer, as_device_data, periodic, support_mask_to_device
from .streaming import BatchPipeline, CoeffArray, KMajorStaging

PROX_CODES = {"nonneg": 0, "l1": 1, "nonneg_l1": 2}


class FISTAHuber:
    """FISTA for the Huber loss of the (weighted) residual with an element-wise prox (module docstring)."""

    clip = True
    weighted = True

    def __init__(self, operator, prox_kind="nonneg", lam=0.0, L=None, tau=None, tv_niter=50, huber_delta=1e-2,
                 support="fov", fused=True, stream_threads=None, fuse_next_forward=True):
        """Arguments as diffractom's FISTAHuber (fista_huber.py:152-...). fused: the update is always fused into the
        adjoint pass (the unfused variant computes the same values with four coefficient arrays); stream_threads is
        accepted (the host copies of the streamed path are pinned DMA copies)."""
        if prox_kind == "nonneg_tv":
            raise NotImplementedError("prox_kind 'nonneg_tv' is not provided (the TV prox is not element-wise)")
        if prox_kind not in PROX_CODES:
            raise ValueError(f"Unknown prox_kind: {prox_kind}")
        self.op = operator
        self.ctx, self.queue = operator.ctx, operator.queue
        self.prox_kind = prox_kind
        self.lam = float(lam)
        if tau is None:
            if L is None:
                raise ValueError("Provide either L or tau")
            self.tau = 1.0 / float(L)
        else:
            self.tau = float(tau)
        self.tv_niter = int(tv_niter)
        self.huber_delta = float(huber_delta)
        self.fused = True
        self.stream_threads = stream_threads
        self.fuse_next_forward = bool(fuse_next_forward)
        self.support_gpu = support_mask_to_device(operator, support, operator.device)
        self.iter_stats, self.final_stats = [], {}

    @on_op_stream
    def run(self, x0_gpu, out_gpu, niter, weights=None, verbose=0, diagnostics_interval=1):
        """As diffractom's FISTAHuber.run (fista_huber.py:279-...): x0_gpu a CUDA tensor (updated in place and
        returned) or a NumPy array (x and y streamed from host memory; updated in place if C-contiguous float32,
        else a converted copy; returned); out_gpu the data b; weights one per segment (N_seg elements) or per data
        point."""
        if getattr(self.op, "coefficient_layout", "dense") == "local":
            return self._run_flat(x0_gpu, out_gpu, niter, weights, verbose, diagnostics_interval)
        t_start = time.perf_counter()
        op = self.op
        dev = op.device
        s = op._s()
        cshape, dshape = tuple(op.coeff_shape), tuple(op.data_shape)
        npix, be, nbt = op.npix, op.batch_elems(), len(op.batches)
        niter = int(niter)
        x_on_gpu = is_device(x0_gpu)
        x_dev = check_device(x0_gpu, cshape, "x0") if x_on_gpu else None
        host_x = None if x_on_gpu else as_host(x0_gpu, cshape, "x0", writeable=True)
        b = as_device_data(out_gpu, dshape, dev)
        w, pw = periodic(weights, dshape, "weights", dev) if self.weighted else (None, 0)
        use_w = pw != 0
        supp = self.support_gpu
        sp = None if supp is None else supp.data_ptr()
        ray = op.support_ray_table(supp) if supp is not None else None
        red = Reducer(op)

        X, Y = CoeffArray(op, "x", x_on_gpu), CoeffArray(op, "y", x_on_gpu)
        pipe = BatchPipeline(op)
        stage = None if x_on_gpu else KMajorStaging(op)
        if x_on_gpu:
            op.to_batches(x_dev, X.dev)
        else:
            stage.load(host_x.reshape(-1), X, pipe)

        def start(ib, sl):                      # x inside the support (padding 0), y = x
            xp = X.ptr(ib, sl)
            _lib.call("dfx_batch_support", xp, None, sp, npix, op.Kstride, op.batches[ib]["K_batch"], 0.0, 3, s)
            if x_on_gpu:
                _lib.call("dfx_copy_f32", xp, Y.ptr(ib, sl), be, s)

        pipe.run([X], [X], start)
        if not x_on_gpu:
            pipe.synchronize()
            Y.host.copy_(X.host)

        g_batch = torch.empty(be, dtype=torch.float32, device=dev)
        fub = int(op._lib.dfx_fista_ls_blocks())
        part = torch.empty(nbt * fub * 3, dtype=torch.float64, device=dev)
        sums = torch.zeros(3, dtype=torch.float64, device=dev)
        Ax = torch.empty(dshape, dtype=torch.float32, device=dev)
        Ax_next = None
        if self.fuse_next_forward and niter > 1:
            free, _ = torch.cuda.mem_get_info(dev)
            if free > Ax.numel() * 4 + (1 << 30):
                Ax_next = torch.empty(dshape, dtype=torch.float32, device=dev)
        code = PROX_CODES[self.prox_kind]
        lt = float(np.float32(self.lam * self.tau))
        tau = self.tau
        t = 1.0
        self.iter_stats = []
        have_ax = False

        def forward_y(into):
            op._fill(into, 0.0)
            pipe.run([Y], [], lambda ib, sl: op._direct_batch_k(Y.ptr(ib, sl), ib, into, ray=ray))

        for it in range(niter):
            if not have_ax:
                forward_y(Ax)
            r2 = red.ls_residual(Ax, b, w, pw, int(self.clip), self.huber_delta)
            fval = 0.5 * r2
            t_new = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t * t))
            beta = (t - 1.0) / t_new
            nxt = Ax_next if (Ax_next is not None and it + 1 < niter) else None
            if nxt is not None:
                op._fill(nxt, 0.0)

            def update(ib, sl, beta=beta, nxt=nxt):
                op._adjoint_batch_k(Ax, ib, g_batch.data_ptr())
                _lib.call("dfx_fista_ls_update", g_batch.data_ptr(), X.ptr(ib, sl), Y.ptr(ib, sl), sp, npix,
                          op.Kstride, op.batches[ib]["K_batch"], float(tau), float(beta), lt, code,
                          part.data_ptr() + 8 * 3 * fub * ib, s)
                if nxt is not None:
                    op._direct_batch_k(Y.ptr(ib, sl), ib, nxt, ray=ray)

            pipe.run([X, Y], [X, Y], update)
            _lib.call("dfx_sum_partials", part.data_ptr(), nbt * fub, 3, sums.data_ptr(), s)
            gsq, xsq, xabs = (float(v) for v in sums.tolist())
            if nxt is not None:
                Ax, Ax_next = nxt, Ax
                have_ax = True
            else:
                have_ax = False
            t = t_new
            gval = self.lam * xabs if self.prox_kind in ("l1", "nonneg_l1") and self.lam != 0.0 else 0.0
            stats = {"iter": it + 1, "f": fval, "g": gval, "obj": fval + gval, "xnorm": float(np.sqrt(xsq)),
                     "gradnorm": float(np.sqrt(gsq)), "beta": beta, "tau": tau, "tv_residual": None,
                     "time": time.perf_counter() - t_start, "weighted": use_w}
            self.iter_stats.append(stats)
            if verbose and ((it + 1) % diagnostics_interval == 0 or it == 0 or it == niter - 1):
                print(f"[iter {it + 1:4d}/{niter}] obj={stats['obj']:.6e}  f={fval:.6e}  g={gval:.6e}  "
                      f"||x||={stats['xnorm']:.6e}  ||grad||={stats['gradnorm']:.6e}  tau={tau:.3e}  "
                      f"beta={beta:.3e}" + ("  (weighted)" if use_w else ""), flush=True)

        last = self.iter_stats[-1] if self.iter_stats else {}
        self.final_stats = {"next_forward_fused": Ax_next is not None, "niter": niter,
                            "final_f": last.get("f"), "final_g": last.get("g"), "final_obj": last.get("obj"),
                            "final_xnorm": last.get("xnorm"), "final_gradnorm": last.get("gradnorm"),
                            "weighted": use_w}
        if x_on_gpu:
            op.from_batches(X.dev, x_dev)
            out = x_dev
        else:
            stage.store(X, host_x.reshape(-1), pipe)
            out = host_x
        pipe.synchronize()
        return out


    def _run_flat(self, x0, out_gpu, niter, weights, verbose, diagnostics_interval):
        """The same iteration on a local-basis operator's flat coefficients (x, y, the gradient: n_coef each, on the
        device; the support is the operator's): forward and adjoint through the operator, the update of the whole
        vector by the same kernel (a single 4-channel "batch" of n_coef / 4 cells)."""
        t_start = time.perf_counter()
        op = self.op
        dev = op.device
        s = op._s()
        n, dshape = int(op.n_coef), tuple(op.data_shape)
        n4 = -(-n // 4) * 4
        x_on_gpu = is_device(x0)
        x_dev = check_device(x0, (n,), "x0") if x_on_gpu else None
        host_x = None if x_on_gpu else as_host(x0, (n,), "x0", writeable=True)
        b = as_device_data(out_gpu, dshape, dev)
        w, pw = periodic(weights, dshape, "weights", dev) if self.weighted else (None, 0)
        red = Reducer(op)
        mask = torch.as_tensor(op.coefficient_mask(), device=dev)
        x = torch.zeros(n4, dtype=torch.float32, device=dev)
        x[:n] = (x_dev if x_on_gpu else torch.as_tensor(host_x, device=dev)) * mask     # inside the support
        y, g = x.clone(), torch.zeros(n4, dtype=torch.float32, device=dev)
        fub = int(op._lib.dfx_fista_ls_blocks())
        part = torch.empty(fub * 3, dtype=torch.float64, device=dev)
        sums = torch.zeros(3, dtype=torch.float64, device=dev)
        Ax = torch.empty(dshape, dtype=torch.float32, device=dev)
        code, lt, tau, t = PROX_CODES[self.prox_kind], float(np.float32(self.lam * self.tau)), self.tau, 1.0
        self.iter_stats = []
        for it in range(int(niter)):
            op.direct_cl(y[:n], Ax)
            fval = 0.5 * red.ls_residual(Ax, b, w, pw, int(self.clip), self.huber_delta)
            t_new = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t * t))
            beta = (t - 1.0) / t_new
            op.adjoint_cl(Ax, g[:n])
            _lib.call("dfx_fista_ls_update", g.data_ptr(), x.data_ptr(), y.data_ptr(), None, n4 // 4, 4, 4,
                      float(tau), float(beta), lt, code, part.data_ptr(), s)
            _lib.call("dfx_sum_partials", part.data_ptr(), fub, 3, sums.data_ptr(), s)
            gsq, xsq, xabs = (float(v) for v in sums.tolist())
            t = t_new
            gval = self.lam * xabs if self.prox_kind in ("l1", "nonneg_l1") and self.lam != 0.0 else 0.0
            stats = {"iter": it + 1, "f": fval, "g": gval, "obj": fval + gval, "xnorm": float(np.sqrt(xsq)),
                     "gradnorm": float(np.sqrt(gsq)), "beta": beta, "tau": tau, "tv_residual": None,
                     "time": time.perf_counter() - t_start, "weighted": pw != 0}
            self.iter_stats.append(stats)
            if verbose and ((it + 1) % diagnostics_interval == 0 or it == 0 or it + 1 == niter):
                print(f"[iter {it + 1:4d}/{niter}] obj={stats['obj']:.6e}  f={fval:.6e}", flush=True)
        last = self.iter_stats[-1] if self.iter_stats else {}
        self.final_stats = {"next_forward_fused": False, "niter": int(niter), "final_f": last.get("f"),
                            "final_g": last.get("g"), "final_obj": last.get("obj"), "final_xnorm": last.get("xnorm"),
                            "final_gradnorm": last.get("gradnorm"), "weighted": pw != 0}
        if x_on_gpu:
            x_dev.copy_(x[:n])
            return x_dev
        host_x[...] = x[:n].cpu().numpy()
        return host_x


class FISTAL2(FISTAHuber):
    """FISTA for 0.5 ||A x - b||^2 with an element-wise prox (fista_l2.py:104-...)."""

    clip = False
    weighted = False

    def __init__(self, operator, prox_kind="nonneg", lam=0.0, L=None, tau=None, tv_niter=50, support="fov",
                 fused=True, stream_threads=None, fuse_next_forward=True):
        super().__init__(operator, prox_kind=prox_kind, lam=lam, L=L, tau=tau, tv_niter=tv_niter, support=support,
                         fused=fused, stream_threads=stream_threads, fuse_next_forward=fuse_next_forward)

    def run(self, x0_gpu, out_gpu, niter, verbose=0, diagnostics_interval=1):
        """As diffractom's FISTAL2.run (fista_l2.py:241-...)."""
        return super().run(x0_gpu, out_gpu, niter, None, verbose, diagnostics_interval)
