"""OSEMPoisson and PDHGPoisson: the Poisson problem of FISTAPoisson / SPDHGPoisson with ordered-subsets EM and with
Chambolle-Pock, on a B200 (diffractom's optimization/osem_poisson.py and optimization/pdhg_poisson.py).

OSEM (Shepp & Vardi 1982, Hudson & Larkin 1994), for the next subset m of a random permutation every epoch:

    x <- x A_m^T(w b / (g mu')) / (A_m^T(w / g) + lam),   mu' = max(A_m x, 0) + bg + eps_counts g

(the EM ratio and w / g from PoissonTerm, the update dfx_osem_update; one sensitivity A_m^T(w / g) per subset kept
with store_sensitivities). PDHG (Chambolle & Pock 2011, diagonal preconditioning of Pock & Chambolle 2011):

    y <- prox_{Sigma F*}(y + Sigma A x_bar);  x_new = max(0, x - T (A^T y + lam));  x_bar = 2 x_new - x

with Sigma = sigma0 / (A 1_S), T = tau0 / (A^T 1_counted), tau0 sigma0 = 1, rho = sigma0 / tau0 (dfx_pdhg_*). Both
run on the operator's direct_cl / adjoint_cl (dense or local coefficients); all their arrays are on the device (a
NumPy x0 is uploaded and the result copied back: the PDHG state is not streamed from host memory).
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .arrays import as_host, check_device, is_device, on_op_stream
from .poisson_term import PoissonTerm
from .solvers import Reducer, as_device_data, periodic, support_mask_to_device
from .streaming import host_copier

__all__ = ["OSEMPoisson", "PDHGPoisson"]

RHO_AUTO = 3e4


def _x_in(op, x0):
    """(device x, host array or None) for a CUDA or NumPy x0."""
    cshape = tuple(op.coeff_shape)
    if is_device(x0):
        return check_device(x0, cshape, "x0"), None
    host = as_host(x0, cshape, "x0", writeable=True)
    x = torch.empty(cshape, dtype=torch.float32, device=op.device)
    host_copier().to_device(host, x)
    return x, host


class OSEMPoisson:
    """Ordered-subsets EM for the Poisson deviance (module docstring; osem_poisson.py:32-185)."""

    def __init__(self, operator, subsets=8, lam=0.0, support="fov", eps_counts=1e-3, seed=0,
                 store_sensitivities=True):
        """As diffractom's OSEMPoisson: subsets an int, a list of angle-index arrays or None (MLEM over all angles);
        lam >= 0 the l1 weight; support "fov" / None / an (Ny, Nx) array (the local basis uses its allowed
        coefficients); seed the subset order."""
        self.op = operator
        self.ctx, self.queue = operator.ctx, operator.queue
        if subsets is None:
            self.subsets, self.M = None, 1
        else:
            self.subsets = operator.set_omega_subsets(subsets)
            self.M = len(self.subsets)
        self.lam = float(lam)
        if self.lam < 0:
            raise ValueError("lam must be >= 0")
        self.eps_counts = float(eps_counts)
        self.rng = np.random.default_rng(seed)
        self.store_sensitivities = bool(store_sensitivities)
        if getattr(operator, "coefficient_layout", "dense") == "local":
            self.mask = torch.as_tensor((np.asarray(operator.coefficient_mask()) > 0).astype(np.uint8),
                                        device=operator.device)
        else:
            self.mask = support_mask_to_device(operator, support, operator.device)
        self.pmask = 0 if self.mask is None else int(self.mask.numel())
        self.iter_stats = []
        self.final_f = None
        self.start_floor_used = None

    def _fwd(self, x, out, m):
        self.op.direct_cl(x, out) if self.subsets is None else self.op.direct_cl(x, out, subset=m)

    def _adj(self, r, out, m):
        self.op.adjoint_cl(r, out) if self.subsets is None else self.op.adjoint_cl(r, out, subset=m)

    @on_op_stream
    def run(self, x0, b, n_epochs, weights=None, gain=None, background=None, start_floor=0.01, verbose=0,
            diagnostics_interval=1, callback=None):
        """As diffractom's OSEMPoisson.run (osem_poisson.py:95-185): a CUDA x0 is updated in place and returned, a
        NumPy x0 gives a new NumPy array; start_floor lifts every allowed coefficient to that fraction of the median
        positive one (a flat start matching the fitted data's total when there is none)."""
        t0 = time.perf_counter()
        op = self.op
        cshape, dshape = tuple(op.coeff_shape), tuple(op.data_shape)
        x, host = _x_in(op, x0)
        fit = None
        if self.subsets is not None:
            fit = np.zeros(dshape[0], bool)
            for s_ in self.subsets:
                fit[np.asarray(s_, np.int64)] = True
        pt = PoissonTerm(None, dshape, as_device_data(b, dshape, op.device), weights, gain, background, fit,
                         self.eps_counts)                # the operator's stream is current here
        pred = torch.zeros(dshape, dtype=torch.float32, device=op.device)
        r = torch.empty_like(pred)
        wg = torch.empty_like(pred)
        pt.weight_over_gain(wg)
        back = torch.empty(cshape, dtype=torch.float32, device=op.device)
        sens = [torch.empty(cshape, dtype=torch.float32, device=op.device)
                for _ in range(self.M if self.store_sensitivities else 1)]
        if self.store_sensitivities:
            for m in range(self.M):
                self._adj(wg, sens[m], m)
        # start (osem_poisson.py:139-160), on the device: the median of the positive allowed coefficients as NumPy's
        # (the mean of the two middle values for an even count, in float64)
        n = int(np.prod(cshape))
        xf = x.reshape(-1)
        allowed = (self.mask.reshape(-1).bool().repeat(n // self.pmask) if self.pmask
                   else torch.ones(n, dtype=torch.bool, device=op.device))
        xf.masked_fill_(~allowed, 0.0)
        if start_floor:
            pos = xf[xf > 0]
            if pos.numel():
                k = pos.numel()
                lo = float(torch.kthvalue(pos, (k + 1) // 2).values.item())
                hi = float(torch.kthvalue(pos, k // 2 + 1).values.item()) if k % 2 == 0 else lo
                floor = float(start_floor) * (0.5 * (lo + hi) if k % 2 == 0 else lo)
            else:
                st = 0.0
                for m in range(self.M):
                    if not self.store_sensitivities:
                        self._adj(wg, sens[0], m)
                    sm = sens[m if self.store_sensitivities else 0]
                    st += float(sm.reshape(-1)[allowed].double().sum().item())
                tot = float(torch.dot(wg.reshape(-1).double(), pt.b.reshape(-1).double()).item())
                if pt.pbg:
                    bgf = pt.bg.double().repeat(int(np.prod(dshape)) // pt.pbg)
                    tot -= float(torch.dot(wg.reshape(-1).double(), bgf).item())
                floor = max(tot, 0.0) / st if st > 0 else 1.0
            xf.copy_(torch.where(allowed, xf.double().clamp(min=floor), torch.zeros((), dtype=torch.float64,
                                                                                      device=op.device)).float())
            self.start_floor_used = floor
        mp = None if self.mask is None else self.mask.data_ptr()
        self.iter_stats = []
        f = None
        for ep in range(int(n_epochs)):
            order = self.rng.permutation(self.M) if self.M > 1 else [0]
            for m in order:
                m = int(m)
                self._fwd(x, pred, m)
                pt.em_ratio(pred, r)
                self._adj(r, back, m)
                if self.store_sensitivities:
                    sm = sens[m]
                else:
                    self._adj(wg, sens[0], m)
                    sm = sens[0]
                _lib.call("dfx_osem_update", x.data_ptr(), back.data_ptr(), sm.data_ptr(), mp, self.pmask,
                          self.lam, n, op._s())
            stats = {"epoch": ep + 1, "time": time.perf_counter() - t0}
            f = None
            if diagnostics_interval and ((ep + 1) % int(diagnostics_interval) == 0 or ep + 1 == int(n_epochs)):
                op.direct_cl(x, pred)
                f = pt.deviance(pred)
                stats["f"] = f
                if verbose:
                    print(f"OSEM epoch {ep + 1}: deviance {f:.6g} ({stats['time']:.1f} s)", flush=True)
            self.iter_stats.append(stats)
            if callback is not None and callback(ep + 1, x if host is None else x.cpu().numpy(), stats):
                break
        if f is None:
            op.direct_cl(x, pred)
            f = pt.deviance(pred)
        self.final_f = f
        if host is None:
            return x
        out = np.empty(cshape, np.float32)
        host_copier().to_host(x, out)
        return out


class PDHGPoisson:
    """Chambolle-Pock for the Poisson deviance (module docstring; pdhg_poisson.py:121-262)."""

    def __init__(self, operator, prox_kind="nonneg", lam=0.0, support="fov", eps_counts=1e-3, rho="auto"):
        if prox_kind not in ("nonneg", "nonneg_l1"):
            raise ValueError("PDHGPoisson supports prox_kind 'nonneg' and 'nonneg_l1'")
        self.op = operator
        self.ctx, self.queue = operator.ctx, operator.queue
        self.lam = float(lam) if prox_kind == "nonneg_l1" else 0.0
        self.eps_counts = float(eps_counts)
        self.rho = rho if rho == "auto" else float(rho)
        self.support_gpu = support_mask_to_device(operator, support, operator.device)
        self.state = None

    def _deviance(self, mu):
        return self.red.deviance(mu, self.b, self.w, self.pw, self.g, self.pg, self.bg, self.pbg, self.eps_counts)

    @on_op_stream
    def run(self, x0, b, niter, weights=None, gain=None, background=None, verbose=0, diagnostics_interval=10,
            callback=None, state=None):
        """As diffractom's PDHGPoisson.run: a CUDA x0 is updated in place and returned, a NumPy x0 updated in place
        (if C-contiguous float32) and returned; state (x_bar, y, it) continues an earlier run."""
        t_start = time.perf_counter()
        op = self.op
        dev, s = op.device, op._s()
        cshape, dshape = tuple(op.coeff_shape), tuple(op.data_shape)
        x, host = _x_in(op, x0)
        self.b = as_device_data(b, dshape, dev)
        self.w, self.pw = periodic(weights, dshape, "weights", dev)
        self.g, self.pg = periodic(gain, dshape, "gain", dev)
        self.bg, self.pbg = periodic(background, dshape, "background", dev)
        self.red = Reducer(op)
        supp = self.support_gpu
        sp, npix = (None, 0) if supp is None else (supp.data_ptr(), int(supp.numel()))
        rho = self.rho
        if rho == "auto":
            sb, sn = self.red.mean_counted(self.b, self.w, self.pw)
            mean_b = sb / max(sn, 1.0)
            rho = RHO_AUTO / mean_b ** 2 if mean_b > 0 else 1.0
        self.rho_used = float(rho)
        tau0, sigma0 = 1.0 / np.sqrt(rho), np.sqrt(rho)
        nx, nd = x.numel(), int(np.prod(dshape))
        f32 = lambda shape: torch.empty(shape, dtype=torch.float32, device=dev)
        xb, T, grad = f32(cshape), f32(cshape), f32(cshape)
        ydual = torch.zeros(dshape, dtype=torch.float32, device=dev)
        sig, Axb, Ax = f32(dshape), f32(dshape), f32(dshape)
        ptr = lambda t: None if t is None else t.data_ptr()
        # row sums A 1_S (Sigma) and column sums A^T 1 over the counted points (T) (pdhg_poisson.py:209-221)
        _lib.call("dfx_support_ones", xb.data_ptr(), sp, npix, nx, s)
        op.direct_cl(xb, Axb)
        _lib.call("dfx_dual_steps", sig.data_ptr(), Axb.data_ptr(), ptr(self.w), self.pw, float(sigma0), nd, s)
        _lib.call("dfx_set_mask_ones", Axb.data_ptr(), ptr(self.w), self.pw, nd, s)
        op.adjoint_cl(Axb, grad)
        _lib.call("dfx_pdhg_primal_steps", T.data_ptr(), grad.data_ptr(), sp, npix, float(tau0), nx, s)
        _lib.call("dfx_project_support", x.data_ptr(), sp, npix, nx, s)
        if state is not None:
            xb.copy_(torch.as_tensor(as_host(state["x_bar"], cshape, "state['x_bar']")))
            ydual.copy_(torch.as_tensor(as_host(state["y"], dshape, "state['y']")))
        else:
            xb.copy_(x)
        op.direct_cl(x, Ax)
        op.direct_cl(xb, Axb)
        t_setup = time.perf_counter() - t_start
        it0 = int(state["it"]) if state is not None else 0
        self.iter_stats = []
        f = self._deviance(Ax)
        for k in range(int(niter)):
            it = it0 + k + 1
            _lib.call("dfx_pdhg_dual_update", ydual.data_ptr(), Axb.data_ptr(), sig.data_ptr(), self.b.data_ptr(),
                      ptr(self.w), self.pw, ptr(self.g), self.pg, ptr(self.bg), self.pbg, self.eps_counts, nd, s)
            op.adjoint_cl(ydual, grad)
            _lib.call("dfx_pdhg_primal_update", x.data_ptr(), xb.data_ptr(), grad.data_ptr(), T.data_ptr(),
                      self.lam, nx, s)
            op.direct_cl(xb, Axb)                        # A x_bar of the next iteration
            _lib.call("dfx_pdhg_average", Ax.data_ptr(), Axb.data_ptr(), nd, s)
            if it % 50 == 0:                             # float32 drift of the recursion
                op.direct_cl(x, Ax)
            f = self._deviance(Ax)
            stats = {"iter": it, "f": f, "rho": self.rho_used, "time": time.perf_counter() - t_start}
            self.iter_stats.append(stats)
            stop = bool(callback(it, x, stats)) if callback is not None else False
            if verbose and (k == 0 or (k + 1) % diagnostics_interval == 0 or k + 1 == niter or stop):
                print(f"[pdhg {it:5d}] f={f:.8e} {time.perf_counter() - t_start:.1f} s", flush=True)
            if stop:
                break
        xb_h, y_h = np.empty(cshape, np.float32), np.empty(dshape, np.float32)
        host_copier().to_host(xb, xb_h)
        host_copier().to_host(ydual, y_h)
        self.state = {"it": it0 + len(self.iter_stats), "x_bar": xb_h, "y": y_h}
        self.final_stats = {"niter": len(self.iter_stats), "final_f": f, "setup_s": t_setup, "rho": self.rho_used,
                            "time": time.perf_counter() - t_start}
        self.b = self.w = self.g = self.bg = None
        if host is None:
            return x
        host_copier().to_host(x, host)
        return host
