"""SPDHGPoisson: stochastic primal-dual hybrid gradient over omega subsets for the Poisson deviance, on a B200.

Drop-in for diffractom's SPDHGPoisson (optimization/spdhg_poisson.py), with the dense total-variation block: the
same arguments, subset schedule (numpy default_rng(seed) permutations, an epoch never starting with the subset that ended
the previous one), step sizes (diagonal preconditioning: S_i = gamma / (A 1_S)_i, T_j = min_m p_m / (gamma (A_m^T
1_counted)_j), gamma = sqrt(rho), rho = 3e4 / mean(b)^2 by default), the same pass structure (one pass over the
orientation batches per iteration: the adjoint of the current subset's dual change, the update of z and x, the
forward of the next subset) and the same state dict.

Iteration, for the next subset m (p_m = 1 / M):
    y_m'  <- prox_{S F_m*}(y_m + S A_m x)            rows of subset m, closed form in float64
    dz    <- A_m^T (y_m' - y_m);  z <- z + dz;  x <- max(0, x - T (z + dz / p_m + lam))
State: x, z, T (coefficient-sized, kept for the whole run in the operator's channel-fastest batch layout, so that
an iteration needs no gather / scatter and the primal step runs in the backprojection's epilogue), y, S, D
(data-sized; D holds A_m x of the next subset and the dual change of the current one) and one batch-sized scratch.
With a NumPy x0, each of x, z, T that does not fit on the device (resident="auto") or is not asked to stay there
(resident="none" or a list of names) lives in pinned host memory in the same batch layout and is streamed through two
device slots on side streams during every pass (spdhg_poisson.py:411-428); the iterates are the same bits either
way. x is converted back to the (K, Ny, Nx) layout for callbacks and at the end; z for the state.

On a local-basis operator (flat coefficients, LocalSinglePhaseForwardOperator) x, z, T are whole vectors on the device
(they scale with the support) and an iteration is the dual step, the subset adjoint, the primal step of the whole
vector and the next subset's forward (spdhg_poisson.py:753-945): the same steps as the fused pass, in four calls.
"""
from __future__ import annotations

import time

import numpy as np
import torch

from . import _lib
from .arrays import as_host, check_device, is_device, on_op_stream
from .solvers import Reducer, as_device_data, periodic, support_mask_to_device
from .orientation_tree import tree_level_arrays
from .streaming import BatchPipeline, CoeffArray, KMajorStaging, host_copier

RHO_AUTO = 3e4
NAMES = ("x", "z", "T")
TV_NAMES = ("qx", "qy")  # the TV dual (tv > 0), after x, z, T
TV_SAFETY = 0.99         # the TV dual step: this fraction of its bound (spdhg_poisson.py:277)
MARGIN_GB = 1.5          # resident="auto": device memory left free (spdhg_poisson.py:278)


class SPDHGPoisson:
    """SPDHG over omega subsets for the Poisson deviance (module docstring)."""

    # the iterates are zero outside the support (projected at set-up, T = 0 there), so the forward projections read
    # the operator's ray table restricted to the support: the same sums without the zero terms
    use_support_table = True
    # CUDA graphs (an operator on its own stream, x on the device, no orientation shards): from the second epoch on, an
    # iteration "dual step of m, then the pass (m, nb)" is replayed as two graphs captured once per subset: the update
    # of m (dual step, adjoint with the primal step) and the forward of nb (row zeroing, forward projections and
    # products). The pass's per-batch interleaving of the two becomes all updates, then all forwards: every batch's
    # forward still reads its updated x and adds into the rows of nb in batch order, so the values are the same bits.
    use_graphs = False
    # With an operator of precision "bf16" the subset iterations run the BF16 tensor-core path (Radon and PF
    # contraction in BF16, float32 accumulation). The other passes follow the precision recipe by default:
    # bf16_steps False: the step sizes S and T come from the float32 operator, as the reference computes them (they
    # agree with float64 ones to 1e-5); True: from the BF16 operator (the one the iterations apply; about a quarter of
    # the set-up time, S and T within 1e-2 of float64).
    bf16_steps = False
    # bf16_diagnostics False: the full forward of a diagnostics epoch (the residual A x, whose rows feed the float64
    # deviance and the next subset) is recomputed with the float32 operator; True: through the BF16 path as well.
    bf16_diagnostics = False
    # T in BF16, rounded toward zero (never above its float32 value, so the steps still meet SPDHG's step condition),
    # kept on the device: with an operator of precision "bf16" and the Fourier-slice projector (whose primal step is
    # its own kernel). "auto" (resident="auto" only): when x and z fit in float32 and T then fits in BF16 but not in
    # float32, instead of streaming T from host memory in every iteration; True: always with such an operator.
    bf16_T = "auto"
    # True: with an operator of precision "bf16" (native projector) and float32 diagnostics, the residual of a
    # diagnostics epoch (the float32 forward A x of the epoch's last x and its float64 deviance) runs on a side stream
    # from a copy of x while the next epoch's iterations go on; the next subset's rows then come from the BF16 forward
    # like every other iteration's, and the objective is read when the run ends. Not with callbacks, printing, TV,
    # shards or streamed state. Off by default: at ti256 the two streams share a GPU that either keeps busy, and the
    # epoch rate stayed the same (1.89 against 1.91 epochs/s) while the iterations' kernels ran half as fast.
    overlap_residual = False

    def __init__(self, operator, subsets=8, prox_kind="nonneg", lam=0.0, support="fov", eps_counts=1e-3, rho="auto",
                 seed=0, resident="auto", tv=0.0, tv_prob=None, tv_tree=None, shards=None):
        """Arguments as diffractom's SPDHGPoisson (spdhg_poisson.py:301-302). resident ("auto", "all", "none" or a
        list of names from ("x", "z", "T")): which coefficient arrays of a run with a NumPy x0 stay on the device;
        the others are streamed from pinned host memory (a CUDA x0 keeps all three on the device). tv > 0: the total
        variation of every orientation's image as one more block of the serial sampling, chosen with probability
        tv_prob (default 1 / (M + 1)); its dual (qx, qy) is two more coefficient arrays, resident or streamed as x, z,
        T (spdhg_poisson.py:20-40, 320-324); not with shards. tv_tree (an orientation_tree.OrientationTree over the
        basis's orientations in the grid's order; local basis only): the hierarchical total variation of its nested
        cells, the leaf level with weight tv leaf_edge and every penalised level with tv edge, their dual steps
        sharing the TV block's (spdhg_poisson.py:322-326, 819-862). shards
        (this package's extension; a sharding.ShardSum): the operator holds one orientation shard of a process
        group, and the forward's data rows are summed over the shards after each pass; every rank passes the same
        seed and subsets."""
        if prox_kind not in ("nonneg", "nonneg_l1"):
            raise ValueError("SPDHGPoisson supports prox_kind 'nonneg' and 'nonneg_l1'")
        if not (resident in ("auto", "all", "none") or set(resident) <= set(NAMES + TV_NAMES)):
            raise ValueError(f"resident must be 'auto', 'all', 'none' or a list of names from {NAMES + TV_NAMES}")
        tv = float(tv)
        if tv < 0:
            raise ValueError("tv must be >= 0")
        if tv_tree is not None and tv <= 0:
            raise ValueError("tv_tree needs tv > 0")
        if tv > 0 and shards is not None:
            raise NotImplementedError("the total-variation block needs all orientations on one device")
        self.op = operator
        self.ctx, self.queue = operator.ctx, operator.queue
        self.subsets = operator.set_omega_subsets(subsets)
        self.M = len(self.subsets)
        self.lam = float(lam) if prox_kind == "nonneg_l1" else 0.0
        self.eps_counts = float(eps_counts)
        self.rho = rho if rho == "auto" else float(rho)
        self.rng = np.random.default_rng(seed)
        self.resident = resident
        self.tv = tv
        self.tv_tree = tv_tree
        self.tv_prob = (1.0 / (self.M + 1) if tv_prob is None else float(tv_prob)) if tv > 0 else 0.0
        if tv > 0 and not 0 < self.tv_prob < 1:
            raise ValueError("tv_prob must be in (0, 1)")
        self._n_tv = max(1, int(round(self.M * self.tv_prob / (1 - self.tv_prob)))) if tv > 0 else 0
        self._names = NAMES + (TV_NAMES if tv > 0 else ())
        # step probabilities: the data subsets (1 - p_tv) / M each, the TV block p_tv (spdhg_poisson.py:349-352)
        self._p_data = (1.0 - self.tv_prob) / self.M
        self._inv_p_data = float(self.M) if tv == 0 else 1.0 / self._p_data
        self._last = None
        self.support_gpu = support_mask_to_device(operator, support, operator.device)
        self.shards = shards
        self.state = None
        self._t16 = False
        self._stage_io = False
        self._side = None
        self._pending = []

    # ---------------------------------------------------------------- schedule
    def _epoch_order(self):
        """A random permutation of the subsets that does not start with the last subset of the previous epoch
        (spdhg_poisson.py:363-371)."""
        perm = self.rng.permutation(self.M)
        if self.M > 1 and int(perm[0]) == self._last:
            perm[[0, 1]] = perm[[1, 0]]
        self._last = int(perm[-1])
        return [int(m) for m in perm]

    def _epoch_sequence(self):
        """The blocks of the next epoch: the subsets and, with tv, the TV block (-1) inserted _n_tv times at random
        places (spdhg_poisson.py:373-381; without tv the random numbers drawn are those of _epoch_order alone)."""
        order = self._epoch_order()
        if self.tv <= 0:
            return order
        n = len(order) + self._n_tv
        tv_at = set(int(i) for i in self.rng.choice(n, self._n_tv, replace=False))
        it = iter(order)
        return [-1 if i in tv_at else next(it) for i in range(n)]

    # ---------------------------------------------------------------- device steps
    def _dual(self, m):
        op = self.op
        e = op._sub[m]
        _lib.call("dfx_spdhg_dual_update", self.y.data_ptr(), self.D.data_ptr(), self.sig.data_ptr(),
                  self.b.data_ptr(), _ptr(self.w), self.pw, _ptr(self.g), self.pg, _ptr(self.bg), self.pbg,
                  self.eps_counts, e["omegas"].data_ptr(), e["n"], op.My * op.N_seg, op._s())

    def _tv_batch(self, ib, s):
        """The TV block on batch ib: its dual step (qx, qy) and D^T of the dual change with the primal step."""
        op = self.op
        Q, R_ = self.QX, self.QY
        _lib.call("dfx_tv_dual", self.X.ptr(ib, s), self.T.ptr(ib, s), Q.ptr(ib, s), R_.ptr(ib, s),
                  self.dqx.data_ptr(), self.dqy.data_ptr(), op.Nx, op.Ny, op.Kstride, float(self.tv),
                  float(TV_SAFETY * self.tv_prob), op._s())
        _lib.call("dfx_tv_adjoint_update", self.dqx.data_ptr(), self.dqy.data_ptr(), self.X.ptr(ib, s),
                  self.Z.ptr(ib, s), self.T.ptr(ib, s), op.Nx, op.Ny, op.Kstride, float(1.0 / self.tv_prob),
                  self.lam, op._s())

    def _arrays(self, upd, tv):
        """(loaded, stored) state arrays of a pass."""
        if tv:
            return [self.X, self.Z, self.T, self.QX, self.QY], [self.X, self.Z, self.QX, self.QY]
        return ([self.X, self.Z, self.T] if upd else [self.X]), ([self.X, self.Z] if upd else [])

    def _pass(self, adj, fwd, tv=False):
        """One pass over the batches: adjoint of subset adj's dual change (in D), z and x updated (tv: the TV block's
        dual step and update instead); then the forward of the new x for subset fwd ("full": all rows) added to D
        (spdhg_poisson.py:430-484)."""
        op = self.op
        if (op.precision == "bf16" and fwd == "full" and adj is None and not tv and self.bf16_diagnostics
                and op.projector != "fft"):
            self._full_forward_bf16()
            return
        if op.precision == "bf16" and fwd != "full":
            self._pass_bf16(adj, fwd, tv)
            return
        sub = None if fwd == "full" else fwd
        X, Z, T = self.X, self.Z, self.T

        def compute(ib, s):
            xp = X.ptr(ib, s)
            if tv:
                self._tv_batch(ib, s)
            elif adj is not None:       # A_m^T of the dual change, z and x updated in the backprojection's epilogue
                op._adjoint_update_batch(self.D, ib, adj, xp, Z.ptr(ib, s), T.ptr(ib, s), self._inv_p_data,
                                         self.lam)
            if fwd is not None:
                op._direct_batch_k(xp, ib, self.D, sub, ray=self._ray)

        self.pipe.run(*self._arrays(adj is not None, tv), compute)
        if fwd is not None:
            self._sum_shards(fwd)

    def _sum_shards(self, fwd):
        """The forward rows just written, summed over the orientation shards (the pass's only exchange)."""
        if self.shards is None:
            return
        op = self.op
        if fwd == "full":
            self.shards.all(self.D, op.stream())
        else:
            self.shards.rows(self.D, op._sub[op._subset(fwd)]["omegas"], op.stream())

    def _full_forward_bf16(self):
        """D = A x on every row through the BF16 path: per angle chunk, the BF16 table forward of every batch's BF16
        x into its columns of the Radon output, then one tensor-core PF product over all orientations."""
        op = self.op
        be = op.batch_elems()
        X = self.X
        for geo, n, om, _ in op._bf16_chunks(None):
            z = op._z(n)

            def compute(ib, s, z=z, n=n, om=om, geo=geo):
                xb = self.xkb.data_ptr() + (2 * ib * be if X.resident else 0)
                if not X.resident:
                    _lib.call("dfx_f32_to_bf16", X.ptr(ib, s), xb, be, op._s())
                op._radon_bf16_image(xb, z.data_ptr() + 2 * ib * op.Kstride, geo, om, n, op.batches[ib]["K_batch"],
                                     ray=self._ray, tiles=self._tiles)

            self.pipe.run([X], [], compute)
            op._pf_tc_forward(z, om, n, self.D)
        self._sum_shards("full")

    def _pass_bf16(self, adj, fwd, tv=False):
        """The pass of an operator with precision "bf16": one tensor-core launch takes the dual change of subset adj
        to the BF16 Radon output of all batches, each batch's backprojection applies the primal step and projects the
        new x for subset fwd into its columns of that output, and one tensor-core launch overwrites subset fwd's data
        rows (full forward passes: _full_forward_bf16). The BF16 copy of x that the forward reads is kept for all
        batches when x is resident, else made per batch (one buffer). With the Fourier-slice projector the forward
        transforms the float32 x (no BF16 copy) and the rows of its output are rounded to BF16."""
        op = self.op
        be = op.batch_elems()
        X, Z, T = self.X, self.Z, self.T
        fft = op.projector == "fft"
        if adj is not None:
            geo, n, zb = op._bf16_adjoint_sino(self.D, adj)

        def compute(ib, s):
            xb = None if fft else self.xkb.data_ptr() + (2 * ib * be if X.resident else 0)
            if tv:                          # the TV block, then the BF16 copy of the new x
                self._tv_batch(ib, s)
                if not fft:
                    _lib.call("dfx_f32_to_bf16", X.ptr(ib, s), xb, be, op._s())
            elif adj is not None:
                op._bf16_update_batch(ib, geo, n, zb, X.ptr(ib, s), Z.ptr(ib, s), T.ptr(ib, s), self._inv_p_data,
                                      self.lam, xb, subset=adj, t_bf16=self._t16)
            elif not X.resident and not fft:
                _lib.call("dfx_f32_to_bf16", X.ptr(ib, s), xb, be, op._s())
            if fwd is not None and fft:
                op._bf16_forward_sino(fwd, ib, X.ptr(ib, s))
            elif fwd is not None:
                op._bf16_forward_sino(fwd, ib, xb, src_bf16=True, ray=self._ray, tiles=self._tiles)

        self.pipe.run(*self._arrays(adj is not None, tv), compute)
        if fwd is not None:
            op._bf16_forward_rows(fwd, self.D)
            self._sum_shards(fwd)

    def _deviance(self, mu):
        return self.red.deviance(mu, self.b, self.w, self.pw, self.g, self.pg, self.bg, self.pbg, self.eps_counts)

    def _tv_value(self):
        """sum_k TV(x_k) (a pass over the batches; float64)."""
        op = self.op
        nb = op._lib.dfx_reduce_scratch_bytes(op.batch_elems())
        total = torch.zeros(len(op.batches), dtype=torch.float64, device=op.device)

        def compute(ib, s):
            scr = op.scratch(nb)
            _lib.call("dfx_tv_value", self.X.ptr(ib, s), self.T.ptr(ib, s), op.Nx, op.Ny, op.Kstride,
                      total.data_ptr() + 8 * ib, scr.data_ptr(), nb, op._s())

        self.pipe.run([self.X, self.T], [], compute)
        return float(total.sum().item())

    # ---------------------------------------------------------------- run
    @on_op_stream
    def run(self, x0, b, n_epochs, weights=None, gain=None, background=None, verbose=0, diagnostics_interval=1,
            callback=None, state=None):
        """As diffractom's SPDHGPoisson.run (spdhg_poisson.py:513-751). x0: a CUDA tensor (updated in place and
        returned) or a NumPy array (updated in place if C-contiguous float32, else converted; returned)."""
        if getattr(self.op, "coefficient_layout", "dense") == "local":
            return self._run_local(x0, b, n_epochs, weights, gain, background, verbose, diagnostics_interval,
                                   callback, state)
        if self.tv_tree is not None:
            raise NotImplementedError("tv_tree needs an operator with the local coefficient layout")
        self._setup(x0, b, weights, gain, background, state)
        self._iterate(n_epochs, verbose, diagnostics_interval, callback, defer_final=True, async_diagnostics=True)
        return self._finish()

    def _setup_data(self, b, weights, gain, background):
        """The data, weights, gain and background on the device, y = 0, the data-sized buffers; returns gamma."""
        op = self.op
        dev, dshape = op.device, tuple(op.data_shape)
        self.b = as_device_data(b, dshape, dev)
        self.w, self.pw = periodic(weights, dshape, "weights", dev)
        self.g, self.pg = periodic(gain, dshape, "gain", dev)
        self.bg, self.pbg = periodic(background, dshape, "background", dev)
        if self.pg and float(self.g.min().item()) <= 0:
            raise ValueError("the gain must be positive everywhere")
        self.red = Reducer(op)
        self.y = torch.zeros(dshape, dtype=torch.float32, device=dev)
        self.sig = torch.empty(dshape, dtype=torch.float32, device=dev)
        self.D = torch.empty(dshape, dtype=torch.float32, device=dev)
        rho = self.rho
        if rho == "auto":
            sb, sn = self.red.mean_counted(self.b, self.w, self.pw)
            mean_b = sb / max(sn, 1.0)
            rho = RHO_AUTO / mean_b ** 2 if mean_b > 0 else 1.0
        self.rho_used = float(rho)
        return np.sqrt(rho)

    def _dual_steps_from_rowsums(self, gamma):
        """S = gamma / (A 1_S) from the row sums in D, the scales; then D = 1 on the counted points (for T)."""
        s = self.op._s()
        rs, rn = self.red.mean_counted(self.D, self.w, self.pw)
        bs, bn = self.red.mean_counted(self.b, self.w, self.pw)
        self.scales = {"row_sum_mean": rs / max(rn, 1.0), "b_mean": bs / max(bn, 1.0),
                       "gain_mean": 1.0 if self.pg == 0 else float(self.g.double().mean().item())}
        _lib.call("dfx_dual_steps", self.sig.data_ptr(), self.D.data_ptr(), _ptr(self.w), self.pw, float(gamma),
                  self.D.numel(), s)
        _lib.call("dfx_set_mask_ones", self.D.data_ptr(), _ptr(self.w), self.pw, self.D.numel(), s)

    # ---------------------------------------------------------------- local basis
    def _run_local(self, x0, b, n_epochs, weights, gain, background, verbose, diagnostics_interval, callback, state):
        """run() on flat coefficients (module docstring); the schedule, steps and state are those of the dense run."""
        t_start = time.perf_counter()
        op = self.op
        dev, s = op.device, op._s()
        n = int(op.n_coef)
        cshape, dshape = (n,), tuple(op.data_shape)
        x_on_gpu = is_device(x0)
        host_x = None if x_on_gpu else as_host(x0, cshape, "x0", writeable=True)
        if x_on_gpu:
            x = check_device(x0, cshape, "x0")
        else:
            x = torch.empty(cshape, dtype=torch.float32, device=dev)
            host_copier().to_device(host_x, x)
        gamma = self._setup_data(b, weights, gain, background)
        # S from the row sums A 1 (1 on the allowed coefficients); T from the subsets' column sums over the counted
        # points (spdhg_poisson.py:799-813)
        ones = torch.as_tensor(np.ascontiguousarray(op.coefficient_mask(), np.float32), device=dev)
        op.direct_cl(ones, self.D)
        del ones
        self._dual_steps_from_rowsums(gamma)
        z = torch.zeros(n, dtype=torch.float32, device=dev)
        T = torch.empty(n, dtype=torch.float32, device=dev)
        dz = torch.empty(n, dtype=torch.float32, device=dev)
        c = float(np.float32(self._p_data / gamma))
        _lib.call("dfx_tinit", T.data_ptr(), n, s)
        for m in range(self.M):
            op.adjoint_cl(self.D, dz, subset=m)
            _lib.call("dfx_tmin", T.data_ptr(), dz.data_ptr(), None, 0, c, n, s)
        _lib.call("dfx_tfinal", T.data_ptr(), n, s)
        _lib.call("dfx_project_support", x.data_ptr(), None, 0, n, s)
        self.resident_used = self._names
        tvq = None
        if self.tv > 0:                 # the TV dual, its change, the patches' neighbour indices (spdhg_poisson.py:814-826)
            f32 = lambda: torch.zeros(n, dtype=torch.float32, device=dev)
            tvq = dict(qx=f32(), qy=f32(), dqx=f32(), dqy=f32(),
                       nbr=[torch.as_tensor(a, device=dev) for a in _patch_neighbours(op)])
            for nm in ("qx", "qy"):
                if state is not None and state.get(nm) is not None:
                    tvq[nm].copy_(torch.as_tensor(as_host(state[nm], cshape, f"state['{nm}']")))
            # the tree's levels: node-pixel arrays, their duals and scratch (spdhg_poisson.py:819-826, 946-978)
            tvq["levels"] = []
            tvq["leaf_edge"] = float(self.tv_tree.leaf_edge) if self.tv_tree is not None else 1.0
            if self.tv_tree is not None:
                if int(self.tv_tree.K) != int(op.K_basis):
                    raise ValueError(f"tv_tree must cover the basis's {op.K_basis} orientations (in the grid's "
                                     f"order), not {self.tv_tree.K}")
                k_, iy_, ix_, pi_ = op._pairs()
                host_levels = tree_level_arrays(k_, iy_, ix_, pi_, int(op.Ny), int(op.Nx), n, T.cpu().numpy(),
                                                self.tv_tree)
                saved = list(state.get("tree_q") or []) if state is not None else []
                for li, hl in enumerate(host_levels):
                    lev = {nm: torch.as_tensor(hl[nm], device=dev)
                           for nm in ("ptr", "idx", "map", "right", "down", "left", "up", "A")}
                    lev.update(n=hl["n"], edge=hl["edge"],
                               qx=torch.zeros(hl["n"], dtype=torch.float32, device=dev),
                               qy=torch.zeros(hl["n"], dtype=torch.float32, device=dev))
                    if li < len(saved):
                        lev["qx"].copy_(torch.as_tensor(as_host(saved[li][0], (hl["n"],), "state['tree_q']")))
                        lev["qy"].copy_(torch.as_tensor(as_host(saved[li][1], (hl["n"],), "state['tree_q']")))
                    tvq["levels"].append(lev)
                if tvq["levels"]:
                    nmax = max(lev["n"] for lev in tvq["levels"])
                    tvq["scr"] = {nm: torch.empty(nmax, dtype=torch.float32, device=dev)
                                  for nm in ("s", "w", "dqx", "dqy")}
            # the leaf level's weight and the dual step shared among the levels
            tvq["lam"] = float(self.tv * tvq["leaf_edge"])
            tvq["ps"] = float(TV_SAFETY * self.tv_prob / (1 + len(tvq["levels"])))
        if state is not None and self.tv > 0 and state.get("z") is None:
            raise ValueError("continuing a TV run needs the state's z")
        if state is not None:
            host_copier().to_device(as_host(state["y"], dshape, "state['y']"), self.y)
            if state.get("z") is not None:
                z.copy_(torch.as_tensor(as_host(state["z"], cshape, "state['z']")))
            else:                                       # z = A^T y of this operator
                op.adjoint_cl(self.y, z)
        t_setup = time.perf_counter() - t_start
        inv_p = self._inv_p_data
        ep0 = int(state["epoch"]) if state is not None else 0
        self.iter_stats = []
        f = float("nan")
        seq = self._epoch_sequence()
        if seq[0] >= 0:
            op.direct_cl(x, self.D, subset=seq[0])
        for e in range(int(n_epochs)):
            ep = ep0 + e + 1
            last = e + 1 == n_epochs
            want_f = (e + 1) % max(1, diagnostics_interval) == 0 or last
            nseq = None
            for j, m in enumerate(seq):
                if m >= 0:
                    self._dual(m)
                    op.adjoint_cl(self.D, dz, subset=m)
                    _lib.call("dfx_spdhg_primal_update", x.data_ptr(), z.data_ptr(), T.data_ptr(), dz.data_ptr(),
                              inv_p, self.lam, n, s)
                else:                                        # the TV block
                    self._tv_block_local(tvq, x, z, T, dz, n, s)
                end_of_epoch = j + 1 == len(seq)
                if not end_of_epoch:
                    nb = seq[j + 1]
                elif not last:
                    nseq = self._epoch_sequence()
                    nb = nseq[0]
                else:
                    nb = None
                m_next = nb if nb is not None and nb >= 0 else None
                if end_of_epoch and want_f:
                    op.direct_cl(x, self.D)                  # every row (the next subset's among them)
                    f = self._deviance(self.D)
                    if self.tv > 0:
                        f += self.tv * self._tv_value_local(tvq, x, T, n, s)
                elif m_next is not None:
                    op.direct_cl(x, self.D, subset=m_next)
            if nseq is not None:
                seq = nseq
            if callback is not None or verbose:
                op.stream().synchronize()
            stats = {"epoch": ep, "f": f if want_f else None, "rho": self.rho_used,
                     "time": time.perf_counter() - t_start}
            self.iter_stats.append(stats)
            stop = False
            if callback is not None:
                if not x_on_gpu:
                    host_copier().to_host(x, host_x)
                stop = bool(callback(ep, x if x_on_gpu else host_x, stats))
            if verbose and want_f:
                print(f"[spdhg epoch {ep:4d}] f={f:.8e} {time.perf_counter() - t_start:.1f} s", flush=True)
            if stop:
                break
        z_host, y_host = np.empty(cshape, np.float32), np.empty(dshape, np.float32)
        host_copier().to_host(z, z_host)
        host_copier().to_host(self.y, y_host)
        self.state = {"epoch": ep0 + len(self.iter_stats), "z": z_host, "y": y_host}
        if tvq is not None:
            self.state.update(qx=tvq["qx"].cpu().numpy(), qy=tvq["qy"].cpu().numpy())
            if tvq["levels"]:
                self.state["tree_q"] = [(lev["qx"].cpu().numpy(), lev["qy"].cpu().numpy()) for lev in tvq["levels"]]
        self.final_stats = {"epochs": len(self.iter_stats), "final_f": f, "setup_s": t_setup, "rho": self.rho_used,
                            "subsets": self.M, "resident": self.resident_used,
                            "time": time.perf_counter() - t_start, "tv": self.tv, "tv_prob": self.tv_prob,
                            "graph_replays": 0, **self.scales}
        if not x_on_gpu:
            host_copier().to_host(x, host_x)
        self.b = self.w = self.g = self.bg = self.y = self.sig = self.D = None
        return x if x_on_gpu else host_x

    def _tv_block_local(self, tvq, x, z, T, dz, n, s):
        """The TV block on flat coefficients: the leaf level's dual step and D^T dq, then per tree level the node-pixel
        sums, their dual step and D^T dq scattered onto the coefficients, and the primal step with the sum
        (spdhg_poisson.py:853-877). Without tree levels the adjoint and the primal step run fused."""
        nb_ = tvq["nbr"]
        inv_p = float(1.0 / self.tv_prob)
        _lib.call("dfx_tv_dual_local", x.data_ptr(), T.data_ptr(), tvq["qx"].data_ptr(), tvq["qy"].data_ptr(),
                  tvq["dqx"].data_ptr(), tvq["dqy"].data_ptr(), nb_[0].data_ptr(), nb_[1].data_ptr(), tvq["lam"],
                  tvq["ps"], n, s)
        if not tvq["levels"]:
            _lib.call("dfx_tv_adjoint_update_local", tvq["dqx"].data_ptr(), tvq["dqy"].data_ptr(), x.data_ptr(),
                      z.data_ptr(), T.data_ptr(), nb_[2].data_ptr(), nb_[3].data_ptr(), inv_p, self.lam, n, s)
            return
        _lib.call("dfx_tv_adjoint_local", tvq["dqx"].data_ptr(), tvq["dqy"].data_ptr(), dz.data_ptr(),
                  nb_[2].data_ptr(), nb_[3].data_ptr(), n, s)
        scr = tvq["scr"]
        for lev in tvq["levels"]:
            nn = lev["n"]
            _lib.call("dfx_tree_sums", x.data_ptr(), lev["ptr"].data_ptr(), lev["idx"].data_ptr(),
                      scr["s"].data_ptr(), nn, s)
            _lib.call("dfx_tv_dual_local", scr["s"].data_ptr(), lev["A"].data_ptr(), lev["qx"].data_ptr(),
                      lev["qy"].data_ptr(), scr["dqx"].data_ptr(), scr["dqy"].data_ptr(), lev["right"].data_ptr(),
                      lev["down"].data_ptr(), float(self.tv * lev["edge"]), tvq["ps"], nn, s)
            _lib.call("dfx_tv_adjoint_local", scr["dqx"].data_ptr(), scr["dqy"].data_ptr(), scr["w"].data_ptr(),
                      lev["left"].data_ptr(), lev["up"].data_ptr(), nn, s)
            _lib.call("dfx_tree_scatter", scr["w"].data_ptr(), lev["map"].data_ptr(), dz.data_ptr(), n, s)
        _lib.call("dfx_spdhg_primal_update", x.data_ptr(), z.data_ptr(), T.data_ptr(), dz.data_ptr(), inv_p,
                  self.lam, n, s)

    def _tv_value_local(self, tvq, x, T, n, s):
        """The penalty over tv: leaf_edge TV(x) + the levels' edge TV(node-pixel sums) (spdhg_poisson.py:842-851)."""
        op = self.op
        nb_ = tvq["nbr"]
        tvs = torch.zeros(1, dtype=torch.float64, device=op.device)
        nbytes = op._lib.dfx_reduce_scratch_bytes(n)
        scr = op.scratch(nbytes)
        _lib.call("dfx_tv_value_local", x.data_ptr(), T.data_ptr(), nb_[0].data_ptr(), nb_[1].data_ptr(), n,
                  tvs.data_ptr(), scr.data_ptr(), nbytes, s)
        v = float(tvs.item()) * tvq["leaf_edge"]
        for lev in tvq["levels"]:
            nn = lev["n"]
            _lib.call("dfx_tree_sums", x.data_ptr(), lev["ptr"].data_ptr(), lev["idx"].data_ptr(),
                      tvq["scr"]["s"].data_ptr(), nn, s)
            nbytes = op._lib.dfx_reduce_scratch_bytes(nn)
            scr = op.scratch(nbytes)
            _lib.call("dfx_tv_value_local", tvq["scr"]["s"].data_ptr(), lev["A"].data_ptr(), lev["right"].data_ptr(),
                      lev["down"].data_ptr(), nn, tvs.data_ptr(), scr.data_ptr(), nbytes, s)
            v += float(tvs.item()) * lev["edge"]
        return v

    @on_op_stream
    def _setup(self, x0, b, weights=None, gain=None, background=None, state=None):
        """Upload, step sizes S and T, support projection, warm start (spdhg_poisson.py:520-662)."""
        self._t_start = time.perf_counter()
        op = self.op
        dev = op.device
        cshape, dshape = tuple(op.coeff_shape), tuple(op.data_shape)
        npix = op.npix
        s = op._s()
        self._x_on_gpu = is_device(x0)
        self._host_x = None if self._x_on_gpu else as_host(x0, cshape, "x0", writeable=True)
        gamma = self._setup_data(b, weights, gain, background)
        supp = self.support_gpu
        sp = None if supp is None else supp.data_ptr()
        p = self._p_data
        # x, z, T in the operator's channel-fastest batch layout for the whole run (batch ib at ib * be): on the device,
        # or in pinned host memory streamed through two device slots
        be = op.batch_elems()
        nbt = len(op.batches)
        if state is not None and self.tv > 0 and state.get("z") is None:
            raise ValueError("continuing a TV run needs the state's z")
        resident = self._choose_resident()
        self.resident_used = tuple(nm for nm in self._names if nm in resident)
        self.X, self.Z = (CoeffArray(op, nm, nm in resident) for nm in NAMES[:2])
        self.T = CoeffArray(op, "T", "T" in resident, torch.bfloat16 if self._t16 else torch.float32)
        self.pipe = BatchPipeline(op)
        # staged host IO (no (K, Ny, Nx) device temporary) when memory is short: some array streamed, or T in BF16
        self._stage = (None if len(resident) == len(self._names) and not self._t16 and not self._stage_io
                       else KMajorStaging(op))
        self.dzk = torch.empty(be, dtype=torch.float32, device=dev)
        self.x = None
        # a host x0 of a resident x is uploaded after the step sizes' passes are queued, on a side stream, so that
        # the copy overlaps them (they do not read x). When some array is streamed, device memory is short of a
        # whole (K, Ny, Nx) array beside the state: host arrays then move through the batch-sized staging buffers
        # (resident arrays included), here and when the run ends.
        upload_x = self.X.resident and not self._x_on_gpu and self._stage is None
        if self._x_on_gpu:
            self.x = x0
            op.to_batches(self.x, self.X.dev)
        elif upload_x:
            self.x = torch.empty(cshape, dtype=torch.float32, device=dev)
            x_alloc = torch.cuda.Event()
            x_alloc.record(op.stream())                 # the side stream writes x after this point only
        else:
            self._stage.load(self._host_x.reshape(-1), self.X, self.pipe)
        if state is not None and state.get("z") is not None:
            z0 = as_host(state["z"], cshape, "state['z']")
            if self.Z.resident and self._stage is None:
                op.to_batches(torch.as_tensor(z0, device=dev), self.Z.dev)
            else:
                self._stage.load(z0.reshape(-1), self.Z, self.pipe)
        elif self.Z.resident:
            op._fill(self.Z.dev, 0.0)
        else:
            self.Z.host.zero_()
        self.QX = self.QY = self.dqx = self.dqy = None
        if self.tv > 0:                                 # the TV dual (state or 0) and its change per batch
            self.QX, self.QY = (CoeffArray(op, nm, nm in resident) for nm in TV_NAMES)
            for arr, nm in ((self.QX, "qx"), (self.QY, "qy")):
                q0 = None if state is None or state.get(nm) is None else as_host(state[nm], cshape, f"state['{nm}']")
                if q0 is None:
                    if arr.resident:
                        op._fill(arr.dev, 0.0)
                    else:
                        arr.host.zero_()
                elif arr.resident and self._stage is None:
                    op.to_batches(torch.as_tensor(q0, device=dev), arr.dev)
                else:
                    self._stage.load(q0.reshape(-1), arr, self.pipe)
            self.dqx = torch.empty(be, dtype=torch.float32, device=dev)
            self.dqy = torch.empty(be, dtype=torch.float32, device=dev)

        self._ray = op.support_ray_table(supp) if supp is not None and self.use_support_table else None
        self._tiles = (op.support_tiles(supp) if supp is not None and self.use_support_table
                       and op.precision == "bf16" else None)
        # S from the row sums A 1_S (spdhg_poisson.py:621-629); with a BF16 operator from the BF16 operator that the
        # iterations apply (the step sizes of the operator in use, at a quarter of the float32 passes' time)
        bf16 = op.precision == "bf16" and self.bf16_steps and op.projector != "fft"
        op._fill(self.D, 0.0)
        if bf16:
            for geo, n, om, a in op._bf16_chunks(None):
                z = op._z(n)
                for ib, bt in enumerate(op.batches):
                    _lib.call("dfx_batch_support", self.dzk.data_ptr(), None, sp, npix, op.Kstride, bt["K_batch"],
                              0.0, 0, s)
                    op._radon_forward_bf16(self.dzk.data_ptr(), ib, z, om, n, row0=a)
                op._pf_tc_forward(z, om, n, self.D)
        elif op.projector == "native":
            # 1_S is the same image in every channel: one Radon transform (the widest batch's channels) serves every
            # batch's PF product, the bits of the batch-by-batch passes
            kbm = max(bt["K_batch"] for bt in op.batches)
            _lib.call("dfx_batch_support", self.dzk.data_ptr(), None, sp, npix, op.Kstride, kbm, 0.0, 0, s)
            op._direct_channel_constant(self.dzk.data_ptr(), kbm, self.D, ray=self._ray)
        else:
            for ib, bt in enumerate(op.batches):
                _lib.call("dfx_batch_support", self.dzk.data_ptr(), None, sp, npix, op.Kstride, bt["K_batch"], 0.0,
                          0, s)
                op._direct_batch_k(self.dzk.data_ptr(), ib, self.D, ray=self._ray)
        self._sum_shards("full")
        self._dual_steps_from_rowsums(gamma)
        # T from the subsets' column sums over the counted points (spdhg_poisson.py:630-643)
        c = float(np.float32(p / gamma))
        T = self.T
        if bf16:
            op._rows_to_bf16(self.D, op._all_omegas, op.N_Omega)

        tk = torch.empty(be, dtype=torch.float32, device=dev) if self._t16 else None

        def t_batch(ib, s_):
            tb, kb = (tk.data_ptr() if self._t16 else T.ptr(ib, s_)), op.batches[ib]["K_batch"]
            _lib.call("dfx_tinit", tb, be, s)
            for m in range(self.M):
                if bf16:                                   # this batch's columns of A_m^T 1_counted, BF16 operator
                    e = op._sub[m]
                    z = op._z(e["n"])
                    op._pf_tc_adjoint(e["omegas"], e["n"], z, ib * op.Kstride, op.Kstride)
                    _lib.call("dfx_radon_backward_bf16", z.data_ptr() + 2 * ib * op.Kstride, op.Ktot,
                              self.dzk.data_ptr(), e["geo"].data_ptr(), e["n"], op.Nx, op.Ny, op.My, op.Kstride, kb,
                              op._kernel_id, int(op.radon_geo.n_taps), s)
                else:
                    op._adjoint_batch_k(self.D, ib, self.dzk.data_ptr(), subset=m)
                _lib.call("dfx_batch_support", tb, self.dzk.data_ptr(), sp, npix, op.Kstride, kb, c, 2, s)
            _lib.call("dfx_tfinal", tb, be, s)           # padding channels were never reached: T = 0 there
            if self._t16:
                _lib.call("dfx_f32_to_bf16_rz", tb, T.ptr(ib, s_), be, s)

        if bf16 and T.resident and not self._t16:
            # subset by subset: one tensor-core PF adjoint for all batches, then every batch's backprojection and
            # running minimum (the same columns as batch by batch, in a twentieth of the PF launches)
            for ib in range(nbt):
                _lib.call("dfx_tinit", T.ptr(ib, None), be, s)
            for m in range(self.M):
                e = op._sub[m]
                z = op._z(e["n"])
                op._pf_tc_adjoint(e["omegas"], e["n"], z)
                for ib, bt in enumerate(op.batches):
                    kb = bt["K_batch"]
                    _lib.call("dfx_radon_backward_bf16", z.data_ptr() + 2 * ib * op.Kstride, op.Ktot,
                              self.dzk.data_ptr(), e["geo"].data_ptr(), e["n"], op.Nx, op.Ny, op.My, op.Kstride, kb,
                              op._kernel_id, int(op.radon_geo.n_taps), s)
                    _lib.call("dfx_batch_support", T.ptr(ib, None), self.dzk.data_ptr(), sp, npix, op.Kstride, kb, c,
                              2, s)
            for ib in range(nbt):
                _lib.call("dfx_tfinal", T.ptr(ib, None), be, s)
        else:
            self.pipe.run([], [T], t_batch)
        if upload_x:
            side = torch.cuda.Stream(dev)
            side.wait_event(x_alloc)                    # not the step sizes' passes queued since
            host_copier().to_device(self._host_x, self.x, stream=side)
            op.stream().wait_stream(side)
            op.to_batches(self.x, self.X.dev)

        def project_x(ib, s_):                          # x on the support, >= 0, padding 0
            _lib.call("dfx_batch_support", self.X.ptr(ib, s_), None, sp, npix, op.Kstride,
                      op.batches[ib]["K_batch"], 0.0, 1, s)

        self.pipe.run([self.X], [self.X], project_x)
        if state is not None:
            host_copier().to_device(as_host(state["y"], dshape, "state['y']"), self.y)
            if state.get("z") is None:
                self.pipe.run([], [self.Z], lambda ib, s_: op._adjoint_batch_k(self.y, ib, self.Z.ptr(ib, s_)))
        # the host arrays the run ends with (z, y, and a NumPy x0 that receives x) have their pages mapped by the
        # copy threads while the device iterates, so that the final downloads run at the copy rate
        self._host_out, self._prefault = None, []
        if self.Z.resident and self._stage is None:
            hc = host_copier()
            z_host, y_host = np.empty(cshape, np.float32), np.empty(dshape, np.float32)
            self._prefault = hc.prefault(z_host, False) + hc.prefault(y_host, False)
            if self.X.resident and not self._x_on_gpu:
                self._prefault += hc.prefault(self._host_x, True)
            self._host_out = (z_host, y_host)
        self._graphs = {}
        self.graph_replays = 0
        self._final_pending = False
        self._t_setup = time.perf_counter() - self._t_start
        self._ep0 = int(state["epoch"]) if state is not None else 0
        self.iter_stats = []
        self._f = float("nan")
        self._seq = self._epoch_sequence()
        self.xkb = None
        if op.precision == "bf16" and op.projector != "fft":   # the BF16 copy of x that the forward projections read
            if self.X.resident:
                self.xkb = torch.empty(nbt * be, dtype=torch.bfloat16, device=dev)
                _lib.call("dfx_f32_to_bf16", self.X.dev.data_ptr(), self.xkb.data_ptr(), nbt * be, s)
            else:
                self.xkb = torch.empty(be, dtype=torch.bfloat16, device=dev)
        if self._seq[0] >= 0:
            op.zero_subset_rows(self.D, self._seq[0])
            self._pass(None, self._seq[0])

    @on_op_stream
    def _iterate(self, n_epochs, verbose=0, diagnostics_interval=1, callback=None, final=True, defer_final=False,
                 async_diagnostics=False):
        """n_epochs epochs (spdhg_poisson.py:664-719). final=False: the last of them is not the run's last (no
        closing full forward unless diagnostics fall there), so that epochs can be run in several calls.
        defer_final (run()): the closing full forward and the objective of the run's last epoch are left to _finish,
        which queues them beside the downloads of x, z and y (same values; the last epoch's "f" is filled in there)."""
        op = self.op
        dev = op.device
        seq = self._seq
        # the closing full forward and objective of the run's last epoch can wait for _finish, which overlaps them
        # with the state's downloads (nobody reads the objective before: no callback, no printing)
        defer = (defer_final and final and callback is None and not verbose and self.tv == 0 and self.X.resident
                 and self.Z.resident and self._stage is None)
        overlap = (async_diagnostics and self.overlap_residual and callback is None and not verbose
                   and op.precision == "bf16"
                   and op.projector != "fft" and not self.bf16_diagnostics and self.tv == 0 and self.shards is None
                   and self._stage is None and not self._graphs_on())
        for e in range(n_epochs):
            ep = self._ep0 + len(self.iter_stats) + 1
            last = final and e + 1 == n_epochs
            want_f = (len(self.iter_stats) + 1) % max(1, diagnostics_interval) == 0 or last
            nseq = None
            for j, blk in enumerate(seq):
                end_of_epoch = j + 1 == len(seq)
                if not end_of_epoch:
                    nb = seq[j + 1]
                elif not last:
                    nseq = self._epoch_sequence()
                    nb = nseq[0]
                else:
                    nb = None
                adj = blk if blk >= 0 else None          # a data subset, or the TV block (-1)
                tvb = adj is None
                m_next = nb if nb is not None and nb >= 0 else None
                full = (end_of_epoch and want_f) or nb is None or (m_next is not None and m_next == adj)
                if overlap and full and end_of_epoch and want_f and m_next is not None and m_next != adj:
                    # this epoch's residual on the side stream; the next subset's rows by the usual pass
                    if adj is not None:
                        self._dual(adj)
                    op.zero_subset_rows(self.D, m_next)
                    self._pass(adj, m_next, tv=tvb)
                    self._residual_async(len(self.iter_stats))
                    continue
                graphed = not full and not tvb and m_next is not None and self._graphs_on()
                if adj is not None and not graphed:
                    self._dual(adj)
                if full:
                    self._pass(adj, None, tv=tvb)
                    if last and end_of_epoch and defer:
                        self._final_pending = True           # _finish runs it beside the downloads
                    elif (end_of_epoch and want_f) or m_next is not None:
                        op._fill(self.D, 0.0)
                        self._pass(None, "full")
                        if end_of_epoch and want_f:
                            self._f = self._deviance(self.D)
                            if self.tv > 0:
                                self._f += self.tv * self._tv_value()
                elif graphed:
                    self._replay(("update", adj), lambda m=adj: (self._dual(m), self._pass(m, None)))
                    self._replay(("forward", m_next), lambda nb=m_next: (op.zero_subset_rows(self.D, nb),
                                                                         self._pass(None, nb)))
                else:
                    if m_next is not None:
                        op.zero_subset_rows(self.D, m_next)
                    self._pass(adj, m_next, tv=tvb)
            if nseq is not None:
                seq = nseq
            self._seq = seq
            if callback is not None or verbose:
                op.stream().synchronize()
            async_f = overlap and want_f and self._pending and self._pending[-1][0] == len(self.iter_stats)
            stats = {"epoch": ep, "f": None if async_f or not want_f else self._f, "rho": self.rho_used,
                     "time": time.perf_counter() - self._t_start}
            self.iter_stats.append(stats)
            stop = False
            if callback is not None:
                self._x_out()
                stop = bool(callback(ep, self.x if self._x_on_gpu else self._host_x, stats))
            if verbose and want_f:
                print(f"[spdhg epoch {ep:4d}] f={self._f:.8e} {time.perf_counter() - self._t_start:.1f} s",
                      flush=True)
            if stop:
                break
        if self._pending:                   # the caller's next work (and its timing) comes after the residuals
            op.stream().wait_event(self._pending[-1][2])

    def _residual_async(self, index):
        """The residual of the current x on the side stream: x copied on the operator's stream (the next update writes
        x), then the float32 full forward of the copy into a separate data buffer and its float64 deviance, with the
        side stream's own batch sinogram and scratch; iter_stats[index]["f"] is filled in by _resolve_pending."""
        op = self.op
        main = op.stream()
        if self._side is None:
            self._side = torch.cuda.Stream(op.device)
            self._x_snap = torch.empty_like(self.X.dev)
            self._D_diag = torch.empty_like(self.D)
            self._side_sino = torch.empty_like(op.coeffs_sino_C)
            self._side_scratch = torch.empty(0, dtype=torch.uint8, device=op.device)
        if self._pending:                   # the previous residual has read its copy of x
            main.wait_event(self._pending[-1][2])
        with torch.cuda.stream(main):
            self._x_snap.copy_(self.X.dev)
        ev = torch.cuda.Event()
        ev.record(main)
        self._side.wait_event(ev)
        out = torch.empty(4, dtype=torch.float64, device=op.device)
        saved = (op.queue, op.coeffs_sino_C, op._scratch)
        op.queue, op.coeffs_sino_C, op._scratch = self._side, self._side_sino, self._side_scratch
        try:
            be = op.batch_elems()
            op._fill(self._D_diag, 0.0)
            for ib in range(len(op.batches)):
                op._direct_batch_k(self._x_snap.data_ptr() + 4 * ib * be, ib, self._D_diag, ray=self._ray)
            self.red.deviance_into(out, self._D_diag, self.b, self.w, self.pw, self.g, self.pg, self.bg, self.pbg,
                                   self.eps_counts)
        finally:
            self._side_scratch = op._scratch
            op.queue, op.coeffs_sino_C, op._scratch = saved
        done = torch.cuda.Event()
        done.record(self._side)
        self._pending.append((index, out, done))

    def _resolve_pending(self):
        """Reads the objectives of the residuals run on the side stream into iter_stats (and into the current
        objective when it is the latest epoch's)."""
        for index, out, done in self._pending:
            done.synchronize()
            f = float(out[0].item())
            if index < len(self.iter_stats):
                self.iter_stats[index]["f"] = f
            if index == len(self.iter_stats) - 1:
                self._f = f
        self._pending = []

    def _graphs_on(self):
        op = self.op
        # a generated BF16 PF is made (or found in its buffers) when a product runs: the host picks, so no graphs
        return (self.use_graphs and len(self.iter_stats) >= 1 and self.shards is None and self._stage is None
                and self.tv == 0 and (op.precision != "bf16" or op.pf_bf16 is not None)
                and torch.cuda.current_stream(op.device) != torch.cuda.default_stream(op.device))

    def _replay(self, key, fn):
        """Replay the graph of key, capturing fn on the current (the operator's) stream the first time."""
        g = self._graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            g.capture_begin(capture_error_mode="thread_local")
            try:
                fn()
            finally:
                g.capture_end()
            self._graphs[key] = g
        g.replay()
        self.graph_replays += 1

    def _wait_prefault(self):
        for f in self._prefault:
            f.result()
        self._prefault = []

    def _x_out(self):
        """x in the (K, Ny, Nx) layout of the caller's array (the CUDA x0, or the NumPy x0's device copy and x0)."""
        self._wait_prefault()
        op = self.op
        if self.x is not None:
            op.from_batches(self.X.dev, self.x)
            if not self._x_on_gpu:
                host_copier().to_host(self.x, self._host_x)
        else:
            self._stage.store(self.X, self._host_x.reshape(-1), self.pipe)

    def _choose_resident(self):
        """The coefficient arrays kept on the device (spdhg_poisson.py:411-428): all of them for a CUDA x0 or
        resident="all"; for "auto" as many of x, z, T (in this order) as fit into the free device memory less the
        streaming buffers and a margin."""
        names = self._names
        op = self.op
        self._stage_io = False
        t16_ok = op.precision == "bf16" and op.projector == "fft" and self.tv == 0
        if self.bf16_T is True and not t16_ok:
            raise ValueError("bf16_T needs an operator of precision 'bf16' with the Fourier-slice projector, no tv")
        self._t16 = self.bf16_T is True
        if self._x_on_gpu or self.resident == "all":
            return set(names)
        if self.resident == "none":
            return set()
        if self.resident != "auto":
            return set(self.resident) & set(names)
        be = op.batch_elems()
        nbytes = 4 * be * len(op.batches)
        free, _ = torch.cuda.mem_get_info(op.device)
        # two slots per streamed array, the k-major staging buffer, the batch scratch and a BF16 batch of x
        staging = (4 * 2 * len(names) + 4 + 4 + 2 + (8 if self.tv > 0 else 0)) * be
        room = max(0, free - staging - MARGIN_GB * 1024 ** 3 - op.lazy_bytes())
        n = int(room // nbytes)
        if n >= len(names):
            # a host x0 of a resident x goes through a (K, Ny, Nx) device copy unless that does not fit as well
            self._stage_io = room < (len(names) + 1) * nbytes
            return set(names)
        if n == 2 and len(names) == 3 and t16_ok and self.bf16_T == "auto" and room >= 2.5 * nbytes:
            self._t16 = True
            return set(names)
        return set(names[:min(n, len(names))])

    @on_op_stream
    def _finish(self):
        op = self.op
        self._resolve_pending()
        if self._final_pending:
            # the closing full forward (writes D only, reads x) and the objective on the operator's stream; x, z and y
            # (final since the last update) converted and downloaded on a side stream meanwhile
            self._final_pending = False
            side = torch.cuda.Stream(op.device)
            side.wait_stream(op.stream())
            op._fill(self.D, 0.0)
            self._pass(None, "full")
            self._wait_prefault()
            z_host, y_host = self._host_out
            with torch.cuda.stream(side):
                if not self._x_on_gpu:
                    op.from_batches(self.X.dev, self.x, stream=side)
                    host_copier().to_host(self.x, self._host_x, stream=side)
                z = torch.empty(op.coeff_shape, dtype=torch.float32, device=op.device)
                op.from_batches(self.Z.dev, z, stream=side)
                host_copier().to_host(z, z_host, stream=side)
                host_copier().to_host(self.y, y_host, stream=side)
            side.synchronize()
            del z
            self._f = self._deviance(self.D)
            if self.iter_stats:
                self.iter_stats[-1]["f"] = self._f
            if self._x_on_gpu:
                op.from_batches(self.X.dev, self.x)
            return self._finish_state(z_host, y_host, {})
        self._x_out()
        if self.Z.resident and self._stage is None:
            z = torch.empty(op.coeff_shape, dtype=torch.float32, device=op.device)
            op.from_batches(self.Z.dev, z)
            z_host = self._host_out[0]
            host_copier().to_host(z, z_host)
            del z
        else:
            z_host = np.empty(op.coeff_shape, np.float32)
            self._stage.store(self.Z, z_host.reshape(-1), self.pipe)
        tv_state = {}
        for arr, nm in ((self.QX, "qx"), (self.QY, "qy")):
            if arr is None:
                continue
            h = np.empty(op.coeff_shape, np.float32)
            if arr.resident and self._stage is None:
                q = torch.empty(op.coeff_shape, dtype=torch.float32, device=op.device)
                op.from_batches(arr.dev, q)
                host_copier().to_host(q, h)
            else:
                self._stage.store(arr, h.reshape(-1), self.pipe)
            tv_state[nm] = h
        self.pipe.synchronize()
        y_host = self._host_out[1] if self._host_out is not None else np.empty(op.data_shape, np.float32)
        host_copier().to_host(self.y, y_host)
        return self._finish_state(z_host, y_host, tv_state)

    def _finish_state(self, z_host, y_host, tv_state):
        self.state = {"epoch": self._ep0 + len(self.iter_stats), "z": z_host, "y": y_host, **tv_state}
        self.final_stats = {"epochs": len(self.iter_stats), "final_f": self._f, "setup_s": self._t_setup,
                            "rho": self.rho_used, "subsets": self.M, "resident": self.resident_used,
                            "time": time.perf_counter() - self._t_start, "tv": self.tv, "tv_prob": self.tv_prob,
                            "graph_replays": self.graph_replays, "T_bf16": self._t16, **self.scales}
        out = self.x if self._x_on_gpu else self._host_x
        self.b = self.w = self.g = self.bg = self.y = self.sig = self.D = None
        self.X = self.Z = self.T = self.dzk = self.xkb = self._stage = self._ray = self._tiles = None
        self.QX = self.QY = self.dqx = self.dqy = None
        self._graphs = {}
        self._side = self._x_snap = self._D_diag = self._side_sino = self._side_scratch = None
        self.x = None
        return out


def _ptr(t):
    return None if t is None else t.data_ptr()


def _patch_neighbours(op):
    """(right, down, left, up) int32 indices of every flat coefficient's neighbour within its patch (a row-major
    h x w box at coff), -1 at the box edges (spdhg_poisson.py:981-999)."""
    P = op._patches
    coff = np.asarray(P["coff"], np.int64)
    h, w = np.asarray(P["h"], np.int64), np.asarray(P["w"], np.int64)
    sizes = h * w
    nc = int(op.n_coef)
    if not (np.array_equal(coff, np.r_[0, np.cumsum(sizes)[:-1]]) and int(sizes.sum()) == nc):
        raise RuntimeError("the local operator's patches are not stored contiguously")
    j = np.arange(nc, dtype=np.int64)
    loc = j - np.repeat(coff, sizes)
    ww, hh = np.repeat(w, sizes), np.repeat(h, sizes)
    r, c = loc // ww, loc % ww
    return [a.astype(np.int32) for a in (np.where(c < ww - 1, j + 1, -1), np.where(r < hh - 1, j + ww, -1),
                                         np.where(c > 0, j - 1, -1), np.where(r > 0, j - ww, -1))]
