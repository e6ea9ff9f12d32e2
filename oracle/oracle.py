"""CPU oracle of diffractom's reconstruction hot path: TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm, as the checker of the CUDA
kernels or as the timed CPU baseline; the package diffractom_b200 never imports it. It wraps oracle/_build/liboracle.so
(the C restatement in oracle.c / oracle_core.h, built by oracle/Makefile) and composes its functions into the operator
and the SPDHG iteration of the reference (functions cite the reference file:line they follow):

  OracleOperator    forward / adjoint of SinglePhaseForwardOperator (SPFO:1646-1728, 1966-2033), full or per angle
                    subset, batch by batch, with the PF matrix evaluated densely (create_pfo_matrix.py:108-199) and
                    compacted into the two CSR copies (pf_kernels.cl:482-548)
  spdhg_reference   SPDHGPoisson.run (optimization/spdhg_poisson.py:513-751) for GPU-resident arrays (float32 state,
                    float64 prox and sums, as the reference), with the TV block
  fista_poisson_reference  FISTAPoisson.run (optimization/fista_poisson.py:414-610) for arrays on the device
  spdhg_reference64 the same loop entirely in float64 (state, data, images, step sizes): the FP64 oracle that the
                    float32 and BF16 paths' errors are stated against
  chambolle_pock_poisson_tv   a float64 primal-dual solve of the Poisson + (hierarchical) TV problem on explicit
                    matrices: the independent optimum the tree-TV tests compare SPDHG's objective with

Parity pins (tests/test_oracle.py): OracleOperator against the reference's float64 ReferenceModel on the golden
fixtures of tests/golden (forward and transpose within 2e-5 of the maximum, as the reference's own
tests/test_differentiable.py:31-40; the PF matrix likewise), and the host geometry against the same fixtures.
"""
from __future__ import annotations

import ctypes
import subprocess
from ctypes import c_double, c_float, c_int, c_int64, c_uint64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        h = ctypes.CDLL(str(LIB))
        P, I, F = c_void_p, c_int, c_float
        for suf in ("_f64", "_f32", "_f64io"):
            getattr(h, "orc_radon_forward" + suf).argtypes = [P, P, P, I, I, I, I, I, I, I, F]
            getattr(h, "orc_radon_backward" + suf).argtypes = [P, P, P, I, I, I, I, I, I, I]
            getattr(h, "orc_spmm_forward" + suf).argtypes = [P, P, P, P, P, P, I, I, I, I, I]
            getattr(h, "orc_spmm_adjoint" + suf).argtypes = [P, P, P, P, P, P, I, I, I, I, I, F, I]
        h.orc_pf_dense.argtypes = [P, P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, I, F, I]
        h.orc_csr_counts.argtypes = [P, I, I, I, P, P]
        h.orc_csr_fill.argtypes = [P, I, I, I, P, P, P, P, P, P]
        h.orc_dual_update_sub.argtypes = [P, P, P, P, P, c_uint64, P, c_uint64, P, c_uint64, F, P, c_uint64,
                                          c_uint64]
        h.orc_spdhg_update.argtypes = [P, P, P, P, F, F, c_uint64]
        h.orc_deviance.argtypes = [P, P, P, c_uint64, P, c_uint64, P, c_uint64, F, c_uint64]
        h.orc_deviance.restype = c_double
        h.orc_num_threads.restype = c_int
        for suf in ("_f32", "_f64"):
            getattr(h, "orc_transpose" + suf).argtypes = [P, P, c_int64, c_int64, c_int64, c_int64]
        _lib = h
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class OracleOperator:
    """The reference operator on the CPU from its host geometry (float32 arrays as the reference uploads them)."""

    def __init__(self, *, coords, poles, axis_start, axis_count, inv_sigma2, norm, quad_w, geo, scale, n_taps,
                 kernel, Nx, Ny, My, cut, batches, intens=None, precision="f64"):
        self.coords = _c(coords, np.float32)
        self.R, self.S, self.C, self.Se, self.P = self.coords.shape[:5]
        self.poles = _c(poles, np.float32)
        self.K, self.A = self.poles.shape[:2]
        self.axis_start = _c(axis_start, np.int32)
        self.axis_count = _c(axis_count, np.float32)
        self.inv_sigma2, self.norm = _c(inv_sigma2, np.float32), _c(norm, np.float32)
        self.quad_w = None if quad_w is None or np.size(quad_w) == 0 else _c(quad_w, np.float32)
        self.intens = None if intens is None else _c(intens, np.float32)
        self.geo = _c(geo, np.float32)
        self.scale, self.n_taps = float(scale), int(n_taps)
        self.kernel = 1 if kernel in ("trapezoid", 1) else 0
        self.Nx, self.Ny, self.My = int(Nx), int(Ny), int(My)
        self.cut = float(cut)
        self.CP = self.C * self.P
        self.batches = [(int(k0), int(kb)) for k0, kb in batches]
        self.suffix = "_" + precision
        self.io = np.float64 if precision == "f64io" else np.float32   # image / data arrays
        self._csr = {}

    @classmethod
    def from_operator(cls, op, precision="f64", batches=None):
        """The oracle of a diffractom_b200 operator (or of its OperatorGeometry): its host arrays and its batches
        (default: the operator's, one batch of all orientations for a bare geometry)."""
        if batches is None:
            batches = ([(b["k_start"], b["K_batch"]) for b in op.batches] if hasattr(op, "batches")
                       else [(0, op.K)])
        return cls(coords=op.coords_cpu, poles=op.poles_cpu, axis_start=op.axis_start_cpu, axis_count=op.axis_count_cpu,
                   inv_sigma2=op.inv_sigma2_cpu, norm=op.norm_factor_cpu, quad_w=op.quad_weights_cpu,
                   geo=op.radon_geo.geo, scale=op.radon_geo.scale, n_taps=op.radon_geo.n_taps, kernel=op.radon_kernel,
                   Nx=op.Nx, Ny=op.Ny, My=op.My, cut=op.pf_cut, batches=batches,
                   intens=None if op.normalized else op.intens_cpu, precision=precision)

    # ---- PF matrix
    def pf_dense(self, k0, kb):
        out = np.empty((self.R, kb, self.C, self.P), np.float32)
        lib().orc_pf_dense(_p(self.coords), _p(self.poles), _p(self.axis_start), _p(self.axis_count),
                           _p(self.inv_sigma2), _p(self.norm), _p(self.quad_w), _p(self.intens), _p(out), self.R, k0,
                           kb, self.C, self.P, self.A, self.S, self.Se, self.cut, int(self.intens is None))
        return out

    def csr(self, k0, kb):
        """Both CSR copies of the batch (adjoint rows r * kb + k over j; forward rows r * CP + j over k)."""
        key = (k0, kb)
        if key not in self._csr:
            pf = _c(self.pf_dense(k0, kb).reshape(self.R, kb, self.CP), np.float32)
            ca = np.empty(self.R * kb, np.int32)
            cf = np.empty(self.R * self.CP, np.int32)
            lib().orc_csr_counts(_p(pf), self.R, kb, self.CP, _p(ca), _p(cf))
            pa = np.zeros(self.R * kb + 1, np.int32)
            np.cumsum(ca, out=pa[1:])
            pfw = np.zeros(self.R * self.CP + 1, np.int32)
            np.cumsum(cf, out=pfw[1:])
            nnz = int(pa[-1])
            cj, va = np.empty(max(nnz, 1), np.uint16), np.empty(max(nnz, 1), np.float32)
            ck, vf = np.empty(max(nnz, 1), np.uint16), np.empty(max(nnz, 1), np.float32)
            lib().orc_csr_fill(_p(pf), self.R, kb, self.CP, _p(pa), _p(cj), _p(va), _p(pfw), _p(ck), _p(vf))
            self._csr[key] = dict(row_ptr_a=pa, col_j=cj[:nnz], val_a=va[:nnz], row_ptr_f=pfw, col_k=ck[:nnz],
                                  val_f=vf[:nnz], nnz=nnz)
        return self._csr[key]

    # ---- operator
    def forward(self, x, subset=None, data=None, accumulate=False):
        """data (R, My, CP) = A x; subset (angle indices): only those rows are written (the others kept from data,
        default zeros); accumulate: A x is added to those rows of data instead (the batched products' beta = 1)."""
        x = _c(x, self.io).reshape(self.K, -1)
        npix = self.Nx * self.Ny
        if data is None:
            data = np.zeros((self.R, self.My, self.CP), self.io)
        else:
            data = _c(data, self.io)
        angles = np.arange(self.R) if subset is None else np.asarray(subset, np.int64)
        if not accumulate:
            data[angles] = 0.0
        om = _c(angles, np.int32)
        geo = _c(self.geo[angles], np.float32)
        L = lib()
        for k0, kb in self.batches:
            img = self._transposed(x[k0:k0 + kb])                # (npix, kb) channel-fastest
            sino = np.empty((len(angles), self.My, kb), self.io)
            getattr(L, "orc_radon_forward" + self.suffix)(_p(img), _p(sino), _p(geo), len(angles), self.Nx, self.Ny,
                                                          self.My, kb, kb, self.kernel, self.scale)
            c = self.csr(k0, kb)
            getattr(L, "orc_spmm_forward" + self.suffix)(_p(sino), _p(c["row_ptr_f"]), _p(c["col_k"]), _p(c["val_f"]),
                                                         _p(data), _p(om), len(angles), self.My, self.CP, kb, 0)
        return data

    def adjoint(self, data, subset=None):
        """coeffs (K, Ny, Nx) = A^T data (subset: the rows of those angles only)."""
        data = _c(data, self.io)
        npix = self.Nx * self.Ny
        angles = np.arange(self.R) if subset is None else np.asarray(subset, np.int64)
        om = _c(angles, np.int32)
        geo = _c(self.geo[angles], np.float32)
        out = np.empty((self.K, npix), self.io)
        alpha = float(np.float32(self.R / np.pi))
        L = lib()
        for k0, kb in self.batches:
            c = self.csr(k0, kb)
            sino = np.empty((len(angles), self.My, kb), self.io)
            getattr(L, "orc_spmm_adjoint" + self.suffix)(_p(data), _p(c["row_ptr_a"]), _p(c["col_j"]),
                                                         _p(c["val_a"]), _p(sino), _p(om), len(angles), self.My, kb,
                                                         self.CP, kb, alpha, 0)
            img = np.empty((npix, kb), self.io)
            getattr(L, "orc_radon_backward" + self.suffix)(_p(sino), _p(img), _p(geo), len(angles), self.Nx, self.Ny,
                                                           self.My, kb, kb, self.kernel)
            self._transposed(img, out=out[k0:k0 + kb])
        return out.reshape(self.K, self.Ny, self.Nx)

    def _transposed(self, a, out=None):
        """a (rows, cols) C-contiguous in the io type -> its transpose (cols, rows), by the oracle's threads."""
        a = _c(a, self.io)
        rows, cols = a.shape
        if out is None:
            out = np.empty((cols, rows), self.io)
        assert out.flags.c_contiguous and out.shape == (cols, rows) and out.dtype == self.io
        fn = lib().orc_transpose_f64 if self.io == np.float64 else lib().orc_transpose_f32
        fn(_p(a), _p(out), rows, cols, cols, rows)
        return out


def periodic(a, n_data, dshape):
    """(array, period) as the solvers take weights / gain / background (fista_poisson.py:287-308)."""
    if a is None:
        return None, 0
    h = np.ascontiguousarray(a, dtype=np.float32).ravel()
    if h.size == 1:
        h = np.full(dshape[-1], float(h[0]), np.float32)
    return h, int(h.size)


def deviance(mu, b, w=None, g=None, bg=None, eps=1e-3):
    """Poisson deviance in float64 (fista_poisson.py:72-113, mode 0)."""
    mu, b = _c(mu, np.float32), _c(b, np.float32)
    w, pw = periodic(w, b.size, b.shape)
    g, pg = periodic(g, b.size, b.shape)
    bg, pbg = periodic(bg, b.size, b.shape)
    return float(lib().orc_deviance(_p(mu), _p(b), _p(w), pw, _p(g), pg, _p(bg), pbg, eps, b.size))


def epoch_order(rng, M, last):
    """SPDHGPoisson._epoch_order (spdhg_poisson.py:363-371): a permutation not starting with the last subset."""
    perm = rng.permutation(M)
    if M > 1 and int(perm[0]) == last:
        perm[[0, 1]] = perm[[1, 0]]
    return [int(m) for m in perm], int(perm[-1])


def epoch_sequence(rng, M, last, n_tv):
    """SPDHGPoisson._epoch_sequence (spdhg_poisson.py:373-381): the epoch's subsets with the TV block (-1) inserted
    n_tv times at random places."""
    order, last = epoch_order(rng, M, last)
    if n_tv == 0:
        return order, last
    n = M + n_tv
    tv_at = set(int(i) for i in rng.choice(n, n_tv, replace=False))
    it = iter(order)
    return [-1 if i in tv_at else next(it) for i in range(n)], last


def _shifted(a, axis):
    """The right (axis 2) or lower (axis 1) neighbour of every pixel of (K, Ny, Nx) a, 0 past the edge."""
    out = np.zeros_like(a)
    if axis == 2:
        out[:, :, :-1] = a[:, :, 1:]
    else:
        out[:, :-1, :] = a[:, 1:, :]
    return out


def tv_dual(x, T, qx, qy, lam, ps):
    """tv_dual_dense (spdhg_poisson.py:110-151) on (K, Ny, Nx) float32 arrays, float32 arithmetic in the kernel's
    order: returns (qx', qy', dqx, dqy)."""
    f = np.float32
    x, T, qx, qy = (np.asarray(a, f) for a in (x, T, qx, qy))
    K, Ny, Nx = x.shape
    vr0 = np.broadcast_to(np.arange(Nx) + 1 < Nx, x.shape)
    vd0 = np.broadcast_to((np.arange(Ny) + 1 < Ny)[:, None], x.shape)
    tr, td, xr, xd = _shifted(T, 2), _shifted(T, 1), _shifted(x, 2), _shifted(x, 1)
    vr = vr0 & (T > 0) & (tr > 0)
    vd = vd0 & (T > 0) & (td > 0)
    m = np.zeros_like(x)
    m = np.where(vr, np.maximum(m, T + tr), m)
    m = np.where(vd, np.maximum(m, T + td), m)
    pos = m > 0
    with np.errstate(divide="ignore", invalid="ignore"):
        st = np.where(pos, f(ps) / (f(4) * m), f(0))
    ax = np.where(vr & pos, qx + st * (xr - x), f(0)).astype(f)
    ay = np.where(vd & pos, qy + st * (xd - x), f(0)).astype(f)
    nrm = np.sqrt(ax * ax + ay * ay)
    big = nrm > f(lam)
    with np.errstate(divide="ignore", invalid="ignore"):
        c = np.where(big, f(lam) / nrm, f(1))
    ax = np.where(big, ax * c, ax).astype(f)
    ay = np.where(big, ay * c, ay).astype(f)
    return ax, ay, (ax - qx).astype(f), (ay - qy).astype(f)


def tv_adjoint(dqx, dqy):
    """tv_adjoint_dense (spdhg_poisson.py:153-165): dz = D^T dq."""
    v = (-dqx - dqy).astype(np.float32)
    v[:, :, 1:] += dqx[:, :, :-1]
    v[:, 1:, :] += dqy[:, :-1, :]
    return v


def tv_value(x, T):
    """tv_value_dense (spdhg_poisson.py:167-181): sum of the float32 gradient norms, float64 sum."""
    f = np.float32
    x, T = np.asarray(x, f), np.asarray(T, f)
    K, Ny, Nx = x.shape
    vr = np.broadcast_to(np.arange(Nx) + 1 < Nx, x.shape) & (T > 0) & (_shifted(T, 2) > 0)
    vd = np.broadcast_to((np.arange(Ny) + 1 < Ny)[:, None], x.shape) & (T > 0) & (_shifted(T, 1) > 0)
    gx = np.where(vr, _shifted(x, 2) - x, f(0)).astype(f)
    gy = np.where(vd, _shifted(x, 1) - x, f(0)).astype(f)
    return float(np.sum(np.sqrt(gx * gx + gy * gy), dtype=np.float64))


def spdhg_reference(op: OracleOperator, subsets, b, n_epochs, x0=None, weights=None, gain=None, background=None,
                    support=None, eps_counts=1e-3, rho="auto", seed=0, lam=0.0, diagnostics_interval=1, tv=0.0,
                    tv_prob=None):
    """SPDHGPoisson.run for arrays on the device (spdhg_poisson.py:513-719, setup 558-662), with the dense
    total-variation block when tv > 0 (spdhg_poisson.py:296-381, 430-484): returns (x, y, z, [deviance per
    diagnostics epoch], rho). The float64 parts (dual prox, deviance, mean) are float64 here as in the reference; the
    operator is the oracle's."""
    L = lib()
    R, My, CP = op.R, op.My, op.CP
    dshape = (R, My, CP)
    b = _c(b, np.float32)
    n = b.size
    row = My * CP
    w, pw = periodic(weights, n, dshape)
    g, pg = periodic(gain, n, dshape)
    bg, pbg = periodic(background, n, dshape)
    M = len(subsets)
    subsets = [np.asarray(s, np.int64) for s in subsets]
    p_tv = (1.0 / (M + 1) if tv_prob is None else float(tv_prob)) if tv > 0 else 0.0
    n_tv = max(1, int(round(M * p_tv / (1 - p_tv)))) if tv > 0 else 0
    p = (1.0 - p_tv) / M
    K, npix = op.K, op.Nx * op.Ny
    supp = np.ones(npix, bool) if support is None else np.asarray(support, bool).ravel()
    wv = np.ones(n, np.float32) if w is None else np.resize(w, n)
    counted = wv != 0
    if rho == "auto":
        sb, sn = float(np.sum(b.ravel()[counted], dtype=np.float64)), float(np.count_nonzero(counted))
        mean_b = sb / max(sn, 1.0)
        rho = 3e4 / mean_b ** 2 if mean_b > 0 else 1.0
    gamma = np.sqrt(rho)
    ones = np.broadcast_to(supp.astype(np.float32), (K, npix)).reshape(K, op.Ny, op.Nx)
    rowsum = op.forward(ones)
    sig = np.where(counted.reshape(dshape) & (rowsum > 0), np.float32(gamma) / np.where(rowsum > 0, rowsum, 1),
                   0).astype(np.float32)
    mask = counted.reshape(dshape).astype(np.float32)
    T = np.full((K, npix), np.inf, np.float32)
    for s in subsets:
        cs = op.adjoint(mask, subset=s).reshape(K, npix)
        upd = supp[None, :] & (cs > 0)
        T = np.where(upd, np.minimum(T, np.float32(p / gamma) / np.where(cs > 0, cs, 1)), T).astype(np.float32)
    T[np.isinf(T)] = 0.0
    x = np.zeros((K, npix), np.float32) if x0 is None else _c(x0, np.float32).reshape(K, npix).copy()
    x[:, ~supp] = 0.0
    x = np.maximum(x, 0)
    z = np.zeros((K, npix), np.float32)
    y = np.zeros(dshape, np.float32)
    D = np.zeros(dshape, np.float32)
    rng = np.random.default_rng(seed)
    last = None
    devs = []
    seq, last = epoch_sequence(rng, M, last, n_tv)
    if seq[0] >= 0:
        D = op.forward(x, subset=subsets[seq[0]], data=D)
    inv_p = np.float32(M) if tv <= 0 else np.float32(1.0 / p)
    qx = np.zeros((K, op.Ny, op.Nx), np.float32)
    qy = np.zeros_like(qx)
    T3 = T.reshape(K, op.Ny, op.Nx)
    for e in range(n_epochs):
        final = e + 1 == n_epochs
        want = (e + 1) % max(1, diagnostics_interval) == 0 or final
        nseq = None
        for j, m in enumerate(seq):
            eoe = j + 1 == len(seq)
            if not eoe:
                nb = seq[j + 1]
            elif not final:
                nseq, last = epoch_sequence(rng, M, last, n_tv)
                nb = nseq[0]
            else:
                nb = None
            if m >= 0:
                om = _c(subsets[m], np.int32)
                L.orc_dual_update_sub(_p(y), _p(D), _p(sig), _p(b), _p(w), pw, _p(g), pg, _p(bg), pbg, eps_counts,
                                      _p(om), row, len(om) * row)
                dz = op.adjoint(D, subset=subsets[m]).reshape(K, npix)
                ip = inv_p
            else:                                   # the TV block
                qx, qy, dqx, dqy = tv_dual(x.reshape(K, op.Ny, op.Nx), T3, qx, qy, tv, np.float32(0.99 * p_tv))
                dz = tv_adjoint(dqx, dqy).reshape(K, npix)
                ip = np.float32(1.0 / p_tv)
            L.orc_spdhg_update(_p(x), _p(z), _p(T), _p(_c(dz, np.float32)), float(ip), float(lam), x.size)
            m_next = nb if nb is not None and nb >= 0 else None
            if (eoe and want) or nb is None or (m_next is not None and m_next == m):
                if (eoe and want) or m_next is not None:
                    D = op.forward(x)
                    if eoe and want:
                        f = deviance(D, b, w, g, bg, eps_counts)
                        if tv > 0:
                            f += tv * tv_value(x.reshape(K, op.Ny, op.Nx), T3)
                        devs.append(f)
            elif m_next is not None:
                D = op.forward(x, subset=subsets[m_next], data=D)
        if nseq is not None:
            seq = nseq
    return x.reshape(K, op.Ny, op.Nx), y, z.reshape(K, op.Ny, op.Nx), devs, rho


def _full64(a, n):
    """A periodic float32 array (weights / gain / background) expanded to n float64 values, or None."""
    if a is None:
        return None
    h = np.ascontiguousarray(a, np.float32).ravel()
    return np.resize(h, n).astype(np.float64)


def deviance64(mu, b, w=None, g=None, bg=None, eps=1e-3):
    """Poisson deviance with every operand in float64 (fista_poisson.py:72-113, mode 0): sum w / g [m - b + b log(b /
    m)], m = max(mu, 0) + bg + eps g, over the points with w != 0."""
    mu = np.asarray(mu, np.float64).ravel()
    b = np.asarray(b, np.float32).ravel().astype(np.float64)
    n = b.size
    wv, gv, bgv = _full64(w, n), _full64(g, n), _full64(bg, n)
    gg = np.ones(n) if gv is None else gv
    m = np.maximum(mu, 0.0) + (0.0 if bgv is None else bgv) + float(np.float32(eps)) * gg
    with np.errstate(divide="ignore", invalid="ignore"):
        term = m - b + np.where(b > 0, b * np.log(np.where(b > 0, b, 1.0) / m), 0.0)
    sc = (1.0 if wv is None else wv) / gg
    live = np.ones(n, bool) if wv is None else wv != 0
    return float(np.sum((sc * term)[live]))


def spdhg_reference64(op: OracleOperator, subsets, b, n_epochs, x0=None, weights=None, gain=None, background=None,
                      support=None, eps_counts=1e-3, rho="auto", seed=0, lam=0.0, diagnostics_interval=1):
    """SPDHGPoisson.run (spdhg_poisson.py:513-719, set-up 558-662) entirely in float64: the operator's forward and
    adjoint with float64 images, sinograms and data (op built with precision "f64io"; the tap weights and PF values
    are the operator's float32 ones), float64 step sizes S and T, dual step (the closed-form prox of
    spdhg_poisson.py:69-91), primal step (spdhg_poisson.py:95-106) and deviance. The same subset schedule
    (default_rng(seed)) as the float32 loops; no TV block. Returns (x, y, z, [deviance per diagnostics epoch], rho,
    {"S": S, "T": T}) with x, z (K, Ny, Nx) and y, S data-shaped, all float64."""
    if op.io is not np.float64:
        raise ValueError("spdhg_reference64 needs an oracle operator of precision 'f64io'")
    R, My, CP = op.R, op.My, op.CP
    dshape = (R, My, CP)
    b32 = np.ascontiguousarray(b, np.float32).reshape(dshape)
    n = b32.size
    b64 = b32.astype(np.float64)
    wv, gv, bgv = _full64(weights, n), _full64(gain, n), _full64(background, n)
    M = len(subsets)
    subsets = [np.asarray(s_, np.int64) for s_ in subsets]
    p = 1.0 / M
    K, npix = op.K, op.Nx * op.Ny
    supp = np.ones(npix, bool) if support is None else np.asarray(support, bool).ravel()
    counted = np.ones(n, bool) if wv is None else wv != 0
    if rho == "auto":
        mean_b = float(np.sum(b64.ravel()[counted])) / max(float(np.count_nonzero(counted)), 1.0)
        rho = 3e4 / mean_b ** 2 if mean_b > 0 else 1.0
    gamma = float(np.sqrt(rho))
    ones = np.broadcast_to(supp.astype(np.float64), (K, npix)).reshape(K, op.Ny, op.Nx)
    rowsum = op.forward(ones).ravel()
    S = np.where(counted & (rowsum > 0), gamma / np.where(rowsum > 0, rowsum, 1.0), 0.0)
    mask = counted.astype(np.float64).reshape(dshape)
    T = np.full((K, npix), np.inf)
    for s_ in subsets:
        cs = op.adjoint(mask, subset=s_).reshape(K, npix)
        upd = supp[None, :] & (cs > 0)
        T = np.where(upd, np.minimum(T, (p / gamma) / np.where(cs > 0, cs, 1.0)), T)
    T[np.isinf(T)] = 0.0
    x = np.zeros((K, npix)) if x0 is None else np.asarray(x0, np.float64).reshape(K, npix).copy()
    x[:, ~supp] = 0.0
    x = np.maximum(x, 0.0)
    z = np.zeros((K, npix))
    y = np.zeros(n)
    D = np.zeros(dshape)
    row = My * CP
    g1 = np.ones(n) if gv is None else gv
    sc_all = (1.0 if wv is None else wv) / g1
    r_all = (0.0 if bgv is None else bgv) + float(np.float32(eps_counts)) * g1
    live_all = counted & (S != 0)

    def dual(m):
        """The Poisson conjugate prox on the rows of subset m; D holds A x there on entry, the dual change on exit."""
        idx = (subsets[m][:, None] * row + np.arange(row)[None, :]).ravel()
        Dv = D.reshape(-1)
        yo, si, sc = y[idx], S[idx], sc_all if np.isscalar(sc_all) else sc_all[idx]
        v = yo + si * Dv[idx] + si * (r_all[idx] if not np.isscalar(r_all) else r_all)
        dd = v - sc
        yn = 0.5 * (v + sc - np.sqrt(dd * dd + 4.0 * si * sc * b64.ravel()[idx]))
        yn = np.where(live_all[idx], yn, 0.0)
        Dv[idx] = yn - yo
        y[idx] = yn

    rng = np.random.default_rng(seed)
    last = None
    devs = []
    seq, last = epoch_sequence(rng, M, last, 0)
    D = op.forward(x, subset=subsets[seq[0]], data=D)
    inv_p = float(M)
    for e in range(n_epochs):
        final = e + 1 == n_epochs
        want = (e + 1) % max(1, diagnostics_interval) == 0 or final
        nseq = None
        for j, m in enumerate(seq):
            eoe = j + 1 == len(seq)
            if not eoe:
                nb = seq[j + 1]
            elif not final:
                nseq, last = epoch_sequence(rng, M, last, 0)
                nb = nseq[0]
            else:
                nb = None
            dual(m)
            dz = op.adjoint(D, subset=subsets[m]).reshape(K, npix)
            z += dz
            zb = z + inv_p * dz
            x = np.where(T > 0, np.maximum(0.0, x - T * (zb + lam)), 0.0)
            if (eoe and want) or nb is None or nb == m:
                if (eoe and want) or nb is not None:
                    D = op.forward(x)
                    if eoe and want:
                        devs.append(deviance64(D, b32, weights, gain, background, eps_counts))
            else:
                D = op.forward(x, subset=subsets[nb], data=D)
        if nseq is not None:
            seq = nseq
    return (x.reshape(K, op.Ny, op.Nx), y.reshape(dshape), z.reshape(K, op.Ny, op.Nx), devs, rho,
            {"S": S.reshape(dshape), "T": T.reshape(K, op.Ny, op.Nx)})


def fista_poisson_reference(op: OracleOperator, b, niter, x0=None, weights=None, gain=None, background=None,
                            support=None, lam=0.0, eps_counts=1e-3, floor_counts=1.0,
                            refresh=(5, 10, 20, 40, 80, 160, 320, 640, 1280, 2560, 5120), refresh_on_failure=True,
                            max_backtracks=60, start="wls", n_start=20):
    """FISTAPoisson.run for arrays on the device (fista_poisson.py:414-610; kernels 60-282): FISTA in the diagonal
    SQS metric D = 1 / A^T(c A 1_S) with descent-lemma backtracking, a metric taken again at y on the first rejected
    step, function-value restarts, metric refreshes with momentum restarts at the iterations in `refresh`, the
    weighted least squares start phase (mode 1) from a zero x0, float32 arrays and float64 sums as the reference.
    Returns (x (K, Ny, Nx) float32, [per-iteration dict: f, obj, theta, backtracks, restart, metric_refresh,
    local_metric], final dict: final_f, final_obj, adjoint_scale, backtracks, restarts)."""
    f32, f64 = np.float32, np.float64
    dshape = (op.R, op.My, op.CP)
    K, npix = op.K, op.Nx * op.Ny
    b = _c(b, f32).ravel()
    n = b.size
    wv = np.ones(n, f32) if weights is None else np.resize(_c(weights, f32).ravel(), n)
    gv = np.ones(n, f32) if gain is None else np.resize(_c(gain, f32).ravel(), n)
    bgv = np.zeros(n, f32) if background is None else np.resize(_c(background, f32).ravel(), n)
    supp = np.ones(npix, bool) if support is None else np.asarray(support, bool).ravel()
    eps = f32(eps_counts)
    floor = f32(floor_counts)
    counted = wv != 0
    fwd = lambda v: op.forward(v.reshape(K, op.Ny, op.Nx)).ravel().astype(f32)
    adj = lambda d: op.adjoint(d.reshape(dshape)).ravel().astype(f32)
    inside = np.broadcast_to(supp, (K, npix)).ravel()

    def data_term(mu, mode, want_grad):
        """f (float64) and, with want_grad, df/dmu (float32): poisson_value_grad (fista_poisson.py:71-101)."""
        sc = wv.astype(f64) / gv.astype(f64)
        bi = b.astype(f64)
        if mode == 0:
            m = np.maximum(mu, f32(0)).astype(f64) + bgv.astype(f64) + f64(eps) * gv.astype(f64)
            with np.errstate(divide="ignore", invalid="ignore"):
                v = m - bi + np.where(bi > 0, bi * np.log(np.where(bi > 0, bi, 1.0) / m), 0.0)
                gr = sc * (1.0 - bi / m)
        else:
            r = mu.astype(f64) + bgv.astype(f64) - bi
            c = sc / np.maximum(bi, f64(floor) * gv.astype(f64))
            v = 0.5 * c * r * r
            gr = c * r
        f = float(np.sum(np.where(counted, sc * v if mode == 0 else v, 0.0)))
        return f, (np.where(counted, gr, 0.0).astype(f32) if want_grad else None)

    state = {"adjoint_scale": 1.0}

    def metric(mu, mode):
        """D (float32): times_curvature, the adjoint, invert_metric (fista_poisson.py:103-134, 170-178, 384-411)."""
        ones = inside.astype(f32)
        u = fwd(ones)
        if mode == 0:
            m = np.maximum(np.maximum(mu, f32(0)) + bgv, floor * gv)
            c = np.where(counted, wv / gv * np.maximum(b, m) / (m * m), f32(0)).astype(f32)
        else:
            c = np.where(counted, wv / (gv * np.maximum(b, floor * gv)), f32(0)).astype(f32)
        u_r = float(np.sum(c.astype(f64) * u.astype(f64) * u.astype(f64)))
        u = (u * c).astype(f32)
        d = adj(u)
        at_u = float(np.sum(np.where(inside, d.astype(f64), 0.0)))
        if u_r > 0 and at_u > 0:
            state["adjoint_scale"] = at_u / u_r
        with np.errstate(divide="ignore"):
            return np.where(inside & (d > 0), f32(1) / d, f32(0)).astype(f32)

    x = np.zeros(K * npix, f32) if x0 is None else _c(x0, f32).ravel().copy()
    x[~inside] = 0
    x = np.maximum(x, f32(0))
    zero_start = float(x.max()) == 0.0
    wls_until = n_start if (start == "wls" and n_start > 0 and zero_start) else 0
    mode = 1 if wls_until else 0
    if zero_start and start == "uniform":
        ones = inside.astype(f32)
        a1 = fwd(ones)
        sb = float(np.sum(wv.astype(f64) * b.astype(f64)))
        sa = float(np.sum(wv.astype(f64) * a1.astype(f64)))
        if sa > 0 and sb > 0:
            x = (ones * f32(sb / sa)).astype(f32)
    t_mom, theta = 1.0, 1.0
    y = x.copy()
    Ax = fwd(x)
    Ay = Ax.copy()
    D = metric(Ax, mode)
    f_x, _ = data_term(Ax, mode, False)
    F_x = f_x + lam * float(np.sum(x.astype(f64)))
    stats = []
    n_bt_total = n_restart = 0
    for k in range(niter):
        it = k + 1
        f_y, gmu = data_term(Ay, mode, True)
        grad = adj(gmu)
        theta = min(1.0, 2.0 * theta)
        n_bt, local = 0, False
        while True:
            xn = np.where(D > 0, np.maximum(f32(0), y - f32(theta) * D * (grad + f32(lam))), f32(0)).astype(f32)
            Axn = fwd(xn)
            f_n, _ = data_term(Axn, mode, False)
            dd = xn.astype(f64) - y.astype(f64)
            lin_adj = float(np.sum(grad.astype(f64) * dd))
            quad_raw = float(np.sum(np.where(D > 0, dd * dd / np.where(D > 0, D, 1).astype(f64), 0.0)))
            xsum = float(np.sum(xn.astype(f64)))
            lin = lin_adj / state["adjoint_scale"]
            quad = quad_raw / (theta * state["adjoint_scale"])
            if f_n <= f_y + lin + 0.5 * quad + 1e-6 * abs(f_y) or quad == 0.0:
                break
            n_bt += 1
            if not local and refresh_on_failure:
                D = metric(fwd(y), mode)
                local, theta = True, 1.0
                continue
            theta *= 0.5
            if n_bt > max_backtracks:
                raise RuntimeError("fista_poisson_reference: no sufficient decrease")
        n_bt_total += n_bt
        F_n = f_n + lam * xsum
        restarted = F_n > F_x
        if restarted:
            t_mom = 1.0
            n_restart += 1
        t_new = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t_mom * t_mom))
        beta = f32((t_mom - 1.0) / t_new)
        t_mom = t_new
        y = (xn + beta * (xn - x)).astype(f32)
        Ay = (Axn + beta * (Axn - Ax)).astype(f32)
        x, Ax = xn, Axn
        f_x, F_x = f_n, F_n
        switch = mode == 1 and it >= wls_until
        if switch:
            mode = 0
            f_x, _ = data_term(Ax, mode, False)
            F_x = f_x + lam * xsum
        refreshed = (it in refresh or switch) and k + 1 < niter and mode == 0
        if refreshed:
            D = metric(Ax, mode)
            t_mom, theta = 1.0, 1.0
            y, Ay = x.copy(), Ax.copy()
        elif it % 50 == 0:
            Ay = fwd(y)
        stats.append({"iter": it, "f": f_n, "obj": F_n, "theta": theta, "backtracks": n_bt, "local_metric": local,
                      "restart": bool(restarted), "metric_refresh": bool(refreshed)})
    final = {"final_f": f_x, "final_obj": F_x, "adjoint_scale": state["adjoint_scale"], "backtracks": n_bt_total,
             "restarts": n_restart}
    return x.reshape(K, op.Ny, op.Nx), stats, final


def fista_ls_reference(op: OracleOperator, b, niter, tau, x0=None, prox="nonneg", lam=0.0, support=None, clip=False,
                       delta=1e-2, weights=None):
    """FISTAL2 / FISTAHuber (fista_l2.py, fista_huber.py with fused_update.py:22-49) in float64 on the oracle
    operator: r = w (A y - b), f = 0.5 sum r^2, r clipped to [-delta, delta] (Huber); x' = prox(y - tau A^T r),
    0 outside the support; y = x' + beta (x' - x); t' = (1 + sqrt(1 + 4 t^2)) / 2, beta = (t - 1) / t'. op should
    be a float64-I/O oracle (precision "f64io"). Returns (x, [f per iteration], [||grad|| per iteration])."""
    K, npix = op.K, op.Nx * op.Ny
    dshape = (op.R, op.My, op.CP)
    b = np.asarray(b, np.float64).reshape(dshape)
    w = None if weights is None else np.resize(np.asarray(weights, np.float64).ravel(), b.size).reshape(dshape)
    supp = np.ones(npix, bool) if support is None else np.asarray(support, bool).ravel()
    x = np.zeros((K, npix)) if x0 is None else np.asarray(x0, np.float64).reshape(K, npix).copy()
    x[:, ~supp] = 0.0
    y = x.copy()
    t = 1.0
    lt = lam * tau
    fs, gs = [], []
    for _ in range(niter):
        r = op.forward(y.reshape(K, op.Ny, op.Nx)).astype(np.float64) - b
        if w is not None:
            r = w * r
        fs.append(0.5 * float(np.sum(r * r)))
        if clip:
            r = np.clip(r, -delta, delta)
        g = op.adjoint(r).reshape(K, npix).astype(np.float64)
        gs.append(float(np.sqrt(np.sum(g * g))))
        t_new = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t * t))
        beta = (t - 1.0) / t_new
        v = y - tau * g
        if prox == "nonneg":
            v = np.maximum(v, 0.0)
        elif prox == "l1":
            v = np.sign(v) * np.maximum(np.abs(v) - lt, 0.0)
        else:
            v = np.maximum(v - lt, 0.0)
        v[:, ~supp] = 0.0
        y = v + beta * (v - x)
        x = v
        t = t_new
    return x.reshape(K, op.Ny, op.Nx), fs, gs


def _data_terms(b, weights, gain, background, dshape, fit=None):
    """Data-shaped float32 (w with unfitted rows 0, g, bg) as the solvers' periodic arrays expand them."""
    n = int(np.prod(dshape))
    w = np.ones(n, np.float32) if weights is None else np.resize(np.asarray(weights, np.float32).ravel(), n)
    g = np.ones(n, np.float32) if gain is None else np.resize(np.asarray(gain, np.float32).ravel(), n)
    bg = np.zeros(n, np.float32) if background is None else np.resize(np.asarray(background, np.float32).ravel(), n)
    w, g, bg = (a.reshape(dshape).copy() for a in (w, g, bg))
    if fit is not None:
        w[~np.asarray(fit, bool)] = 0.0
    return w, g, bg


def osem_reference(op: OracleOperator, subsets, b, n_epochs, x0, weights=None, gain=None, background=None,
                   support=None, eps_counts=1e-3, seed=0, lam=0.0, start_floor=0.01):
    """OSEMPoisson.run (optimization/osem_poisson.py:95-185) on the oracle operator, float32 arithmetic in the
    reference's order: returns (x, final deviance)."""
    dshape = (op.R, op.My, op.CP)
    K, npix = op.K, op.Nx * op.Ny
    f = np.float32
    b = _c(b, f).reshape(dshape)
    M = 1 if subsets is None else len(subsets)
    fit = None
    if subsets is not None:
        fit = np.zeros(op.R, bool)
        for s_ in subsets:
            fit[np.asarray(s_, np.int64)] = True
    w, g, bg = _data_terms(b, weights, gain, background, dshape, fit)
    eps = f(eps_counts)
    with np.errstate(divide="ignore", invalid="ignore"):
        wg = np.where(w != 0, w / g, f(0)).astype(f)
    sub = (lambda m: None) if subsets is None else (lambda m: subsets[m])
    sens = [op.adjoint(wg, subset=sub(m)).reshape(K, npix).astype(f) for m in range(M)]
    allowed = np.ones((K, npix), bool) if support is None else np.broadcast_to(np.asarray(support, bool).ravel(),
                                                                               (K, npix))
    x = np.where(allowed, _c(x0, f).reshape(K, npix), f(0)).astype(f)
    if start_floor:
        pos = x[x > 0]
        if pos.size:
            floor = float(start_floor) * float(np.median(pos.astype(np.float64)))
        else:
            st = sum(float(sm[allowed].sum(dtype=np.float64)) for sm in sens)
            tot = float(np.sum(wg.astype(np.float64) * b)) - float(np.sum(wg.astype(np.float64) * bg))
            floor = max(tot, 0.0) / st if st > 0 else 1.0
        x = np.where(allowed, np.maximum(x.astype(np.float64), floor), 0.0).astype(f)
    rng = np.random.default_rng(seed)
    for _ in range(int(n_epochs)):
        order = rng.permutation(M) if M > 1 else [0]
        for m in order:
            m = int(m)
            pred = op.forward(x.reshape(K, op.Ny, op.Nx), subset=sub(m)).astype(f)
            mu = (np.maximum(pred, f(0)) + bg) + eps * g
            with np.errstate(divide="ignore", invalid="ignore"):
                r = np.where(w != 0, (w / g) * (b / mu), f(0)).astype(f)
            back = op.adjoint(r, subset=sub(m)).reshape(K, npix).astype(f)
            s = sens[m]
            with np.errstate(divide="ignore", invalid="ignore"):
                upd = np.where(s > 0, (x * back) / (s + f(lam)), x).astype(f)
            x = np.where(allowed, upd, f(0)).astype(f)
    pred = op.forward(x.reshape(K, op.Ny, op.Nx))
    return x.reshape(K, op.Ny, op.Nx), deviance(pred, b, w, g, bg, eps_counts)


def pdhg_reference(op: OracleOperator, b, niter, x0=None, weights=None, gain=None, background=None, support=None,
                   eps_counts=1e-3, rho="auto", lam=0.0):
    """PDHGPoisson.run for device arrays (optimization/pdhg_poisson.py:159-262) on the oracle operator: float32 state,
    the dual prox in float64; returns (x, [deviance per iteration], rho)."""
    dshape = (op.R, op.My, op.CP)
    K, npix = op.K, op.Nx * op.Ny
    f = np.float32
    b = _c(b, f).reshape(dshape)
    w, g, bg = _data_terms(b, weights, gain, background, dshape)
    counted = w != 0
    if rho == "auto":
        mean_b = float(np.sum(b[counted], dtype=np.float64)) / max(float(np.count_nonzero(counted)), 1.0)
        rho = 3e4 / mean_b ** 2 if mean_b > 0 else 1.0
    tau0, sigma0 = f(1.0 / np.sqrt(rho)), f(np.sqrt(rho))
    supp = np.ones(npix, bool) if support is None else np.asarray(support, bool).ravel()
    ones = np.broadcast_to(supp.astype(f), (K, npix)).reshape(K, op.Ny, op.Nx)
    rowsum = op.forward(ones).astype(f)
    with np.errstate(divide="ignore", invalid="ignore"):
        sig = np.where(counted & (rowsum > 0), sigma0 / rowsum, f(0)).astype(f)
        colsum = op.adjoint(counted.astype(f)).reshape(K, npix).astype(f)
        T = np.where(supp[None, :] & (colsum > 0), tau0 / colsum, f(0)).astype(f)
    x = np.maximum(_c(x0 if x0 is not None else np.zeros((K, npix), f), f).reshape(K, npix), f(0))
    x[:, ~supp] = 0.0
    xb = x.copy()
    y = np.zeros(dshape, f)
    Ax = op.forward(x.reshape(K, op.Ny, op.Nx)).astype(f)
    Axb = Ax.copy()
    s64 = np.where(counted, w.astype(np.float64) / g, 0.0)
    r64 = bg.astype(np.float64) + np.float64(f(eps_counts)) * g
    devs = []
    for it in range(1, int(niter) + 1):
        v = y.astype(np.float64) + sig.astype(np.float64) * Axb + sig.astype(np.float64) * r64
        d = v - s64
        yn = 0.5 * (v + s64 - np.sqrt(d * d + 4.0 * sig.astype(np.float64) * s64 * b))
        y = np.where(counted & (sig != 0), yn, 0.0).astype(f)
        grad = op.adjoint(y).reshape(K, npix).astype(f)
        xn = np.where(T > 0, np.maximum(f(0), x - T * (grad + f(lam))), f(0)).astype(f)
        xb = (f(2) * xn - x).astype(f)
        x = xn
        Axb = op.forward(xb.reshape(K, op.Ny, op.Nx)).astype(f)
        Ax = (f(0.5) * (Axb + Ax)).astype(f)
        if it % 50 == 0:
            Ax = op.forward(x.reshape(K, op.Ny, op.Nx)).astype(f)
        devs.append(deviance(Ax, b, w, g, bg, eps_counts))
    return x.reshape(K, op.Ny, op.Nx), devs, rho


def chambolle_pock_poisson_tv(A, D, b, gain, tv, free, eps=1e-3, n_iter=20000):
    """The minimiser of sum_i (mu_i - b_i log mu_i) / g + tv sum_p |(D x)_p| over x >= 0 (x_j = 0 where not free),
    mu = A x + eps g, by the diagonally preconditioned primal-dual method of Pock and Chambolle (ICCV 2011, alpha = 1:
    sigma_i = 1 / sum_j |K_ij|, tau_j = 1 / sum_i |K_ij|, K = [A; D]) in float64 on the explicit matrices. D: sparse,
    two rows (right, down) per penalty term p, already scaled by the term's weight; the dual of the Poisson rows is
    the prox of sigma F*, F(u) = (u + r - b log(u + r)) / g, r = eps g: the smaller root of
    y^2 - (c + v') y + v' c - sigma c b = 0, c = 1 / g, v' = v + sigma r; the TV rows are projected onto |q_p| <= tv.
    The independent check of the optimum the reference's tests/test_tree_tv.py:69-91 makes."""
    import scipy.sparse as sp
    K = sp.vstack([sp.csr_matrix(A), sp.csr_matrix(D)]).tocsr()
    KT = K.T.tocsr()
    absK = abs(K)
    sig = 1.0 / np.maximum(np.asarray(absK.sum(axis=1)).ravel(), 1e-30)
    tau = 1.0 / np.maximum(np.asarray(absK.sum(axis=0)).ravel(), 1e-30)
    tau[~np.asarray(free, bool)] = 0.0
    nA = A.shape[0]
    b = np.asarray(b, np.float64).ravel()
    c, r = 1.0 / gain, eps * gain
    sa = sig[:nA]
    x = np.zeros(A.shape[1])
    xb = x.copy()
    y = np.zeros(K.shape[0])
    for _ in range(n_iter):
        v = y + sig * (K @ xb)
        vp = v[:nA] + sa * r
        y[:nA] = 0.5 * ((c + vp) - np.sqrt((vp - c) ** 2 + 4.0 * sa * c * b))
        if tv > 0:
            q = v[nA:].reshape(-1, 2)
            y[nA:] = (q / np.maximum(1.0, np.hypot(q[:, 0], q[:, 1]) / tv)[:, None]).ravel()
        else:                                    # |q_p| <= 0
            y[nA:] = 0.0
        xn = np.maximum(0.0, x - tau * (KT @ y))
        xb = 2.0 * xn - x
        x = xn
    return x


def poisson_tv_objective(A, D, x, b, gain, tv, eps=1e-3):
    """sum (mu - b + b log(b / mu)) / g + tv sum_p |(D x)_p|, mu = max(A x, 0) + eps g (the solver's objective)."""
    b = np.asarray(b, np.float64).ravel()
    mu = np.maximum(A @ x, 0.0) + eps * gain
    dev = np.sum((mu - b + np.where(b > 0, b * np.log(np.where(b > 0, b, 1.0) / mu), 0.0)) / gain)
    g = (D @ x).reshape(-1, 2)
    return float(dev + tv * np.hypot(g[:, 0], g[:, 1]).sum())
