"""The hierarchical total variation of SPDHGPoisson (tv_tree=, local basis) on the GPU, as the reference's
tests/test_tree_tv.py checks it: its kernels (node-pixel sums, D^T dq on the node-pixels, the scatter) bit for bit
against NumPy float32; one radius is the plain TV (weight tv r / 2) bit for bit; a long run reaches the optimum of an
independent float64 primal-dual solve on the explicit matrices (objective within 1e-3, the solver's own objective
within 1e-4 of NumPy's); the tree duals are kept in the state and a run resumes from it."""
import ctypes

import numpy as np
import pytest

from conftest import case_inputs

torch = pytest.importorskip("torch")

RADII = (90.0, 45.0, 20.0)           # two penalised levels (edges 22.5, 12.5) over the diff case's 12 orientations


def _box_problem(K, Ny, Nx, seed=3, box=(3, 9, 4, 10)):
    """Every orientation allowed in one box of pixels; the true coefficients two half planes per orientation."""
    y0, y1, x0, x1 = box
    mask = np.zeros((K, Ny, Nx), bool)
    mask[:, y0:y1, x0:x1] = True
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[:Ny, :Nx]
    x_true = np.zeros((K, Ny, Nx), np.float32)
    for k in range(K):
        a = rng.uniform(0, np.pi)
        x_true[k] = rng.uniform(0.5, 1.5) * ((np.cos(a) * (xx - (x0 + x1) / 2) + np.sin(a) * (yy - (y0 + y1) / 2)) > 0)
    return mask, x_true * mask


def _tree_rows(k, iy, ix, pi, Ny, Nx, n_coef, tree, free):
    """The penalty's rows on the flat coefficients (scipy CSR): per level (the leaves as single-orientation cells
    with the leaf edge, then tree.levels()) and per (cell, pixel) holding free coefficients, the right and down
    differences of the cell's sums, scaled by the level's edge; two rows per (cell, pixel)."""
    from scipy.sparse import coo_matrix
    K = tree.K
    rows, cols, vals, base = [], [], [], 0
    for cell, edge in [(np.arange(K), tree.leaf_edge)] + tree.levels():
        members = {}
        for kk, y, x, j in zip(k, iy, ix, pi):
            if free[j]:
                members.setdefault((int(cell[kk]), int(y), int(x)), []).append(int(j))
        for (c, y, x), js in members.items():
            for comp, (dy, dx) in enumerate(((0, 1), (1, 0))):
                other = members.get((c, y + dy, x + dx))
                if other is not None:
                    r = base + 2 * ((c * Ny + y) * Nx + x) + comp
                    rows += [r] * (len(js) + len(other))
                    cols += js + other
                    vals += [-edge] * len(js) + [edge] * len(other)
        base += 2 * (int(cell.max()) + 1) * Ny * Nx
    return coo_matrix((vals, (rows, cols)), shape=(base, n_coef)).tocsr()


def _local_problem(golden, gain=0.02):
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport
    d = golden("diff_auto_trapezoid")
    cfg, mat, grid = case_inputs(d)
    mats, _ = grid.leaf_arrays()
    mask, x_true = _box_problem(len(mats), int(cfg["Ny"]), int(cfg["Nx"]))
    lop = LocalSinglePhaseForwardOperator(cfg, mat, grid, 1e-5, LocalSupport.from_mask(mask), normalized=True,
                                          quadrature=d["quadrature"], radon_kernel=d["kernel"], split_patches=False)
    assert lop.K == len(mats)                            # every orientation in the box, one patch each
    rng = np.random.default_rng(3)
    b = (rng.poisson(np.maximum(lop.direct(lop.from_dense(x_true)), 0) / gain) * gain).astype(np.float32)
    return lop, b, gain, np.asarray(mats, np.float64)


@pytest.mark.gpu
def test_tree_kernels_equal_numpy():
    from diffractom_b200 import _lib
    rng = np.random.default_rng(0)
    n, nn = 5000, 1300
    x = rng.random(n).astype(np.float32)
    owner = rng.integers(-1, nn, n)                      # -1: a coefficient in no node-pixel
    order = np.argsort(owner[owner >= 0], kind="stable")
    idx = np.flatnonzero(owner >= 0)[order].astype(np.int32)
    ptr = np.concatenate([[0], np.cumsum(np.bincount(owner[owner >= 0], minlength=nn))]).astype(np.int32)
    want_s = np.zeros(nn, np.float32)
    for j in range(nn):
        a = np.float32(0)
        for p in range(ptr[j], ptr[j + 1]):
            a = np.float32(a + x[idx[p]])
        want_s[j] = a
    dqx = rng.normal(size=nn).astype(np.float32)
    dqy = rng.normal(size=nn).astype(np.float32)
    left = np.where(rng.random(nn) < 0.7, rng.integers(0, nn, nn), -1).astype(np.int32)
    up = np.where(rng.random(nn) < 0.7, rng.integers(0, nn, nn), -1).astype(np.int32)
    v = (-dqx - dqy).astype(np.float32)
    v = np.where(left >= 0, v + dqx[np.maximum(left, 0)], v).astype(np.float32)
    want_w = np.where(up >= 0, v + dqy[np.maximum(up, 0)], v).astype(np.float32)
    mp = owner.astype(np.int32)
    dz = rng.normal(size=n).astype(np.float32)
    want_dz = np.where(mp >= 0, dz + want_w[np.maximum(mp, 0)], dz).astype(np.float32)
    dev = lambda a: torch.as_tensor(a, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    xd, ptrd, idxd, s = dev(x), dev(ptr), dev(idx), torch.empty(nn, device="cuda")
    _lib.call("dfx_tree_sums", xd.data_ptr(), ptrd.data_ptr(), idxd.data_ptr(), s.data_ptr(), nn, st)
    w = torch.empty(nn, device="cuda")
    dqxd, dqyd, leftd, upd, mpd, dzd = dev(dqx), dev(dqy), dev(left), dev(up), dev(mp), dev(dz)   # held while used
    _lib.call("dfx_tv_adjoint_local", dqxd.data_ptr(), dqyd.data_ptr(), w.data_ptr(), leftd.data_ptr(),
              upd.data_ptr(), nn, st)
    _lib.call("dfx_tree_scatter", w.data_ptr(), mpd.data_ptr(), dzd.data_ptr(), n, st)
    assert np.array_equal(s.cpu().numpy(), want_s)
    assert np.array_equal(w.cpu().numpy(), want_w)
    assert np.array_equal(dzd.cpu().numpy(), want_dz)


@pytest.mark.gpu
def test_single_radius_is_the_plain_tv(golden):
    from diffractom_b200 import OrientationTree, SPDHGPoisson
    lop, b, gain, mats = _local_problem(golden)
    tree = OrientationTree(mats, None, (4.0,))
    x0 = np.zeros(lop.coeff_shape, np.float32)
    a = SPDHGPoisson(lop, subsets=3, tv=3.0, seed=2)
    xa = a.run(x0.copy(), b, 15, gain=gain, diagnostics_interval=5)
    c = SPDHGPoisson(lop, subsets=3, tv=1.5, tv_tree=tree, seed=2)
    xc = c.run(x0.copy(), b, 15, gain=gain, diagnostics_interval=5)
    assert np.array_equal(xc, xa)
    assert "tree_q" not in c.state and np.array_equal(c.state["qx"], a.state["qx"])
    fa = [s["f"] for s in a.iter_stats if s["f"] is not None]
    fc = [s["f"] for s in c.iter_stats if s["f"] is not None]
    np.testing.assert_allclose(fc, fa, rtol=1e-12)


@pytest.mark.gpu
def test_tree_tv_reaches_the_optimum(golden):
    """3000 epochs of SPDHG with the hierarchical TV against 30000 float64 primal-dual iterations on the explicit A
    (columns of the operator) and the explicit penalty rows (the reference's tests/test_tree_tv.py:69-91)."""
    import scipy.sparse as sp
    from diffractom_b200 import OrientationTree, SPDHGPoisson
    from oracle.oracle import chambolle_pock_poisson_tv, poisson_tv_objective
    lop, b, gain, mats = _local_problem(golden)
    tree = OrientationTree(mats, None, RADII)
    assert len(tree.levels()) == 2 and tree.n_nodes[1] < lop.K_basis
    n = int(lop.n_coef)
    cols = []
    e = torch.zeros(n, device="cuda")
    for j in range(n):
        e.zero_()
        e[j] = 1.0
        cols.append(sp.csc_matrix(lop.direct(e).cpu().numpy().astype(np.float64).reshape(-1, 1)))
    A = sp.hstack(cols).tocsr()
    free = np.asarray(abs(A).sum(axis=0)).ravel() > 0
    k, iy, ix, pi = lop._pairs()
    D = _tree_rows(k, iy, ix, pi, int(lop.Ny), int(lop.Nx), n, tree, free)
    bb = b.ravel().astype(np.float64)
    tv = 0.06
    x_ref = chambolle_pock_poisson_tv(A, D, bb, gain, tv, free, n_iter=30000)
    f_ref = poisson_tv_objective(A, D, x_ref, bb, gain, tv)
    sp_ = SPDHGPoisson(lop, subsets=4, tv=tv, tv_tree=tree, seed=1)
    x = sp_.run(np.zeros(lop.coeff_shape, np.float32), b, 3000, gain=gain, diagnostics_interval=3000)
    f = poisson_tv_objective(A, D, x.astype(np.float64), bb, gain, tv)
    assert f <= f_ref * (1 + 1e-3), (f, f_ref)
    assert abs(sp_.final_stats["final_f"] - f) <= 1e-4 * f, (sp_.final_stats["final_f"], f)


@pytest.mark.gpu
def test_tree_state_resumes_and_misuse_raises(golden):
    from diffractom_b200 import OrientationTree, SinglePhaseForwardOperator, SPDHGPoisson
    lop, b, gain, mats = _local_problem(golden)
    tree = OrientationTree(mats, None, RADII)
    kw = dict(subsets=3, tv=0.06, tv_tree=tree, seed=4)
    a = SPDHGPoisson(lop, **kw)
    xa = a.run(np.zeros(lop.coeff_shape, np.float32), b, 4, gain=gain, diagnostics_interval=4)
    tq = a.state["tree_q"]
    assert len(tq) == 2 and all(q[0].shape == q[1].shape and q[0].dtype == np.float32 for q in tq)
    assert any(np.abs(q[0]).max() > 0 for q in tq)
    c = SPDHGPoisson(lop, **kw)
    xc = c.run(np.zeros(lop.coeff_shape, np.float32), b, 2, gain=gain, diagnostics_interval=4)
    xc = c.run(xc, b, 2, gain=gain, diagnostics_interval=4, state=c.state)
    assert c.state["epoch"] == 4 and np.isfinite(xc).all()
    assert np.array_equal(xc, xa)                        # the same schedule and steps as the unbroken run
    for (p, q), (r, s) in zip(c.state["tree_q"], tq):
        assert np.array_equal(p, r) and np.array_equal(q, s)
    with pytest.raises(ValueError):
        SPDHGPoisson(lop, subsets=3, tv_tree=tree)
    with pytest.raises(ValueError):                      # a tree over other orientations
        SPDHGPoisson(lop, subsets=3, tv=0.06, tv_tree=OrientationTree(mats[:5], None, RADII)).run(
            np.zeros(lop.coeff_shape, np.float32), b, 1, gain=gain)
    d = golden("diff_auto_trapezoid")
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    pf_mode="sparse")
    with pytest.raises(NotImplementedError):
        SPDHGPoisson(op, subsets=3, tv=0.06, tv_tree=tree).run(np.zeros(op.coeff_shape, np.float32),
                                                              np.zeros(op.data_shape, np.float32), 1)
