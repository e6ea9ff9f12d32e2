"""SPDHGPoisson's total-variation block on the GPU: the TV kernels (dual step, adjoint with the primal step, value)
bit for bit against the oracle's float32 restatement of the reference's kernels (spdhg_poisson.py:110-181); a TV run
against the oracle's loop (same schedule with the TV block at the same places, same steps): iterates, dual variable
and objective; the streamed TV state equals the resident one bit for bit; a resumed run continues the TV dual."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _problem(golden, name="adj_0_360", seed=7, precision="fp32"):
    from diffractom_b200 import SinglePhaseForwardOperator
    d = golden(name)
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    precision=precision)
    rng = np.random.default_rng(seed)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(x_true) * 50).astype(np.float32)
    return op, b


def _to_k(a, kstride):
    """(K, Ny, Nx) -> channel-fastest (Ny * Nx, kstride), padding channels 0."""
    K = a.shape[0]
    out = np.zeros((a.shape[1] * a.shape[2], kstride), np.float32)
    out[:, :K] = a.reshape(K, -1).T
    return out


def test_tv_kernels_equal_oracle():
    from diffractom_b200 import _lib
    from oracle.oracle import tv_adjoint, tv_dual, tv_value
    rng = np.random.default_rng(0)
    K, Ny, Nx, ks = 13, 9, 11, 16
    x = rng.random((K, Ny, Nx)).astype(np.float32)
    T = (rng.random((K, Ny, Nx)) * (rng.random((K, Ny, Nx)) < 0.8)).astype(np.float32)
    qx = (rng.normal(size=(K, Ny, Nx)) * 0.3).astype(np.float32)
    qy = (rng.normal(size=(K, Ny, Nx)) * 0.3).astype(np.float32)
    z = rng.normal(size=(K, Ny, Nx)).astype(np.float32)
    lam, ps, ip, l1 = np.float32(0.4), np.float32(0.99 * 0.2), np.float32(5.0), np.float32(0.01)
    dev = lambda a: torch.as_tensor(_to_k(a, ks), device="cuda")
    xk, Tk, qxk, qyk, zk = dev(x), dev(T), dev(qx), dev(qy), dev(z)
    dqx, dqy = torch.empty_like(xk), torch.empty_like(xk)
    s = torch.cuda.current_stream().cuda_stream
    import ctypes
    st = ctypes.c_void_p(s)
    _lib.call("dfx_tv_dual", xk.data_ptr(), Tk.data_ptr(), qxk.data_ptr(), qyk.data_ptr(), dqx.data_ptr(),
              dqy.data_ptr(), Nx, Ny, ks, float(lam), float(ps), st)
    rqx, rqy, rdx, rdy = tv_dual(x, T, qx, qy, lam, ps)
    for got, want in ((qxk, rqx), (qyk, rqy), (dqx, rdx), (dqy, rdy)):
        assert np.array_equal(got.cpu().numpy(), _to_k(want, ks))
    _lib.call("dfx_tv_adjoint_update", dqx.data_ptr(), dqy.data_ptr(), xk.data_ptr(), zk.data_ptr(), Tk.data_ptr(),
              Nx, Ny, ks, float(ip), float(l1), st)
    dz = tv_adjoint(rdx, rdy)
    z2 = (z + dz).astype(np.float32)
    zb = (z2 + ip * dz).astype(np.float32)
    x2 = np.where(T > 0, np.maximum(np.float32(0), x - T * (zb + l1)), 0).astype(np.float32)
    assert np.array_equal(zk.cpu().numpy()[:, :K], _to_k(z2, ks)[:, :K])
    assert np.array_equal(xk.cpu().numpy(), _to_k(x2, ks))
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    nb = _lib.lib().dfx_reduce_scratch_bytes(Ny * Nx * ks)
    scr = torch.empty(nb, dtype=torch.uint8, device="cuda")
    _lib.call("dfx_tv_value", xk.data_ptr(), Tk.data_ptr(), Nx, Ny, ks, out.data_ptr(), scr.data_ptr(), nb, st)
    want = tv_value(x2, T)
    assert abs(float(out.item()) - want) <= 1e-12 * want


def test_spdhg_tv_matches_oracle(golden):
    from diffractom_b200 import SPDHGPoisson
    from oracle.oracle import OracleOperator, spdhg_reference
    op, b = _problem(golden)
    tv = 0.05
    sp = SPDHGPoisson(op, subsets=3, seed=1, tv=tv)
    assert sp._n_tv == 1 and abs(sp.tv_prob - 0.25) < 1e-15
    x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 4, diagnostics_interval=2).cpu().numpy()
    orc = OracleOperator.from_operator(op)
    xr, yr, zr, devs, rho = spdhg_reference(orc, op.omega_subsets, b, 4, support=op.support_mask(), seed=1,
                                            diagnostics_interval=2, tv=tv)
    f = [s["f"] for s in sp.iter_stats if s["f"] is not None]
    assert len(f) == len(devs) == 2
    np.testing.assert_allclose(f, devs, rtol=1e-5)
    assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
    assert np.abs(sp.state["y"] - yr).max() <= 1e-4 * np.abs(yr).max()
    assert set(sp.state) >= {"qx", "qy", "z", "y"} and np.abs(sp.state["qx"]).max() <= tv * (1 + 1e-6)
    assert sp.final_stats["tv"] == tv and sp.final_stats["tv_prob"] == sp.tv_prob
    # a TV run differs from the plain one
    plain = SPDHGPoisson(op, subsets=3, seed=1).run(torch.zeros(op.coeff_shape, device="cuda"), b, 4).cpu().numpy()
    assert not np.allclose(plain, x)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_spdhg_tv_streamed_equals_resident_and_resumes(golden, precision):
    from diffractom_b200 import SPDHGPoisson
    op, b = _problem(golden, "al5_small", seed=3, precision=precision)
    kw = dict(subsets=4, seed=2, tv=0.02, tv_prob=0.3)
    a = SPDHGPoisson(op, **kw)
    xa = a.run(np.zeros(op.coeff_shape, np.float32), b, 3, diagnostics_interval=3)
    s = SPDHGPoisson(op, resident="none", **kw)
    xs = s.run(np.zeros(op.coeff_shape, np.float32), b, 3, diagnostics_interval=3)
    assert s.resident_used == () and set(a.resident_used) == {"x", "z", "T", "qx", "qy"}
    assert np.array_equal(xa, xs)
    for k in ("qx", "qy", "z", "y"):
        assert np.array_equal(a.state[k], s.state[k]), k
    assert [t["f"] for t in a.iter_stats] == [t["f"] for t in s.iter_stats]
    # a run resumed from its state (z, y, qx, qy) continues; a TV state without z is refused
    c = SPDHGPoisson(op, **kw)
    xc = c.run(np.zeros(op.coeff_shape, np.float32), b, 2, diagnostics_interval=3)
    xc = c.run(xc, b, 1, diagnostics_interval=3, state=c.state)
    assert np.isfinite(xc).all() and c.state["epoch"] == 3
    with pytest.raises(ValueError):
        SPDHGPoisson(op, **kw).run(np.zeros(op.coeff_shape, np.float32), b, 1, state={"y": a.state["y"], "epoch": 1})


def test_local_basis_tv_equals_dense_tv(golden):
    """The TV block on a local basis (neighbours within the patches) with every orientation allowed in the whole field
    of view takes the dense TV run's steps bit for bit; the objective with tv TV(x) agrees to float64 rounding."""
    from diffractom_b200 import SPDHGPoisson
    from test_gpu_local import _everywhere_pair
    loc, inner, oi = _everywhere_pair(golden)
    rng = np.random.default_rng(8)
    x0 = rng.random((loc.K_basis, loc.Ny, loc.Nx)).astype(np.float32)
    mu = inner.direct(torch.as_tensor(x0[oi], device="cuda")).cpu().numpy()
    b = rng.poisson(np.maximum(mu, 0) * 3 + 0.5).astype(np.float32)
    xs = np.full((loc.K_basis, loc.Ny, loc.Nx), 0.5, np.float32)
    kw = dict(subsets=3, seed=2, tv=0.05)
    sl = SPDHGPoisson(loc, **kw)
    xl = sl.run(torch.as_tensor(loc.from_dense(xs), device="cuda"), b, 3)
    sd = SPDHGPoisson(inner, **kw)
    xd = sd.run(torch.as_tensor(xs[oi], device="cuda"), b, 3)
    assert np.array_equal(loc.to_dense(xl)[oi], xd.cpu().numpy())
    assert np.array_equal(sl.state["y"], sd.state["y"])
    np.testing.assert_allclose([s["f"] for s in sl.iter_stats], [s["f"] for s in sd.iter_stats], rtol=1e-12)
    fov = inner.support_mask()
    assert np.array_equal(loc.to_dense(sl.state["qx"])[oi][:, fov], sd.state["qx"][:, fov])
