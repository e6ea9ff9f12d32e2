"""The local-basis operator on the GPU: forward and adjoint equal those of SinglePhaseForwardOperator over the same
orientations (the operator's Z-order) applied to the zero-extended coefficients, bit for bit, with single and split
patches; subsets; the coefficient conversions."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _support(K, Ny, Nx, seed=1):
    from diffractom_b200.local import LocalSupport
    rng = np.random.default_rng(seed)
    mask = np.zeros((K, Ny, Nx), bool)
    for k in range(K):
        if k % 5 == 3:
            continue                                           # unused orientations
        cy, cx = rng.integers(0, Ny), rng.integers(0, Nx)
        mask[k, max(0, cy - 3):cy + 4, max(0, cx - 2):cx + 3] = True
        if k % 4 == 0:                                         # a second, far blob: split patches
            mask[k, (cy + Ny // 2) % Ny, (cx + Nx // 2) % Nx] = True
    return LocalSupport.from_mask(mask)


@pytest.mark.parametrize("split", [True, False])
def test_local_operator_equals_dense_inner_operator(golden, split):
    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.local import LocalSinglePhaseForwardOperator
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    mats, sig = grid.leaf_arrays()
    sup = _support(len(mats), int(cfg["Ny"]), int(cfg["Nx"]))
    loc = LocalSinglePhaseForwardOperator(cfg, mat, grid, 1e-5, sup, normalized=True, quadrature=d["quadrature"],
                                          split_patches=split)
    oi = loc.orientation_index
    inner = SinglePhaseForwardOperator(cfg, mat, MatrixGrid(mats[oi], sig[oi]), 1e-5, normalized=True,
                                       quadrature=d["quadrature"])
    assert [b["K_batch"] for b in inner.batches] == [b["K_batch"] for b in loc.batches] and len(loc.batches) > 1
    assert loc.coeff_shape == (loc.n_coef,) and loc.n_coef < loc.K_basis * loc.Nx * loc.Ny
    rng = np.random.default_rng(2)
    x = rng.random(loc.n_coef).astype(np.float32) * loc.coefficient_mask()
    dense = loc.to_dense(x)
    assert np.array_equal(loc.from_dense(dense), x)
    k, iy, ix, v = loc.to_coo(x)
    assert np.array_equal(dense[k, iy, ix], v)
    fwd = loc.direct(torch.as_tensor(x, device="cuda")).cpu().numpy()
    ref = inner.direct(torch.as_tensor(dense[oi], device="cuda")).cpu().numpy()
    assert np.array_equal(fwd, ref)
    assert np.array_equal(loc.direct(x), fwd)                 # NumPy in, NumPy out
    y = rng.standard_normal(loc.data_shape).astype(np.float32)
    adj = loc.adjoint(torch.as_tensor(y, device="cuda")).cpu().numpy()
    full = np.zeros((loc.K_basis, loc.Ny, loc.Nx), np.float32)
    full[oi] = inner.adjoint(torch.as_tensor(y, device="cuda")).cpu().numpy()
    assert np.array_equal(adj, loc.from_dense(full))
    assert not adj[loc.coefficient_mask() == 0].any()
    # subsets: the rows of a subset, and its adjoint
    loc.set_omega_subsets(3)
    inner.set_omega_subsets(3)
    d1 = torch.zeros(loc.data_shape, device="cuda")
    d2 = torch.zeros(loc.data_shape, device="cuda")
    loc.direct_cl(torch.as_tensor(x, device="cuda"), d1, subset=2)
    inner.direct_cl(torch.as_tensor(dense[oi], device="cuda"), d2, subset=2)
    assert torch.equal(d1, d2)
    a1 = torch.empty(loc.coeff_shape, device="cuda")
    loc.adjoint_cl(torch.as_tensor(y, device="cuda"), a1, subset=1)
    a2 = torch.empty(inner.coeff_shape, device="cuda")
    inner.adjoint_cl(torch.as_tensor(y, device="cuda"), a2, subset=1)
    full[oi] = a2.cpu().numpy()
    assert np.array_equal(a1.cpu().numpy(), loc.from_dense(full))



@pytest.mark.parametrize("prox_kind", ["nonneg", "l1"])
def test_fista_on_the_local_operator(golden, prox_kind):
    """FISTAL2 on the local operator (flat coefficients, the update kernel over the whole vector) against the same
    iteration written as float32 tensor operations through the operator's direct / adjoint: every step is a
    correctly rounded float32 operation, so the iterates agree bit for bit; a NumPy x0 returns the same values."""
    from diffractom_b200 import FISTAL2, estimate_L_power
    from diffractom_b200.local import LocalSinglePhaseForwardOperator
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    mats, _ = grid.leaf_arrays()
    sup = _support(len(mats), int(cfg["Ny"]), int(cfg["Nx"]), seed=4)
    loc = LocalSinglePhaseForwardOperator(cfg, mat, grid, 1e-5, sup, normalized=True, quadrature=d["quadrature"])
    rng = np.random.default_rng(5)
    m = loc.coefficient_mask()
    b = loc.direct(torch.as_tensor(rng.random(loc.n_coef).astype(np.float32) * m, device="cuda"))
    L = estimate_L_power(loc, niter=20, verbose=0)
    lam, niter = (0.0, 8) if prox_kind == "nonneg" else (1e-3, 8)
    sol = FISTAL2(loc, prox_kind=prox_kind, lam=lam, L=L)
    x0 = torch.as_tensor(rng.random(loc.n_coef).astype(np.float32), device="cuda")
    got = sol.run(x0.clone(), b, niter).cpu().numpy()
    f = [s_["f"] for s_ in sol.iter_stats]
    tau, lt = np.float32(1.0 / L), np.float32(lam / L)
    x = x0 * torch.as_tensor(m, device="cuda")
    y, t = x.clone(), 1.0
    for _ in range(niter):
        r = loc.direct(y) - b
        g = loc.adjoint(r)
        t_new = 0.5 * (1.0 + np.sqrt(1.0 + 4.0 * t * t))
        beta = np.float32((t - 1.0) / t_new)
        v = y - g * float(tau)
        if prox_kind == "nonneg":
            v = torch.clamp_min(v, 0.0)
        else:
            a = v.abs() - float(lt)
            v = torch.where(a > 0, torch.copysign(a, v), torch.zeros_like(v))
        y = v + (v - x) * float(beta)
        x, t = v, t_new
    assert np.array_equal(got, x.cpu().numpy())
    assert f[-1] < f[0] and not got[m == 0].any()
    host = FISTAL2(loc, prox_kind=prox_kind, lam=lam, L=L).run(x0.cpu().numpy(), b.cpu().numpy(), niter)
    assert isinstance(host, np.ndarray) and np.array_equal(host, got)


def _everywhere_pair(golden):
    """The local operator on the global basis (every orientation everywhere in the field of view) and the dense
    operator over the same orientations in the local operator's order."""
    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    mats, sig = grid.leaf_arrays()
    sup = LocalSupport.everywhere(len(mats), (int(cfg["Ny"]), int(cfg["Nx"])))
    loc = LocalSinglePhaseForwardOperator(cfg, mat, grid, 1e-5, sup, normalized=True, quadrature=d["quadrature"])
    oi = loc.orientation_index
    inner = SinglePhaseForwardOperator(cfg, mat, MatrixGrid(mats[oi], sig[oi]), 1e-5, normalized=True,
                                       quadrature=d["quadrature"])
    assert len(oi) == len(mats) and np.array_equal(loc.support.to_mask().any(0), inner.support_mask())
    return loc, inner, oi


def test_solvers_on_the_global_local_basis_equal_dense_runs(golden):
    """SPDHGPoisson and FISTAL2 on the local operator with every orientation allowed in the whole field of view take
    the same steps as the dense solvers (support "fov") on the dense operator: the iterates, the dual variable and
    the objective agree bit for bit (the fused and the separate primal steps round alike)."""
    from diffractom_b200 import FISTAL2, SPDHGPoisson, estimate_L_power
    loc, inner, oi = _everywhere_pair(golden)
    rng = np.random.default_rng(8)
    x0 = rng.random((loc.K_basis, loc.Ny, loc.Nx)).astype(np.float32)
    mu = inner.direct(torch.as_tensor(x0[oi], device="cuda")).cpu().numpy()
    b = rng.poisson(np.maximum(mu, 0) * 3 + 0.5).astype(np.float32)
    xs = torch.full((loc.K_basis, loc.Ny, loc.Nx), 0.5, device="cuda")
    sp_l = SPDHGPoisson(loc, subsets=3, seed=2)
    xl = sp_l.run(torch.as_tensor(loc.from_dense(xs.cpu().numpy()), device="cuda"), b, 3)
    sp_d = SPDHGPoisson(inner, subsets=3, seed=2)
    xd = sp_d.run(xs[oi].contiguous(), b, 3)
    assert np.array_equal(loc.to_dense(xl)[oi], xd.cpu().numpy())
    assert np.array_equal(sp_l.state["y"], sp_d.state["y"])
    fov = inner.support_mask()                 # z outside the support: the dense run's only (no coefficients there)
    assert np.array_equal(loc.to_dense(sp_l.state["z"])[oi][:, fov], sp_d.state["z"][:, fov])
    assert [s["f"] for s in sp_l.iter_stats] == [s["f"] for s in sp_d.iter_stats]
    # warm start from the state, NumPy x0
    xh = loc.to_dense(xl)
    xl2 = SPDHGPoisson(loc, subsets=3, seed=5).run(loc.from_dense(xh), b, 1, state=sp_l.state)
    xd2 = SPDHGPoisson(inner, subsets=3, seed=5).run(np.ascontiguousarray(xh[oi]), b, 1, state=sp_d.state)
    assert np.array_equal(loc.to_dense(xl2)[oi], xd2)

    L = estimate_L_power(inner, niter=10, verbose=0)
    bl = torch.as_tensor(mu, device="cuda")
    fl = FISTAL2(loc, L=L)
    yl = fl.run(torch.as_tensor(loc.from_dense(x0), device="cuda"), bl, 6)
    fd = FISTAL2(inner, L=L)
    yd = fd.run(torch.as_tensor(x0[oi], device="cuda"), bl, 6)
    assert np.array_equal(loc.to_dense(yl)[oi], yd.cpu().numpy())
    assert [s["f"] for s in fl.iter_stats] == [s["f"] for s in fd.iter_stats]
