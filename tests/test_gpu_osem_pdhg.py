"""OSEMPoisson and PDHGPoisson on the GPU against the oracle's restatements of the reference loops (same subsets,
schedule, start and steps): iterates to 1e-4 of the largest and deviances to 1e-5; the local basis; NumPy inputs."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _problem(golden, name="adj_0_360", seed=7):
    from diffractom_b200 import SinglePhaseForwardOperator
    d = golden(name)
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"])
    rng = np.random.default_rng(seed)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(x_true) * 50).astype(np.float32)
    return op, b


@pytest.mark.parametrize("subsets,lam", [(3, 0.0), (None, 0.05)])
def test_osem_matches_oracle(golden, subsets, lam):
    from diffractom_b200 import OSEMPoisson
    from oracle.oracle import OracleOperator, osem_reference
    op, b = _problem(golden)
    rng = np.random.default_rng(2)
    x0 = (rng.random(op.coeff_shape) * 0.1).astype(np.float32)
    bg = np.full(op.N_seg, 0.2, np.float32)
    em = OSEMPoisson(op, subsets=subsets, lam=lam, seed=3)
    x = em.run(torch.as_tensor(x0, device="cuda"), b, 3, background=bg).cpu().numpy()
    orc = OracleOperator.from_operator(op)
    subs = None if subsets is None else op.omega_subsets
    xr, fr = osem_reference(orc, subs, b, 3, x0, background=bg, support=op.support_mask(), seed=3, lam=lam)
    assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
    assert abs(em.final_f / fr - 1) < 1e-5
    f = [s_["f"] for s_ in em.iter_stats]
    assert f[-1] < f[0]
    xn = OSEMPoisson(op, subsets=subsets, lam=lam, seed=3).run(x0, b, 3, background=bg)   # NumPy in, new NumPy out
    assert isinstance(xn, np.ndarray) and np.array_equal(xn, x) and not np.array_equal(x0, xn)


def test_osem_flat_start_and_local_basis(golden):
    from diffractom_b200 import OSEMPoisson
    from diffractom_b200.local import LocalSinglePhaseForwardOperator, LocalSupport
    op, b = _problem(golden)
    em = OSEMPoisson(op, subsets=3, seed=0)
    x = em.run(np.zeros(op.coeff_shape, np.float32), b, 2)
    assert em.start_floor_used > 0 and np.isfinite(x).all() and x[:, ~op.support_mask()].max() == 0
    d = golden("adj_0_360")
    cfg, mat, grid = case_inputs(d)
    sup = LocalSupport.everywhere(op.K, (op.Ny, op.Nx))
    loc = LocalSinglePhaseForwardOperator(cfg, mat, grid, 1e-5, sup, normalized=True, quadrature=d["quadrature"])
    oi = loc.orientation_index
    xl = OSEMPoisson(loc, subsets=3, seed=0).run(np.zeros(loc.n_coef, np.float32), b, 2)
    # on the global basis the local operator is the dense one over the same orientations: the same EM steps
    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.grid import MatrixGrid
    mats, sig = grid.leaf_arrays()
    dense = SinglePhaseForwardOperator(cfg, mat, MatrixGrid(mats[oi], sig[oi]), 1e-5, normalized=True,
                                       quadrature=d["quadrature"])
    xd = OSEMPoisson(dense, subsets=3, seed=0).run(np.zeros(dense.coeff_shape, np.float32), b, 2)
    assert np.abs(loc.to_dense(xl)[oi] - xd).max() <= 1e-5 * np.abs(xd).max()


def test_pdhg_matches_oracle(golden):
    from diffractom_b200 import PDHGPoisson
    from oracle.oracle import OracleOperator, pdhg_reference
    op, b = _problem(golden)
    w = (np.random.default_rng(4).random(op.N_seg) > 0.1).astype(np.float32)
    pd = PDHGPoisson(op, prox_kind="nonneg_l1", lam=0.01)
    x = pd.run(torch.zeros(op.coeff_shape, device="cuda"), b, 8, weights=w).cpu().numpy()
    orc = OracleOperator.from_operator(op)
    xr, devs, rho = pdhg_reference(orc, b, 8, weights=w, support=op.support_mask(), lam=0.01)
    assert abs(pd.rho_used / rho - 1) < 1e-12
    np.testing.assert_allclose([s_["f"] for s_ in pd.iter_stats], devs, rtol=1e-5)
    assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
    assert devs[-1] < devs[0]
    # continuing from the state equals one longer run
    a = PDHGPoisson(op)
    xa = a.run(np.zeros(op.coeff_shape, np.float32), b, 6)
    c = PDHGPoisson(op)
    xc = c.run(np.zeros(op.coeff_shape, np.float32), b, 4)
    xc = c.run(xc, b, 2, state=c.state)
    assert np.array_equal(xa, xc) and c.state["it"] == 6
