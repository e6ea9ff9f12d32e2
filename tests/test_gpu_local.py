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
