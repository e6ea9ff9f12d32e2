"""The forward operator as a torch.autograd.Function: gradients are the hand-written adjoint, checked against float64
finite differences of the oracle's forward model, the adjoint identity on 100 random pairs at the shape of the
differentiable configuration (bcc Fe, 128 x 128 pixels, 180 angles, 133 translations, 120 eta bins, 5 rings,
K = 5000, 5 % support), a batch of slices, the subset form, and an operator whose PF matrix is generated again in
every call (memory-bounded: nothing stored, or only some batches) giving the same values and gradients."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def make_operator(d, **kw):
    from diffractom_b200 import SinglePhaseForwardOperator
    cfg, mat, grid = case_inputs(d)
    kw.setdefault("max_gb", 1e-5)
    return SinglePhaseForwardOperator(cfg, mat, grid, normalized=True, quadrature=d["quadrature"],
                                      radon_kernel=d["kernel"], **kw)


def test_gradient_is_adjoint_and_matches_float64_finite_differences(golden):
    from diffractom_b200.autograd import forward_operator
    from oracle.oracle import OracleOperator
    d = golden("al5_small")
    op = make_operator(d)
    rng = np.random.default_rng(3)
    x0 = (rng.random(op.coeff_shape) * op.support_mask()[None]).astype(np.float32)
    w = rng.standard_normal(op.data_shape).astype(np.float32)
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    y = forward_operator(op, x)
    loss = (y * torch.as_tensor(w, device="cuda")).sum()
    loss.backward()
    grad = x.grad.cpu().numpy()
    assert np.array_equal(grad, op.adjoint(torch.as_tensor(w, device="cuda")).cpu().numpy())
    orc = OracleOperator.from_operator(op, precision="f64io")       # float64 images and data
    x64 = x0.astype(np.float64)
    h = 1e-6
    for seed in range(3):
        dr = np.random.default_rng(100 + seed).standard_normal(op.coeff_shape)
        fp = float(np.dot(orc.forward(x64 + h * dr).ravel(), w.ravel().astype(np.float64)))
        fm = float(np.dot(orc.forward(x64 - h * dr).ravel(), w.ravel().astype(np.float64)))
        fd = (fp - fm) / (2 * h)
        an = float(np.dot(grad.ravel().astype(np.float64), dr.ravel()))
        assert abs(an - fd) <= 1e-5 * abs(fd), (an, fd)


def _fe_config_operator(K=5000, **kw):
    from diffractom_b200 import Grid, Material, SinglePhaseForwardOperator
    cfg = dict(Nx=128, Ny=128, My=133, N_Omega=180, angle_range=[0, 180], cor_offset=0.0, N_eta=120,
               eta_angle_range=[0, 360], energy=12.398 / 0.3, k_direction_0=[0, 0, 1], p_direction_0=[1, 0, 0],
               detector_direction_origin=[0, -1, 0], detector_direction_positive_90=[0, 0, -1])
    mat = Material.from_lattice_parameters(a=2.87, symmetry_group="cubic", wavelength_A=0.3,
                                           hkl_list=[[1, 1, 0], [2, 0, 0], [2, 1, 1], [2, 2, 0], [3, 1, 0]])
    grid = Grid.from_random_fundamental_zone(K, mat.crystal_system, np.deg2rad(3.0), seed=4)
    return SinglePhaseForwardOperator(cfg, mat, grid, 0.5, normalized=True, **kw)


def test_adjoint_identity_100_pairs_and_slice_batch():
    from diffractom_b200.autograd import forward_operator
    op = _fe_config_operator()
    g = torch.Generator(device="cuda").manual_seed(9)
    supp = torch.as_tensor(op.support_mask(), device="cuda")
    worst = 0.0
    for _ in range(100):
        x = (torch.rand(op.coeff_shape, generator=g, device="cuda") < 0.05) * supp * \
            torch.rand(op.coeff_shape, generator=g, device="cuda")
        x.requires_grad_(True)
        yv = torch.rand(op.data_shape, generator=g, device="cuda")   # non-negative, as the reference's test
        ax = forward_operator(op, x)
        (aty,) = torch.autograd.grad(ax, x, grad_outputs=yv)
        lhs = float((ax.double() * yv.double()).sum())
        rhs = float((x.detach().double() * aty.double()).sum())
        worst = max(worst, abs(lhs / rhs - 1))
    assert worst < 1e-5, worst
    xs = torch.rand((4, *op.coeff_shape), generator=g, device="cuda") * supp
    xs.requires_grad_(True)
    ys = forward_operator(op, xs)
    assert ys.shape == (4, *op.data_shape)
    assert torch.equal(ys[2], op.direct(xs[2].detach()))
    gy = torch.randn(ys.shape, generator=g, device="cuda")
    ys.backward(gy)
    assert torch.equal(xs.grad[1], op.adjoint(gy[1]))


def test_subset_rows_and_their_gradient(golden):
    from diffractom_b200.autograd import forward_operator
    d = golden("adj_0_360")
    op = make_operator(d)
    subs = op.set_omega_subsets(3)
    rng = np.random.default_rng(5)
    x = torch.tensor((rng.random(op.coeff_shape) * op.support_mask()[None]).astype(np.float32), device="cuda",
                     requires_grad=True)
    y = forward_operator(op, x, subset=1)
    full = op.direct(x.detach())
    rows = torch.as_tensor(subs[1], device="cuda")
    others = torch.as_tensor(np.setdiff1d(np.arange(op.N_Omega), subs[1]), device="cuda")
    assert torch.equal(y[rows], full[rows]) and torch.all(y[others] == 0)
    gy = torch.as_tensor(rng.standard_normal(op.data_shape).astype(np.float32), device="cuda")
    y.backward(gy)
    ref = torch.empty(op.coeff_shape, device="cuda")
    op.adjoint_cl(gy, ref, subset=1)
    assert torch.equal(x.grad, ref)
    with pytest.raises(TypeError):
        forward_operator(op, x.detach().double())
    with pytest.raises(ValueError):
        forward_operator(op, torch.zeros((2, 3), device="cuda"))


def test_memory_bounded_operator_gives_the_same_values_and_gradients():
    """At the Fe configuration (K = 5000), an operator that keeps no PF matrix (pf_mode "generated": the blocks are
    made again in every call) and one that stores only the first batches (a storage budget below the matrix) give
    the stored operator's forward values and gradients bit for bit."""
    from diffractom_b200.autograd import forward_operator
    stored = _fe_config_operator(pf_mode="sparse")
    assert stored.pf_storage == "both"
    both, adj, ptr_f, batch_adj = stored.sparse_estimates(stored.sparse_fill_first)
    part_gb = (len(stored.batches) * ptr_f + batch_adj[0] + 1) / 1024.0 ** 3
    ops = [_fe_config_operator(pf_mode="generated"),
           _fe_config_operator(pf_mode="auto", sparse_max_gb=part_gb, sparse_max_fill=1.0, sparse_max_fill_partial=1.0)]
    assert ops[0].pf_storage == "none" and ops[1].pf_storage.startswith("adjoint, 1 of")
    g = torch.Generator(device="cuda").manual_seed(21)
    supp = torch.as_tensor(stored.support_mask(), device="cuda")
    x0 = (torch.rand(stored.coeff_shape, generator=g, device="cuda") < 0.05) * supp * \
        torch.rand(stored.coeff_shape, generator=g, device="cuda")
    gy = torch.rand(stored.data_shape, generator=g, device="cuda")
    out = []
    for op in [stored] + ops:
        x = x0.clone().requires_grad_(True)
        y = forward_operator(op, x)
        y.backward(gy)
        out.append((y.detach(), x.grad))
    for y, gx in out[1:]:
        assert torch.equal(y, out[0][0]) and torch.equal(gx, out[0][1])
