"""PoissonTerm on the device against the float32 / float64 NumPy expressions of the reference's kernels
(optimization/poisson_term.py:36-78), and OrientationRefiner: with noise-free data of the true coefficients, one
Gauss-Newton step from orientations turned by 0.3 deg brings them most of the way back and lowers the deviance; a
run() alternates steps and refits."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _op(d, grid=None, **kw):
    from diffractom_b200 import SinglePhaseForwardOperator
    cfg, mat, g = case_inputs(d)
    return SinglePhaseForwardOperator(cfg, mat, grid if grid is not None else g, 1e-5, normalized=True,
                                      quadrature=d["quadrature"], radon_kernel=d["kernel"], pf_mode="sparse", **kw)


def test_poisson_term_matches_numpy():
    from diffractom_b200.poisson_term import PoissonTerm
    rng = np.random.default_rng(0)
    shape = (6, 5, 8)
    b = rng.poisson(20, shape).astype(np.float32)
    pred = (rng.random(shape) * 30 - 2).astype(np.float32)
    w = (rng.random(8) > 0.2).astype(np.float32)
    g = (rng.random(40) + 0.5).astype(np.float32)
    bg = (rng.random(8) * 2).astype(np.float32)
    fit = np.array([1, 1, 0, 1, 0, 1], bool)
    eps, floor = np.float32(1e-3), np.float32(0.25)
    pt = PoissonTerm(None, shape, torch.as_tensor(b, device="cuda"), w, g, bg, fit_rows=fit, eps_counts=eps)
    pd = torch.as_tensor(pred, device="cuda")
    wf = np.broadcast_to(w, shape) * fit[:, None, None]
    gf = np.broadcast_to(g.reshape(5, 8), shape)
    bgf = np.broadcast_to(bg, shape)
    mu = (np.maximum(pred, 0) + bgf) + eps * gf
    with np.errstate(divide="ignore", invalid="ignore"):
        r_ref = np.where(wf != 0, (wf / gf) * (np.float32(1) - b / mu), 0).astype(np.float32)
        c_ref = np.where(wf != 0, wf / (gf * np.maximum(mu, floor * gf)), 0).astype(np.float32)
        em_ref = np.where(wf != 0, (wf / gf) * (b / mu), 0).astype(np.float32)
    r, c, e = (torch.empty(shape, device="cuda") for _ in range(3))
    pt.grad_curv(pd, r, c, floor)
    assert np.array_equal(r.cpu().numpy(), r_ref) and np.array_equal(c.cpu().numpy(), c_ref)
    pt.em_ratio(pd, e)
    assert np.array_equal(e.cpu().numpy(), em_ref)
    pt.weight_over_gain(e)
    assert np.array_equal(e.cpu().numpy(), np.where(wf != 0, wf / gf, 0).astype(np.float32))
    m64 = np.maximum(pred, 0).astype(np.float64) + bgf + np.float64(eps) * gf.astype(np.float64)
    term = m64 - b + np.where(b > 0, b * np.log(np.where(b > 0, b, 1) / m64), 0)
    dev = float(np.sum(np.where(wf != 0, wf.astype(np.float64) / gf * term, 0)))
    assert abs(pt.deviance(pd) - dev) <= 1e-12 * abs(dev)
    assert pt.n_points() == int(np.count_nonzero(wf))


def _misorientation_deg(A, B):
    R = np.einsum("kji,kjl->kil", A, B)
    return np.degrees(np.arccos(np.clip((np.trace(R, axis1=1, axis2=2) - 1) / 2, -1, 1)))


def test_gauss_newton_step_recovers_orientations(golden):
    from diffractom_b200.differentiable import rotate_orientations
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.refine import OrientationRefiner
    d = golden("diff_auto_trapezoid")
    truth = _op(d)
    rng = np.random.default_rng(1)
    x = (rng.random(truth.coeff_shape) * truth.support_mask()[None] * 2).astype(np.float32)
    b = truth.direct(x) * np.float32(50.0)
    axes = rng.normal(size=(truth.K, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    U_true = np.asarray(truth.grid_rot_cpu, np.float64)
    U0 = rotate_orientations(U_true, np.radians(0.3) * axes)
    op = _op(d, grid=MatrixGrid(U0, d["sigma64"]))
    xs = x * np.float32(50.0)
    # the widths of this case are 6 deg: the width bounds must hold them (the step clips the widths in any case)
    ref = OrientationRefiner(op, b, max_rot_deg=1.0, refine_sigma=False, sigma_max_deg=10.0)
    before = np.median(_misorientation_deg(U_true, np.asarray(op.grid_rot_cpu, np.float64)))
    info = ref.step(xs)
    after = np.median(_misorientation_deg(U_true, np.asarray(op.grid_rot_cpu, np.float64)))
    assert info["alpha"] > 0 and info["f"] < 0.5 * info["f0"]
    assert after < 0.5 * before, (before, after)
    assert abs(ref.loss(xs) - info["f"]) <= 1e-9 * info["f"]      # the operator holds the accepted parameters


def test_refiner_run_alternates_with_refits(golden):
    from diffractom_b200 import SPDHGPoisson
    from diffractom_b200.differentiable import rotate_orientations
    from diffractom_b200.grid import MatrixGrid
    from diffractom_b200.refine import OrientationRefiner
    d = golden("diff_auto_trapezoid")
    truth = _op(d)
    rng = np.random.default_rng(2)
    x = (rng.random(truth.coeff_shape) * truth.support_mask()[None] * 2).astype(np.float32)
    b = rng.poisson(truth.direct(x) * 50.0).astype(np.float32)
    U0 = rotate_orientations(np.asarray(truth.grid_rot_cpu, np.float64), np.radians(0.2) * rng.normal(size=(truth.K, 3)))
    op = _op(d, grid=MatrixGrid(U0, d["sigma64"]))
    x0 = torch.full(op.coeff_shape, 50.0, device="cuda")
    x0 = SPDHGPoisson(op, subsets=4, seed=0).run(x0, b, 20)
    ref = OrientationRefiner(op, b, max_rot_deg=0.5, sigma_max_deg=10.0)
    solve = lambda xx: SPDHGPoisson(op, subsets=4, seed=1).run(xx, b, 5)
    ref.run(x0, solve, 3)
    h = ref.history
    assert [s["step"] for s in h] == [1, 2, 3]
    assert all(s["f"] <= s["f0"] for s in h) and h[0]["alpha"] > 0
    assert h[-1]["f_fit"] < h[0]["f0"]
