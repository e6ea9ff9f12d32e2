"""FISTAL2 / FISTAHuber on the GPU against the float64 oracle loop (oracle.fista_ls_reference, the reference's
iteration with the fused update): iterates, objective and gradient norms for the element-wise proxes, weights and the
Huber clip; the streamed (NumPy) path and the unfused next forward give the same bits as the device path."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _problem(golden, name="al5_small", seed=3):
    from diffractom_b200 import SinglePhaseForwardOperator, estimate_L_power
    d = golden(name)
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"])
    rng = np.random.default_rng(seed)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.25) * op.support_mask()[None]
              ).astype(np.float32)
    b = (op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy()
         + 0.01 * rng.standard_normal(op.data_shape)).astype(np.float32)
    L = estimate_L_power(op, niter=30, verbose=0)
    return op, b, L


@pytest.mark.parametrize("solver, prox, lam, weighted", [
    ("l2", "nonneg", 0.0, False), ("l2", "l1", 2e-3, False), ("huber", "nonneg_l1", 1e-3, True),
    ("huber", "nonneg", 0.0, False)])
def test_fista_ls_matches_float64_loop(golden, solver, prox, lam, weighted):
    from diffractom_b200 import FISTAHuber, FISTAL2
    from oracle.oracle import OracleOperator, fista_ls_reference
    op, b, L = _problem(golden)
    orc = OracleOperator.from_operator(op, precision="f64io")
    niter = 12
    w = np.linspace(0.5, 1.5, op.N_seg).astype(np.float32) if weighted else None
    delta = float(0.3 * np.abs(b).max())
    if solver == "l2":
        sol = FISTAL2(op, prox_kind=prox, lam=lam, L=L)
        x = sol.run(torch.zeros(op.coeff_shape, device="cuda"), b, niter).cpu().numpy()
    else:
        sol = FISTAHuber(op, prox_kind=prox, lam=lam, L=L, huber_delta=delta)
        x = sol.run(torch.zeros(op.coeff_shape, device="cuda"), b, niter, weights=w).cpu().numpy()
    xr, fr, gr = fista_ls_reference(orc, b, niter, 1.0 / L, prox=prox, lam=lam, support=op.support_mask(),
                                    clip=solver == "huber", delta=delta, weights=w)
    assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
    np.testing.assert_allclose([s["f"] for s in sol.iter_stats], fr, rtol=1e-4)
    np.testing.assert_allclose([s["gradnorm"] for s in sol.iter_stats], gr, rtol=1e-4)
    assert sol.final_stats["niter"] == niter and sol.final_stats["next_forward_fused"]
    assert np.all(x[:, ~op.support_mask()] == 0)
    if prox != "l1":
        assert x.min() >= 0


def test_fista_ls_streamed_and_unfused_forward_equal_device(golden):
    from diffractom_b200 import FISTAHuber
    op, b, L = _problem(golden, seed=5)
    runs = []
    for kw, x0 in (({}, torch.zeros(op.coeff_shape, device="cuda")), ({}, np.zeros(op.coeff_shape, np.float32)),
                   ({"fuse_next_forward": False}, torch.zeros(op.coeff_shape, device="cuda"))):
        sol = FISTAHuber(op, L=L, huber_delta=0.05, **kw)
        x = sol.run(x0, b, 6)
        runs.append((x.cpu().numpy() if torch.is_tensor(x) else x, [s["f"] for s in sol.iter_stats],
                     [s["xnorm"] for s in sol.iter_stats]))
    for r in runs[1:]:
        assert np.array_equal(r[0], runs[0][0]) and r[1] == runs[0][1] and r[2] == runs[0][2]


def test_fista_ls_arguments(golden):
    from diffractom_b200 import FISTAHuber, FISTAL2
    op, b, L = _problem(golden)
    with pytest.raises(ValueError):
        FISTAL2(op)
    with pytest.raises(NotImplementedError):
        FISTAHuber(op, prox_kind="nonneg_tv", L=L)
    with pytest.raises(ValueError):
        FISTAHuber(op, prox_kind="tv", L=L)
