"""FISTAPoisson on the GPU: its objective against scipy's L-BFGS-B minimum of the same Poisson deviance on the
oracle operator (as the reference tests its solvers against L-BFGS-B, tests/test_poisson.py:100-130), SPDHG reaching
FISTA's minimiser (tests/test_subsets.py:130-145), resume from state, and argument errors."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _problem(golden, name="diff_midpoint_hat", seed=7, gain=0.05):
    from diffractom_b200 import SinglePhaseForwardOperator
    d = golden(name)
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    radon_kernel=d["kernel"], pf_mode="sparse")
    rng = np.random.default_rng(seed)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.3) * op.support_mask()[None]
              ).astype(np.float32)
    b = (rng.poisson(op.direct(x_true) / gain) * gain).astype(np.float32)
    return op, b, gain


def _lbfgs_minimum(op, b, gain, eps=1e-3):
    """min over x >= 0 (support) of the deviance, float64, with the oracle's A and A^T."""
    from scipy.optimize import minimize

    from oracle.oracle import OracleOperator
    orc = OracleOperator.from_operator(op)
    supp = np.broadcast_to(op.support_mask()[None], op.coeff_shape).ravel()
    bd = b.astype(np.float64).ravel()
    sc = 1.0 / gain
    epsg = float(np.float32(eps)) * gain

    def fg(xf):
        x = np.zeros(op.coeff_shape, np.float32)
        x.ravel()[supp] = xf
        mu = orc.forward(x).astype(np.float64).ravel()
        m = np.maximum(mu, 0) + epsg
        f = sc * np.sum(m - bd + np.where(bd > 0, bd * np.log(np.where(bd > 0, bd, 1) / m), 0))
        gmu = sc * (1 - bd / m) * (mu > 0)
        g = orc.adjoint(gmu.reshape(op.data_shape).astype(np.float32)).astype(np.float64).ravel()[supp]
        return f, g
    n = int(supp.sum())
    res = minimize(fg, np.full(n, 0.01), jac=True, method="L-BFGS-B", bounds=[(0, None)] * n,
                   options=dict(maxiter=5000, maxfun=10000, ftol=1e-14, gtol=1e-10))
    return float(res.fun)


def test_fista_reaches_lbfgs_minimum(golden):
    from diffractom_b200.fista import FISTAPoisson
    op, b, gain = _problem(golden)
    fista = FISTAPoisson(op)
    fista.run(torch.zeros(op.coeff_shape, device="cuda"), b, niter=800, gain=gain)
    f = fista.final_stats["final_f"]
    f_ref = _lbfgs_minimum(op, b, gain)
    assert f <= f_ref * (1 + 1e-4)
    assert abs(fista.final_stats["adjoint_scale"] - 1) < 1e-4


def test_spdhg_reaches_fista_minimum(golden):
    from diffractom_b200 import SPDHGPoisson
    from diffractom_b200.fista import FISTAPoisson
    op, b, gain = _problem(golden, "adj_0_360")
    ref = FISTAPoisson(op)
    ref.run(torch.zeros(op.coeff_shape, device="cuda"), b, niter=1500, gain=gain)
    f_ref = ref.final_stats["final_f"]
    sp = SPDHGPoisson(op, subsets=4)
    sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, n_epochs=600, gain=gain, diagnostics_interval=100)
    assert sp.final_stats["final_f"] <= f_ref * (1 + 2e-3)


def test_fista_resume_and_numpy(golden):
    from diffractom_b200.fista import FISTAPoisson
    op, b, gain = _problem(golden, seed=3)
    one = FISTAPoisson(op)
    x1 = one.run(np.zeros(op.coeff_shape, np.float32), b, niter=40, gain=gain)
    two = FISTAPoisson(op)
    x2 = two.run(np.zeros(op.coeff_shape, np.float32), b, niter=25, gain=gain)
    x2 = two.run(x2, b, niter=15, gain=gain, state=two.state)
    assert two.state["it"] == 40
    # the resumed run recomputes A y from y (float32 rounding differs from the running combination)
    np.testing.assert_allclose(x2, x1, rtol=2e-4, atol=1e-4 * np.abs(x1).max())
    with pytest.raises(ValueError):
        FISTAPoisson(op, prox_kind="l1")
    with pytest.raises(ValueError):
        FISTAPoisson(op).run(np.zeros(op.coeff_shape, np.float32), b, 1, gain=np.zeros(op.N_seg, np.float32))


@pytest.mark.parametrize("start,gain", [("wls", 0.05), ("uniform", None), ("x0", 0.05)])
def test_fista_poisson_iterates_match_the_oracle_loop(golden, start, gain):
    """FISTAPoisson against oracle.fista_poisson_reference (the reference's loop, fista_poisson.py:414-610, on the
    oracle operator with float32 arrays and float64 sums) iteration by iteration: the same backtracking, restart
    and metric-refresh decisions, every iteration's deviance to 1e-5 and the final x to 1e-4 of its maximum; through
    the weighted least squares start, the switch to the deviance and two metric refreshes."""
    from diffractom_b200 import FISTAPoisson
    from oracle.oracle import OracleOperator, fista_poisson_reference
    op, b, g = _problem(golden, seed=11)
    gain = None if gain is None else g
    rng = np.random.default_rng(5)
    x0 = (np.zeros(op.coeff_shape, np.float32) if start != "x0" else
          (rng.random(op.coeff_shape) * op.support_mask()[None]).astype(np.float32))
    fs = FISTAPoisson(op, start=start, n_start=4)
    x = fs.run(torch.as_tensor(x0, device="cuda"), b, 12, gain=gain).cpu().numpy()
    orc = OracleOperator.from_operator(op)
    xr, st, fin = fista_poisson_reference(orc, b, 12, x0=x0, gain=gain, support=op.support_mask(), start=start,
                                          n_start=4)
    keys = ("backtracks", "restart", "metric_refresh", "local_metric")
    assert [[s[k] for k in keys] for s in fs.iter_stats] == [[s[k] for k in keys] for s in st]
    np.testing.assert_allclose([s["f"] for s in fs.iter_stats], [s["f"] for s in st], rtol=1e-5)
    assert abs(fs.final_stats["adjoint_scale"] / fin["adjoint_scale"] - 1) < 1e-5
    assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
