"""Parity at the first benchmark configuration (al99: 99 x 99 pixels, 180 angles, 103 translations, 180 eta bins, 5
rings of cubic Al, 1000 orientations at sigma 3 deg, 30 grains, mean 100 counts; SPDHG with 10 subsets, 20 epochs)
against the oracle's float64 restatement of the reference loop (oracle.spdhg_reference64: float64 state, data,
images, step sizes, prox and deviance; the same subset schedule):

  float32 path   coefficients within 1e-4 relative (2-norm), every epoch's deviance within 1e-5 relative;
                 its step sizes S and T within 1e-5 relative of the float64 ones
  BF16 path      every epoch's deviance within 1e-3 relative of the float64 loop's, with the default passes (step
                 sizes and diagnostics forward through the BF16 operator) and with the float32 ones (step sizes and a
                 float32 residual once per epoch); the coefficient error is reported

The inputs are the bench's al99 workload (seeded synthetic phantom and Poisson counts)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

EPOCHS, SUBSETS = 20, 10


@pytest.fixture(scope="module")
def al99():
    import bench
    from diffractom_b200 import SinglePhaseForwardOperator
    from oracle.oracle import OracleOperator, spdhg_reference64
    torch.cuda.set_device(0)
    cfg, mat, grid, w = bench.make_problem("al99")
    op = SinglePhaseForwardOperator(cfg, mat, grid, w["max_gb"], normalized=True, precision="bf16")
    op.precision = "fp32"
    b = bench.counts(op, bench.phantom(op, w, seed=1), w["mean_counts"]).cpu().numpy()
    op.set_omega_subsets(SUBSETS)
    orc = OracleOperator.from_operator(op, precision="f64io")
    x64, y64, z64, devs64, rho64, steps64 = spdhg_reference64(orc, op.omega_subsets, b, EPOCHS,
                                                              support=op.support_mask(), seed=0)
    return dict(op=op, b=b, x64=x64, devs64=np.asarray(devs64), rho64=rho64, steps64=steps64)


def _rel(a, ref):
    return float(np.linalg.norm(np.asarray(a, np.float64) - ref) / np.linalg.norm(ref))


def _run(op, b, precision, **switches):
    from diffractom_b200 import SPDHGPoisson
    op.precision = precision
    sp = SPDHGPoisson(op, subsets=SUBSETS, seed=0)
    for k, v in switches.items():
        setattr(sp, k, v)
    x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, EPOCHS, diagnostics_interval=1).cpu().numpy()
    op.precision = "fp32"
    return x, np.array([s["f"] for s in sp.iter_stats]), sp.rho_used


def _steps(op, b, precision, bf16_steps):
    """(S, T) of the solver's set-up for the operator in the given precision, T in the (K, Ny, Nx) layout."""
    from diffractom_b200 import SPDHGPoisson
    op.precision = precision
    sp = SPDHGPoisson(op, subsets=SUBSETS, seed=0)
    sp.bf16_steps = bf16_steps
    sp._setup(torch.zeros(op.coeff_shape, device="cuda"), b)
    T = torch.empty(op.coeff_shape, dtype=torch.float32, device="cuda")
    op.from_batches(sp.T.dev, T)
    S = sp.sig.cpu().numpy()
    T = T.cpu().numpy()
    sp._finish()
    op.precision = "fp32"
    return S, T


def test_fp32_spdhg_matches_the_float64_loop(al99):
    op, b = al99["op"], al99["b"]
    x, devs, rho = _run(op, b, "fp32")
    assert abs(rho / al99["rho64"] - 1) < 1e-12
    e_x = _rel(x, al99["x64"])
    e_f = np.abs(devs - al99["devs64"]) / al99["devs64"]
    print(f"al99 FP32 vs FP64: coefficients {e_x:.3e}, deviance max over epochs {e_f.max():.3e} "
          f"(final {e_f[-1]:.3e})")
    assert len(devs) == EPOCHS
    assert e_x <= 1e-4
    assert e_f.max() <= 1e-5


@pytest.mark.parametrize("fp32_passes", [False, True], ids=["bf16-passes", "fp32-residual-and-steps"])
def test_bf16_spdhg_deviance_within_1e3_of_the_float64_loop(al99, fp32_passes):
    op, b = al99["op"], al99["b"]
    sw = dict(bf16_steps=not fp32_passes, bf16_diagnostics=not fp32_passes)
    x, devs, _ = _run(op, b, "bf16", **sw)
    e_x = _rel(x, al99["x64"])
    e_f = np.abs(devs - al99["devs64"]) / al99["devs64"]
    print(f"al99 BF16 ({'float32' if fp32_passes else 'BF16'} step sizes and residual) vs FP64: coefficients "
          f"{e_x:.3e}, deviance max over epochs {e_f.max():.3e} (final {e_f[-1]:.3e})")
    assert e_f.max() <= 1e-3
    assert e_x <= 5e-2


@pytest.mark.parametrize("precision,bf16_steps", [("fp32", False), ("bf16", True)], ids=["fp32", "bf16"])
def test_step_sizes_against_float64(al99, precision, bf16_steps):
    """S = gamma / (A 1_S) and T = min_m p / (gamma A_m^T 1_counted) of each operator against the float64 ones: the
    float32 operator's to 1e-5 relative, the BF16 operator's (BF16 Radon output and PF) to 1e-2."""
    op, b = al99["op"], al99["b"]
    S, T = _steps(op, b, precision, bf16_steps)
    S64, T64 = al99["steps64"]["S"], al99["steps64"]["T"]
    assert np.array_equal(S > 0, S64 > 0) and np.array_equal(T > 0, T64 > 0)
    eS = float(np.max(np.abs(S - S64)[S64 > 0] / S64[S64 > 0]))
    eT = float(np.max(np.abs(T - T64)[T64 > 0] / T64[T64 > 0]))
    print(f"al99 step sizes of the {precision} operator vs float64: S max relative {eS:.3e}, T {eT:.3e}")
    tol = 1e-5 if precision == "fp32" else 1e-2
    assert eS <= tol and eT <= tol
