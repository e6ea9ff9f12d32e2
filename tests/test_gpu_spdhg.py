"""SPDHGPoisson on the GPU against the oracle's float64-prox restatement of the reference loop (same subsets, same
random schedule, same step sizes): iterates and deviances; reproducibility, resume from state and the NumPy path."""
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


def test_spdhg_matches_oracle(golden):
    from diffractom_b200 import SPDHGPoisson
    from oracle.oracle import OracleOperator, spdhg_reference
    op, b = _problem(golden)
    sp = SPDHGPoisson(op, subsets=3, seed=1)
    x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 4, diagnostics_interval=2).cpu().numpy()
    orc = OracleOperator.from_operator(op)
    xr, yr, zr, devs, rho = spdhg_reference(orc, op.omega_subsets, b, 4, support=op.support_mask(), seed=1,
                                            diagnostics_interval=2)
    assert abs(sp.rho_used / rho - 1) < 1e-12
    f = [s["f"] for s in sp.iter_stats if s["f"] is not None]
    assert len(f) == len(devs) == 2
    np.testing.assert_allclose(f, devs, rtol=1e-5)
    assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
    assert np.abs(sp.state["y"] - yr).max() <= 1e-4 * np.abs(yr).max()


def test_spdhg_reproducible_resumed_and_numpy(golden):
    from diffractom_b200 import SPDHGPoisson
    op, b = _problem(golden, "al5_small", seed=9)
    ref = SPDHGPoisson(op, subsets=3, seed=1)
    x_ref = ref.run(torch.zeros(op.coeff_shape, device="cuda"), b, 6, diagnostics_interval=2).cpu().numpy()
    f_ref = [s["f"] for s in ref.iter_stats]
    again = SPDHGPoisson(op, subsets=3, seed=1)
    x2 = again.run(np.zeros(op.coeff_shape, np.float32), b, 6, diagnostics_interval=2)
    assert np.array_equal(x2, x_ref)
    assert [s["f"] for s in again.iter_stats] == f_ref
    two = SPDHGPoisson(op, subsets=3, seed=1)
    x = two.run(np.zeros(op.coeff_shape, np.float32), b, 4, diagnostics_interval=4)
    x = two.run(x, b, 2, diagnostics_interval=2, state=two.state)
    assert two.state["epoch"] == 6
    np.testing.assert_allclose(x, x_ref, rtol=1e-5, atol=1e-6 * np.abs(x_ref).max())


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_spdhg_streamed_state_equals_resident(golden, precision):
    """x, z, T streamed from pinned host memory through two device slots (any mix, resident= as in the reference's
    test_spdhg_streamed_and_resumed) give the iterates, deviances and state of the device-resident run bit for bit;
    a callback sees the same x; a run resumed from the state of a streamed run matches too."""
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    kw = {} if precision == "fp32" else {"precision": "bf16"}
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"], **kw)
    assert len(op.batches) > 2
    rng = np.random.default_rng(9)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy() * 50).astype(np.float32)
    seen = {}

    def cb(key):
        def f(ep, x, stats):
            seen.setdefault(key, []).append(np.array(x.cpu().numpy() if torch.is_tensor(x) else x, copy=True))
        return f

    ref = SPDHGPoisson(op, subsets=3, seed=1)
    x_ref = ref.run(torch.zeros(op.coeff_shape, device="cuda"), b, 5, diagnostics_interval=2,
                    callback=cb("ref")).cpu().numpy()
    f_ref = [s["f"] for s in ref.iter_stats]
    assert ref.resident_used == ("x", "z", "T")
    for resident in ("none", ["x"], ["x", "z"], ["z", "T"], ["T"], "all"):
        sp = SPDHGPoisson(op, subsets=3, seed=1, resident=resident)
        x = sp.run(np.zeros(op.coeff_shape, np.float32), b, 5, diagnostics_interval=2, callback=cb(str(resident)))
        want = {"none": (), "all": ("x", "z", "T")}.get(resident) if isinstance(resident, str) else \
            tuple(n for n in ("x", "z", "T") if n in resident)
        assert sp.final_stats["resident"] == want
        assert np.array_equal(x, x_ref), resident
        assert [s["f"] for s in sp.iter_stats] == f_ref, resident
        assert np.array_equal(sp.state["z"], ref.state["z"]) and np.array_equal(sp.state["y"], ref.state["y"])
        assert all(np.array_equal(a, r) for a, r in zip(seen[str(resident)], seen["ref"]))

    def resumed(resident):
        sp = SPDHGPoisson(op, subsets=3, seed=1, resident=resident)
        x1 = sp.run(np.zeros(op.coeff_shape, np.float32), b, 3, diagnostics_interval=3)
        x1 = sp.run(x1, b, 2, diagnostics_interval=2, state=sp.state)
        assert sp.state["epoch"] == 5
        return x1, sp.state

    xa, sa = resumed("all")
    xn, sn = resumed("none")
    assert np.array_equal(xa, xn) and np.array_equal(sa["z"], sn["z"]) and np.array_equal(sa["y"], sn["y"])


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_support_ray_table_gives_the_same_iterates(golden, precision):
    """The forward projections of SPDHG read the ray table restricted to the support (the iterates are zero outside
    it): fewer taps, the iterates and deviances of the full table bit for bit."""
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    kw = {} if precision == "fp32" else {"precision": "bf16"}
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"], **kw)
    rng = np.random.default_rng(2)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.3) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy() * 40).astype(np.float32)
    runs = []
    for use in (False, True):
        sp = SPDHGPoisson(op, subsets=3, seed=4)
        sp.use_support_table = use
        x0 = torch.as_tensor(rng.random(op.coeff_shape).astype(np.float32), device="cuda")   # non-zero outside
        x0.copy_(torch.as_tensor(np.random.default_rng(7).random(op.coeff_shape).astype(np.float32)))
        x = sp.run(x0, b, 3, diagnostics_interval=1).cpu().numpy()
        runs.append((x, [s["f"] for s in sp.iter_stats], sp.state["y"]))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1] and np.array_equal(runs[0][2], runs[1][2])
    supp = torch.as_tensor(op.support_mask().astype(np.uint8).ravel(), device="cuda")
    assert op.support_ray_table(supp)[2] < op.ray_taps


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_spdhg_cuda_graphs_equal_plain_iterations(golden, precision):
    """use_graphs: from the second epoch on the iterations replay captured CUDA graphs (update of subset m, forward of
    subset nb); iterates, deviances and state equal the plain run bit for bit, and the graphs were replayed."""
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    kw = {} if precision == "fp32" else {"precision": "bf16"}
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    queue=torch.cuda.Stream(), **kw)
    rng = np.random.default_rng(3)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy() * 50).astype(np.float32)
    runs = []
    for graphs in (False, True):
        sp = SPDHGPoisson(op, subsets=4, seed=2)
        sp.use_graphs = graphs
        x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 5, diagnostics_interval=2).cpu().numpy()
        runs.append((x, [s["f"] for s in sp.iter_stats], sp.state["z"], sp.state["y"],
                     sp.final_stats["graph_replays"]))
    (x0, f0, z0, y0, n0), (x1, f1, z1, y1, n1) = runs
    assert n0 == 0 and n1 > 0
    assert np.array_equal(x0, x1) and f0 == f1 and np.array_equal(z0, z1) and np.array_equal(y0, y1)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_deferred_closing_forward_equals_the_plain_one(golden, precision):
    """run() without callback or printing leaves the last epoch's closing full forward and objective to _finish
    (beside the downloads); with a callback it runs inside the epoch loop. Both give the same final objective, x, z
    and y bit for bit, and the same per-epoch objectives."""
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    d = golden("al5_small")
    cfg, mat, grid = case_inputs(d)
    kw = {} if precision == "fp32" else {"precision": "bf16"}
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"], **kw)
    rng = np.random.default_rng(4)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    b = rng.poisson(op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy() * 50).astype(np.float32)
    runs = []
    for cb in (None, lambda ep, x, stats: False):
        sp = SPDHGPoisson(op, subsets=3, seed=2)
        sp.overlap_residual = False     # a callback keeps the residual in line; compare like with like
        x = sp.run(np.zeros(op.coeff_shape, np.float32), b, 3, diagnostics_interval=1, callback=cb)
        runs.append((x, sp.state, sp.final_stats["final_f"], [s["f"] for s in sp.iter_stats]))
    (x0, s0, f0, fs0), (x1, s1, f1, fs1) = runs
    assert f0 == f1 and fs0 == fs1
    assert np.array_equal(x0, x1)
    assert np.array_equal(s0["z"], s1["z"]) and np.array_equal(s0["y"], s1["y"])
