"""The serving loop on the GPU: requests of uneven size (pixels, angles, orientations, cubic and hexagonal) give the
same coefficients alone and in the mix (bit for bit: every request runs its own kernels in its own order on its own
stream), all finish, and the statistics report p50 / p99 latency."""
import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _requests(golden):
    from diffractom_b200 import SinglePhaseForwardOperator
    from diffractom_b200.serving import Request
    out = []
    for i, name in enumerate(["al5_small", "ti8_small", "adj_0_360"]):
        d = golden(name)
        cfg, mat, grid = case_inputs(d)
        op = SinglePhaseForwardOperator(cfg, mat, grid, 0.5, normalized=True, pf_mode="sparse")
        rng = np.random.default_rng(20 + i)
        x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
                  ).astype(np.float32)
        b = rng.poisson(op.direct(x_true) * 40).astype(np.float32)
        op.free_memory()
        out.append(Request(cfg, mat, grid, b, subsets=3, max_epochs=12, tol=1e-4))
    return out


def _serve(reqs, slots):
    from diffractom_b200.serving import ReconstructionServer
    srv = ReconstructionServer(device=0, max_slots=slots, hbm_budget_gb=20).start()
    for r in reqs:
        srv.submit(r)
    assert srv.wait_all(timeout=600)
    srv.stop()
    return srv


def test_results_alone_equal_results_in_the_mix(golden):
    alone = []
    for r in _requests(golden):
        srv = _serve([r], 1)
        assert r.error is None, r.error
        alone.append(r)
    mixed = _requests(golden)
    srv = _serve(mixed, 3)
    for a, m in zip(alone, mixed):
        assert m.error is None, m.error
        assert m.epochs == a.epochs and m.deviance == a.deviance
        assert np.array_equal(m.result, a.result)
    st = srv.stats()
    assert st["requests"] == 3 and st["failed"] == 0
    assert 0 < st["p50_s"] <= st["p99_s"]
    # the three ran concurrently: each was admitted before the first one finished
    first_done = min(r.finished for r in mixed)
    assert all(r.admitted < first_done for r in mixed)
