"""K-sharded SPDHG on one GPU: two orientation shards, each with its own operator (built on its shard of the grid)
and its own stream, driven by two host threads; their exchange is a host-side sum of the forward rows that stands
in for the NCCL all-reduce of ShardSum (the threads meet at a host barrier, so no kernel waits for another). The
shards' iterates, concatenated, and their deviances match the single-operator run; a one-rank NCCL process group
runs the ShardSum path itself."""
import threading

import numpy as np
import pytest

from conftest import case_inputs

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


class _Shared:
    def __init__(self, world):
        self.world = world
        self.bar = threading.Barrier(world, timeout=120)
        self.slots = [None] * world
        self.res = None


class ThreadShardSum:
    """ShardSum's interface for ranks that are threads of one process on one GPU."""

    def __init__(self, shared, rank):
        self.sh, self.rank = shared, rank

    def _sum(self, t, stream):
        sh = self.sh
        stream.synchronize()
        sh.slots[self.rank] = t
        sh.bar.wait()
        if self.rank == 0:
            acc = sh.slots[0].clone()
            for o in sh.slots[1:]:
                acc += o
            torch.cuda.synchronize()
            sh.res = acc
        sh.bar.wait()
        with torch.cuda.stream(stream):
            t.copy_(sh.res)
        stream.synchronize()
        sh.bar.wait()

    def all(self, data, stream=None):
        self._sum(data, stream or torch.cuda.current_stream())

    def rows(self, data, omegas, stream=None):
        stream = stream or torch.cuda.current_stream()
        flat = data.view(data.shape[0], -1)
        with torch.cuda.stream(stream):
            packed = flat.index_select(0, omegas)
        self._sum(packed, stream)
        with torch.cuda.stream(stream):
            flat.index_copy_(0, omegas.long(), packed)


def _problem(d, precision):
    from diffractom_b200 import SinglePhaseForwardOperator
    cfg, mat, grid = case_inputs(d)
    op = SinglePhaseForwardOperator(cfg, mat, grid, 1e-5, normalized=True, quadrature=d["quadrature"],
                                    precision=precision)
    rng = np.random.default_rng(9)
    x_true = (rng.random(op.coeff_shape) * (rng.random(op.coeff_shape) < 0.2) * op.support_mask()[None]
              ).astype(np.float32)
    op.precision = "fp32"
    b = rng.poisson(op.direct(torch.as_tensor(x_true, device="cuda")).cpu().numpy() * 50).astype(np.float32)
    op.precision = precision
    return op, b, cfg, mat, grid


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_sharded_spdhg_matches_single_operator(golden, precision):
    from diffractom_b200 import SinglePhaseForwardOperator, SPDHGPoisson
    from diffractom_b200.sharding import shard_grid
    d = golden("al5_small")
    op, b, cfg, mat, grid = _problem(d, precision)
    ref = SPDHGPoisson(op, subsets=3, seed=1)
    x_ref = ref.run(torch.zeros(op.coeff_shape, device="cuda"), b, 4, diagnostics_interval=2).cpu().numpy()
    f_ref = [s["f"] for s in ref.iter_stats if s["f"] is not None]
    world = 2
    shared = _Shared(world)
    out, errs = [None] * world, []

    def rank_main(r):
        try:
            torch.cuda.set_device(0)
            op_r = SinglePhaseForwardOperator(cfg, mat, shard_grid(grid, r, world), 1e-5, normalized=True,
                                              quadrature=d["quadrature"], precision=precision,
                                              queue=torch.cuda.Stream())
            sp = SPDHGPoisson(op_r, subsets=3, seed=1, shards=ThreadShardSum(shared, r))
            x = sp.run(torch.zeros(op_r.coeff_shape, device="cuda"), b, 4, diagnostics_interval=2)
            op_r.stream().synchronize()
            out[r] = (x.cpu().numpy(), [s["f"] for s in sp.iter_stats if s["f"] is not None], sp.state["y"])
        except BaseException as e:                      # noqa: BLE001 - reported by the main thread
            errs.append(e)
            shared.bar.abort()

    th = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    x = np.concatenate([o[0] for o in out])
    tol_x = 1e-4 if precision == "fp32" else 1e-3
    assert np.abs(x - x_ref).max() <= tol_x * np.abs(x_ref).max()
    assert out[0][1] == out[1][1]                       # every rank computes the same deviances
    np.testing.assert_allclose(out[0][1], f_ref, rtol=1e-5)
    assert np.array_equal(out[0][2], out[1][2])          # and the same dual variable


def test_shard_sum_over_a_one_rank_nccl_group(golden):
    """ShardSum itself (NCCL, one rank): the sharded run of one shard reproduces the unsharded run bit for bit."""
    import os
    import socket
    import torch.distributed as dist
    from diffractom_b200 import SPDHGPoisson
    from diffractom_b200.sharding import ShardSum
    d = golden("al5_small")
    op, b, *_ = _problem(d, "fp32")
    ref = SPDHGPoisson(op, subsets=3, seed=1)
    x_ref = ref.run(torch.zeros(op.coeff_shape, device="cuda"), b, 3, diagnostics_interval=3).cpu().numpy()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    import datetime
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    try:
        sp = SPDHGPoisson(op, subsets=3, seed=1, shards=ShardSum())
        x = sp.run(torch.zeros(op.coeff_shape, device="cuda"), b, 3, diagnostics_interval=3).cpu().numpy()
        assert sp.shards.total(2.5) == 2.5
    finally:
        dist.destroy_process_group()
    assert np.array_equal(x, x_ref)
    assert [s["f"] for s in sp.iter_stats] == [s["f"] for s in ref.iter_stats]
