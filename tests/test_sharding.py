"""Orientation sharding on the CPU: the partition of K over ranks, and the shards' exchange step (ShardSum) over a
gloo process group of two ranks, with the CPU oracle as the per-shard operator: the forward of each rank's shard
operator (built on its shard of the grid), summed over the ranks (subset rows, or all rows), equals the forward of
the whole grid."""
import os
import socket

import numpy as np
import pytest

from conftest import GOLDEN, case_inputs

torch = pytest.importorskip("torch")


def test_shard_range_partitions_K():
    from diffractom_b200.sharding import shard_range
    for K in (1, 2, 7, 1000, 20001):
        for world in (1, 2, 3, 8):
            if world > K:
                continue
            r = [shard_range(K, i, world) for i in range(world)]
            assert r[0][0] == 0 and r[-1][1] == K
            assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_shard_grid_keeps_rotations_and_widths():
    from diffractom_b200.grid import Grid
    from diffractom_b200.sharding import shard_grid
    g = Grid.from_random_fundamental_zone(11, "cubic", np.deg2rad(3.0), seed=4)
    parts = [shard_grid(g, r, 3) for r in range(3)]
    assert np.array_equal(np.concatenate([p.matrices for p in parts]), g.matrices)
    assert np.array_equal(np.concatenate([p.sigmas for p in parts]), g.sigmas)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir, case):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from conftest import load_case
        from diffractom_b200.geometry import OperatorGeometry
        from diffractom_b200.sharding import ShardSum, shard_grid, shard_range
        from oracle.oracle import OracleOperator
        d = load_case(case)
        cfg, mat, grid = case_inputs(d)
        K = len(grid)
        k0, k1 = shard_range(K, rank, world)
        g = OperatorGeometry(cfg, mat, shard_grid(grid, rank, world), normalized=True, quadrature=d["quadrature"],
                             radon_kernel=d["kernel"])
        orc = OracleOperator.from_operator(g, batches=[(0, k1 - k0)], precision="f64")
        rng = np.random.default_rng(3)
        x = rng.random((K, g.Ny, g.Nx)).astype(np.float32)         # the same full x on every rank
        sub = np.arange(1, orc.R, 3)
        part = orc.forward(x[k0:k1]).astype(np.float32)
        keep = rng.random(part.shape).astype(np.float32)            # rows outside the subset: left alone
        rows = keep.copy()
        rows[sub] = part[sub]
        summed = ShardSum()
        full = torch.from_numpy(part.copy())
        summed.all(full)
        tr = torch.from_numpy(rows)
        summed.rows(tr, torch.as_tensor(sub, dtype=torch.int32))
        tot = summed.total(float(rank + 1))
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), full=full.numpy(), rows=tr.numpy(), keep=keep, tot=tot)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("case", ["al5_small", "ti8_small"])
def test_shard_sum_of_shard_forwards_equals_whole_forward(tmp_path, case):
    import torch.multiprocessing as mp
    from conftest import load_case
    from diffractom_b200.geometry import OperatorGeometry
    from oracle.oracle import OracleOperator
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), case), nprocs=world, join=True,
                       start_method="spawn")
    d = load_case(case)
    cfg, mat, grid = case_inputs(d)
    g = OperatorGeometry(cfg, mat, grid, normalized=True, quadrature=d["quadrature"], radon_kernel=d["kernel"])
    whole = OracleOperator.from_operator(g, batches=[(0, len(grid))], precision="f64")
    rng = np.random.default_rng(3)
    x = rng.random((len(grid), g.Ny, g.Nx)).astype(np.float32)
    ref = whole.forward(x)
    sub = np.arange(1, whole.R, 3)
    res = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    scale = np.abs(ref).max()
    for r in res:
        assert np.abs(r["full"] - ref).max() <= 1e-6 * scale
        assert np.array_equal(r["full"], res[0]["full"])          # the same bits on every rank
        assert np.abs(r["rows"][sub] - ref[sub]).max() <= 1e-6 * scale
        others = np.setdiff1d(np.arange(whole.R), sub)
        assert np.array_equal(r["rows"][others], r["keep"][others])
        assert float(r["tot"]) == 3.0
