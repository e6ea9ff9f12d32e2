"""Orientation sharding over several GPUs (one process per GPU, torch.distributed over NCCL).

The forward operator is a sum over orientations, A x = sum_k A_k x_k, and the solvers' coefficient state (x, z, T
of SPDHG) is per orientation. So K splits into contiguous shards, one per rank; each rank builds its own
SinglePhaseForwardOperator on its shard of the grid and keeps its shard's coefficients. The adjoint needs no
exchange (A_k^T reads the replicated data rows only). The forward's exchange is one all-reduce of the data rows the
pass wrote: the rows of the next subset in an SPDHG iteration (R/M angles x My x N_eta N_rings floats), or all rows
for the full forward of the step sizes and of the diagnostics. The dual update, the deviance and the subset schedule
then run redundantly on every rank on identical data (an all-reduce leaves the same bits on all ranks).

ShardSum is that exchange; SPDHGPoisson(..., shards=ShardSum(group)) uses it. The ranks take the same collective
steps in the same order (the schedule comes from the same seed on every rank).
"""
from __future__ import annotations

import numpy as np
import torch

from .grid import MatrixGrid, grid_arrays


def shard_range(K: int, rank: int, world: int):
    """(k0, k1): the contiguous orientations of a rank; shard sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for {world} ranks")
    base, extra = divmod(int(K), world)
    k0 = rank * base + min(rank, extra)
    return k0, k0 + base + (1 if rank < extra else 0)


def shard_grid(grid, rank: int, world: int) -> MatrixGrid:
    """The rank's orientations of a grid (rotations and kernel widths as the grid holds them), as a grid the
    operator accepts."""
    if hasattr(grid, "leaf_arrays"):
        mats, sig = (np.asarray(a) for a in grid.leaf_arrays())
    else:
        mats, sig = grid_arrays(grid)
    k0, k1 = shard_range(len(mats), rank, world)
    if k1 <= k0:
        raise ValueError(f"{len(mats)} orientations cannot be split over {world} ranks")
    return MatrixGrid(mats[k0:k1], sig[k0:k1])


class ShardSum:
    """Sum of data rows over the orientation shards of a process group: all(data) for a whole data array,
    rows(data, omegas) for the rows of some angles (packed into one contiguous buffer, all-reduced, unpacked).
    Collectives run ordered with the given stream (the operator's), so the caller's kernel order is kept."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self._buf = None

    def all(self, data: torch.Tensor, stream=None):
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.dist.all_reduce(data, group=self.group)

    def rows(self, data: torch.Tensor, omegas: torch.Tensor, stream=None):
        """data (R, ...) float32: rows omegas (int32 or int64 indices, on data's device) summed over the ranks."""
        R = data.shape[0]
        flat = data.view(R, -1)
        n = int(omegas.numel())
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            need = n * flat.shape[1]
            if self._buf is None or self._buf.numel() < need or self._buf.device != data.device:
                self._buf = torch.empty(need, dtype=data.dtype, device=data.device)
            packed = self._buf[:need].view(n, flat.shape[1])
            torch.index_select(flat, 0, omegas, out=packed)
            self.dist.all_reduce(packed, group=self.group)
            flat.index_copy_(0, omegas.long() if omegas.dtype != torch.int64 else omegas, packed)

    def total(self, value: float) -> float:
        """Sum of a host scalar over the ranks (float64)."""
        nccl = str(self.dist.get_backend(self.group)).lower() == "nccl"
        dev = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
        t = torch.tensor([value], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, group=self.group)
        return float(t.item())


class _nullctx:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False
