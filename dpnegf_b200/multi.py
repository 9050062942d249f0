"""Work items over ranks: one process per GPU, no data-path collective.

A batch of (device, k-point, energy) items is independent item by item, so
ranks split the cost-sorted queue and each runs its share through the same
persistent launch as a single GPU would.  The only exchange is one all-reduce
(sum) of the per-item result vectors at the end (T(E), DOS, densities, or their
k-weighted sums), which is how the reference's runner adds k-point
contributions on the host (runner/NEGF.py:904-906).
"""
from typing import Callable, Sequence

import numpy as np
import torch
import torch.distributed as dist


def shard(costs: Sequence[float], world: int, rank: int) -> np.ndarray:
    """Item indices owned by ``rank``: longest-processing-time assignment of the
    cost-sorted queue (each item goes to the rank with the least work so far;
    ties to the lower rank), returned in queue order.  Every item is owned by
    exactly one rank and the per-rank work differs by at most one item's cost."""
    costs = np.asarray(costs, dtype=np.float64).reshape(-1)
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside a world of {world}")
    order = np.argsort(-costs, kind="stable")
    load = np.zeros(world)
    owner = np.empty(len(costs), dtype=np.int64)
    for i in order:
        r = int(np.argmin(load))
        owner[i] = r
        load[r] += costs[i]
    mine = np.nonzero(owner == rank)[0]
    return mine[np.argsort(-costs[mine], kind="stable")]


def run_sharded(costs: Sequence[float], compute: Callable[[np.ndarray], torch.Tensor], out_shape,
                dtype=torch.float64, device="cpu", group=None) -> torch.Tensor:
    """Compute every item once over all ranks and give every rank the full result.

    ``compute(idx)`` returns the results of items ``idx`` (first dimension
    ``len(idx)``); ``out_shape`` is the shape of the full result (first dimension
    = number of items).  Without an initialised process group this is a plain
    single-process call.
    """
    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    idx = shard(costs, world, rank)
    out = torch.zeros(out_shape, dtype=dtype, device=device)
    if len(idx):
        out[torch.as_tensor(idx, device=device)] = compute(idx).to(device=device, dtype=dtype)
    if world > 1:
        dist.all_reduce(out, op=dist.ReduceOp.SUM, group=group)
    return out
