"""Several GPUs: independent beams, one process per GPU, no data-path collective.

Beams (E, theta, phi systems) are independent, so a batch shards by beam:
each rank builds a plan over its own contiguous slice and solves it alone.
The only collectives are on the host side of the measurement (max of the
per-rank device times) and, for callers that want every intensity on one
rank, a gather of the per-beam results after the solves.  Nothing here waits
on another GPU inside a kernel.
"""

from __future__ import annotations

import torch
import torch.distributed as dist


def shard_bounds(n_items: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of a contiguous split of n_items over world ranks (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard(items: list, rank: int, world: int) -> list:
    lo, hi = shard_bounds(len(items), rank, world)
    return items[lo:hi]


def max_over_ranks(value: float, device: torch.device | str = "cpu") -> float:
    """Max of a per-rank scalar (a device time) over the process group; the value
    itself when no group is initialised."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(local: list, world: int) -> list | None:
    """Concatenate every rank's list of per-beam results on rank 0 (rank order,
    so the order of the unsharded batch is restored); None on other ranks."""
    if not (dist.is_available() and dist.is_initialized()) or world == 1:
        return list(local)
    out = [None] * world if dist.get_rank() == 0 else None
    dist.gather_object(local, out, dst=0)
    if out is None:
        return None
    return [x for part in out for x in part]


def sharded_sweep(conditions: list, config, *, solve=None) -> list | None:
    """A sweep of many beams over one potential split across the ranks of the
    process group: rank r solves its contiguous slice of ``conditions`` on its
    own GPU (``get_scattering_matrices``, one batched plan) and rank 0 gets
    every beam's |S|^2 grid back in the order of ``conditions``; other ranks
    get None.  Without a process group it is ``get_scattering_matrices``.
    ``solve(conditions, config) -> list`` replaces the per-rank solve (the
    host-side tests run the sharding and the gather without a GPU)."""
    if solve is None:
        from .api import get_scattering_matrices as solve
    if not (dist.is_available() and dist.is_initialized()):
        return list(solve(conditions, config))
    world, rank = dist.get_world_size(), dist.get_rank()
    mine = shard(list(conditions), rank, world)
    local = list(solve(mine, config)) if mine else []
    return gather_to_rank0(local, world)
