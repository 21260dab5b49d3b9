"""Multi-rank host logic on CPU (gloo, world size 2): beam sharding, the
max-over-ranks timing and the gather of per-beam results."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from multiscat_b200.replicas import (gather_to_rank0, max_over_ranks, shard, shard_bounds,
                                     sharded_sweep)


def test_shard_bounds_cover_every_item_once():
    for n in (0, 1, 5, 512, 513):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_bounds(n, r, world)
                seen.extend(range(lo, hi))
                assert hi - lo in (n // world, n // world + 1)
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shard_bounds(4, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        beams = list(range(11))
        mine = shard(beams, rank, world)
        t = max_over_ranks(1.5 + rank)                    # per-rank "device time"
        results = [b * 10 for b in mine]                  # per-beam results
        gathered = gather_to_rank0(results, world)
        out[rank] = (mine, t, gathered)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == [0, 1, 2, 3, 4, 5] and res[1][0] == [6, 7, 8, 9, 10]
    assert res[0][1] == res[1][1] == 2.5                  # max over ranks
    assert res[0][2] == [b * 10 for b in range(11)]       # rank order restored on rank 0
    assert res[1][2] is None


def test_single_process_helpers_without_group():
    assert max_over_ranks(3.0) == 3.0
    assert gather_to_rank0([1, 2], 1) == [1, 2]
    assert torch.tensor([1.0]).item() == 1.0


def _fake_solve(conditions, config):
    """Stands in for the per-rank GPU solve: one result per condition."""
    return [(c.incident_energy, config.precision, os.getpid()) for c in conditions]


def _sweep_worker(rank: int, world: int, port: int, out):
    import math
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        from multiscat_b200 import OptimizationConfig
        from tests.test_api_host import _sweep_conditions
        conds = _sweep_conditions(7)
        res = sharded_sweep(conds, OptimizationConfig(precision=1e-6), solve=_fake_solve)
        out[rank] = None if res is None else [(r[0], r[1], r[2]) for r in res]
        out[f"e{rank}"] = [c.incident_energy for c in conds]
        assert math.isfinite(conds[0].incident_energy)
    finally:
        dist.destroy_process_group()


def test_sharded_sweep_splits_beams_and_gathers_in_order():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_sweep_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[1] is None
    got = res[0]
    assert [r[0] for r in got] == res["e0"]                   # every beam once, in order
    assert all(r[1] == 1e-6 for r in got)
    pids = [r[2] for r in got]
    assert len(set(pids[:4])) == 1 and len(set(pids[4:])) == 1 and pids[0] != pids[4]
