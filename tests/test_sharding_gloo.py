"""Multi-process host logic of the walker-sharded path on CPU: two `gloo`
ranks shard a mixed-density walker list, each evaluates its shard (a seeded
stand-in per walker takes the place of one GPU's engine call), and the timing
max / result gather reproduce the single-process answer."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from y3_cluster_cpp_b200 import sharding


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_partition_and_balance():
    dens = [1, 2, 4, 4, 1, 2, 2, 1, 4, 1, 1, 2]
    for world in (1, 2, 3, 4):
        parts = [sharding.shard_walkers(dens, r, world) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(dens)))          # every walker exactly once
        loads = [sum(sharding.DENSITY_COST[dens[i]] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sharding.DENSITY_COST.values())
    assert sharding.shard_walkers([], 0, 2) == []


def _tiny_eval(idx):
    """Deterministic stand-in for a per-walker evaluation (one number per bin)."""
    rng = np.random.default_rng(1000 + idx)
    return rng.standard_normal(12)


def _worker(rank, world, port, dens, out_q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = sharding.shard_walkers(dens, rank, world)
        n_max = max(len(sharding.shard_walkers(dens, r, world)) for r in range(world))
        local = np.full((n_max, 13), np.nan)
        for j, i in enumerate(mine):
            local[j, 0] = i
            local[j, 1:] = _tiny_eval(i)
        t_max = sharding.max_over_ranks(float(rank + 1))
        n_tot = sharding.sum_over_ranks(float(len(mine)))
        gathered = sharding.gather_results(local, rank, world)
        if rank == 0:
            out_q.put((t_max, n_tot, [g.tolist() for g in gathered]))
    finally:
        dist.destroy_process_group()


def test_gloo_world2_shard_gather():
    dens = [4, 1, 2, 2, 4, 1, 1]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, dens, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        t_max, n_tot, gathered = q.get(timeout=120)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert t_max == 2.0
    assert n_tot == len(dens)
    rows = np.concatenate([np.asarray(g) for g in gathered])
    rows = rows[~np.isnan(rows[:, 0])]
    rows = rows[np.argsort(rows[:, 0])]
    assert rows[:, 0].tolist() == list(range(len(dens)))
    ref = np.stack([_tiny_eval(i) for i in range(len(dens))])
    np.testing.assert_array_equal(rows[:, 1:], ref)
