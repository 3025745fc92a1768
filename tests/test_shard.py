"""Sharding of independent solves over ranks (pyom2_b200/shard.py), on the
CPU: the partition, and the gather of every rank's results over a gloo
process group of world size 2 (the solver itself is replaced by a host
function; the GPU path calls the batch kernel in its place)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from pyom2_b200 import shard


def test_partition_is_deterministic_and_balanced():
    rng = np.random.default_rng(0)
    dims = [(int(rng.integers(128, 1025)), int(rng.integers(128, 769))) for _ in range(64)]
    costs = [shard.solve_cost(nx, ny) for nx, ny in dims]
    for world in (1, 2, 4, 8):
        owner = shard.partition(costs, world)
        assert owner == shard.partition(costs, world)
        assert set(owner) <= set(range(world))
        loads = np.bincount(owner, weights=costs, minlength=world)
        # LPT bound: no rank above the average by more than the largest job
        assert loads.max() <= np.mean(loads) + max(costs) + 1e-9


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        shapes = [(6 + k % 3, 5 + k % 4) for k in range(n)]
        forcs = [np.asfortranarray(np.full(s, float(k + 1))) for k, s in enumerate(shapes)]
        sols = [np.zeros(s, order="F") for s in shapes]
        costs = [float(a * b) for a, b in shapes]

        def solve_subset(idx):
            out = {}
            for k in idx:
                sols[k][...] = 2.0 * forcs[k] + rank * 0.0  # the "solve"
                out[k] = {"iterations": 10 + k, "rank": rank}
            return out

        infos, owner = shard.run_sharded(n, costs, solve_subset, shard.make_gather(sols), rank, world)
        ok = all(np.array_equal(sols[k], 2.0 * forcs[k]) for k in range(n))
        ok = ok and all(infos[k]["iterations"] == 10 + k and infos[k]["rank"] == owner[k] for k in range(n))
        q.put((rank, ok, owner))
    finally:
        dist.destroy_process_group()


def test_sharded_results_reach_every_rank_gloo():
    world, n = 2, 9
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    assert all(ok for _, ok, _ in res)
    owners = [o for _, _, o in res]
    assert owners[0] == owners[1] and set(owners[0]) == {0, 1}
