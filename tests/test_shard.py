"""Sharding of independent solves over ranks (pyom2_b200/shard.py), on the
CPU: the partition, and the gather of every rank's results over a gloo
process group of world size 2.  Each rank solves its share of small closed
basins with the oracle's congrad_streamfunction (the GPU path calls the batch
solver in its place); after the gather every rank holds every solution and
info, equal bit for bit to its own oracle solve of the same problem."""
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


def _problems(n):
    """n small closed basins with islands, their forcing and zero first guess."""
    from pyom2_b200 import synth
    return [synth.basin(20 + 4 * (k % 3), 14 + 3 * (k % 4), 500 + k, 0.2, 1 + k % 3, nz=4) for k in range(n)]


def _oracle_solve(oracle, W):
    O = oracle.Oracle(W.M.copy())
    O.streamfunction_init(maxipp=10**6, maxq=10**6)
    cf = O.make_coeff_streamfunction()
    x = np.zeros(W.M.shape2d, order="F")
    r = O.congrad_streamfunction(cf, W.forc, x)
    return x, r


def _worker(rank, world, port, n, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    from oracle import oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ws = _problems(n)
        sols = [np.zeros(w.M.shape2d, order="F") for w in ws]
        costs = [shard.solve_cost(w.M.nx, w.M.ny) for w in ws]

        def solve_subset(idx):
            out = {}
            for k in idx:
                x, r = _oracle_solve(oracle, ws[k])
                sols[k][...] = x
                out[k] = {"iterations": int(r["iterations"]), "converged": bool(r["converged"]), "rank": rank}
            return out

        infos, owner = shard.run_sharded(n, costs, solve_subset, shard.make_gather(sols), rank, world)
        ok = True
        for k in range(n):  # every rank now holds every solve: check against a local oracle solve
            x, r = _oracle_solve(oracle, ws[k])
            ok = ok and np.array_equal(sols[k], x) and infos[k]["iterations"] == int(r["iterations"])
            ok = ok and infos[k]["converged"] and infos[k]["rank"] == owner[k]
        q.put((rank, ok, owner))
    finally:
        dist.destroy_process_group()


def test_sharded_results_reach_every_rank_gloo():
    from oracle import oracle
    oracle.build()  # before the workers start, so they only load it
    world, n = 2, 7
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
