"""Independent solves over several GPUs: one process per GPU, each rank runs
its share of the solves through one batch call
(``congrad_streamfunction_batch``: resident solves side by side, or the
work-queue kernel), then every rank receives every result.

A single solve does not shard (its per-iteration halo exchange and scalar
all-reduces would be dominated by NVLink latency), but the units the
reference runs one after another do: the per-island ``psin`` solves
(streamfct_init.f90:272-287), unevenly sized grids, ensemble members.  There
is no collective on the data path; the only exchange is the final gather
(``torch.distributed.broadcast`` from each solve's owner, NCCL for CUDA
tensors, gloo for host tensors).
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(costs, world):
    """Deterministic longest-processing-time assignment of solves to ranks:
    solves sorted by decreasing cost (ties by index) go to the least loaded
    rank (ties by rank).  Returns ``owner[k]`` for every solve."""
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    owner = [0] * len(costs)
    for k in order:
        load, r = heapq.heappop(heap)
        owner[k] = r
        heapq.heappush(heap, (load + float(costs[k]), r))
    return owner


def solve_cost(nx, ny):
    """Cost model of one solve: Jacobi-PCG iterations grow about linearly with
    the grid extent, the work per iteration with the points."""
    return float(nx) * float(ny) * max(nx, ny)


def run_sharded(n, costs, solve_subset, gather, rank, world):
    """Generic driver.  ``solve_subset(indices)`` solves this rank's share and
    returns ``{k: result}``; ``gather(k, owner, local_result_or_None)`` makes
    solve k's result known on every rank and returns it.  Returns the list of
    all n results (in solve order) and the owner list."""
    owner = partition(costs, world)
    mine = [k for k in range(n) if owner[k] == rank]
    local = solve_subset(mine) if mine else {}
    out = []
    for k in range(n):
        out.append(gather(k, owner[k], local.get(k)))
    return out, owner


def make_gather(sols, group=None):
    """Gather function for :func:`run_sharded`: solve k's solution array is
    broadcast from its owner into every rank's ``sols[k]`` (in place), and its
    result object with it."""
    import torch
    import torch.distributed as dist

    def src(owner):
        return dist.get_global_rank(group, owner) if group is not None else owner

    def gather(k, owner, info):
        s = sols[k]
        # Fortran-ordered arrays: their transpose is the contiguous buffer
        t = s.T if isinstance(s, torch.Tensor) else torch.from_numpy(np.asarray(s).T)
        assert t.is_contiguous(), "solutions must be Fortran-ordered"
        dist.broadcast(t, src=src(owner), group=group)
        box = [info]
        dist.broadcast_object_list(box, src=src(owner), group=group)
        return box[0]

    return gather


def congrad_streamfunction_batch_sharded(contexts, forcs, sols, eps=1e-12, max_it=1000000, rtol=0.0, group=None):
    """``external.congrad_streamfunction_batch`` over all ranks of the process
    group: solve k runs on rank ``partition(...)[k]``; afterwards every rank
    holds every solution (``sols`` updated in place) and every info dict.
    ``sols`` are Fortran-ordered float64 CUDA tensors (NCCL) or numpy arrays
    (gloo).  Returns (infos, owner)."""
    import torch.distributed as dist
    from . import external

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    costs = [solve_cost(em.M.nx, em.M.ny) for em in contexts]

    def solve_subset(idx):
        infos = external.congrad_streamfunction_batch([contexts[k] for k in idx], [forcs[k] for k in idx],
                                                      [sols[k] for k in idx], eps=eps, max_it=max_it, rtol=rtol)
        return {k: info for k, info in zip(idx, infos)}

    return run_sharded(len(contexts), costs, solve_subset, make_gather(sols, group), rank, world)
