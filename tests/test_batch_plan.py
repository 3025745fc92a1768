"""The host planner of the resident batch (pyomgpu_plan_batch: list
scheduling of rigid gangs of blocks plus a local search over the order), on
the CPU.  What the multi-solve kernel relies on:

* every job gets exactly its number of distinct blocks;
* no block serves two jobs at once under the planned durations;
* every block's jobs, taken by rank, are in planned-start order -- one total
  order for all blocks, so gangs never wait on one another in a cycle;
* the local search never lengthens the plan, and on a batch shaped like
  config 2 it packs the blocks to well above 80 %.
"""
import ctypes as C

import numpy as np
import pytest

from pyom2_b200 import _abi

NSM = 148


def plan(blocks, est, tries=400):
    L = _abi.load()
    n = len(blocks)
    b = np.ascontiguousarray(blocks, dtype=np.int32)
    e = np.ascontiguousarray(est, dtype=np.float64)
    rank = np.zeros(n, dtype=np.int32)
    start = np.zeros(n)
    gang = np.zeros((n, NSM), dtype=np.int32)
    span = C.c_double()
    _abi.check(L.pyomgpu_plan_batch(NSM, n, b.ctypes.data, e.ctypes.data, int(tries), rank.ctypes.data,
                                    start.ctypes.data, gang.ctypes.data, C.byref(span)))
    return rank, start, gang, span.value


def batches():
    rng = np.random.default_rng(3)
    # config 2 shaped: 64 grids of 128-1024 x 128-768 points, ~7000 points per block
    pts = rng.integers(128, 1025, 64) * rng.integers(128, 769, 64)
    b2 = np.maximum(1, np.ceil(pts / 7000.0)).astype(int)
    yield "c2-like", b2, np.sqrt(pts) * (8.0 + rng.uniform(-1, 1, 64))
    yield "equal", np.full(20, 136), np.full(20, 10.0)
    yield "small", rng.integers(1, 12, 30), rng.uniform(1, 5, 30)
    yield "mixed", rng.integers(1, NSM + 1, 40), rng.uniform(0.5, 20, 40)
    yield "two", np.array([100, 60]), np.array([3.0, 2.0])


@pytest.mark.parametrize("name,blocks,est", list(batches()), ids=lambda x: x if isinstance(x, str) else "")
def test_plan_invariants(name, blocks, est):
    rank, start, gang, span = plan(blocks, est)
    n = len(blocks)
    assert sorted(rank) == list(range(n))
    busy = {b: [] for b in range(NSM)}
    for k in range(n):
        g = gang[k][gang[k] >= 0]
        assert len(g) == blocks[k] and len(set(g.tolist())) == blocks[k] and g.min() >= 0 and g.max() < NSM
        assert np.all(np.diff(g) > 0)  # ascending: piece q on the q-th block
        assert np.all(gang[k][blocks[k]:] == -1)
        for blk in g:
            busy[blk].append((start[k], start[k] + est[k], rank[k]))
    for blk, iv in busy.items():
        iv.sort(key=lambda x: x[2])  # the order the block runs its jobs in
        for (s0, e0, _), (s1, e1, _) in zip(iv, iv[1:]):
            assert s1 >= e0 - 1e-9 * max(1.0, e0), (name, blk)  # by rank = by start, never overlapping
    assert span >= max(start + est) - 1e-9 and span <= (start + est).max() + 1e-9


@pytest.mark.parametrize("name,blocks,est", list(batches()), ids=lambda x: x if isinstance(x, str) else "")
def test_search_never_lengthens_and_packs(name, blocks, est):
    _, _, _, greedy = plan(blocks, est, tries=0)
    _, _, _, searched = plan(blocks, est, tries=400)
    assert searched <= greedy + 1e-9
    lower = max(float((blocks * est).sum()) / NSM, float(est.max()))
    if name == "c2-like":
        assert lower / searched > 0.8, lower / searched


def test_bad_arguments():
    L = _abi.load()
    b = np.array([NSM + 1], dtype=np.int32)
    e = np.array([1.0])
    assert L.pyomgpu_plan_batch(NSM, 1, b.ctypes.data, e.ctypes.data, 0, None, None, None, None) == _abi.EINVAL
