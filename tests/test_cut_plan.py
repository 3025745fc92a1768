"""The piece cut of the on-chip-resident kernel (pyomgpu_plan_cut: res_cut with
the fitted iteration-time estimate), on the host only.

MEASURED holds the iteration times of the 1440x720 FP64 solve (1869
iterations to 2e-11, one B200, CUDA events) under every cut of that grid that
fits at 16 points per thread; the estimate was fitted to them.  MEASURED32
holds whole mixed-precision solves (FP32 resident correction solves, 2755
and 4270 inner iterations) under five cuts of each grid.
"""
import ctypes as C

import numpy as np
import pytest

from pyom2_b200 import _abi

CAP = 225 * 1024  # dynamic shared memory a resident block may use (B200: ~227 KB less static)
NSM = 148

# (npx, npy): us per iteration
MEASURED = {
    (37, 4): 9.62, (6, 23): 9.14, (6, 24): 9.10, (9, 15): 9.00, (9, 16): 8.91, (12, 12): 8.89,
    (15, 9): 9.01, (16, 9): 9.09, (18, 8): 8.97, (24, 6): 9.27, (28, 5): 9.33, (29, 5): 9.38,
    (36, 4): 9.37, (45, 3): 9.56, (46, 3): 9.59, (47, 3): 10.23, (48, 3): 10.22, (49, 3): 10.04,
}

# grid: {(npx, npy): ms per mixed-precision solve}
MEASURED32 = {
    (1440, 720): {(37, 4): 24.93, (9, 16): 23.50, (12, 12): 23.43, (6, 24): 23.85, (8, 18): 31.95},
    (2048, 1024): {(49, 3): 58.81, (37, 4): 57.00, (9, 16): 55.79, (18, 8): 56.25, (13, 11): 54.60},
}


@pytest.fixture(scope="module")
def L():
    return _abi.load()


def plan(L, nx, ny, maxb=NSM, cap=CAP, p=0, dense=False, fp32=False):
    out = np.zeros(5, dtype=np.int32)
    est = C.c_double(0.0)
    _abi.check(L.pyomgpu_plan_cut(nx, ny, maxb, cap, p, int(dense), int(fp32), out.ctypes.data, C.byref(est)))
    return tuple(int(v) for v in out), est.value


def res_smem_bytes(w, h):
    """Dynamic shared memory of a w x h piece (cg_res.cuh res_smem_bytes)."""
    words = (w + 2) * (h + 2) + (w + 1) * h + w * (h + 1) + 2 * h + 6 * (w + h)
    return 8 * ((words + 1) // 2 * 2 + 8 * (w + h))


def test_headline_grid_takes_a_near_fastest_measured_cut(L):
    (npx, npy, w, h, p), est = plan(L, 1440, 720)
    assert (npx, npy, p) == (9, 16, 16) and (w, h) == (160, 45)
    assert (npx, npy) in MEASURED
    assert MEASURED[(npx, npy)] <= 1.01 * min(MEASURED.values())
    assert abs(est * 1e-3 - MEASURED[(npx, npy)]) < 0.25


@pytest.mark.parametrize("nx,ny", [(1440, 720), (670, 372), (1010, 280), (185, 438), (2048, 1024), (64, 64)])
@pytest.mark.parametrize("dense", [False, True])
def test_cut_invariants(L, nx, ny, dense):
    (npx, npy, w, h, p), est = plan(L, nx, ny, p=16 if dense else 0, dense=dense)
    if npx == 0:
        assert (nx, ny) == (2048, 1024)  # too large for FP64 pieces on 148 SMs
        return
    assert npx * npy <= NSM
    assert w == -(-nx // npx) and h == -(-ny // npy)
    assert p in (4, 8, 16) and w * (-(-h // p)) <= 480 and w + h <= 480
    assert res_smem_bytes(w, h) <= CAP
    assert est > 3000.0
    if dense:
        (fx, fy, *_), est_fast = plan(L, nx, ny, p=16)
        assert npx * npy * est <= fx * fy * est_fast + 1e-6


@pytest.mark.parametrize("grid", sorted(MEASURED32))
def test_fp32_cut_avoids_the_slow_measured_cuts(L, grid):
    """The FP32 choice is a 16-point cut where one fits and a compact one
    otherwise: within 3 % of the fastest of the five measured cuts, where the
    narrow pieces the points-only estimate chose ran 4-5 % slower and 32
    points per thread where 16 fit ran 36 % slower."""
    (npx, npy, w, h, p), est = plan(L, *grid, fp32=True)
    ms = MEASURED32[grid]
    best = min(ms.values())
    assert p == (16 if grid == (1440, 720) else 32)
    assert w >= 100  # no narrow column pieces
    if (npx, npy) in ms:
        assert ms[(npx, npy)] <= 1.03 * best
    assert ms[(37, 4)] > 1.03 * best  # the narrow cut is measurably slower
    assert est > 3000.0


def test_no_fit_and_bad_arguments(L):
    cut, est = plan(L, 1440, 720, maxb=20)
    assert cut == (0, 0, 0, 0, 0) and est == 0.0
    out = np.zeros(5, dtype=np.int32)
    assert L.pyomgpu_plan_cut(1440, 720, NSM, CAP, 5, 0, 0, out.ctypes.data, None) == _abi.EINVAL
    assert L.pyomgpu_plan_cut(1440, 720, NSM, CAP, 32, 0, 0, out.ctypes.data, None) == _abi.EINVAL
    assert L.pyomgpu_plan_cut(1440, 720, NSM, CAP, 8, 0, 1, out.ctypes.data, None) == _abi.EINVAL
    assert L.pyomgpu_plan_cut(1, 720, NSM, CAP, 0, 0, 0, out.ctypes.data, None) == _abi.EINVAL
    assert L.pyomgpu_plan_cut(1440, 720, 400, CAP, 0, 0, 0, out.ctypes.data, None) == _abi.EINVAL
    assert L.pyomgpu_plan_cut(1440, 720, NSM, CAP, 0, 0, 0, None, None) == _abi.EINVAL
