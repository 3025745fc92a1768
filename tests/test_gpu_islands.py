"""GPU island labelling and perimeter tracing (csrc/islands_gpu.cu) against
the host restatement of isleperim / streamfct_init (csrc/islands.cpp, itself
bit-exact with the oracle in tests/test_abi.py): the same island count,
max_boundary, boundary points, directions and lengths, or the same error, on
the benchmark grids and on raw random land masks (seam-crossing masses,
collisions, lakes) in both cyclic settings."""
import time

import numpy as np
import pytest

from pyom2_b200 import _abi, external, synth
from pyom2_b200.model import ModelState

pytestmark = pytest.mark.gpu
LIM = dict(maxipp=10**6, maxq=10**6)


def both(M):
    out = []
    for gpu in (False, True):
        try:
            out.append(("ok", external.island_boundaries(M, gpu=gpu, **LIM)))
        except _abi.PyOMGPUError as e:
            out.append(("err", e.code, str(e).split(":")[-1]))
    return out


def same(a, b):
    if a[0] != b[0]:
        return False
    if a[0] == "err":
        return a[1] == b[1]
    return all(np.array_equal(x, y) for x, y in zip(a[1], b[1]))


def grids():
    yield "c0", synth.config0().M
    yield "cyc96", synth._global_like(96, 48, -80.0, 80.0, 13, n_land_masses=6, mask_sigma=4.0, depth_sigma=4.0).M
    for k, (nx, ny) in enumerate([(40, 32), (64, 48), (130, 70)]):
        yield f"basin{k}", synth.basin(nx, ny, 300 + k, 0.25, 6).M
    yield "channel", synth.config4(1004, nx=64, ny=64, nz=4).M
    yield "c1", synth.config1().M


@pytest.mark.parametrize("name,M", list(grids()))
def test_gpu_islands_match_host(name, M):
    h, g = both(M)
    assert h[0] == "ok" and same(h, g), name


def raw_grid(seed):
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(12, 90)), int(rng.integers(12, 60))
    cyc = bool(rng.integers(0, 2))
    M = ModelState(nx, ny, 2, enable_cyclic_x=cyc)
    noise = synth.smooth_field(rng, (nx, ny), float(rng.uniform(1.0, 4.0)), (cyc, False))
    land = noise < np.quantile(noise, float(rng.uniform(0.1, 0.5)))
    M.kbot[2:nx + 2, 2:ny + 2] = np.where(land, 0, 1)
    return M


@pytest.mark.parametrize("seed", range(40))
def test_gpu_islands_match_host_on_raw_masks(seed):
    """Unprocessed masks: lakes, one-cell straits and collisions included; the
    tracing may fail on them in the reference, and must then fail the same way."""
    M = raw_grid(seed)
    h, g = both(M)
    assert same(h, g), (seed, h[0], g[0], h[1] if h[0] == "err" else None, g[1] if g[0] == "err" else None)


def test_gpu_islands_are_faster_on_the_large_grid():
    M = synth.config3().M
    external.island_boundaries(M, gpu=True, **LIM)  # warm-up (module load)
    t0 = time.perf_counter()
    g = external.island_boundaries(M, gpu=True, **LIM)
    tg = time.perf_counter() - t0
    t0 = time.perf_counter()
    h = external.island_boundaries(M, **LIM)
    th = time.perf_counter() - t0
    assert all(np.array_equal(x, y) for x, y in zip(h, g))
    print(f"2048x1024 island set-up: host {th * 1e3:.1f} ms, GPU {tg * 1e3:.1f} ms")
