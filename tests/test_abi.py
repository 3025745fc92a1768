"""The C ABI library on the CPU: it loads, exports every declared entry
point, and its host-side island code (labelling and perimeter tracing)
agrees bit for bit with the oracle."""
import os
import re

import numpy as np
import pytest

from pyom2_b200 import _abi, external, synth

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "pyomgpu.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(pyomgpu_\w+)\s*\(", txt)))


def test_exports_every_declared_symbol(lib):
    names = declared()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_abi.EXPORTS)
    assert lib.pyomgpu_version() >= 1


def _worlds():
    yield "c0", synth.config0()
    yield "small_cyclic", synth._global_like(96, 48, -80.0, 80.0, 7, n_land_masses=6, mask_sigma=4.0,
                                             depth_sigma=4.0)
    yield "cyclic_b", synth._global_like(128, 64, -70.0, 70.0, 21, n_land_masses=10, mask_sigma=3.0,
                                         depth_sigma=4.0)
    for k, (nx, ny) in enumerate([(40, 32), (64, 48)]):
        yield f"basin{k}", synth.basin(nx, ny, 300 + k, 0.25, 4)


@pytest.mark.parametrize("name,W", list(_worlds()))
def test_isleperim_matches_oracle(lib, oracle_lib, name, W):
    M = W.M
    kmt = np.where(M.kbot > 0, 5, 0).astype(np.int32)
    for cyc in (False, True):
        mp, n, nip = external.isleperim(kmt, cyc, maxipp=10**6, maxq=10**6)
        rc, mp2, n2, nip2, _ = oracle_lib.Oracle(M).isleperim(kmt, cyc, maxipp=10**6, maxq=10**6)
        assert rc == 0 and n == n2
        assert np.array_equal(mp, mp2)
        assert np.array_equal(nip, nip2)


@pytest.mark.parametrize("name,W", list(_worlds()))
def test_island_boundaries_match_oracle(lib, oracle_lib, name, W):
    M = W.M
    b, d, nr = external.island_boundaries(M, maxipp=10**6, maxq=10**6)
    O = oracle_lib.Oracle(M)
    rc, am, nisle, maxb = O.island_map(maxipp=10**6, maxq=10**6)
    assert rc == 0
    rc, b2, d2, nr2 = O.island_trace(am, nisle, maxb, maxipp=10**6, maxq=10**6)
    assert rc == 0
    assert np.array_equal(nr, nr2)
    assert np.array_equal(b, b2)
    assert np.array_equal(d, d2)


def test_island_limits_are_errors(lib):
    W = synth.config0()
    with pytest.raises(_abi.PyOMGPUError) as e:
        external.island_boundaries(W.M, maxipp=10)
    assert e.value.code == _abi.EISLAND
    with pytest.raises(_abi.PyOMGPUError) as e:
        external.island_boundaries(W.M, maxq=8)
    assert e.value.code == _abi.EISLAND


def test_no_gpu_fails_loudly(lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    W = synth.config0()
    with pytest.raises(_abi.PyOMGPUError) as e:
        external.ExternalMode(W.M)
    assert e.value.code in (_abi.ECUDA, _abi.ENOMEM)
