"""Config 4 inputs on the CPU: the channel grid (two land masses, the walls,
so one island unknown) and the seeded tendency sequence (reproducible,
masked, wind stress on the top level only)."""
import numpy as np

from pyom2_b200 import synth
from pyom2_b200.sequence import TAUX, TendencySequence


def test_channel_grid_and_islands(oracle_lib):
    W = synth.config4(1004, nx=64, ny=64, nz=8)
    M = W.M
    assert M.enable_cyclic_x and not M.enable_cyclic_y
    rc, allmap, nisle, maxb = oracle_lib.Oracle(M).island_map(maxipp=10**6, maxq=10**6)
    assert rc == 0 and nisle == 2
    # the ridge: shallower columns near the seeded longitude, full depth away from it
    kb = M.kbot[2:-2, 2]
    assert kb.max() > kb.min() >= 1


def test_tendency_sequence_is_seeded_and_masked():
    W = synth.config4(1004, nx=48, ny=32, nz=6)
    M = W.M
    a, b = TendencySequence(M, 2, 9), TendencySequence(M, 2, 9)
    for _ in range(3):
        a.advance()
        b.advance()
    fa, fb = a.host_fields(1), b.host_fields(1)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)
    du, dv, rho = fa
    assert np.all(du[M.maskU == 0] == 0) and np.all(dv[M.maskV == 0] == 0)
    wind_top = a.wind[:, :, -1]
    assert np.abs(wind_top).max() <= TAUX / M.dzt[-1] * (1 + 1e-12)
    assert not a.wind[:, :, :-1].any()
    # members differ, consecutive steps are close (AR(1) with correlation 0.98)
    assert not np.array_equal(a.host_fields(0)[0], a.host_fields(1)[0])
    prev = a.coef.copy()
    a.advance()
    assert np.linalg.norm(a.coef - prev) < 0.5 * np.linalg.norm(prev)
