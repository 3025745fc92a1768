"""The momentum tendencies on the GPU (pyomgpu_momentum_tendencies,
pyomgpu_vertical_velocity) against the reference's own momentum routine run
through the Fortran-subset translator (tests/golden/make_ref_golden.py,
fixture ref_f90_momentum.npz): a 32 x 24 x 6 re-entrant channel with the
reference channel set-up's friction (harmonic with cos scaling, linear
bottom, implicit vertical with a seeded viscosity), one call of momentum
(momentum.f90:4-168), which ends with solve_streamfunction.

The tendency kernels evaluate the reference's expressions in its order
without FMA contraction, so w, du, dv, du_mix and dv_mix must equal the
reference's bit for bit on the interior points (the reference also writes
some halo points of du_mix, which the step never reads there).  The solve
that follows runs the GPU's CG (other reduction order): its iteration count
within one and psi, dpsi, u, v within 1e-9 relative, as the other step
tests.
"""
import os
import sys
import warnings

import numpy as np
import pytest

from pyom2_b200.external import ExternalMode

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
from ref_cases import MOMENTUM_CASE, MOMENTUM_OUT_3D, momentum_state  # noqa: E402

IN = (slice(2, -2), slice(2, -2))


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_momentum_matches_reference_source():
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_f90_momentum.npz"))
    W = MOMENTUM_CASE[1]()
    M = W.M
    momentum_state(M, 31)
    E = ExternalMode(M)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(maxipp=10**6, maxq=10**6)
    tau, tp1 = M.tau - 1, M.taup1 - 1
    E.vertical_velocity(M, level=M.tau)
    w = M.w[:, :, :, tau]
    assert np.array_equal(w[1:, 1:], g["w_tau"][1:, 1:]), float(np.abs(w[1:, 1:] - g["w_tau"][1:, 1:]).max())
    E.momentum(M)
    for n in MOMENTUM_OUT_3D:
        a = getattr(M, n)
        a = a[:, :, :, tau] if a.ndim == 4 else a
        b = g[n]
        assert np.array_equal(a[IN], b[IN]), (n, float(np.abs(a[IN] - b[IN]).max()), float(np.abs(b[IN]).max()))
    info = E.solve_streamfunction(M)
    assert abs(M.congr_itts - int(g["itts"])) <= 1, (M.congr_itts, int(g["itts"]))
    for n in ("psi", "dpsi"):
        assert rel(getattr(M, n)[:, :, tp1][IN], g[n][IN]) < 1e-9, n
    for n in ("u", "v"):
        assert rel(getattr(M, n)[:, :, :, tp1][IN], g[n + "_taup1"][IN]) < 1e-9, n
    E.close()


def test_ensemble_with_momentum_physics_matches_the_host_path():
    """Two steps of a member of the channel ensemble (device tensors, the
    model's own tendencies, the reference's stop) equal the same steps run
    through ExternalMode on host arrays: momentum, solve_streamfunction, the
    cyclic halos and vertical_velocity of the new level."""
    from pyom2_b200 import synth
    from pyom2_b200.sequence import ChannelEnsemble, channel_physics

    W = synth.config4(1004, nx=48, ny=32, nz=6)
    ens = ChannelEnsemble(W, members=2, seed=1004)
    M = W.M.copy()
    channel_physics(M)
    rho = ens.seq.host_fields(1)[2]
    for lev in range(3):
        M.rho[..., lev] = rho
    E = ExternalMode(M)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(maxipp=10**6, maxq=10**6)
    for step in range(2):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            ens.step("ref")
            E.momentum(M)
            E.solve_streamfunction(M)
        E.vertical_velocity(M, level=M.taup1)
        M.taum1, M.tau, M.taup1 = M.tau, M.taup1, M.taum1
        h = ens.host_state(1, names=("u", "v", "w", "psi", "dpsi"))
        for n in ("u", "v", "w", "psi", "dpsi"):
            assert np.array_equal(h[n], getattr(M, n)), (step, n, float(np.abs(h[n] - getattr(M, n)).max()))
    assert np.abs(M.u).max() > 0
    ens.close()
    E.close()
