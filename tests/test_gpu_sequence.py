"""Config 4 on the GPU: consecutive solve_streamfunction steps of an ensemble
of re-entrant channel runs (pyom2_b200/sequence.py) against the oracle's
solve_streamfunction on the same synthetic tendency sequence, and the
alternative solvers (one batched launch for all members, FP64 and mixed
FP32/FP64 PCG, learned FCG) against each other."""
import warnings

import numpy as np
import pytest

from pyom2_b200 import synth
from pyom2_b200.sequence import ChannelEnsemble, TendencySequence

pytestmark = pytest.mark.gpu
LIMITS = dict(maxipp=10**6, maxq=10**6)


def small_channel(seed=1004):
    # the config-4 channel (same extent and cell aspect) on a coarser grid, so that the oracle runs in seconds
    return synth.config4(seed, nx=96, ny=96, nz=8)


def test_sequence_matches_oracle(oracle_lib):
    W = small_channel()
    M = W.M
    members, steps = 2, 3
    ens = ChannelEnsemble(W, members=members, seed=1004)
    seq = TendencySequence(M, members, 1004 + 7)  # the same inputs, generated on the host
    Mo = [M.copy() for _ in range(members)]
    Os = [oracle_lib.Oracle(m) for m in Mo]
    for m, O in enumerate(Os):
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)
            O.streamfunction_init(**LIMITS)
    cf = Os[0].make_coeff_streamfunction()
    for step in range(steps):
        seq.advance()
        inputs = [seq.host_fields(m) for m in range(members)]
        infos = ens.step("ref", host_inputs=inputs)
        for m in range(members):
            Mm = Mo[m]
            du, dv, rho = inputs[m]
            Mm.du[..., Mm.tau - 1] = du
            Mm.dv[..., Mm.tau - 1] = dv
            Mm.rho[..., Mm.tau - 1] = rho
            assert Os[m].solve_streamfunction(Mm, cf) == 0
            assert abs(infos[m]["iterations"] - Mm.congr_itts) <= 1, (step, m, infos[m]["iterations"], Mm.congr_itts)
            Mm.taum1, Mm.tau, Mm.taup1 = Mm.tau, Mm.taup1, Mm.taum1
    for m in range(members):
        g = ens.host_state(m)
        for n in ("psi", "dpsi", "u", "v"):
            a, b = g[n], getattr(Mo[m], n)
            assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), (m, n)
        assert np.allclose(g["dpsin"], Mo[m].dpsin, rtol=1e-9, atol=0), m
    ens.close()


def test_solvers_agree_on_the_sequence():
    """Every solver reaches the FP64 true residual 1e-10 at every step, warm
    started from the reference's first guess; after a few steps their psi
    agree to 1e-8."""
    W = small_channel(1005)
    res = {}
    for method in ("batch", "pcg64", "mixed32", "fcg"):
        ens = ChannelEnsemble(W, members=3, seed=1005)
        for step in range(4):
            infos = ens.step(method, rtol=1e-10)
            assert all(i["status"] == 0 for i in infos), (method, step, infos)
            assert all(i["rel_residual"] <= 1e-10 for i in infos), (method, step)
        res[method] = [ens.host_state(m)["psi"] for m in range(3)]
        ens.close()
    for method in ("pcg64", "mixed32", "fcg"):
        for m in range(3):
            a, b = res[method][m], res["batch"][m]
            assert np.abs(a - b).max() <= 1e-8 * np.abs(b).max(), (method, m)


def test_batched_reference_stop_matches_sequential():
    """All members in one work-queue launch with the reference's own stop
    (congr_epsilon): the same states as the per-member congrad path."""
    W = small_channel(1006)
    out = {}
    for method in ("ref", "batch_ref"):
        ens = ChannelEnsemble(W, members=3, seed=1006)
        its = []
        for step in range(3):
            infos = ens.step(method)
            its.append([i["iterations"] for i in infos])
        out[method] = ([ens.host_state(m) for m in range(3)], its)
        ens.close()
    for step_its_a, step_its_b in zip(out["ref"][1], out["batch_ref"][1]):
        assert all(abs(a - b) <= 1 for a, b in zip(step_its_a, step_its_b))
    for m in range(3):
        for n in ("psi", "dpsi", "u"):
            a, b = out["batch_ref"][0][m][n], out["ref"][0][m][n]
            assert np.abs(a - b).max() <= 1e-9 * np.abs(b).max(), (m, n)
