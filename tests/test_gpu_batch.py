"""GPU parity of the batch (pyomgpu_congrad_streamfunction_batch): many
congrad_streamfunction solves in one call, each checked against a separate
oracle solve on the same inputs (solve_streamfct.f90:153-327), on both
engines: the work-queue kernel ("queue") and groups of SMs running resident
solves side by side ("resident").

Tolerances as in test_gpu_parity: solutions to 1e-10 relative, iteration
counts within one (dot products are summed in another order).
"""
import ctypes as C
import warnings

import numpy as np
import pytest

from pyom2_b200 import _abi, external, synth
from pyom2_b200.external import ExternalMode

pytestmark = pytest.mark.gpu

RTOL_SOL = 1e-10
LIMITS = dict(maxipp=10**6, maxq=10**6)


def rel(a, b, mask=None):
    a, b = np.asarray(a), np.asarray(b)
    if mask is not None:
        a, b = a[mask], b[mask]
    n = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return d / n if n > 0 else d


def worlds():
    return [
        synth.config0(),
        synth._global_like(96, 48, -80.0, 80.0, 13, n_land_masses=6, mask_sigma=4.0, depth_sigma=4.0, name="cyc96"),
        synth.basin(72, 40, 5, 0.2, 3),
        synth.basin(50, 90, 6, 0.35, 6),
        synth.basin(130, 64, 7, 0.15, 2),
    ]


@pytest.fixture(scope="module")
def batch_set(oracle_lib):
    out = []
    for W in worlds():
        Mo = W.M.copy()
        O = oracle_lib.Oracle(Mo)
        ro = O.streamfunction_init(**LIMITS)
        E = ExternalMode(W.M)
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)  # one psin solve of cyc96 reaches max_it in both
            it = E.streamfunction_init(**LIMITS)
        assert W.M.nisle == Mo.nisle
        # the psin solves of streamfunction_init run through the batch kernel
        assert np.abs(it - ro["psin_iterations"]).max() <= 1, (W.name, it, ro["psin_iterations"])
        for k in range(W.M.nisle):
            assert rel(W.M.psin[:, :, k], Mo.psin[:, :, k]) < 1e-9, (W.name, k)
        out.append((W, O, E))
    return out


def entries(batch_set, seed=3):
    """Solve list: every world once with its own forcing and a random first
    guess, the first two worlds a second time with another forcing."""
    rng = np.random.default_rng(seed)
    ents = []
    for W, O, E in batch_set:
        ents.append((W, O, E, W.forc, np.asfortranarray(rng.standard_normal(W.M.shape2d) * 1e3)))
    for W, O, E in batch_set[:2]:
        f2 = np.asfortranarray(W.forc * rng.uniform(0.5, 2.0) + np.roll(W.forc, 3, axis=1))
        ents.append((W, O, E, f2, np.zeros(W.M.shape2d, order="F")))
    return ents


ENGINES = ["queue", "resident"]


@pytest.mark.parametrize("engine", ENGINES)
def test_batch_matches_separate_oracle_solves(batch_set, engine):
    ents = entries(batch_set)
    sols = [s0.copy(order="F") for *_, s0 in ents]
    infos = external.congrad_streamfunction_batch([e[2] for e in ents], [e[3] for e in ents], sols, kernel=engine)
    for (W, O, E, f, s0), sg, info in zip(ents, sols, infos):
        cf = O.make_coeff_streamfunction()
        so = s0.copy(order="F")
        ro = O.congrad_streamfunction(cf, f, so)
        assert info["status"] == ro["status"] and bool(info["converged"]) == bool(ro["converged"]), (W.name, info, ro)
        assert abs(info["iterations"] - ro["iterations"]) <= 1, (W.name, info, ro)
        assert rel(sg, so) < RTOL_SOL, W.name


@pytest.mark.parametrize("engine", ENGINES)
def test_batch_equals_single_call_statistics(batch_set, engine):
    """The batch gives each solve the iteration count of a separate GPU call."""
    ents = entries(batch_set, seed=4)
    sols = [s0.copy(order="F") for *_, s0 in ents]
    infos = external.congrad_streamfunction_batch([e[2] for e in ents], [e[3] for e in ents], sols, kernel=engine)
    for (W, O, E, f, s0), sb, ib in zip(ents, sols, infos):
        s1 = s0.copy(order="F")
        it, conv, i1 = E.congrad_streamfunction(f, s1)
        assert abs(ib["iterations"] - it) <= 1 and bool(ib["converged"]) == conv
        assert rel(sb, s1) < RTOL_SOL


@pytest.mark.parametrize("engine", ENGINES)
def test_batch_rtol_and_torch(batch_set, engine):
    import torch
    ents = entries(batch_set, seed=5)
    sols = [np.zeros(W.M.shape2d, order="F") for W, *_ in ents]
    infos = external.congrad_streamfunction_batch([e[2] for e in ents], [e[3] for e in ents], sols, eps=0.0,
                                                  rtol=1e-10, kernel=engine)
    for (W, O, E, f, _), s, info in zip(ents, sols, infos):
        assert info["status"] == 0 and info["rel_residual"] <= 1e-10, (W.name, info)
        cf = O.make_coeff_streamfunction()
        assert O.rel_residual(cf, O.make_inv_sfc(cf), f, s) <= 1.5e-10
    # device tensors give the same bits as host arrays
    dev = [torch.zeros(tuple(reversed(W.M.shape2d)), dtype=torch.float64, device="cuda").T for W, *_ in ents]
    fdev = [torch.from_numpy(np.ascontiguousarray(f.T)).cuda().T for *_, f, _ in ents]
    external.congrad_streamfunction_batch([e[2] for e in ents], fdev, dev, eps=0.0, rtol=1e-10)
    for d, s in zip(dev, sols):
        assert np.array_equal(d.cpu().numpy(), s)
    torch.cuda.synchronize()


@pytest.mark.parametrize("engine", ENGINES)
def test_batch_statuses_are_per_solve(batch_set, engine):
    """A NaN forcing stops its own solve with status NaN; the others converge."""
    ents = entries(batch_set, seed=6)[:4]
    _abi.check(_abi.load().pyomgpu_set_batch_kernel(ents[0][2]._ctx, external._BATCH_KERNELS[engine]))
    bad = ents[1][3].copy(order="F")
    bad[10, 10] = np.nan
    forcs = [e[3] for e in ents]
    forcs[1] = bad
    sols = [e[4].copy(order="F") for e in ents]
    L = _abi.load()
    n = len(ents)
    VP = C.c_void_p * n
    infos = (_abi.SolveInfo * n)()
    rc = L.pyomgpu_congrad_streamfunction_batch(VP(*[e[2]._ctx for e in ents]), n,
                                                VP(*[f.ctypes.data for f in forcs]),
                                                VP(*[s.ctypes.data for s in sols]), 1e-12, 100000, 0.0, infos, None)
    assert rc == _abi.NAN
    assert infos[1].status == _abi.NAN and not infos[1].converged
    for k in (0, 2, 3):
        assert infos[k].status == _abi.OK and infos[k].converged
    # max_it reached by every solve: iterations = max_it + 1, status MAXITER (solve_streamfct.f90:303)
    sols = [e[4].copy(order="F") for e in ents]
    with pytest.warns(RuntimeWarning):
        infos = external.congrad_streamfunction_batch([e[2] for e in ents], [e[3] for e in ents], sols, max_it=5)
    assert all(i["status"] == _abi.MAXITER and i["iterations"] == 6 for i in infos)


@pytest.mark.parametrize("engine", ENGINES)
def test_batch_timeout_then_usable(batch_set, engine):
    """The stall hook makes the first barrier (queue) or the first reduction
    of every solve (resident) await one block more than there are, so every
    wait runs into its time limit: the call ends with PYOMGPU_TIMEOUT and the
    context stays usable."""
    W, O, E = batch_set[1]
    E.set_sync_timeout(1e-3)
    E.inject_barrier_stall(True)
    f = [W.forc] * 8
    sols = [np.zeros(W.M.shape2d, order="F") for _ in f]
    try:
        with pytest.raises(_abi.PyOMGPUError) as e:
            external.congrad_streamfunction_batch([E] * 8, f, sols, kernel=engine)
        assert e.value.code == _abi.TIMEOUT
    finally:
        E.set_sync_timeout(2.0)
    sols = [np.zeros(W.M.shape2d, order="F") for _ in f]
    infos = external.congrad_streamfunction_batch([E] * 8, f, sols, kernel=engine)
    assert all(i["converged"] for i in infos)
    for s in sols[1:]:
        assert np.array_equal(s, sols[0])


def test_batch_with_a_grid_beyond_the_resident_engine(batch_set):
    """A batch holding a grid too large for the on-chip engine (2100 x 1000,
    no islands): the resident engine refuses it with EINVAL, the automatic
    engine runs the whole batch on the work-queue kernel, and every solve
    reaches the residual."""
    big = synth.basin(2100, 1000, 911, 0.2, 0, nz=4)
    Eb = ExternalMode(big.M)
    Eb.streamfunction_init(**LIMITS)
    assert Eb.resident_layout() is None
    W, O, E = batch_set[2]
    ems, forcs = [Eb, E], [big.forc, W.forc]
    sols = [np.zeros(big.M.shape2d, order="F"), np.zeros(W.M.shape2d, order="F")]
    with pytest.raises(_abi.PyOMGPUError) as e:
        external.congrad_streamfunction_batch(ems, forcs, sols, eps=0.0, rtol=1e-10, kernel="resident")
    assert e.value.code == _abi.EINVAL
    sols = [np.zeros(big.M.shape2d, order="F"), np.zeros(W.M.shape2d, order="F")]
    infos = external.congrad_streamfunction_batch(ems, forcs, sols, eps=0.0, rtol=1e-10, kernel="auto")
    assert all(i["status"] == 0 and i["rel_residual"] <= 1e-10 for i in infos), infos
    cf = O.make_coeff_streamfunction()
    assert O.rel_residual(cf, O.make_inv_sfc(cf), W.forc, sols[1]) <= 1.5e-10
    Eb.close()
