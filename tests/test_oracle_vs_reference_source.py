"""The oracle against golden vectors computed by the reference's own Fortran
source (tests/golden/make_ref_golden.py runs pyOM2's routines through the
Fortran-subset translator oracle/f90sub.py; no Fortran compiler exists in
this image).  This is what pins the oracle -- and through it every GPU
parity test -- to the reference.

Expected agreement: bit for bit.  The oracle (oracle/pyom_oracle.c, built
without FMA contraction) and the synthetic-input generator (pyom2_b200/
synth.py's calc_grid / calc_topo) follow the reference's operation order, so
grid metrics, masks, island lists, psin, line_psin, the CG iterates and
iteration counts, and whole time steps of solve_streamfunction and
solve_pressure must be identical, and are.  The one third-party routine,
LAPACK's DGESV, is scipy's LAPACK in the fixtures and the oracle's own LU with
partial pivoting in the oracle: for the 4x4 island system of the second
cyclic96 step the island values dpsin differ by rounding (held to 1e-12
relative), and psi, u, v, which take them in, to 1e-13.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from ref_cases import CASES, GRID_OUT, MOMENTUM_CASE, NH_CASES, PRESSURE, STEP_OUT_3D, digest, random_state  # noqa: E402

LIMITS = dict(maxipp=10**6, maxq=10**6)


def fixture(name):
    return np.load(os.path.join(HERE, "golden", f"ref_f90_{name}.npz"))


def same(g, key, a, rtol=0.0):
    """a equals the reference's array stored under key (whole, or digest +
    norm when large); rtol > 0 allows a relative difference."""
    a = np.asarray(a)
    if key in g:
        b = g[key]
        assert a.shape == b.shape, (key, a.shape, b.shape)
        if rtol == 0.0:
            assert np.array_equal(a, b), (key, float(np.abs(a - b).max()))
        else:
            d = np.linalg.norm((a - b).astype(np.float64))
            assert d <= rtol * max(np.linalg.norm(b.astype(np.float64)), 1e-300), (key, d)
        return
    if rtol == 0.0:
        assert digest(a) == str(g[key + "__digest"]), (key, float(np.linalg.norm(a)), float(g[key + "__norm"]))
    else:
        n = float(g[key + "__norm"])
        assert abs(np.linalg.norm(a.astype(np.float64)) - n) <= rtol * n, key
        s = g[key + "__sample"]
        flat = a.reshape(-1, order="F")[:: max(1, a.size // 500)]
        assert np.linalg.norm(flat - s) <= rtol * max(np.linalg.norm(s), 1e-300), key


@pytest.mark.parametrize("name", list(CASES))
def test_inputs_and_grid_match_reference(name):
    """synth's restatement of calc_grid / calc_topo gives the reference's
    grid metrics, depths and masks bit for bit; the seeded inputs are the
    ones the fixture was made from."""
    g = fixture(name)
    W = CASES[name]()
    assert digest(W.forc) == str(g["forc__digest"])
    assert digest(W.M.kbot) == str(g["kbot__digest"])
    for n in GRID_OUT:
        same(g, "grid_" + n, getattr(W.M, n))


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_streamfunction_init_matches_reference(oracle_lib, name):
    g = fixture(name)
    W = CASES[name]()
    M = W.M
    O = oracle_lib.Oracle(M)
    O.streamfunction_init(**LIMITS)
    assert M.nisle == int(g["nisle"])
    nb = M.boundary.shape[1]
    # the reference sizes its lists 20 x the largest perimeter; the oracle keeps the same
    same(g, "boundary", M.boundary)
    same(g, "line_dir", M.line_dir)
    same(g, "nr_boundary", M.nr_boundary)
    same(g, "psin", M.psin)
    same(g, "line_psin", M.line_psin)
    assert nb == g["boundary"].shape[1] if "boundary" in g else True


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_congrad_matches_reference(oracle_lib, name):
    g = fixture(name)
    W = CASES[name]()
    M = W.M
    O = oracle_lib.Oracle(M)
    O.streamfunction_init(**LIMITS)
    cf = O.make_coeff_streamfunction()
    sol = np.zeros(M.shape2d, order="F")
    r = O.congrad_streamfunction(cf, W.forc, sol)
    assert r["iterations"] == int(g["sol_iterations"]) and r["converged"] == bool(g["sol_converged"])
    same(g, "sol", sol)


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_solve_streamfunction_steps_match_reference(oracle_lib, name):
    g = fixture(name)
    W = CASES[name]()
    M = W.M
    O = oracle_lib.Oracle(M)
    O.streamfunction_init(**LIMITS)
    random_state(M, 4)
    for step in range(2):
        O.solve_streamfunction(M)
        assert M.congr_itts == int(g[f"step{step}_itts"]), step
        tp1 = M.taup1 - 1
        # dpsin comes from DGESV (the oracle's LU vs the fixture's LAPACK): identical for the
        # 1x1 system of c0 and in the first step of cyclic96, rounding-level apart in its second
        # step, and psi, u, v take it in
        exact = name == "c0" or step == 0
        same(g, f"step{step}_dpsin", M.dpsin, rtol=0.0 if exact else 1e-12)
        same(g, f"step{step}_dpsi", M.dpsi[:, :, tp1])
        same(g, f"step{step}_psi", M.psi[:, :, tp1], rtol=0.0 if exact else 1e-13)
        for n in STEP_OUT_3D:
            same(g, f"step{step}_{n}", getattr(M, n), rtol=0.0 if exact else 1e-13)
        M.taum1, M.tau, M.taup1 = M.tau, M.taup1, M.taum1


@pytest.mark.parametrize("case", PRESSURE, ids=lambda c: f"{c[0]}-{'free' if c[1] else 'rigid'}")
def test_oracle_solve_pressure_matches_reference(oracle_lib, case):
    g = fixture("pressure")
    name, free, max_it = case
    W = CASES[name]()
    M = W.M
    M.enable_free_surface = free
    if max_it is not None:
        M.congr_max_iterations = max_it
    random_state(M, 5)
    O = oracle_lib.Oracle(M)
    O.solve_pressure(M)
    key = f"{name}_{'free' if free else 'rigid'}"
    assert M.congr_itts == int(g[key + "_itts"])
    same(g, key + "_psi", M.psi[:, :, M.taup1 - 1])
    for n in ("u", "v"):
        same(g, f"{key}_{n}", getattr(M, n))


@pytest.mark.parametrize("name", list(NH_CASES))
def test_oracle_non_hydrostatic_matches_reference(oracle_lib, name):
    """congrad_non_hydro from the seeded first guess and one step of
    solve_non_hydrostatic (non_hydrostatic.f90:5-63,146-242): grid and masks,
    iterates and iteration counts, u, v, w and p_non_hydro bit for bit."""
    from pyom2_b200 import synth

    g = fixture("nh")
    W = NH_CASES[name]()
    M = W.M
    for n in GRID_OUT:
        same(g, f"{name}_grid_{n}", getattr(M, n))
    O = oracle_lib.Oracle3D(M)
    cf = O.make_coeff()
    p = W.p0.copy(order="F")
    r = O.congrad(cf, W.forc, p)
    assert r["iterations"] == int(g[f"{name}_cg_iterations"])
    same(g, f"{name}_cg_p", p)
    synth.nonhydro_state(W, 21)
    O.solve_non_hydrostatic(M)
    assert M.congr_itts_non_hydro == int(g[f"{name}_step_itts"])
    for n in ("u", "v", "w", "p_non_hydro"):
        same(g, f"{name}_step_{n}", getattr(M, n))


def test_channel_grid_matches_reference():
    """synth's grid of the momentum case, with the metric term tantr and the
    box areas of calc_grid (numerics.f90:147-167), is the reference's bit for
    bit."""
    g = fixture("momentum")
    W = MOMENTUM_CASE[1]()
    assert digest(W.M.kbot) == str(g["kbot__digest"])
    for n in GRID_OUT + ("tantr", "area_t", "area_u", "area_v"):
        same(g, "grid_" + n, getattr(W.M, n))
