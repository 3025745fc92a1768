"""GPU parity: every entry point of libpyomgpu.so against the CPU oracle on
the same seeded inputs.  Floating-point tolerances are stated per test; the
integer island set-up must match bit for bit.

Tolerances.  The GPU solvers run the reference algorithm in FP64 but sum the
dot products in a different order (tree reduction) and apply the operator in
face-coupling form, so iterates differ from the oracle at rounding level.
A converged solution is required to match the oracle's to 1e-10 relative
(the parity bar of this path); iteration counts may differ by one when a
stopping test sits on its threshold.
"""
import numpy as np
import pytest

from pyom2_b200 import _abi, external, synth
from pyom2_b200.external import ExternalMode

pytestmark = pytest.mark.gpu

RTOL_SOL = 1e-10


def rel(a, b, mask=None):
    a = np.asarray(a)
    b = np.asarray(b)
    if mask is not None:
        a, b = a[mask], b[mask]
    d = np.linalg.norm(a - b)
    n = np.linalg.norm(b)
    return d / n if n > 0 else d


def small_cyclic(seed=13, nx=96, ny=48, masses=6):
    return synth._global_like(nx, ny, -80.0, 80.0, seed, n_land_masses=masses, mask_sigma=4.0, depth_sigma=4.0,
                              name="small")


WORLDS = {
    "c0": lambda: synth.config0(),
    "cyclic96": lambda: small_cyclic(),
    "cyclic200": lambda: small_cyclic(seed=9, nx=200, ny=100, masses=10),
}


def setup(name, oracle_lib, limits=dict(maxipp=10**6, maxq=10**6)):
    W = WORLDS[name]()
    Mg = W.M
    Mo = W.M.copy()
    O = oracle_lib.Oracle(Mo)
    O.streamfunction_init(**limits)
    E = ExternalMode(Mg)
    it = E.streamfunction_init(**limits)
    return W, Mg, Mo, O, E, it


@pytest.mark.parametrize("name", list(WORLDS))
def test_streamfunction_init(oracle_lib, name):
    W, Mg, Mo, O, E, it = setup(name, oracle_lib)
    assert Mg.nisle == Mo.nisle
    assert np.array_equal(Mg.boundary, Mo.boundary)
    assert np.array_equal(Mg.line_dir, Mo.line_dir)
    assert np.array_equal(Mg.nr_boundary, Mo.nr_boundary)
    assert Mg.nisle >= 2
    for k in range(Mg.nisle):
        assert rel(Mg.psin[:, :, k], Mo.psin[:, :, k]) < 1e-9, k
    # line_psin holds circulations around each island; entries that cancel to
    # rounding level are compared against the matrix scale
    scale = np.abs(Mo.line_psin).max()
    assert np.abs(Mg.line_psin - Mo.line_psin).max() <= 1e-8 * scale


@pytest.mark.parametrize("name", list(WORLDS))
def test_congrad_streamfunction(oracle_lib, name):
    W, Mg, Mo, O, E, _ = setup(name, oracle_lib)
    cf = O.make_coeff_streamfunction()
    rng = np.random.default_rng(1)
    sol0 = np.asfortranarray(rng.standard_normal(Mg.shape2d) * 1e3)
    so = sol0.copy(order="F")
    ro = O.congrad_streamfunction(cf, W.forc, so)
    sg = sol0.copy(order="F")
    it, conv, info = E.congrad_streamfunction(W.forc, sg)
    assert conv == ro["converged"]
    assert abs(it - ro["iterations"]) <= 1
    assert rel(sg, so) < RTOL_SOL
    # the halo is left as the reference leaves it (set once at entry)
    assert np.array_equal(sg[:2], so[:2]) or rel(sg[:2], so[:2]) < RTOL_SOL


def test_autotuned_kernel_matches_oracle(oracle_lib):
    """After the autotuner picks a tile shape and grid, congrad_streamfunction
    still follows the oracle (solution to 1e-10, iterations within one) and
    solve_rtol still reaches the 1e-10 true residual."""
    W, Mg, Mo, O, E, _ = setup("cyclic200", oracle_lib)
    tx, ty, grid, us = E.autotune(iterations=50)
    assert tx in (32, 64, 96, 128) and ty in (8, 16, 24, 32) and grid >= 1 and us > 0
    cf = O.make_coeff_streamfunction()
    rng = np.random.default_rng(2)
    sol0 = np.asfortranarray(rng.standard_normal(Mg.shape2d) * 1e3)
    so = sol0.copy(order="F")
    ro = O.congrad_streamfunction(cf, W.forc, so)
    sg = sol0.copy(order="F")
    it, conv, info = E.congrad_streamfunction(W.forc, sg)
    assert conv == ro["converged"] and abs(it - ro["iterations"]) <= 1
    assert rel(sg, so) < RTOL_SOL
    s2 = np.zeros(Mg.shape2d, order="F")
    info = E.solve_rtol(W.forc, s2, rtol=1e-10, precision=_abi.PREC_F64)
    assert info["status"] == 0 and info["rel_residual"] <= 1e-10


def test_congrad_torch_in_place(oracle_lib):
    import torch
    W, Mg, Mo, O, E, _ = setup("cyclic96", oracle_lib)
    s_np = np.zeros(Mg.shape2d, order="F")
    E.congrad_streamfunction(W.forc, s_np)
    f_t = torch.from_numpy(np.ascontiguousarray(W.forc.T)).cuda().T
    s_t = torch.zeros(tuple(reversed(Mg.shape2d)), dtype=torch.float64, device="cuda").T
    E.congrad_streamfunction(f_t, s_t)
    assert np.array_equal(s_t.cpu().numpy(), s_np)


@pytest.mark.parametrize("name", ["c0", "cyclic96"])
@pytest.mark.parametrize("free_surface", [False, True])
def test_congrad_surf_press(oracle_lib, name, free_surface):
    W = WORLDS[name]()
    M = W.M
    M.enable_free_surface = free_surface
    M.dt_mom = 1800.0
    O = oracle_lib.Oracle(M)
    cf = O.make_coeff_surf_press()
    E = ExternalMode(M)
    rng = np.random.default_rng(2)
    forc = np.asfortranarray(rng.standard_normal(M.shape2d) * M.maskT[:, :, -1] * 1e-9)
    forc[:2] = forc[-2:] = 0
    forc[:, :2] = forc[:, -2:] = 0
    m = M.maskT[:, :, -1] > 0
    if not free_surface:
        # Neumann problem: A = D^-1 S with D the T-cell area, so a solvable
        # right-hand side has zero area-weighted mean
        area = M.dxt[:, None] * M.dyt[None, :] * M.cost[None, :]
        forc[m] -= (area * forc)[m].sum() / area[m].sum()
    psi0 = np.asfortranarray(rng.standard_normal(M.shape2d))
    po = psi0.copy(order="F")
    ro = O.congrad_surf_press(cf, forc, po)
    pg = psi0.copy(order="F")
    it, info = E.congrad_surf_press(forc, pg)
    assert abs(it - ro["iterations"]) <= 1
    assert info["status"] == ro["status"]
    if free_surface:
        assert rel(pg, po) < RTOL_SOL
    else:
        # The singular problem cannot reach the absolute step 1e-12 on a psi of
        # O(1e2): both solvers stagnate in rounding noise and stop on the
        # divergence test (checked above).  Compare the iterates before the
        # stagnation, modulo the constant null vector.
        po = psi0.copy(order="F")
        O.congrad_surf_press(cf, forc, po, max_it=300)
        pg = psi0.copy(order="F")
        E.congrad_surf_press(forc, pg, max_it=300)
        dg = pg[m] - pg[m].mean()
        do = po[m] - po[m].mean()
        assert np.linalg.norm(dg - do) / np.linalg.norm(do) < RTOL_SOL


@pytest.mark.parametrize("name", list(WORLDS))
def test_apply_op_and_inverse(oracle_lib, name):
    W = WORLDS[name]()
    M = W.M
    O = oracle_lib.Oracle(M)
    E = ExternalMode(M)
    cf = O.make_coeff_streamfunction()
    rng = np.random.default_rng(3)
    p = np.asfortranarray(rng.standard_normal(M.shape2d))
    ro = O.apply_op(cf, p)
    rg = E.apply_op(p)
    scale = np.abs(cf).max() * np.abs(p).max()
    assert np.abs(rg - ro).max() <= 1e-14 * scale
    Zo = O.make_inv_sfc(cf)
    Zg = E.make_inv_sfc()
    assert np.array_equal(Zo == 0, Zg == 0)
    assert rel(Zg, Zo) < 1e-14
    M.enable_free_surface = True
    cfs = O.make_coeff_surf_press()
    E2 = ExternalMode(M)
    assert np.abs(E2.apply_op(p, "surf_press") - O.apply_op(cfs, p)).max() <= 1e-14 * np.abs(cfs).max() * 4


@pytest.mark.parametrize("name", list(WORLDS))
def test_line_integral(oracle_lib, name):
    W, Mg, Mo, O, E, _ = setup(name, oracle_lib)
    for k in range(1, Mg.nisle + 1):
        a = E.line_integral(k, W.fpx, W.fpy)
        b = O.line_integral(k, W.fpx, W.fpy)
        assert abs(a - b) <= 1e-12 * max(1e-30, np.abs(W.fpx).max() * 1e6)


def random_state(M, seed):
    rng = np.random.default_rng(seed)
    X, Y = M.shape2d
    nz = M.nz
    M.dt_mom = 1200.0
    for n in ("u", "v", "du", "dv"):
        getattr(M, n)[...] = rng.standard_normal((X, Y, nz, 3)) * 1e-3 * M.maskU[..., None]
    M.rho[...] = (rng.standard_normal((X, Y, nz, 3)) * 0.1 + 1.0) * M.maskT[..., None]
    M.du_mix[...] = rng.standard_normal((X, Y, nz)) * 1e-6 * M.maskU
    M.dv_mix[...] = rng.standard_normal((X, Y, nz)) * 1e-6 * M.maskV
    M.dpsi[...] = rng.standard_normal((X, Y, 3)) * 1e2
    M.psi[...] = rng.standard_normal((X, Y, 3)) * 1e4
    if M.dpsin is not None:
        M.dpsin[...] = rng.standard_normal(M.dpsin.shape) * 10


@pytest.mark.parametrize("name", ["c0", "cyclic96"])
def test_solve_streamfunction_step(oracle_lib, name):
    W, Mg, Mo, O, E, _ = setup(name, oracle_lib)
    random_state(Mg, 4)
    random_state(Mo, 4)
    for step in range(2):
        rc = O.solve_streamfunction(Mo)
        assert rc in (0, 1, 2)
        E.solve_streamfunction(Mg)
        assert abs(Mg.congr_itts - Mo.congr_itts) <= 1
        for n in ("dpsi", "psi", "u", "v", "du", "dv", "p_hydro", "dpsin"):
            assert rel(getattr(Mg, n), getattr(Mo, n)) < 1e-9, (step, n)
        for M in (Mg, Mo):
            M.taum1, M.tau, M.taup1 = M.tau, M.taup1, M.taum1


@pytest.mark.parametrize("name", ["c0", "cyclic96"])
@pytest.mark.parametrize("free_surface", [False, True])
def test_solve_pressure_step(oracle_lib, name, free_surface):
    W = WORLDS[name]()
    Mg = W.M
    Mg.enable_free_surface = free_surface
    random_state(Mg, 5)
    Mo = Mg.copy()
    O = oracle_lib.Oracle(Mo)
    E = ExternalMode(Mg)
    m = Mg.maskT[:, :, -1] > 0
    if not free_surface:  # stop the singular problem before it stagnates in rounding noise
        Mg.congr_max_iterations = Mo.congr_max_iterations = 300
    for step in range(2 if free_surface else 1):
        O.solve_pressure(Mo)
        E.solve_pressure(Mg)
        assert abs(Mg.congr_itts - Mo.congr_itts) <= 1
        if free_surface:
            assert rel(Mg.psi, Mo.psi) < 1e-9, step
        else:  # psi is defined up to a constant; the velocities are not
            pg = Mg.psi[:, :, Mg.taup1 - 1][m]
            po = Mo.psi[:, :, Mo.taup1 - 1][m]
            assert np.linalg.norm((pg - pg.mean()) - (po - po.mean())) / np.linalg.norm(po - po.mean()) < 1e-7
        # velocities take the gradient of psi; for the singular problem the
        # rounding-level psi differences after 300 iterations reach ~1e-9 there
        tol = 1e-9 if free_surface else 1e-8
        for n in ("u", "v", "du", "dv", "p_hydro"):
            assert rel(getattr(Mg, n), getattr(Mo, n)) < tol, (step, n)
        for M in (Mg, Mo):
            M.taum1, M.tau, M.taup1 = M.tau, M.taup1, M.taum1


@pytest.mark.parametrize("name", list(WORLDS))
@pytest.mark.parametrize("precision", [_abi.PREC_F64, _abi.PREC_F32])
def test_solve_rtol_reaches_1e10(oracle_lib, name, precision):
    """Solved to the residual the benchmark uses (2e-11, which on these
    operators leaves a solution error below 1e-10), the solution matches the
    oracle's tight (1e-14) solution to 1e-10 relative."""
    W, Mg, Mo, O, E, _ = setup(name, oracle_lib)
    sol = np.zeros(Mg.shape2d, order="F")
    info = E.solve_rtol(W.forc, sol, rtol=2e-11, precision=precision)
    assert info["status"] == 0 and info["rel_residual"] <= 2e-11, info
    cf = O.make_coeff_streamfunction()
    Z = O.make_inv_sfc(cf)
    assert O.rel_residual(cf, Z, W.forc, sol) <= 3e-11
    so = np.zeros(Mg.shape2d, order="F")
    O.congrad_streamfunction(cf, W.forc, so, eps=0.0, max_it=100000, rtol=1e-14)
    O.setcyclic_xy(so)
    assert rel(sol, so, Z != 0) < 1e-10


def test_status_nan_maxiter_timeout(oracle_lib):
    W, Mg, Mo, O, E, _ = setup("c0", oracle_lib)
    bad = W.forc.copy(order="F")
    bad[10, 10] = np.nan
    with pytest.raises(_abi.PyOMGPUError) as e:
        E.congrad_streamfunction(bad, np.zeros(Mg.shape2d, order="F"))
    assert e.value.code == _abi.NAN
    with pytest.warns(RuntimeWarning):
        it, conv, info = E.congrad_streamfunction(W.forc, np.zeros(Mg.shape2d, order="F"), max_it=3)
    assert it == 4 and not conv and info["status"] == _abi.MAXITER
    ro = O.congrad_streamfunction(O.make_coeff_streamfunction(), W.forc, np.zeros(Mg.shape2d, order="F"), max_it=3)
    assert ro["iterations"] == 4 and ro["status"] == 1
    E.set_sync_timeout(1e-3)
    E.inject_barrier_stall(True)
    with pytest.raises(_abi.PyOMGPUError) as e:
        E.congrad_streamfunction(W.forc, np.zeros(Mg.shape2d, order="F"))
    assert e.value.code == _abi.TIMEOUT
    E.set_sync_timeout(2.0)
    s = np.zeros(Mg.shape2d, order="F")
    it, conv, _ = E.congrad_streamfunction(W.forc, s)  # the context is still usable
    assert conv and it > 10
