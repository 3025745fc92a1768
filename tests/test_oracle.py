"""Pins the CPU oracle (a C restatement of the reference path) without a
Fortran compiler: manufactured solutions, hand-built island maps, operator
identities, LAPACK known answers and the committed golden fixture."""
import os

import numpy as np
import pytest

from pyom2_b200 import synth
from pyom2_b200.model import CONGR_EPSILON, PI_F, f32

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "c0_oracle.npz")


def small_world(seed=7, nx=96, ny=48, masses=6):
    return synth._global_like(nx, ny, -80.0, 80.0, seed, n_land_masses=masses, mask_sigma=4.0, depth_sigma=4.0,
                              name="small")


def test_fortran_literal_constants():
    # main_module.f90:13,19,52,189 are default-real literals stored in real*8
    assert PI_F == 3.1415927410125732
    assert CONGR_EPSILON == f32(1e-12) and CONGR_EPSILON != 1e-12


def test_operator_row_sums_and_symmetry(oracle_lib):
    W = synth.config0()
    O = oracle_lib.Oracle(W.M)
    cf = O.make_coeff_streamfunction()
    M = W.M
    I = slice(2, M.nx + 2)
    J = slice(2, M.ny + 2)
    rs = cf.sum(axis=(2, 3))[I, J]
    assert np.abs(rs).max() <= 1e-15 * np.abs(cf[I, J, 1, 1]).max()
    # A = D^-1 S with D = dxu dyu cosu and S symmetric (face couplings)
    D = M.dxu[:, None] * M.dyu[None, :] * M.cosu[None, :]
    E = cf[:, :, 2, 1] * D
    Wc = cf[:, :, 0, 1] * D
    N = cf[:, :, 1, 2] * D
    S = cf[:, :, 1, 0] * D
    e = E[2:M.nx + 1, J]
    w = Wc[3:M.nx + 2, J]
    assert np.allclose(e, w, rtol=1e-13, atol=0)
    n = N[I, 2:M.ny + 1]
    s = S[I, 3:M.ny + 2]
    assert np.allclose(n, s, rtol=1e-13, atol=0)


@pytest.mark.parametrize("cyclic", [False, True])
def test_manufactured_solution(oracle_lib, cyclic):
    W = small_world() if cyclic else synth.config0()
    M = W.M
    O = oracle_lib.Oracle(M)
    O.streamfunction_init(max_it=1, maxipp=10**6, maxq=10**6)
    cf = O.make_coeff_streamfunction()
    Z = O.make_inv_sfc(cf)
    rng = np.random.default_rng(5)
    xs = np.asfortranarray(np.where(Z != 0, rng.standard_normal(M.shape2d), 0.0))
    O.setcyclic_xy(xs)
    b = O.apply_op(cf, xs)
    x = np.zeros(M.shape2d, order="F")
    r = O.congrad_streamfunction(cf, b, x, eps=0.0, max_it=20000, rtol=1e-13)
    assert r["converged"]
    O.setcyclic_xy(x)
    err = np.linalg.norm((x - xs)[2:-2, 2:-2]) / np.linalg.norm(xs[2:-2, 2:-2])
    assert err < 1e-7, err
    assert O.rel_residual(cf, Z, b, x) < 1e-12


def test_surf_press_manufactured(oracle_lib):
    W = synth.config0()
    M = W.M
    O = oracle_lib.Oracle(M)
    cf = O.make_coeff_surf_press(free_surface=True, grav=M.grav, dt_mom=3600.0)
    mask = M.maskT[:, :, -1]
    rng = np.random.default_rng(3)
    xs = np.asfortranarray(rng.standard_normal(M.shape2d) * mask)
    xs[:2] = xs[-2:] = 0
    xs[:, :2] = xs[:, -2:] = 0
    b = O.apply_op(cf, xs)
    x = np.zeros(M.shape2d, order="F")
    r = O.congrad_surf_press(cf, b, x, eps=0.0, max_it=5000, rtol=1e-13)
    assert r["converged"]
    err = np.linalg.norm((x - xs) * mask) / np.linalg.norm(xs)
    assert err < 1e-8, err


def test_isleperim_hand_map(oracle_lib):
    # 12 x 9 map (imt x jmt), 1 = land in kmt terms means kmt == 0
    land = np.zeros((12, 9), dtype=bool)
    land[:, 0] = land[:, -1] = True          # southern / northern walls
    land[0, :] = land[-1, :] = True          # western / eastern walls -> one mass with the walls
    land[4:6, 3:5] = True                    # an interior 2x2 island
    land[8, 5] = True                        # a single-cell island
    kmt = np.where(land, 0, 5).astype(np.int32)
    O = oracle_lib.Oracle(synth.config0().M)
    rc, mp, nisle, nippts, nerr = O.isleperim(kmt, cyclic=False)
    assert rc == 0 and nisle == 3
    # masses are numbered in scan order: north row first, then west->east, south
    assert mp[0, 8] == 1                     # the walls
    assert mp[8, 5] == 2                     # first interior mass met scanning down from the north
    assert mp[4, 3] == 3
    # perimeter cells carry -label; ocean not next to land stays 0
    assert mp[7, 4] == -2 and mp[3, 2] == -3 and mp[6, 6] == 0
    assert nippts[1] == 8                    # ring around a single cell
    assert nippts[2] == 12                   # ring around a 2x2 block


def test_isleperim_cyclic_wrap(oracle_lib):
    # an island crossing the periodic seam must be a single mass
    imt, jmt = 14, 8
    land = np.zeros((imt, jmt), dtype=bool)
    land[:, 0] = land[:, -1] = True
    # periodic columns are positions 2..imt-1 (island_module.f90:71-77); land on
    # both sides of the seam must form one mass
    land[[1, imt - 2], 3] = True
    land[0, :] = land[imt - 2, :]
    land[imt - 1, :] = land[1, :]
    kmt = np.where(land, 0, 5).astype(np.int32)
    O = oracle_lib.Oracle(synth.config0().M)
    rc, mp, nisle, nippts, nerr = O.isleperim(kmt, cyclic=True)
    assert rc == 0 and nisle == 3            # north wall, the seam island, south wall
    labs = {int(mp[i, 3]) for i in (1, imt - 2)}
    assert len(labs) == 1 and labs.pop() > 0


def test_trace_of_the_c0_island(oracle_lib):
    W = synth.config0()
    O = oracle_lib.Oracle(W.M)
    O.streamfunction_init(max_it=1)
    M = W.M
    assert M.nisle == 2
    n = M.nr_boundary[1]
    pts = {(int(M.boundary[1, k, 0]), int(M.boundary[1, k, 1])) for k in range(n)}
    ring = {(i, j) for i in range(18, 23) for j in range(18, 23) if i in (18, 22) or j in (18, 22)}
    assert pts == ring and n == 16
    # consecutive points are unit steps along line_dir (boundary(n+1) =
    # boundary(n) + line_dir(n), streamfct_init.f90:230-254) and the walk closes
    for k in range(n):
        a = M.boundary[1, k]
        b = M.boundary[1, (k + 1) % n]
        d = M.line_dir[1, k]
        assert abs(int(a[0]) - int(b[0])) + abs(int(a[1]) - int(b[1])) == 1
        assert tuple(b - a) == tuple(d)


def test_dgesv_known_answers(oracle_lib):
    import scipy.linalg.lapack as lapack
    O = oracle_lib.Oracle(synth.config0().M)
    rng = np.random.default_rng(11)
    for n in (1, 2, 5, 19):
        a = rng.standard_normal((n, n)) + n * np.eye(n) * 0.1
        b = rng.standard_normal(n)
        info, x = O.dgesv(a, b)
        lu, piv, xr, info_r = lapack.dgesv(a, b)
        assert info == 0 and info_r == 0
        assert np.allclose(x, xr, rtol=1e-12, atol=1e-12)
    a = np.array([[1.0, 2.0], [2.0, 4.0]])
    info, _ = O.dgesv(a, np.ones(2))
    assert info == 2


def test_psin_partition_of_unity(oracle_lib):
    W = synth.config0()
    M = W.M
    O = oracle_lib.Oracle(M)
    O.streamfunction_init(eps=1e-20, max_it=5000)
    Z = O.make_inv_sfc(O.make_coeff_streamfunction())
    tot = M.psin.sum(axis=2)
    assert np.abs(tot - 1.0)[Z != 0].max() < 1e-8
    # the velocity of sum(psin) vanishes, so every row of line_psin sums to 0
    assert np.abs(M.line_psin.sum(axis=1)).max() < 1e-8 * np.abs(M.line_psin).max()


def test_golden_fixture(oracle_lib):
    g = np.load(GOLDEN)
    W = synth.config0()
    M = W.M
    assert np.array_equal(W.forc, g["forc"])
    O = oracle_lib.Oracle(M)
    O.streamfunction_init()
    assert np.array_equal(M.boundary, g["boundary"])
    assert np.array_equal(M.line_dir, g["line_dir"])
    assert np.array_equal(M.psin, g["psin"])
    assert np.array_equal(M.line_psin, g["line_psin"])
    cf = O.make_coeff_streamfunction()
    sol = np.zeros(M.shape2d, order="F")
    r = O.congrad_streamfunction(cf, W.forc, sol)
    assert r["iterations"] == int(g["iterations"])
    assert np.array_equal(sol, g["sol"])
