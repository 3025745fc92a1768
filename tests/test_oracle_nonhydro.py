"""Known-answer checks that pin the CPU oracle of the non-hydrostatic pressure
solve (oracle/pyom_oracle.c: o_make_coeff_non_hydro, o_apply_op_3d, o_dot_3d,
o_absmax_3d, o_congrad_non_hydro; non_hydrostatic.f90:70-322).

No Fortran compiler exists here, so the reference cannot be run beside the
oracle.  The oracle is pinned instead by
  * a second, independent restatement in numpy/Python of the same routines
    (the 27-entry coefficient array built by the reference's loops, the
    operator applied in its (kk, jj, ii) order, dot products summed in its
    (k, j, i) order), which must agree bit for bit, CG iterations included;
  * operator identities: constant fields are in the null space (no-flux
    walls), the operator is symmetric on a uniform Cartesian grid, and its
    stencil on a smooth field is the 7-point Laplacian;
  * manufactured solutions: forcing = A x* is solved back to x*.
"""
import numpy as np
import pytest

from pyom2_b200 import synth

I0 = 2  # Python index of Fortran i = 1


def py_make_coeff(M):
    """non_hydrostatic.f90:70-138 transcribed loop by loop."""
    nx, ny, nz = M.nx, M.ny, M.nz
    X, Y = M.shape2d
    cf = np.zeros((X, Y, nz, 3, 3, 3), order="F")
    for k in range(nz):
        for j in range(I0, ny + I0):
            for i in range(I0, nx + I0):
                c2 = M.cost[j] ** 2
                mp, mm = M.maskU[i, j, k], M.maskU[i - 1, j, k]
                cf[i, j, k, 1, 1, 1] -= mp / M.dxu[i] / M.dxt[i] / c2
                cf[i, j, k, 2, 1, 1] += mp / M.dxu[i] / M.dxt[i] / c2
                cf[i, j, k, 1, 1, 1] -= mm / M.dxu[i - 1] / M.dxt[i] / c2
                cf[i, j, k, 0, 1, 1] += mm / M.dxu[i - 1] / M.dxt[i] / c2
                mp, mm = M.maskV[i, j, k], M.maskV[i, j - 1, k]
                cf[i, j, k, 1, 1, 1] -= mp / M.dyu[j] / M.dyt[j] * M.cosu[j] / M.cost[j]
                cf[i, j, k, 1, 2, 1] += mp / M.dyu[j] / M.dyt[j] * M.cosu[j] / M.cost[j]
                cf[i, j, k, 1, 1, 1] -= mm / M.dyu[j - 1] / M.dyt[j] * M.cosu[j - 1] / M.cost[j]
                cf[i, j, k, 1, 0, 1] += mm / M.dyu[j - 1] / M.dyt[j] * M.cosu[j - 1] / M.cost[j]
    for k in range(nz):
        for j in range(I0, ny + I0):
            for i in range(I0, nx + I0):
                if k < nz - 1:
                    mp = M.maskW[i, j, k]
                    cf[i, j, k, 1, 1, 1] -= mp / M.dzw[k] / M.dzt[k]
                    cf[i, j, k, 1, 1, 2] += mp / M.dzw[k] / M.dzt[k]
                if k > 0:
                    mm = M.maskW[i, j, k - 1]
                    cf[i, j, k, 1, 1, 1] -= mm / M.dzw[k - 1] / M.dzt[k]
                    cf[i, j, k, 1, 1, 0] += mm / M.dzw[k - 1] / M.dzt[k]
    return cf


def py_apply(M, cf, p):
    """non_hydrostatic.f90:247-276, vectorised over cells, same per-cell order."""
    nx, ny, nz = M.nx, M.ny, M.nz
    res = np.zeros_like(p)
    I = slice(I0, nx + I0)
    J = slice(I0, ny + I0)
    for kk in (-1, 0, 1):
        for jj in (-1, 0, 1):
            for ii in (-1, 0, 1):
                for k in range(nz):
                    kp = min(nz - 1, max(0, k + kk))
                    res[I, J, k] = res[I, J, k] + cf[I, J, k, ii + 1, jj + 1, kk + 1] * \
                        p[I0 + ii:nx + I0 + ii, I0 + jj:ny + I0 + jj, kp]
    return res


def py_dot(M, a, b):
    s = 0.0
    for k in range(M.nz):
        for j in range(I0, M.ny + I0):
            for i in range(I0, M.nx + I0):
                s = s + a[i, j, k] * b[i, j, k] * M.maskT[i, j, k]
    return s


def py_absmax(M, a):
    s = 0.0
    for k in range(M.nz):
        for j in range(I0, M.ny + I0):
            for i in range(I0, M.nx + I0):
                s = max(abs(a[i, j, k] * M.maskT[i, j, k]), s)
    return s


def py_congrad(M, cf, forc, pnh, eps, max_it):
    """non_hydrostatic.f90:146-242, returns (n, status)."""
    res = py_apply(M, cf, pnh)
    I = slice(I0, M.nx + I0)
    J = slice(I0, M.ny + I0)
    res[I, J] = forc[I, J] - res[I, J]
    p = res.copy(order="F")
    synth.setcyclic_xy(M, p)
    rsold = py_dot(M, res, res)
    if rsold == 0.0:
        return 0, 0
    rs_min = step1 = 0.0
    for n in range(1, max_it + 1):
        Ap = py_apply(M, cf, p)
        fxa = py_dot(M, p, Ap)
        if fxa == 0.0:
            return n, 0
        alpha = rsold / fxa
        pnh[...] = pnh + alpha * p
        res = res - alpha * Ap
        rsnew = py_dot(M, res, res)
        p = np.asfortranarray(res + rsnew / rsold * p)
        synth.setcyclic_xy(M, p)
        rsold = rsnew
        if n == 1:
            rs_min = abs(rsnew)
        elif n > 2:
            rs_min = min(rs_min, abs(rsnew))
            if abs(rsnew) > 100.0 * rs_min:
                return n, 2
        smax = py_absmax(M, p)
        step = abs(alpha) * smax
        if n == 1:
            step1 = step
            if step < eps:
                return n, 0
        elif step < eps:
            rate = np.exp(np.log(step / step1) / (n - 1))
            est = step * rate / (1.0 - rate)
            if est < eps:
                return n, 0
    return max_it + 1, 1


def tiny(cyclic_x, seed, ny=5):
    return synth.nonhydro_tank(10, ny, 6, seed, cyclic_x=cyclic_x, dx=0.5, first_guess=True)


@pytest.mark.parametrize("cyclic_x,ny", [(False, 5), (True, 5), (True, 1)])
def test_coefficients_and_operator_bit_exact(oracle_lib, cyclic_x, ny):
    W = tiny(cyclic_x, 11, ny)
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    assert np.array_equal(cf, py_make_coeff(W.M))
    rng = np.random.default_rng(1)
    p = np.asfortranarray(rng.standard_normal(O.shape))
    assert np.array_equal(O.apply_op(cf, p), py_apply(W.M, cf, p))
    assert O.dot(p, p) == py_dot(W.M, p, p)
    assert O.absmax(p) == py_absmax(W.M, p)


@pytest.mark.parametrize("cyclic_x,ny", [(False, 5), (True, 5), (True, 1)])
def test_congrad_bit_exact_against_python_restatement(oracle_lib, cyclic_x, ny):
    W = tiny(cyclic_x, 12, ny)
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    for eps, max_it in ((1e-9, 500), (0.0, 7)):
        p1 = W.p0.copy(order="F")
        p2 = W.p0.copy(order="F")
        info = O.congrad(cf, W.forc, p1, eps=eps, max_it=max_it)
        n, st = py_congrad(W.M, cf, W.forc, p2, eps, max_it)
        assert (info["iterations"], info["status"]) == (n, st)
        assert np.array_equal(p1, p2)
    assert info["status"] == 1 and info["iterations"] == 8


def test_operator_identities(oracle_lib):
    W = synth.nonhydro_tank(24, 20, 10, 3, dx=0.25)
    M = W.M
    O = oracle_lib.Oracle3D(M)
    cf = O.make_coeff()
    # no-flux walls: constants are in the null space
    one = np.asfortranarray(np.ones(O.shape))
    a1 = O.apply_op(cf, one)
    assert np.abs(a1).max() <= 1e-12 * np.abs(cf).max()
    # uniform Cartesian grid: A is symmetric in the maskT inner product
    rng = np.random.default_rng(2)
    u = np.asfortranarray(rng.standard_normal(O.shape) * M.maskT)
    v = np.asfortranarray(rng.standard_normal(O.shape) * M.maskT)
    lhs, rhs = O.dot(u, O.apply_op(cf, v)), O.dot(O.apply_op(cf, u), v)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # away from walls the stencil is the 7-point Laplacian (dx = dy = dz = 0.25)
    x = np.arange(O.shape[0])[:, None, None] * 0.25
    y = np.arange(O.shape[1])[None, :, None] * 0.25
    z = np.arange(O.shape[2])[None, None, :] * 0.25
    f = np.asfortranarray(x ** 2 + 2 * y ** 2 + 3 * z ** 2)
    af = O.apply_op(cf, f)
    wet7 = (M.maskT > 0)
    for sh in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
        wet7 = wet7 & (np.roll(M.maskT, sh, axis=(0, 1, 2)) > 0)
    wet7[:, :, 0] = wet7[:, :, -1] = False
    wet7[:I0 + 1] = wet7[-I0 - 1:] = False
    wet7[:, :I0 + 1] = wet7[:, -I0 - 1:] = False
    assert wet7.sum() > 100
    assert np.allclose(af[wet7], 12.0, rtol=1e-9)


@pytest.mark.parametrize("cyclic_x", [False, True])
def test_manufactured_solution(oracle_lib, cyclic_x):
    W = synth.nonhydro_tank(20, 16, 8, 5, cyclic_x=cyclic_x)
    M = W.M
    O = oracle_lib.Oracle3D(M)
    cf = O.make_coeff()
    rng = np.random.default_rng(3)
    xs = np.asfortranarray(rng.standard_normal(O.shape) * M.maskT)
    O.setcyclic_xyz(xs)
    forc = O.apply_op(cf, xs)
    p = np.zeros(O.shape, order="F")
    info = O.congrad(cf, forc, p, eps=1e-11, max_it=5000)
    assert info["status"] == 0, info
    O.setcyclic_xyz(p)
    # defined up to a constant per connected wet region; the tank is one region
    m = M.maskT > 0
    d = (p - xs)[m]
    assert np.abs(d - d.mean()).max() < 1e-7 * np.abs(xs[m]).max()


def test_zero_forcing_stops_at_once(oracle_lib):
    W = tiny(False, 13)
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    p = np.zeros(O.shape, order="F")
    info = O.congrad(cf, np.zeros(O.shape, order="F"), p)
    assert info["iterations"] == 0 and info["status"] == 0 and not p.any()


def test_maskW_follows_calc_topo():
    W = tiny(False, 14)
    M = W.M
    assert np.array_equal(M.maskW[:, :, :-1], np.minimum(M.maskT[:, :, :-1], M.maskT[:, :, 1:]))
    assert np.array_equal(M.maskW[:, :, -1], M.maskT[:, :, -1])


def test_forcing_is_in_the_range(oracle_lib):
    """The synthetic forcing is a divergence of a masked velocity: its volume
    integral over the wet cells vanishes, so the singular Neumann problem is
    consistent."""
    W = synth.nonhydro_tank(30, 20, 12, 7)
    M = W.M
    vol = M.dxt[:, None, None] * M.dyt[None, :, None] * M.dzt[None, None, :] * M.cost[None, :, None]
    s = np.sum((W.forc * vol)[2:-2, 2:-2])
    assert abs(s) < 1e-10 * np.sum(np.abs(W.forc * vol))
