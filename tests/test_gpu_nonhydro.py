"""GPU parity of the non-hydrostatic pressure solve against the CPU oracle
(non_hydrostatic.f90:70-322).

* apply_op_3D: bit-identical to the oracle (the compact operator rebuilds the
  reference's coefficients and sums in its order without fused multiply-adds).
* congrad_non_hydro: the dot products are reduced in another order than the
  reference's sequential loop, so the iteration counts may differ by one
  where the stopping estimate crosses eps within rounding, and CG iterates,
  which amplify the rounding of alpha and beta over hundreds of iterations,
  agree with the oracle's at the same iteration to 1e-7 relative (max norm
  over the wet cells) -- far inside the solve's own accuracy (eps = 1e-9
  absolute on fields of size 1e-3, i.e. 1e-6 relative).  Statuses are equal.
"""
import warnings

import numpy as np
import pytest

from pyom2_b200 import _abi, synth
from pyom2_b200.non_hydrostatic import NonHydrostatic, congrad_non_hydro

pytestmark = pytest.mark.gpu

CASES = [
    ("tank_60x60x20", dict(nx=60, ny=60, nz=20, seed=1, cyclic_x=False)),
    ("xz_64x1x64_cyclic", dict(nx=64, ny=1, nz=64, seed=2, cyclic_x=True)),
    ("tank_97x33x17_cyclic", dict(nx=97, ny=33, nz=17, seed=3, cyclic_x=True)),
    ("tank_40x36x9_guess", dict(nx=40, ny=36, nz=9, seed=4, cyclic_x=False, first_guess=True)),
]


def world(kw):
    kw = dict(kw)
    return synth.nonhydro_tank(kw.pop("nx"), kw.pop("ny"), kw.pop("nz"), kw.pop("seed"), **kw)


def rel_max(a, b, m):
    return np.abs((a - b)[m]).max() / max(np.abs(b[m]).max(), 1e-300)


@pytest.mark.parametrize("name,kw", CASES)
def test_apply_op_3d_bit_exact(oracle_lib, name, kw):
    W = world(kw)
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    nh = NonHydrostatic(W.M)
    rng = np.random.default_rng(5)
    p = np.asfortranarray(rng.standard_normal(O.shape))
    assert np.array_equal(nh.apply_op_3d(p), O.apply_op(cf, p))
    nh.close()


@pytest.mark.parametrize("name,kw", CASES)
def test_congrad_non_hydro_matches_oracle(oracle_lib, name, kw):
    W = world(kw)
    M = W.M
    O = oracle_lib.Oracle3D(M)
    cf = O.make_coeff()
    nh = NonHydrostatic(M)
    eps = 1e-9
    p_gpu = W.p0.copy(order="F")
    it, info = nh.congrad_non_hydro(W.forc, p_gpu, eps=eps, max_it=5000)
    p_cpu = W.p0.copy(order="F")
    io = O.congrad(cf, W.forc, p_cpu, eps=eps, max_it=5000)
    assert info["status"] == io["status"] == 0, (info, io)
    assert abs(it - io["iterations"]) <= 1, (it, io["iterations"])
    p_same = W.p0.copy(order="F")
    O.congrad(cf, W.forc, p_same, eps=0.0, max_it=it)  # oracle stopped where the GPU stopped
    m = M.maskT > 0
    assert rel_max(p_gpu, p_same, m) < 1e-7
    # halos follow the whole-array update of the reference
    assert rel_max(p_gpu, p_same, np.ones_like(m)) < 1e-7
    nh.close()


def test_max_iterations_and_zero_forcing(oracle_lib):
    W = world(CASES[0][1])
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    nh = NonHydrostatic(W.M)
    p = W.p0.copy(order="F")
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        it, info = nh.congrad_non_hydro(W.forc, p, eps=1e-30, max_it=12)
    assert info["status"] == _abi.MAXITER and it == 13
    assert any("max iterations" in str(r.message) for r in rec)
    po = W.p0.copy(order="F")
    io = O.congrad(cf, W.forc, po, eps=1e-30, max_it=12)
    assert io["status"] == 1 and io["iterations"] == 13
    assert rel_max(p, po, W.M.maskT > 0) < 1e-10
    z = np.zeros(O.shape, order="F")
    p0 = np.zeros(O.shape, order="F")
    it, info = nh.congrad_non_hydro(z, p0)
    assert it == 0 and info["status"] == 0 and not p0.any()
    nh.close()


def test_device_tensors_in_place_and_model_entry(oracle_lib):
    import torch
    W = world(CASES[1][1])
    M = W.M
    nh = NonHydrostatic(M)
    p_host = W.p0.copy(order="F")
    nh.congrad_non_hydro(W.forc, p_host, eps=1e-9)
    to_dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).cuda().T
    f_t, p_t = to_dev(W.forc), to_dev(W.p0)
    nh.congrad_non_hydro(f_t, p_t, eps=1e-9)
    assert np.array_equal(p_t.cpu().numpy(), p_host)
    # module-level call on the model arrays (p_non_hydro(:,:,:,taup1), congr_itts_non_hydro)
    M.congr_epsilon_non_hydro = 1e-9
    M.p_non_hydro[..., M.taup1 - 1] = W.p0
    it = congrad_non_hydro(M, W.forc)
    assert it == M.congr_itts_non_hydro > 0
    assert np.array_equal(M.p_non_hydro[..., M.taup1 - 1], p_host)
    nh.close()


def test_barrier_timeout_is_reported_and_handle_survives():
    W = world(CASES[0][1])
    nh = NonHydrostatic(W.M)
    nh.set_sync_timeout(0.2)
    nh.inject_barrier_stall(True)
    p = W.p0.copy(order="F")
    with pytest.raises(_abi.PyOMGPUError) as e:
        nh.congrad_non_hydro(W.forc, p, eps=1e-9)
    assert e.value.code == _abi.TIMEOUT
    p = W.p0.copy(order="F")
    it, info = nh.congrad_non_hydro(W.forc, p, eps=1e-9)
    assert info["status"] == 0 and it > 0
    nh.close()


@pytest.mark.parametrize("blocks", [1, 7, 64])
def test_grid_size_changes_only_rounding(oracle_lib, blocks):
    W = world(CASES[2][1])
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    nh = NonHydrostatic(W.M)
    nh.set_grid(blocks)
    p = W.p0.copy(order="F")
    it, info = nh.congrad_non_hydro(W.forc, p, eps=1e-9, max_it=5000)
    po = W.p0.copy(order="F")
    io = O.congrad(cf, W.forc, po, eps=1e-9, max_it=5000)
    assert info["status"] == 0 and abs(it - io["iterations"]) <= 1
    nh.close()


@pytest.mark.parametrize("cyclic_x,itt", [(False, 1), (True, 0)])
def test_solve_non_hydrostatic_step_matches_oracle(oracle_lib, cyclic_x, itt):
    """The whole step (non_hydrostatic.f90:5-63) on the GPU against the
    oracle's: same iteration count within one, u, v, w and p_non_hydro at all
    three levels within 1e-7 of their size (the CG iterate's rounding)."""
    from pyom2_b200.non_hydrostatic import solve_non_hydrostatic
    W = synth.nonhydro_state(synth.nonhydro_tank(48, 20, 12, 6, cyclic_x=cyclic_x), 9)
    M = W.M
    M.itt = itt
    M.congr_epsilon_non_hydro = 1e-10
    Mo = M.copy()
    O = oracle_lib.Oracle3D(Mo)
    rc = O.solve_non_hydrostatic()
    assert rc == 0
    info = solve_non_hydrostatic(M)
    assert info["status"] == 0
    assert abs(M.congr_itts_non_hydro - Mo.congr_itts_non_hydro) <= 1
    for n in ("u", "v", "w", "p_non_hydro"):
        a, b = getattr(M, n), getattr(Mo, n)
        assert np.abs(a - b).max() <= 1e-7 * np.abs(b).max(), n
    # fields the step does not touch are untouched
    assert np.array_equal(M.u[..., M.tau - 1], Mo.u[..., Mo.tau - 1])


@pytest.mark.parametrize("name,kw", [CASES[1], CASES[3]])
def test_single_block_kernel_matches_oracle_and_bricks(oracle_lib, name, kw):
    """Small grids run in one block with the fields in shared memory; the
    result follows the oracle as the brick kernel's does."""
    W = world(kw)
    O = oracle_lib.Oracle3D(W.M)
    cf = O.make_coeff()
    nh = NonHydrostatic(W.M)
    out = {}
    for variant in (1, 2):
        nh.set_variant(variant)
        p = W.p0.copy(order="F")
        it, info = nh.congrad_non_hydro(W.forc, p, eps=1e-9, max_it=5000)
        io = O.congrad(cf, W.forc, W.p0.copy(order="F"), eps=1e-9, max_it=5000)
        assert info["status"] == 0 and abs(it - io["iterations"]) <= 1, (variant, it, io)
        ps = W.p0.copy(order="F")
        O.congrad(cf, W.forc, ps, eps=0.0, max_it=it)
        assert rel_max(p, ps, np.ones(p.shape, bool)) < 1e-7, variant
        out[variant] = (it, p)
    # max-iteration semantics on the single-block kernel too
    p = W.p0.copy(order="F")
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        it, info = nh.congrad_non_hydro(W.forc, p, eps=1e-30, max_it=9)
    assert info["status"] == _abi.MAXITER and it == 10
    nh.close()
