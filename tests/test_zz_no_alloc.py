"""The allocation-free streamfunction solve, pyomgpu_congrad_streamfunction_noalloc.

It serves callers that cannot call cudaMalloc -- a host program whose
device memory is already claimed by its own pool, code running where new
device allocations are forbidden, or a time loop that must not allocate --
by solving in a static device array the library reserves at load time.  The
test calls it through the C ABI with only caller-owned inputs and outputs
and checks it against the context entry point (pyomgpu_congrad_streamfunction)
on two calls in a row: the second call finds the first call's data in the
shared scratch array and must not depend on it.  Kept in its own file, named
to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_SOL = 1e-10  # the parity tolerance of the GPU tests


def _world():
    from pyom2_b200 import synth
    return synth._global_like(96, 48, -80.0, 80.0, 13, n_land_masses=6, mask_sigma=4.0, depth_sigma=4.0,
                              name="small")


def _dev_f(a, dev):
    """Fortran-ordered CUDA copy of a numpy array (C order of the transpose)."""
    import torch
    a = np.asarray(a)
    if a.ndim == 1:
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).to(dev)


def test_noalloc_solve_matches_context_solve():
    import torch

    from pyom2_b200 import _abi
    from pyom2_b200.external import ExternalMode

    L = _abi.load()
    dev = torch.device("cuda")
    W = _world()
    M = W.M
    E = ExternalMode(M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6)
    assert M.nisle >= 2
    pi = np.concatenate([M.boundary[k, :M.nr_boundary[k], 0] for k in range(M.nisle)]).astype(np.int32)
    pj = np.concatenate([M.boundary[k, :M.nr_boundary[k], 1] for k in range(M.nisle)]).astype(np.int32)
    keep = {n: _dev_f(getattr(M, n), dev) for n in ("dxt", "dxu", "dyt", "dyu", "cost", "cosu", "hur", "hvr")}
    bi = torch.from_numpy(pi).to(dev)
    bj = torch.from_numpy(pj).to(dev)
    g = _abi.Grid()
    g.nx, g.ny, g.onx = M.nx, M.ny, M.onx
    g.enable_cyclic_x, g.enable_cyclic_y = int(M.enable_cyclic_x), int(M.enable_cyclic_y)
    for n, t in keep.items():
        setattr(g, n, t.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    rng = np.random.default_rng(17)
    forcs = [W.forc, np.asfortranarray(W.forc * 0.5 + rng.standard_normal(M.shape2d) * 1e-15)]
    firsts = [np.zeros(M.shape2d, order="F"), np.asfortranarray(rng.standard_normal(M.shape2d) * 1e2)]
    for call in range(2):
        ref = firsts[call].copy(order="F")
        it_ref, conv_ref, _ = E.congrad_streamfunction(forcs[call], ref)
        f_d = _dev_f(forcs[call], dev)
        s_d = _dev_f(firsts[call], dev)
        info = _abi.SolveInfo()
        rc = L.pyomgpu_congrad_streamfunction_noalloc(
            C.byref(g), C.c_void_p(bi.data_ptr()), C.c_void_p(bj.data_ptr()), int(pi.size),
            C.c_void_p(f_d.data_ptr()), C.c_void_p(s_d.data_ptr()), float(M.congr_epsilon),
            int(M.congr_max_iterations), C.byref(info), stream)
        assert rc == _abi.OK, _abi.last_error()
        assert info.iterations == it_ref and bool(info.converged) == conv_ref
        sol = s_d.cpu().numpy().T
        err = np.linalg.norm(sol - ref) / np.linalg.norm(ref)
        assert err < RTOL_SOL, (call, err)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    from pyom2_b200 import _abi

    L = _abi.load()
    dev = torch.device("cuda")
    small = torch.zeros(16, dtype=torch.float64, device=dev)
    g = _abi.Grid()
    g.nx, g.ny, g.onx = 4000, 4000, 2
    for n in ("dxt", "dxu", "dyt", "dyu", "cost", "cosu", "hur", "hvr"):
        setattr(g, n, small.data_ptr())
    info = _abi.SolveInfo()
    rc = L.pyomgpu_congrad_streamfunction_noalloc(C.byref(g), None, None, 0, C.c_void_p(small.data_ptr()),
                                                  C.c_void_p(small.data_ptr()), 1e-12, 10, C.byref(info), None)
    assert rc == _abi.EINVAL
    assert "scratch" in _abi.last_error()
