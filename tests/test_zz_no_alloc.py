"""The allocation-free streamfunction solve, pyomgpu_congrad_streamfunction_noalloc.

It serves callers that cannot call cudaMalloc -- a host program whose
device memory is already claimed by its own pool, code running where new
device allocations are forbidden, or a time loop that must not allocate --
by solving in a static device array the library holds.  The test calls it
through the C ABI with only caller-owned inputs and outputs and checks it
against the context entry point (pyomgpu_congrad_streamfunction) on two calls
in a row: a larger grid, then a smaller one with another pitch, so the second
call finds the first call's data in the shared scratch array and must not
depend on it; free device memory must not drop across the second call.  Kept
in its own file, named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_SOL = 1e-10  # the parity tolerance of the GPU tests


def _world(nx, ny, seed):
    from pyom2_b200 import synth
    return synth._global_like(nx, ny, -80.0, 80.0, seed, n_land_masses=6, mask_sigma=4.0, depth_sigma=4.0,
                              name="small")


def _dev_f(a, dev):
    """Fortran-ordered CUDA copy of a numpy array (C order of the transpose)."""
    import torch
    a = np.asarray(a)
    if a.ndim == 1:
        return torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    return torch.from_numpy(np.ascontiguousarray(np.asfortranarray(a).T)).to(dev)


def _case(W, forc, first, dev):
    """Everything one no-alloc call needs, on the device, plus the context
    entry point's result on the same inputs."""
    import torch

    from pyom2_b200 import _abi
    from pyom2_b200.external import ExternalMode

    M = W.M
    E = ExternalMode(M)
    E.streamfunction_init(maxipp=10**6, maxq=10**6)
    assert M.nisle >= 2
    ref = first.copy(order="F")
    it_ref, conv_ref, _ = E.congrad_streamfunction(forc, ref)
    pi = np.concatenate([M.boundary[k, :M.nr_boundary[k], 0] for k in range(M.nisle)]).astype(np.int32)
    pj = np.concatenate([M.boundary[k, :M.nr_boundary[k], 1] for k in range(M.nisle)]).astype(np.int32)
    keep = {n: _dev_f(getattr(M, n), dev) for n in ("dxt", "dxu", "dyt", "dyu", "cost", "cosu", "hur", "hvr")}
    keep["bi"] = torch.from_numpy(pi).to(dev)
    keep["bj"] = torch.from_numpy(pj).to(dev)
    keep["f"] = _dev_f(forc, dev)
    keep["s"] = _dev_f(first, dev)
    g = _abi.Grid()
    g.nx, g.ny, g.onx = M.nx, M.ny, M.onx
    g.enable_cyclic_x, g.enable_cyclic_y = int(M.enable_cyclic_x), int(M.enable_cyclic_y)
    for n in ("dxt", "dxu", "dyt", "dyu", "cost", "cosu", "hur", "hvr"):
        setattr(g, n, keep[n].data_ptr())
    E.close()
    return dict(M=M, g=g, keep=keep, nbnd=int(pi.size), ref=ref, it=it_ref, conv=conv_ref)


def test_noalloc_solve_matches_context_solve():
    import torch

    from pyom2_b200 import _abi

    L = _abi.load()
    dev = torch.device("cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(17)
    WA, WB = _world(128, 64, 7), _world(96, 48, 13)  # the second call's grid is smaller: another pitch
    cases = [_case(WA, WA.forc, np.zeros(WA.M.shape2d, order="F"), dev),
             _case(WB, np.asfortranarray(WB.forc * 0.5 + rng.standard_normal(WB.M.shape2d) * 1e-15),
                   np.asfortranarray(rng.standard_normal(WB.M.shape2d) * 1e2), dev)]
    torch.cuda.synchronize()
    for call, c in enumerate(cases):
        k, M = c["keep"], c["M"]
        info = _abi.SolveInfo()
        free0 = torch.cuda.mem_get_info()[0]
        rc = L.pyomgpu_congrad_streamfunction_noalloc(
            C.byref(c["g"]), C.c_void_p(k["bi"].data_ptr()), C.c_void_p(k["bj"].data_ptr()), c["nbnd"],
            C.c_void_p(k["f"].data_ptr()), C.c_void_p(k["s"].data_ptr()), float(M.congr_epsilon),
            int(M.congr_max_iterations), C.byref(info), stream)
        free1 = torch.cuda.mem_get_info()[0]
        assert rc == _abi.OK, _abi.last_error()
        if call == 1:  # set-up done by the first call: the second takes no device memory
            assert free1 >= free0, (free0, free1)
        assert info.iterations == c["it"] and bool(info.converged) == c["conv"], (call, info.iterations, c["it"])
        sol = k["s"].cpu().numpy().T
        err = np.linalg.norm(sol - c["ref"]) / np.linalg.norm(c["ref"])
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
