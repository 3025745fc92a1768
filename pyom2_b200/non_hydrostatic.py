"""Python mirror of pyOM2's non-hydrostatic pressure solve on the B200 library.

=============================================  ====================================================
reference (file:line)                          here
=============================================  ====================================================
make_coeff_non_hydro (non_hydrostatic.f90:70)  :class:`NonHydrostatic` (operator built once, kept)
congrad_non_hydro (non_hydrostatic.f90:146)    :meth:`NonHydrostatic.congrad_non_hydro`,
                                               :func:`congrad_non_hydro`
apply_op_3D (non_hydrostatic.f90:247)          :meth:`NonHydrostatic.apply_op_3d`
solve_non_hydrostatic (non_hydrostatic.f90:5)  :meth:`NonHydrostatic.solve_non_hydrostatic`,
                                               :func:`solve_non_hydrostatic`
=============================================  ====================================================

Arrays are Fortran-ordered float64 (nx+4, ny+4, nz) buffers: numpy (host,
copied by the library) or torch CUDA tensors in the same memory order (used
in place).  As in the reference, exceeding the iteration limit or the
divergence test is a warning; a NaN estimate raises :class:`PyOMGPUError`.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np

from . import _abi
from ._abi import PyOMGPUError
from .external import _f64, _from_device_f, _host, _is_torch, _ptr, _stream, _to_device_f, _torch_like


class NonHydrostatic:
    """Operator and work buffers of the 3-D solve for one model grid (the
    SAVE'd ``cf`` of congrad_non_hydro lives here, on the GPU)."""

    def __init__(self, M):
        L = _abi.load()
        self.M = M
        self.shape = (M.nx + 2 * M.onx, M.ny + 2 * M.onx, M.nz)
        self._keep = {}

        def host(name, arr):
            x = _f64(_host(arr))
            self._keep[name] = x
            return x.ctypes.data

        g = _abi.Grid3D()
        g.nx, g.ny, g.nz, g.onx = M.nx, M.ny, M.nz, M.onx
        g.enable_cyclic_x = int(bool(M.enable_cyclic_x))
        g.enable_cyclic_y = int(bool(M.enable_cyclic_y))
        for n in ("dxt", "dxu", "dyt", "dyu", "cost", "cosu", "dzt", "dzw", "maskT", "maskU", "maskV", "maskW"):
            setattr(g, n, host(n, getattr(M, n)))
        h = C.c_void_p()
        _abi.check(L.pyomgpu_nh_create(C.byref(g), C.byref(h)))
        self._h = h
        self._L = L

    def close(self):
        if getattr(self, "_h", None):
            self._L.pyomgpu_nh_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_sync_timeout(self, seconds: float):
        _abi.check(self._L.pyomgpu_nh_set_sync_timeout(self._h, float(seconds)))

    def inject_barrier_stall(self, enable: bool = True):
        """Failure-detection test hook: the next solve's first grid barrier
        can never complete, so it ends with PYOMGPU_TIMEOUT."""
        _abi.check(self._L.pyomgpu_nh_inject_barrier_stall(self._h, int(bool(enable))))

    def set_grid(self, blocks: int):
        """Blocks of the CG launch (0 = automatic)."""
        _abi.check(self._L.pyomgpu_nh_set_grid(self._h, int(blocks)))

    def set_brick(self, ty: int, kc: int):
        """Brick shape 32 x ty x kc of the CG sweeps ((0, 0) = automatic)."""
        _abi.check(self._L.pyomgpu_nh_set_brick(self._h, int(ty), int(kc)))

    def set_stages(self, stages: int):
        """TMA pipeline depth of the CG sweeps (2..4; 0 = automatic)."""
        _abi.check(self._L.pyomgpu_nh_set_stages(self._h, int(stages)))

    def set_variant(self, variant: int):
        """CG kernel: 1 grid-wide bricks, 2 one block resident in shared memory
        (small grids), 0 automatic."""
        _abi.check(self._L.pyomgpu_nh_set_variant(self._h, int(variant)))

    def apply_op_3d(self, p):
        """non_hydrostatic.f90:247-276: ``res = A p`` over the interior, zero halo."""
        res = np.zeros(self.shape, order="F") if not _is_torch(p) else _torch_like(p)
        _abi.check(self._L.pyomgpu_apply_op_3d(self._h, _ptr(p, self.shape), _ptr(res, self.shape, True), _stream()))
        return res

    def congrad_non_hydro(self, forc, p, eps=None, max_it=None):
        """non_hydrostatic.f90:146-242 in place on ``p`` (= p_non_hydro(:,:,:,taup1)).
        Returns (iterations, info dict)."""
        info = _abi.SolveInfo()
        rc = self._L.pyomgpu_congrad_non_hydro(
            self._h, _ptr(forc, self.shape), _ptr(p, self.shape, True),
            float(self.M.congr_epsilon_non_hydro if eps is None else eps),
            int(self.M.congr_max_itts_non_hydro if max_it is None else max_it), C.byref(info), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        if rc == _abi.MAXITER:
            warnings.warn("congrad_non_hydro: max iterations exceeded", RuntimeWarning, stacklevel=2)
        elif rc == _abi.DIVERGED:
            warnings.warn("congrad_non_hydro: non hydrostatic solver diverging", RuntimeWarning, stacklevel=2)
        return info.iterations, info.as_dict()


    def solve_non_hydrostatic(self, M=None):
        """non_hydrostatic.f90:5-63 on the model arrays u, v, w, dw, dw_mix,
        p_non_hydro (numpy host arrays are copied to the GPU and back; torch
        CUDA tensors are updated in place).  Sets M.congr_itts_non_hydro and
        returns the solve's info dict."""
        import torch
        M = M or self.M
        dev = torch.device("cuda")
        D = {n: _to_device_f(getattr(M, n), dev) for n in ("u", "v", "w", "dw", "dw_mix", "p_non_hydro")}
        s = _abi.State3D()
        s.taum1, s.tau, s.taup1, s.itt = int(M.taum1), int(M.tau), int(M.taup1), int(M.itt)
        s.congr_max_itts_non_hydro = int(M.congr_max_itts_non_hydro)
        s.dt_mom, s.AB_eps = float(M.dt_mom), float(M.AB_eps)
        s.congr_epsilon_non_hydro = float(M.congr_epsilon_non_hydro)
        for n, t in D.items():
            setattr(s, n, C.c_void_p(t.data_ptr()))
        info = _abi.SolveInfo()
        rc = self._L.pyomgpu_solve_non_hydrostatic(self._h, C.byref(s), C.byref(info), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        if rc == _abi.MAXITER:
            warnings.warn("solve_non_hydrostatic: max iterations exceeded", RuntimeWarning, stacklevel=2)
        elif rc == _abi.DIVERGED:
            warnings.warn("solve_non_hydrostatic: non hydrostatic solver diverging", RuntimeWarning, stacklevel=2)
        for n in ("u", "v", "w", "p_non_hydro"):
            a = getattr(M, n)
            if not _is_torch(a):
                a[...] = _from_device_f(D[n])
        M.congr_itts_non_hydro = int(s.congr_itts_non_hydro)
        return info.as_dict()


_CACHE = {}


def _nh_for(M):
    key = id(M)
    nh = _CACHE.get(key)
    if nh is None or nh.M is not M:
        nh = NonHydrostatic(M)
        _CACHE[key] = nh
    return nh


def congrad_non_hydro(M, forc):
    """Module-level form of the reference call
    ``congrad_non_hydro(is_pe-onx, ..., nz, forc, congr_itts_non_hydro)``:
    updates ``M.p_non_hydro(:,:,:,taup1)`` in place and sets
    ``M.congr_itts_non_hydro``."""
    p = M.p_non_hydro[:, :, :, M.taup1 - 1]
    if not _is_torch(p) and not p.flags.f_contiguous:
        raise PyOMGPUError(_abi.EINVAL, "p_non_hydro(:,:,:,taup1) must be contiguous")
    it, _ = _nh_for(M).congrad_non_hydro(forc, p)
    M.congr_itts_non_hydro = it
    return it


def solve_non_hydrostatic(M):
    """Module-level form of the reference call ``solve_non_hydrostatic``
    (momentum.f90:167): updates M's u, v, w and p_non_hydro in place."""
    return _nh_for(M).solve_non_hydrostatic(M)
