"""Python mirror of pyOM2's external-mode routines on the B200 library.

pyOM2 calls these Fortran routines through its f2py module (py_src/pyOM.py:48-50,
151; for_src/main/momentum.f90:157-168).  The functions here keep their names,
argument meaning and in-place behaviour on the model arrays:

=====================================  =================================================
reference (file:line)                  here
=====================================  =================================================
streamfunction_init (streamfct_init.f90:7)   :func:`streamfunction_init`
solve_streamfunction (solve_streamfct.f90:10) :func:`solve_streamfunction`
congrad_streamfunction (solve_streamfct.f90:153) :meth:`ExternalMode.congrad_streamfunction`
solve_pressure (solve_pressure.f90:10)          :func:`solve_pressure`
congrad_surf_press (solve_pressure.f90:137)      :meth:`ExternalMode.congrad_surf_press`
apply_op (solve_pressure.f90:254)                :meth:`ExternalMode.apply_op`
make_inv_sfc (solve_streamfct.f90:381)           :meth:`ExternalMode.make_inv_sfc`
line_integral (streamfct_init.f90:311)           :meth:`ExternalMode.line_integral`
isleperim (island_module.f90:7)                  :func:`isleperim`
=====================================  =================================================

Arrays are the Fortran-ordered float64 buffers pyOM2 keeps in
``main_module``: numpy arrays (host; copied to the GPU and back by the
library) or torch CUDA tensors with the same memory order (used in place).
The reference stops the process on a NaN estimate or a singular island
system; here :class:`PyOMGPUError` is raised.  Exceeding the iteration limit
or the divergence test is a warning, as in the reference, which prints and
carries on.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np

from . import _abi
from ._abi import PyOMGPUError


def _stream():
    try:
        import torch
        if torch.cuda.is_available():
            return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    except Exception:  # pragma: no cover
        pass
    return None


def _is_torch(a):
    return type(a).__module__.startswith("torch")


def _ptr(a, shape=None, writable=False):
    """Address of a Fortran-ordered float64 array (numpy host or torch CUDA)."""
    if a is None:
        return None
    if _is_torch(a):
        import torch
        if a.dtype != torch.float64 or not a.is_cuda:
            raise PyOMGPUError(_abi.EINVAL, "torch arrays must be float64 CUDA tensors")
        if not a.permute(*reversed(range(a.dim()))).is_contiguous():
            raise PyOMGPUError(_abi.EINVAL, "torch arrays must have Fortran memory order")
        if shape is not None and tuple(a.shape) != tuple(shape):
            raise PyOMGPUError(_abi.EINVAL, f"shape {tuple(a.shape)} != {tuple(shape)}")
        return C.c_void_p(a.data_ptr())
    if not isinstance(a, np.ndarray) or a.dtype != np.float64:
        raise PyOMGPUError(_abi.EINVAL, "arrays must be float64")
    if a.ndim > 1 and not a.flags.f_contiguous:
        raise PyOMGPUError(_abi.EINVAL, "numpy arrays must be Fortran-ordered (as f2py exposes them)")
    if shape is not None and tuple(a.shape) != tuple(shape):
        raise PyOMGPUError(_abi.EINVAL, f"shape {tuple(a.shape)} != {tuple(shape)}")
    if writable and not a.flags.writeable:
        raise PyOMGPUError(_abi.EINVAL, "array is read-only")
    return C.c_void_p(a.ctypes.data)


def _f64(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _warn_status(rc, where):
    if rc == _abi.MAXITER:
        warnings.warn(f"{where}: max iterations exceeded", RuntimeWarning, stacklevel=3)
    elif rc == _abi.DIVERGED:
        warnings.warn(f"{where}: solver diverging", RuntimeWarning, stacklevel=3)


class ExternalMode:
    """Solver context for one model grid (the SAVE'd ``cf`` and the island
    arrays of the reference live here, on the GPU)."""

    def __init__(self, M):
        L = _abi.load()
        self.M = M
        self.shape = (M.nx + 2 * M.onx, M.ny + 2 * M.onx)
        self._keep = {}

        def host(name, arr):
            if arr is None:
                return None
            x = _f64(arr)
            self._keep[name] = x
            return x.ctypes.data

        g = _abi.Grid()
        g.nx, g.ny, g.onx = M.nx, M.ny, M.onx
        g.enable_cyclic_x = int(bool(M.enable_cyclic_x))
        g.enable_cyclic_y = int(bool(M.enable_cyclic_y))
        g.enable_free_surface = int(bool(getattr(M, "enable_free_surface", False)))
        g.grav = float(getattr(M, "grav", 9.81))
        g.dt_mom = float(getattr(M, "dt_mom", 1.0))
        for n in ("dxt", "dxu", "dyt", "dyu", "cost", "cosu", "hur", "hvr", "hu", "hv"):
            setattr(g, n, host(n, _host(getattr(M, n))))
        g.maskT_top = host("maskT_top", _host(M.maskT)[:, :, -1])
        g.maskU_top = host("maskU_top", _host(M.maskU)[:, :, -1])
        g.maskV_top = host("maskV_top", _host(M.maskV)[:, :, -1])
        ctx = C.c_void_p()
        _abi.check(L.pyomgpu_ctx_create(C.byref(g), C.byref(ctx)))
        self._ctx = ctx
        self._L = L
        self.nisle = 0

    def close(self):
        if getattr(self, "_ctx", None):
            self._L.pyomgpu_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set_sync_timeout(self, seconds: float):
        _abi.check(self._L.pyomgpu_set_sync_timeout(self._ctx, float(seconds)))

    def autotune(self, iterations: int = 200):
        """Pick the solve kernel's tile shape and grid for this grid by timing
        candidates on the GPU; returns (tile_x, tile_y, grid, us_per_iteration)."""
        tx, ty, gr, us = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        _abi.check(self._L.pyomgpu_autotune(self._ctx, int(iterations), C.byref(tx), C.byref(ty), C.byref(gr),
                                            C.byref(us), _stream()))
        return tx.value, ty.value, gr.value, us.value

    def inject_barrier_stall(self, enable: bool = True):
        """Failure-detection test hook: the next solve's first grid barrier
        can never complete, so it ends with PYOMGPU_TIMEOUT."""
        _abi.check(self._L.pyomgpu_inject_barrier_stall(self._ctx, int(bool(enable))))

    def set_cg_kernel(self, kernel: str = "auto"):
        """CG kernel of the streamfunction solves: ``"tiled"`` (any grid),
        ``"resident"`` (one piece of the grid per SM, held on chip for the
        whole solve, two reductions per iteration as the reference),
        ``"resident1"`` (the same with one reduction per iteration) or
        ``"auto"``; the resident ones raise on a grid that does not fit."""
        code = {"auto": 0, "tiled": 1, "resident": 2, "resident1": 3}[kernel]
        _abi.check(self._L.pyomgpu_set_cg_kernel(self._ctx, code))
        self._cg_kernel = kernel

    def resident_kernel_name(self):
        """Name of the resident kernel instance the current choice launches."""
        lay = self.resident_layout()
        if lay is None:
            return None
        single = getattr(self, "_cg_kernel", "auto") == "resident1"
        return f"cg_res{'1' if single else ''}_kernel<{lay[2]}>"

    def resident_layout(self, fp32: bool = False):
        """(pieces in x, pieces in y, points per thread) of the resident
        kernel on this grid (``fp32``: of the FP32 one that runs the
        mixed-precision correction solves), or None when the grid does not fit."""
        a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
        fn = self._L.pyomgpu_resident_layout32 if fp32 else self._L.pyomgpu_resident_layout
        rc = fn(self._ctx, C.byref(a), C.byref(b), C.byref(c))
        if rc == _abi.EINVAL:
            return None
        _abi.check(rc)
        return a.value, b.value, c.value

    # ---- islands -----------------------------------------------------------------
    def streamfunction_init(self, M=None, mnisle=0, maxipp=0, maxq=0, eps=None, max_it=None, psin_rtol=0.0,
                            psin_weighted=False):
        """streamfct_init.f90:7-304; fills ``nisle, boundary, line_dir,
        nr_boundary, psin, dpsin, line_psin`` of the model (allocated here,
        :87-93).  ``mnisle/maxipp/maxq`` = 0 keep the reference's limits.
        ``psin_rtol`` > 0 solves the psin problems to that residual relative
        to the initial one instead of the reference's stop, with cell-area
        weighted products if ``psin_weighted`` (pyomgpu_set_psin_solve)."""
        M = M or self.M
        _abi.check(self._L.pyomgpu_set_psin_solve(self._ctx, float(psin_rtol), int(bool(psin_weighted))))
        kbot = np.asfortranarray(_host(M.kbot), dtype=np.int32)
        rc = self._L.pyomgpu_streamfunction_init(
            self._ctx, C.c_void_p(kbot.ctypes.data), int(mnisle), int(maxipp), int(maxq),
            float(M.congr_epsilon if eps is None else eps),
            int(M.congr_max_iterations if max_it is None else max_it), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        _warn_status(rc, "streamfunction_init")
        nisle, maxb = C.c_int32(), C.c_int32()
        _abi.check(self._L.pyomgpu_island_sizes(self._ctx, C.byref(nisle), C.byref(maxb)))
        M.allocate_islands(nisle.value, maxb.value) if hasattr(M, "allocate_islands") else _alloc_islands(
            M, nisle.value, maxb.value)
        iters = np.zeros(max(1, nisle.value), dtype=np.int32)
        _abi.check(self._L.pyomgpu_get_islands(
            self._ctx, C.c_void_p(M.boundary.ctypes.data), C.c_void_p(M.line_dir.ctypes.data),
            C.c_void_p(M.nr_boundary.ctypes.data), _ptr(M.psin), C.c_void_p(M.line_psin.ctypes.data),
            C.c_void_p(iters.ctypes.data), _stream()))
        self.nisle = nisle.value
        M.congr_itts = int(iters[-1]) if nisle.value else 0
        return iters[:nisle.value].copy()

    def set_islands(self, M=None, with_psin=True):
        """Use island arrays computed elsewhere (e.g. by the Fortran
        streamfunction_init) for make_inv_sfc and the island correction."""
        M = M or self.M
        b = np.asfortranarray(M.boundary, dtype=np.int32)
        d = np.asfortranarray(M.line_dir, dtype=np.int32)
        nr = np.ascontiguousarray(M.nr_boundary, dtype=np.int32)
        s = _abi.Islands(int(M.nisle), int(b.shape[1]), b.ctypes.data, d.ctypes.data, nr.ctypes.data)
        psin = _ptr(M.psin) if with_psin and M.psin is not None else None
        lps = _f64(M.line_psin) if with_psin and M.line_psin is not None else None
        _abi.check(self._L.pyomgpu_set_islands(self._ctx, C.byref(s), psin,
                                               None if lps is None else C.c_void_p(lps.ctypes.data), _stream()))
        self.nisle = int(M.nisle)

    # ---- solvers --------------------------------------------------------------------
    def congrad_streamfunction(self, forc, sol, eps=None, max_it=None):
        """solve_streamfct.f90:153-327 in place on ``sol``; returns
        ``(iterations, converged, info)``."""
        info = _abi.SolveInfo()
        rc = self._L.pyomgpu_congrad_streamfunction(
            self._ctx, _ptr(forc, self.shape), _ptr(sol, self.shape, True),
            float(self.M.congr_epsilon if eps is None else eps),
            int(self.M.congr_max_iterations if max_it is None else max_it), C.byref(info), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        _warn_status(rc, "congrad_streamfunction")
        return info.iterations, bool(info.converged), info.as_dict()

    def congrad_surf_press(self, forc, psi, eps=None, max_it=None):
        """solve_pressure.f90:137-249 in place on ``psi`` (= psi(:,:,taup1))."""
        info = _abi.SolveInfo()
        rc = self._L.pyomgpu_congrad_surf_press(
            self._ctx, _ptr(forc, self.shape), _ptr(psi, self.shape, True),
            float(self.M.congr_epsilon if eps is None else eps),
            int(self.M.congr_max_iterations if max_it is None else max_it), C.byref(info), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        _warn_status(rc, "congrad_surf_press")
        return info.iterations, info.as_dict()

    def solve_rtol(self, forc, sol, rtol=1e-10, precision=_abi.PREC_F64, max_it=1000000):
        """Solve to FP64 true relative residual ``rtol`` (measurement entry)."""
        info = _abi.SolveInfo()
        rc = self._L.pyomgpu_solve_rtol(self._ctx, _ptr(forc, self.shape), _ptr(sol, self.shape, True),
                                        float(rtol), int(precision), int(max_it), C.byref(info), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        return info.as_dict()

    # ---- operator utilities -------------------------------------------------------------
    def apply_op(self, p, op="streamfunction"):
        """solve_pressure.f90:254-274: ``res = A p`` over the interior, zero halo."""
        res = np.zeros(self.shape, order="F") if not _is_torch(p) else _torch_like(p)
        code = _abi.OP_SURF_PRESS if op == "surf_press" else _abi.OP_STREAMFUNCTION
        _abi.check(self._L.pyomgpu_apply_op(self._ctx, code, _ptr(p, self.shape), _ptr(res, self.shape, True),
                                            _stream()))
        return res

    def make_inv_sfc(self):
        """Z of solve_streamfct.f90:381-422 (zero halo, zero on perimeters)."""
        Z = np.zeros(self.shape, order="F")
        _abi.check(self._L.pyomgpu_get_inv_diag(self._ctx, _ptr(Z), _stream()))
        return Z

    def line_integral(self, isle, uloc, vloc):
        """streamfct_init.f90:311-377 for island ``isle`` (1-based)."""
        out = C.c_double()
        _abi.check(self._L.pyomgpu_line_integral(self._ctx, int(isle), _ptr(uloc, self.shape),
                                                 _ptr(vloc, self.shape), C.byref(out), _stream()))
        return out.value

    # ---- one step on device arrays ------------------------------------------------------
    def _state(self, D, M):
        s = _abi.State()
        s.nz = M.nz
        s.taum1, s.tau, s.taup1 = int(M.taum1), int(M.tau), int(M.taup1)
        s.congr_max_iterations = int(M.congr_max_iterations)
        s.dt_mom, s.AB_eps, s.grav, s.rho_0 = float(M.dt_mom), float(M.AB_eps), float(M.grav), float(M.rho_0)
        s.congr_epsilon = float(M.congr_epsilon)
        for n in ("dzt", "dzw", "maskT", "maskU", "maskV", "rho", "u", "v", "du", "dv", "du_mix", "dv_mix",
                  "p_hydro", "psi", "dpsi", "dpsin"):
            t = D.get(n)
            setattr(s, n, None if t is None else t.data_ptr())
        return s

    def _run_step(self, M, fn, names_out):
        import torch
        dev = torch.device("cuda")
        D = {}
        for n in ("dzt", "dzw", "maskT", "maskU", "maskV", "rho", "u", "v", "du", "dv", "du_mix", "dv_mix",
                  "p_hydro", "psi", "dpsi", "dpsin"):
            a = getattr(M, n, None)
            if a is None:
                continue
            D[n] = _to_device_f(a, dev)
        s = self._state(D, M)
        info = _abi.SolveInfo()
        rc = fn(self._ctx, C.byref(s), C.byref(info), _stream())
        _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
        _warn_status(rc, fn.__name__)
        for n in names_out:
            a = getattr(M, n, None)
            if a is None:
                continue
            if _is_torch(a):
                continue  # updated in place
            a[...] = _from_device_f(D[n])
        M.congr_itts = int(s.congr_itts)
        return info.as_dict()

    def solve_streamfunction(self, M=None):
        """solve_streamfct.f90:10-120 on the model arrays."""
        M = M or self.M
        if self.nisle != int(getattr(M, "nisle", 0)):
            raise PyOMGPUError(_abi.ESTATE, "streamfunction_init / set_islands first")
        return self._run_step(M, self._L.pyomgpu_solve_streamfunction,
                              ("du", "dv", "u", "v", "p_hydro", "psi", "dpsi", "dpsin"))

    def solve_pressure(self, M=None):
        """solve_pressure.f90:10-82 on the model arrays."""
        M = M or self.M
        return self._run_step(M, self._L.pyomgpu_solve_pressure, ("du", "dv", "u", "v", "p_hydro", "psi"))

    _MOM_IN = ("dzt", "dzw", "tantr", "maskT", "maskU", "maskV", "maskW", "coriolis_t", "area_t", "area_u", "area_v",
               "surface_taux", "surface_tauy", "kappaM", "u", "v", "w", "du", "dv", "du_mix", "dv_mix")

    def _momentum_struct(self, M):
        import torch
        dev = torch.device("cuda")
        D = {n: _to_device_f(getattr(M, n), dev) for n in self._MOM_IN}
        kb = M.kbot
        D["kbot"] = kb if _is_torch(kb) else torch.from_numpy(
            np.ascontiguousarray(np.asfortranarray(kb, dtype=np.int32).T)).to(dev)
        m = _abi.Momentum()
        m.nz, m.taum1, m.tau, m.taup1 = int(M.nz), int(M.taum1), int(M.tau), int(M.taup1)
        m.coord_degree = int(bool(M.coord_degree))
        m.enable_hor_friction = int(bool(M.enable_hor_friction))
        m.enable_hor_friction_cos_scaling = int(bool(M.enable_hor_friction_cos_scaling))
        m.hor_friction_cospower = int(M.hor_friction_cosPower)
        m.enable_bottom_friction = int(bool(M.enable_bottom_friction))
        m.enable_implicit_vert_friction = int(bool(M.enable_implicit_vert_friction))
        m.dt_mom, m.A_h, m.r_bot = float(M.dt_mom), float(M.A_h), float(M.r_bot)
        for n, t in D.items():
            setattr(m, n, t.data_ptr())
        return m, D

    def momentum(self, M=None):
        """momentum.f90:4-152 up to the external-mode solve (Coriolis, metric
        terms, wind stress, advection, implicit vertical friction with
        M.kappaM, harmonic and linear bottom friction as enabled on M):
        writes du, dv at tau, du_mix and dv_mix (pyomgpu_momentum_tendencies).
        Host arrays are copied in and out; CUDA tensors are used in place."""
        M = M or self.M
        m, D = self._momentum_struct(M)
        _abi.check(self._L.pyomgpu_momentum_tendencies(self._ctx, C.byref(m), _stream()))
        for n in ("du", "dv", "du_mix", "dv_mix", "u", "v"):
            a = getattr(M, n)
            if not _is_torch(a):
                a[...] = _from_device_f(D[n])

    def vertical_velocity(self, M=None, level=None):
        """The end of the reference's step for ``level`` (default taup1): the
        cyclic halos of u, v (main.f90:114-117), then vertical_velocity.f90:
        w(:,:,:,level) from u, v at level.  Host arrays u, v, w are written
        back; CUDA tensors are updated in place."""
        M = M or self.M
        m, D = self._momentum_struct(M)
        lev = int(M.taup1 if level is None else level)
        _abi.check(self._L.pyomgpu_vertical_velocity(self._ctx, C.byref(m), lev, _stream()))
        for n in ("u", "v", "w"):
            a = getattr(M, n)
            if not _is_torch(a):
                a[...] = _from_device_f(D[n])


# ---------------------------------------------------------------------------
def _host(a):
    if _is_torch(a):
        return a.detach().cpu().numpy()
    return a


def _torch_like(p):
    import torch
    return torch.zeros(tuple(reversed(p.shape)), dtype=torch.float64, device=p.device).permute(
        *reversed(range(p.dim())))


def _to_device_f(a, dev):
    """Fortran-ordered CUDA tensor view of ``a`` (torch tensors pass through)."""
    import torch
    if _is_torch(a):
        _ptr(a)
        return a
    a = np.asfortranarray(a)
    t = torch.from_numpy(np.ascontiguousarray(a.T)).to(dev)  # C-order of the transpose == F-order of a
    return t


def _from_device_f(t):
    return np.asfortranarray(t.cpu().numpy().T)


def _alloc_islands(M, nisle, maxb):
    X, Y = M.nx + 2 * M.onx, M.ny + 2 * M.onx
    M.nisle = nisle
    M.boundary = np.zeros((nisle, maxb, 2), dtype=np.int32, order="F")
    M.line_dir = np.zeros((nisle, maxb, 2), dtype=np.int32, order="F")
    M.nr_boundary = np.zeros(nisle, dtype=np.int32)
    M.psin = np.zeros((X, Y, nisle), order="F")
    M.dpsin = np.zeros((nisle, 3), order="F")
    M.line_psin = np.zeros((nisle, nisle), order="F")


def _ctx_for(M) -> ExternalMode:
    em = getattr(M, "_pyomgpu", None)
    if em is None:
        em = ExternalMode(M)
        M._pyomgpu = em
    return em


# ---- module-level functions with the reference names (operate on M's state) ----------
def streamfunction_init(M, **kw):
    return _ctx_for(M).streamfunction_init(M, **kw)


def solve_streamfunction(M):
    return _ctx_for(M).solve_streamfunction(M)


def solve_pressure(M):
    return _ctx_for(M).solve_pressure(M)


def congrad_streamfunction(M, forc, sol):
    it, conv, _ = _ctx_for(M).congrad_streamfunction(forc, sol)
    M.congr_itts = it
    return it, conv


def congrad_surf_press(M, forc):
    psi = M.psi[:, :, M.taup1 - 1]
    view = psi if _is_torch(psi) or psi.flags.f_contiguous else None
    if view is None:
        raise PyOMGPUError(_abi.EINVAL, "psi(:,:,taup1) must be contiguous")
    it, _ = _ctx_for(M).congrad_surf_press(forc, view)
    M.congr_itts = it
    return it


_BATCH_KERNELS = {"auto": 0, "queue": 1, "resident": 2}


def congrad_streamfunction_batch(contexts, forcs, sols, eps=1e-12, max_it=1000000, rtol=0.0, kernel=None):
    """Many congrad_streamfunction solves (solve_streamfct.f90:153-327) in one
    call: solve k on ``contexts[k]`` (an :class:`ExternalMode`; repeats
    allowed) with ``forcs[k]`` (None = zero forcing) and ``sols[k]`` updated
    in place.  The reference runs such solves one after another
    (streamfct_init.f90:272-287).  ``rtol`` > 0 adds the relative-residual
    stop.  ``kernel`` ("auto", "queue" = the work-queue kernel, "resident" =
    groups of SMs running on-chip solves side by side) is stored on
    ``contexts[0]`` for this and later calls; None keeps its setting.
    Returns one info dict per solve."""
    L = _abi.load()
    n = len(contexts)
    if n < 1 or len(forcs) != n or len(sols) != n:
        raise PyOMGPUError(_abi.EINVAL, "contexts, forcs and sols must have the same non-zero length")
    if kernel is not None:
        if kernel not in _BATCH_KERNELS:
            raise ValueError(f"kernel must be one of {sorted(_BATCH_KERNELS)}")
        _abi.check(L.pyomgpu_set_batch_kernel(contexts[0]._ctx, _BATCH_KERNELS[kernel]))
    VP = C.c_void_p * n
    ctx = VP(*[em._ctx for em in contexts])
    fp = VP(*[None if f is None else _ptr(f, em.shape).value for em, f in zip(contexts, forcs)])
    sp = VP(*[_ptr(s, em.shape, True).value for em, s in zip(contexts, sols)])
    infos = (_abi.SolveInfo * n)()
    rc = L.pyomgpu_congrad_streamfunction_batch(ctx, n, fp, sp, float(eps), int(max_it), float(rtol), infos,
                                                _stream())
    _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
    _warn_status(rc, "congrad_streamfunction_batch")
    return [i.as_dict() for i in infos]


def batch_schedule(owner, count):
    """Diagnostics of the last resident batch whose first context was
    ``owner``: per solve (call order) its device start and end in ms after
    the earliest start, and the SMs it used."""
    L = _abi.load()
    st, en = np.zeros(count), np.zeros(count)
    bl = np.zeros(count, dtype=np.int32)
    _abi.check(L.pyomgpu_batch_schedule(owner._ctx, int(count), C.c_void_p(st.ctypes.data),
                                        C.c_void_p(en.ctypes.data), C.c_void_p(bl.ctypes.data)))
    return st, en, bl


def island_boundaries(M, mnisle=0, maxipp=0, maxq=0, gpu=False):
    """Island labels and traced perimeters (streamfct_init.f90:35-267):
    returns (boundary, line_dir, nr_boundary) in the reference layout.  On
    the host (the flood-fill restatement) or, with ``gpu``, on the GPU."""
    L = _abi.load()
    kbot = np.asfortranarray(_host(M.kbot), dtype=np.int32)
    n, mb = C.c_int32(), C.c_int32()
    args = (int(M.nx), int(M.ny), int(bool(M.enable_cyclic_x)), C.c_void_p(kbot.ctypes.data), int(mnisle),
            int(maxipp), int(maxq))
    fn = L.pyomgpu_island_boundaries_gpu if gpu else L.pyomgpu_island_boundaries
    tail = (_stream(),) if gpu else ()
    _abi.check(fn(*args, C.byref(n), C.byref(mb), None, None, None, *tail))
    b = np.zeros((n.value, mb.value, 2), dtype=np.int32, order="F")
    d = np.zeros_like(b)
    nr = np.zeros(n.value, dtype=np.int32)
    _abi.check(fn(*args, C.byref(n), C.byref(mb), C.c_void_p(b.ctypes.data), C.c_void_p(d.ctypes.data),
                  C.c_void_p(nr.ctypes.data), *tail))
    return b, d, nr


def isleperim(kmt, cyclic, mnisle=0, maxipp=0, maxq=0):
    """island_module.f90:7-127 on an (imt, jmt) int map: returns (map, nisle, nippts)."""
    L = _abi.load()
    k = np.asfortranarray(kmt, dtype=np.int32)
    imt, jmt = k.shape
    mp = np.zeros_like(k)
    n = C.c_int32()
    cap = mnisle if mnisle > 0 else 1000
    nip = np.zeros(cap + 2, dtype=np.int32)
    _abi.check(L.pyomgpu_isleperim(C.c_void_p(k.ctypes.data), imt, jmt, int(bool(cyclic)), int(mnisle), int(maxipp),
                                   int(maxq), C.c_void_p(mp.ctypes.data), C.byref(n), C.c_void_p(nip.ctypes.data)))
    return mp, n.value, nip[:n.value].copy()
