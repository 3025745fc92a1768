"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle is a plain-C FP64 restatement of pyOM2's external-mode solve
(pyom_oracle.c).  Only tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of bench.py import this module; the product package never does.

Parity status: pinned to the reference's own source.  No Fortran compiler
exists in this image, so tests/golden/make_ref_golden.py runs pyOM2's Fortran
routines through the Fortran-subset translator oracle/f90sub.py and commits
their outputs; tests/test_oracle_vs_reference_source.py holds this oracle to
them bit for bit (rounding level only where LAPACK's DGESV enters).
Known-answer tests (manufactured solutions, hand-built island maps, operator
identities) and further committed fixtures check it as well.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

# limits of the reference (streamfct_init.f90:16, island_module.f90:22)
MNISLE, MAXIPP, MAXQ = 1000, 20000, 10000


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "pyom_oracle.c")
    deps = [src, os.path.join(HERE, "pyom_oracle_mt.c"), os.path.join(HERE, "pyom_oracle.h"),
            os.path.join(HERE, "Makefile")]
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < max(map(os.path.getmtime, deps)):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


class OGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("cyclic_x", C.c_int), ("cyclic_y", C.c_int),
                ("dxt", C.c_void_p), ("dxu", C.c_void_p), ("dyt", C.c_void_p), ("dyu", C.c_void_p),
                ("cost", C.c_void_p), ("cosu", C.c_void_p)]


class OGrid3(C.Structure):
    _fields_ = [("g", OGrid), ("nz", C.c_int), ("dzt", C.c_void_p), ("dzw", C.c_void_p), ("maskT", C.c_void_p),
                ("maskU", C.c_void_p), ("maskV", C.c_void_p), ("maskW", C.c_void_p)]


class OState3(C.Structure):
    _fields_ = [("taum1", C.c_int), ("tau", C.c_int), ("taup1", C.c_int), ("itt", C.c_int),
                ("dt_mom", C.c_double), ("AB_eps", C.c_double), ("congr_epsilon_non_hydro", C.c_double),
                ("congr_max_itts_non_hydro", C.c_int), ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("dw", C.c_void_p), ("dw_mix", C.c_void_p), ("p_non_hydro", C.c_void_p),
                ("congr_itts_non_hydro", C.c_int), ("status", C.c_int)]


class OIslands(C.Structure):
    _fields_ = [("nisle", C.c_int), ("max_boundary", C.c_int), ("boundary", C.c_void_p),
                ("line_dir", C.c_void_p), ("nr_boundary", C.c_void_p)]


class OInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("status", C.c_int),
                ("estimated_error", C.c_double)]


class OState(C.Structure):
    _fields_ = [("nz", C.c_int), ("taum1", C.c_int), ("tau", C.c_int), ("taup1", C.c_int),
                ("enable_free_surface", C.c_int),
                ("dt_mom", C.c_double), ("AB_eps", C.c_double), ("grav", C.c_double), ("rho_0", C.c_double),
                ("congr_epsilon", C.c_double), ("congr_max_iterations", C.c_int),
                ("dzt", C.c_void_p), ("dzw", C.c_void_p),
                ("hu", C.c_void_p), ("hv", C.c_void_p), ("hur", C.c_void_p), ("hvr", C.c_void_p),
                ("maskT", C.c_void_p), ("maskU", C.c_void_p), ("maskV", C.c_void_p),
                ("rho", C.c_void_p), ("u", C.c_void_p), ("v", C.c_void_p), ("du", C.c_void_p),
                ("dv", C.c_void_p), ("du_mix", C.c_void_p), ("dv_mix", C.c_void_p),
                ("p_hydro", C.c_void_p), ("psi", C.c_void_p), ("dpsi", C.c_void_p),
                ("psin", C.c_void_p), ("dpsin", C.c_void_p), ("line_psin", C.c_void_p),
                ("congr_itts", C.c_int), ("status", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        d, i, v, p = C.c_double, C.c_int, None, C.c_void_p
        sig = {
            "o_setcyclic_xy": (v, [p, p]),
            "o_make_coeff_streamfunction": (v, [p, p, p, p]),
            "o_make_coeff_surf_press": (v, [p, p, p, p, i, d, d, p]),
            "o_apply_op": (v, [p, p, p, p]),
            "o_make_inv_sfc": (v, [p, p, p, p]),
            "o_dot_sfc": (d, [p, p, p]),
            "o_absmax_sfc": (d, [p, p]),
            "o_dot_sfp": (d, [p, p, p, p]),
            "o_absmax_sfp": (d, [p, p, p]),
            "o_congrad_streamfunction": (i, [p, p, p, p, p, d, i, d, p]),
            "o_congrad_surf_press": (i, [p, p, p, p, p, d, i, d, p]),
            "o_congrad_streamfunction_mt": (i, [p, p, p, p, p, d, i, d, i, p]),
            "o_max_threads": (i, []),
            "o_rel_residual": (d, [p, p, p, p, p]),
            "o_isleperim": (i, [p, p, i, i, i, i, i, i, p, p, p, p, p, p]),
            "o_island_map": (i, [p, p, i, i, i, p, p, p]),
            "o_island_trace": (i, [p, p, i, i, i, i, i, p, p, p]),
            "o_line_integral": (d, [p, p, i, p, p, p]),
            "o_psin_solve": (i, [p, p, p, d, i, d, i, p, p]),
            "o_congrad_streamfunction_w": (i, [p, p, p, p, p, d, i, d, p]),
            "o_line_psin": (i, [p, p, p, p, p, p, p, p]),
            "o_dgesv": (i, [i, p, p, p]),
            "o_solve_streamfunction": (i, [p, p, p, p]),
            "o_solve_pressure": (i, [p, p, p]),
            "o_setcyclic_xyz": (v, [p, p]),
            "o_make_coeff_non_hydro": (v, [p, p]),
            "o_apply_op_3d": (v, [p, p, p, p]),
            "o_dot_3d": (d, [p, p, p]),
            "o_absmax_3d": (d, [p, p]),
            "o_congrad_non_hydro": (i, [p, p, p, p, d, i, p]),
            "o_solve_non_hydrostatic": (i, [p, p, p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(_lib, name)
            f.restype = res
            f.argtypes = args
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _f64(a):
    a = np.asarray(a)
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim <= 1), "need F-ordered float64"
    return a


class Oracle:
    """Oracle bound to one model grid (a :class:`pyom2_b200.model.ModelState`)."""

    def __init__(self, M):
        self.M = M
        self._keep = [np.ascontiguousarray(x) for x in (M.dxt, M.dxu, M.dyt, M.dyu, M.cost, M.cosu)]
        k = self._keep
        self.g = OGrid(M.nx, M.ny, int(M.enable_cyclic_x), int(M.enable_cyclic_y),
                       _p(k[0]), _p(k[1]), _p(k[2]), _p(k[3]), _p(k[4]), _p(k[5]))
        self.gp = C.byref(self.g)
        self.shape = M.shape2d

    # --- operators --------------------------------------------------------------
    def make_coeff_streamfunction(self):
        cf = np.zeros(self.shape + (3, 3), order="F")
        lib().o_make_coeff_streamfunction(self.gp, _p(_f64(self.M.hur)), _p(_f64(self.M.hvr)), _p(cf))
        return cf

    def make_coeff_surf_press(self, free_surface=None, grav=None, dt_mom=None):
        M = self.M
        cf = np.zeros(self.shape + (3, 3), order="F")
        maskM = np.asfortranarray(M.maskT[:, :, -1])
        fs = M.enable_free_surface if free_surface is None else free_surface
        lib().o_make_coeff_surf_press(self.gp, _p(_f64(M.hu)), _p(_f64(M.hv)), _p(maskM), int(fs),
                                      float(M.grav if grav is None else grav),
                                      float(M.dt_mom if dt_mom is None else dt_mom), _p(cf))
        return cf

    def apply_op(self, cf, p):
        res = np.zeros(self.shape, order="F")
        lib().o_apply_op(self.gp, _p(cf), _p(_f64(p)), _p(res))
        return res

    def islands_struct(self, M=None):
        M = M or self.M
        if M.nisle == 0 or M.boundary is None:
            return None, None
        keep = (np.asfortranarray(M.boundary, dtype=np.int32), np.asfortranarray(M.line_dir, dtype=np.int32),
                np.ascontiguousarray(M.nr_boundary, dtype=np.int32))
        s = OIslands(int(M.nisle), int(M.boundary.shape[1]), _p(keep[0]), _p(keep[1]), _p(keep[2]))
        return s, keep

    def make_inv_sfc(self, cf):
        Z = np.zeros(self.shape, order="F")
        s, keep = self.islands_struct()
        lib().o_make_inv_sfc(self.gp, _p(cf), C.byref(s) if s is not None else None, _p(Z))
        return Z

    def setcyclic_xy(self, a):
        lib().o_setcyclic_xy(self.gp, _p(_f64(a)))

    # --- solvers ----------------------------------------------------------------
    def congrad_streamfunction(self, cf, forc, sol, eps=None, max_it=None, rtol=0.0):
        """Runs the CG in place on ``sol``; returns an info dict."""
        M = self.M
        s, keep = self.islands_struct()
        info = OInfo()
        lib().o_congrad_streamfunction(self.gp, _p(cf), C.byref(s) if s is not None else None,
                                       _p(_f64(forc)), _p(_f64(sol)),
                                       float(M.congr_epsilon if eps is None else eps),
                                       int(M.congr_max_iterations if max_it is None else max_it),
                                       float(rtol), C.byref(info))
        return dict(iterations=info.iterations, converged=bool(info.converged), status=info.status,
                    estimated_error=info.estimated_error)

    def congrad_streamfunction_w(self, cf, forc, sol, eps=0.0, max_it=10**6, rtol=0.0):
        """congrad_streamfunction with cell-area-weighted inner products (exact
        Jacobi-PCG on the symmetric S = D A), in place on ``sol``."""
        s, keep = self.islands_struct()
        info = OInfo()
        lib().o_congrad_streamfunction_w(self.gp, _p(cf), C.byref(s) if s is not None else None,
                                         _p(_f64(forc)), _p(_f64(sol)), float(eps), int(max_it), float(rtol),
                                         C.byref(info))
        return dict(iterations=info.iterations, converged=bool(info.converged), status=info.status,
                    estimated_error=info.estimated_error)

    def congrad_streamfunction_mt(self, cf, forc, sol, eps=None, max_it=None, rtol=0.0, threads=0):
        """congrad_streamfunction as the reference's MPI build runs it on
        ``threads`` processes (row bands, partial sums combined in rank order),
        on OpenMP threads; in place on ``sol``.  For timing the reference
        algorithm on the host cores."""
        M = self.M
        s, keep = self.islands_struct()
        info = OInfo()
        lib().o_congrad_streamfunction_mt(self.gp, _p(cf), C.byref(s) if s is not None else None,
                                          _p(_f64(forc)), _p(_f64(sol)),
                                          float(M.congr_epsilon if eps is None else eps),
                                          int(M.congr_max_iterations if max_it is None else max_it),
                                          float(rtol), int(threads), C.byref(info))
        return dict(iterations=info.iterations, converged=bool(info.converged), status=info.status,
                    estimated_error=info.estimated_error)

    def congrad_surf_press(self, cf, forc, psi, eps=None, max_it=None, rtol=0.0):
        M = self.M
        maskM = np.asfortranarray(M.maskT[:, :, -1])
        info = OInfo()
        lib().o_congrad_surf_press(self.gp, _p(cf), _p(maskM), _p(_f64(forc)), _p(_f64(psi)),
                                   float(M.congr_epsilon if eps is None else eps),
                                   int(M.congr_max_iterations if max_it is None else max_it),
                                   float(rtol), C.byref(info))
        return dict(iterations=info.iterations, converged=bool(info.converged), status=info.status,
                    estimated_error=info.estimated_error)

    def rel_residual(self, cf, Z, forc, sol):
        return lib().o_rel_residual(self.gp, _p(cf), _p(Z), _p(_f64(forc)), _p(_f64(sol)))

    # --- islands ------------------------------------------------------------------
    def island_map(self, mnisle=MNISLE, maxipp=MAXIPP, maxq=MAXQ):
        M = self.M
        allmap = np.zeros(self.shape, dtype=np.int32, order="F")
        nisle = C.c_int(0)
        maxb = C.c_int(0)
        kbot = np.asfortranarray(M.kbot, dtype=np.int32)
        rc = lib().o_island_map(self.gp, _p(kbot), mnisle, maxipp, maxq, _p(allmap), C.byref(nisle), C.byref(maxb))
        return rc, allmap, nisle.value, maxb.value

    def island_trace(self, allmap, nisle, max_boundary, mnisle=MNISLE, maxipp=MAXIPP, maxq=MAXQ):
        b = np.zeros((nisle, max_boundary, 2), dtype=np.int32, order="F")
        d = np.zeros((nisle, max_boundary, 2), dtype=np.int32, order="F")
        nr = np.zeros(nisle, dtype=np.int32)
        rc = lib().o_island_trace(self.gp, _p(allmap), nisle, max_boundary, mnisle, maxipp, maxq, _p(b), _p(d),
                                  _p(nr))
        return rc, b, d, nr

    def isleperim(self, kmt, cyclic, mnisle=MNISLE, maxipp=MAXIPP, maxq=MAXQ):
        kmt = np.asfortranarray(kmt, dtype=np.int32)
        imt, jmt = kmt.shape
        mp = np.zeros_like(kmt)
        nisle = C.c_int(0)
        nerr = C.c_int(0)
        nippts = np.zeros(mnisle + 2, dtype=np.int32)
        iofs = np.zeros(mnisle + 2, dtype=np.int32)
        iperm = np.zeros(maxipp + 2, dtype=np.int32)
        jperm = np.zeros(maxipp + 2, dtype=np.int32)
        rc = lib().o_isleperim(_p(kmt), _p(mp), imt, jmt, int(cyclic), mnisle, maxipp, maxq, C.byref(nisle),
                               _p(nippts), _p(iofs), _p(iperm), _p(jperm), C.byref(nerr))
        return rc, mp, nisle.value, nippts[1:nisle.value + 1].copy(), nerr.value

    def line_integral(self, isle, uloc, vloc):
        s, keep = self.islands_struct()
        err = C.c_int(0)
        v = lib().o_line_integral(self.gp, C.byref(s), int(isle), _p(_f64(uloc)), _p(_f64(vloc)), C.byref(err))
        if err.value:
            raise RuntimeError("line integral: missing line_dir")
        return v

    def streamfunction_init(self, eps=None, max_it=None, mnisle=MNISLE, maxipp=MAXIPP, maxq=MAXQ, psin_rtol=0.0,
                            psin_weighted=False):
        """streamfct_init.f90:7-304 on the oracle; fills M's island arrays.
        ``psin_rtol`` > 0: the psin solves stop at that residual relative to
        the initial one (reference stop off), with cell-area-weighted inner
        products if ``psin_weighted`` (not in the reference)."""
        M = self.M
        rc, allmap, nisle, maxb = self.island_map(mnisle, maxipp, maxq)
        if rc:
            raise RuntimeError(f"island map failed ({rc})")
        rc, b, d, nr = self.island_trace(allmap, nisle, maxb, mnisle, maxipp, maxq)
        if rc:
            raise RuntimeError(f"island trace failed ({rc})")
        M.allocate_islands(nisle, maxb)
        M.boundary[...] = b
        M.line_dir[...] = d
        M.nr_boundary[...] = nr
        cf = self.make_coeff_streamfunction()
        s, keep = self.islands_struct()
        iters = np.zeros(nisle, dtype=np.int32)
        if psin_rtol > 0:
            eps, max_it = 0.0, max(10**6, max_it or 0)
        st = lib().o_psin_solve(self.gp, _p(cf), C.byref(s), float(M.congr_epsilon if eps is None else eps),
                                int(M.congr_max_iterations if max_it is None else max_it), float(psin_rtol),
                                int(bool(psin_weighted)), _p(M.psin), _p(iters))
        mU = np.asfortranarray(M.maskU[:, :, -1])
        mV = np.asfortranarray(M.maskV[:, :, -1])
        err = lib().o_line_psin(self.gp, C.byref(s), _p(M.psin), _p(_f64(M.hur)), _p(_f64(M.hvr)), _p(mU), _p(mV),
                                _p(M.line_psin))
        if err:
            raise RuntimeError("line_psin: missing line_dir")
        return dict(allmap=allmap, psin_iterations=iters, status=st)

    def dgesv(self, a, b):
        a = np.asfortranarray(a, dtype=np.float64).copy(order="F")
        b = np.ascontiguousarray(b, dtype=np.float64).copy()
        n = a.shape[0]
        ipiv = np.zeros(n, dtype=np.int32)
        info = lib().o_dgesv(n, _p(a), _p(ipiv), _p(b))
        return info, b

    def _state(self, M):
        keep = []

        def P(a, dtype=np.float64):
            if a is None:
                return None
            assert a.dtype == dtype and (a.flags.f_contiguous or a.ndim <= 1)
            keep.append(a)
            return a.ctypes.data

        s = OState()
        s.nz = M.nz
        s.taum1, s.tau, s.taup1 = M.taum1, M.tau, M.taup1
        s.enable_free_surface = int(M.enable_free_surface)
        s.dt_mom, s.AB_eps, s.grav, s.rho_0 = M.dt_mom, M.AB_eps, M.grav, M.rho_0
        s.congr_epsilon, s.congr_max_iterations = M.congr_epsilon, M.congr_max_iterations
        for name in ("dzt", "dzw", "hu", "hv", "hur", "hvr", "maskT", "maskU", "maskV", "rho", "u", "v", "du",
                     "dv", "du_mix", "dv_mix", "p_hydro", "psi", "dpsi", "psin", "dpsin", "line_psin"):
            setattr(s, name, P(getattr(M, name)))
        return s, keep

    def solve_streamfunction(self, M=None, cf=None):
        M = M or self.M
        cf = self.make_coeff_streamfunction() if cf is None else cf
        s, keep = self._state(M)
        isl, keep2 = self.islands_struct(M)
        rc = lib().o_solve_streamfunction(self.gp, _p(cf), C.byref(isl) if isl is not None else None, C.byref(s))
        M.congr_itts = s.congr_itts
        return rc

    def solve_pressure(self, M=None, cf=None):
        M = M or self.M
        cf = self.make_coeff_surf_press() if cf is None else cf
        s, keep = self._state(M)
        rc = lib().o_solve_pressure(self.gp, _p(cf), C.byref(s))
        M.congr_itts = s.congr_itts
        return rc


class Oracle3D:
    """Oracle of the non-hydrostatic pressure solve (non_hydrostatic.f90) bound
    to one model state (3-D fields (nx+4, ny+4, nz), Fortran order)."""

    def __init__(self, M):
        if M.nz < 2:
            raise ValueError("make_coeff_non_hydro reads maskW(:,:,nz-1): nz >= 2")
        self.M = M
        self.o2 = Oracle(M)
        self._keep = [np.ascontiguousarray(M.dzt), np.ascontiguousarray(M.dzw)] + \
            [np.asfortranarray(getattr(M, n)) for n in ("maskT", "maskU", "maskV", "maskW")]
        k = self._keep
        self.g = OGrid3(self.o2.g, M.nz, *[_p(a) for a in k])
        self.gp = C.byref(self.g)
        self.shape = M.shape2d + (M.nz,)

    def make_coeff(self):
        cf = np.zeros(self.shape + (3, 3, 3), order="F")
        lib().o_make_coeff_non_hydro(self.gp, _p(cf))
        return cf

    def apply_op(self, cf, p):
        res = np.zeros(self.shape, order="F")
        lib().o_apply_op_3d(self.gp, _p(cf), _p(_f64(p)), _p(res))
        return res

    def dot(self, a, b):
        return lib().o_dot_3d(self.gp, _p(_f64(a)), _p(_f64(b)))

    def absmax(self, a):
        return lib().o_absmax_3d(self.gp, _p(_f64(a)))

    def setcyclic_xyz(self, a):
        lib().o_setcyclic_xyz(self.gp, _p(_f64(a)))

    def congrad(self, cf, forc, p, eps=None, max_it=None):
        """congrad_non_hydro in place on ``p`` (p_non_hydro(:,:,:,taup1))."""
        M = self.M
        info = OInfo()
        lib().o_congrad_non_hydro(self.gp, _p(cf), _p(_f64(forc)), _p(_f64(p)),
                                  float(M.congr_epsilon_non_hydro if eps is None else eps),
                                  int(M.congr_max_itts_non_hydro if max_it is None else max_it), C.byref(info))
        return dict(iterations=info.iterations, converged=bool(info.converged), status=info.status,
                    estimated_error=info.estimated_error)

    def solve_non_hydrostatic(self, M=None, cf=None):
        """non_hydrostatic.f90:5-63 in place on M's u, v, w, p_non_hydro;
        sets M.congr_itts_non_hydro and returns the solver status."""
        M = M or self.M
        cf = self.make_coeff() if cf is None else cf
        keep = []

        def P(a):
            assert a.dtype == np.float64 and a.flags.f_contiguous
            keep.append(a)
            return a.ctypes.data

        s = OState3()
        s.taum1, s.tau, s.taup1, s.itt = M.taum1, M.tau, M.taup1, int(M.itt)
        s.dt_mom, s.AB_eps = float(M.dt_mom), float(M.AB_eps)
        s.congr_epsilon_non_hydro = float(M.congr_epsilon_non_hydro)
        s.congr_max_itts_non_hydro = int(M.congr_max_itts_non_hydro)
        for n in ("u", "v", "w", "dw", "dw_mix", "p_non_hydro"):
            setattr(s, n, P(getattr(M, n)))
        rc = lib().o_solve_non_hydrostatic(self.gp, _p(cf), C.byref(s))
        M.congr_itts_non_hydro = s.congr_itts_non_hydro
        return rc
