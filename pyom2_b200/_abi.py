"""ctypes binding of ``libpyomgpu.so`` (declarations in include/pyomgpu.h).

The library is the only compute path: if it cannot be loaded, or no CUDA
device is present, every solver call raises :class:`PyOMGPUError`.  There is
no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyomgpu.so")

OK, MAXITER, DIVERGED, NAN, TIMEOUT, SINGULAR = 0, 1, 2, 3, 4, 5
EINVAL, ECUDA, ENOMEM, EISLAND, ESTATE = -1, -2, -3, -4, -5
OP_STREAMFUNCTION, OP_SURF_PRESS = 0, 1
PREC_F64, PREC_F32 = 64, 32

STATUS_NAMES = {OK: "ok", MAXITER: "max iterations exceeded", DIVERGED: "solver diverging",
                NAN: "estimated error is NaN", TIMEOUT: "device grid-barrier time-out",
                SINGULAR: "island system singular (lapack info not zero)", EINVAL: "invalid argument",
                ECUDA: "CUDA error", ENOMEM: "out of device memory", EISLAND: "island set-up failed",
                ESTATE: "missing state"}

# every symbol include/pyomgpu.h declares
EXPORTS = ("pyomgpu_version", "pyomgpu_last_error", "pyomgpu_ctx_create", "pyomgpu_ctx_destroy",
           "pyomgpu_set_sync_timeout", "pyomgpu_inject_barrier_stall", "pyomgpu_set_cg_kernel", "pyomgpu_set_batch_kernel", "pyomgpu_batch_schedule", "pyomgpu_plan_batch", "pyomgpu_plan_cut",
           "pyomgpu_resident_layout", "pyomgpu_resident_layout32", "pyomgpu_resident_trace", "pyomgpu_set_psin_solve",
           "pyomgpu_momentum_tendencies", "pyomgpu_vertical_velocity", "pyomgpu_autotune", "pyomgpu_isleperim",
           "pyomgpu_island_boundaries", "pyomgpu_island_boundaries_gpu", "pyomgpu_streamfunction_init",
           "pyomgpu_island_sizes", "pyomgpu_get_islands", "pyomgpu_set_islands",
           "pyomgpu_congrad_streamfunction", "pyomgpu_congrad_streamfunction_noalloc",
           "pyomgpu_congrad_streamfunction_batch",
           "pyomgpu_congrad_surf_press", "pyomgpu_solve_rtol",
           "pyomgpu_apply_op", "pyomgpu_get_inv_diag", "pyomgpu_line_integral",
           "pyomgpu_solve_streamfunction", "pyomgpu_solve_pressure",
           "pyomgpu_solve_streamfunction_begin", "pyomgpu_solve_streamfunction_end",
           "pyomgpu_conv3x3_bf16", "pyomgpu_precond_num_params", "pyomgpu_precond_create",
           "pyomgpu_precond_destroy", "pyomgpu_precond_rebind", "pyomgpu_precond_set_params", "pyomgpu_precond_get_params",
           "pyomgpu_precond_get_grads", "pyomgpu_precond_apply", "pyomgpu_precond_train_step",
           "pyomgpu_unet_forward_backward", "pyomgpu_solve_fcg",
           "pyomgpu_nh_create", "pyomgpu_nh_destroy", "pyomgpu_nh_set_sync_timeout",
           "pyomgpu_nh_inject_barrier_stall", "pyomgpu_nh_set_grid", "pyomgpu_nh_set_brick", "pyomgpu_nh_set_stages", "pyomgpu_nh_set_variant",
           "pyomgpu_apply_op_3d",
           "pyomgpu_congrad_non_hydro", "pyomgpu_solve_non_hydrostatic")


class PyOMGPUError(RuntimeError):
    def __init__(self, code, msg=""):
        self.code = code
        super().__init__(f"[{code}] {STATUS_NAMES.get(code, 'error')}: {msg}")


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("onx", C.c_int32),
                ("enable_cyclic_x", C.c_int32), ("enable_cyclic_y", C.c_int32),
                ("enable_free_surface", C.c_int32), ("grav", C.c_double), ("dt_mom", C.c_double),
                ("dxt", C.c_void_p), ("dxu", C.c_void_p), ("dyt", C.c_void_p), ("dyu", C.c_void_p),
                ("cost", C.c_void_p), ("cosu", C.c_void_p), ("hur", C.c_void_p), ("hvr", C.c_void_p),
                ("hu", C.c_void_p), ("hv", C.c_void_p), ("maskT_top", C.c_void_p),
                ("maskU_top", C.c_void_p), ("maskV_top", C.c_void_p)]


class Grid3D(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("onx", C.c_int32),
                ("enable_cyclic_x", C.c_int32), ("enable_cyclic_y", C.c_int32),
                ("dxt", C.c_void_p), ("dxu", C.c_void_p), ("dyt", C.c_void_p), ("dyu", C.c_void_p),
                ("cost", C.c_void_p), ("cosu", C.c_void_p), ("dzt", C.c_void_p), ("dzw", C.c_void_p),
                ("maskT", C.c_void_p), ("maskU", C.c_void_p), ("maskV", C.c_void_p), ("maskW", C.c_void_p)]


class State3D(C.Structure):
    _fields_ = [("taum1", C.c_int32), ("tau", C.c_int32), ("taup1", C.c_int32), ("itt", C.c_int32),
                ("congr_max_itts_non_hydro", C.c_int32), ("congr_itts_non_hydro", C.c_int32),
                ("dt_mom", C.c_double), ("AB_eps", C.c_double), ("congr_epsilon_non_hydro", C.c_double),
                ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p), ("dw", C.c_void_p),
                ("dw_mix", C.c_void_p), ("p_non_hydro", C.c_void_p)]


class Islands(C.Structure):
    _fields_ = [("nisle", C.c_int32), ("max_boundary", C.c_int32), ("boundary", C.c_void_p),
                ("line_dir", C.c_void_p), ("nr_boundary", C.c_void_p)]


class Momentum(C.Structure):
    """pyomgpu_momentum (include/pyomgpu.h)."""
    _fields_ = [("nz", C.c_int32), ("taum1", C.c_int32), ("tau", C.c_int32), ("taup1", C.c_int32),
                ("coord_degree", C.c_int32), ("enable_hor_friction", C.c_int32),
                ("enable_hor_friction_cos_scaling", C.c_int32), ("hor_friction_cospower", C.c_int32),
                ("enable_bottom_friction", C.c_int32), ("enable_implicit_vert_friction", C.c_int32),
                ("dt_mom", C.c_double), ("A_h", C.c_double), ("r_bot", C.c_double)] + [
        (n, C.c_void_p) for n in ("dzt", "dzw", "tantr", "maskT", "maskU", "maskV", "maskW", "kbot", "coriolis_t",
                                  "area_t", "area_u", "area_v", "surface_taux", "surface_tauy", "kappaM", "u", "v",
                                  "w", "du", "dv", "du_mix", "dv_mix")]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("converged", C.c_int32), ("status", C.c_int32),
                ("outer_iterations", C.c_int32), ("estimated_error", C.c_double),
                ("rel_residual", C.c_double), ("device_ms", C.c_double),
                ("kernel_launches", C.c_int32), ("fcg_iterations", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class State(C.Structure):
    _fields_ = [("nz", C.c_int32), ("taum1", C.c_int32), ("tau", C.c_int32), ("taup1", C.c_int32),
                ("congr_max_iterations", C.c_int32), ("congr_itts", C.c_int32),
                ("dt_mom", C.c_double), ("AB_eps", C.c_double), ("grav", C.c_double), ("rho_0", C.c_double),
                ("congr_epsilon", C.c_double),
                ("dzt", C.c_void_p), ("dzw", C.c_void_p), ("maskT", C.c_void_p), ("maskU", C.c_void_p),
                ("maskV", C.c_void_p), ("rho", C.c_void_p), ("u", C.c_void_p), ("v", C.c_void_p),
                ("du", C.c_void_p), ("dv", C.c_void_p), ("du_mix", C.c_void_p), ("dv_mix", C.c_void_p),
                ("p_hydro", C.c_void_p), ("psi", C.c_void_p), ("dpsi", C.c_void_p), ("dpsin", C.c_void_p)]


_lib = None


def load(path: str = LIB_PATH):
    """Load the library and declare the signatures (no GPU needed)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise PyOMGPUError(ESTATE, f"{path} is missing; run `python -m pyom2_b200.build`")
    L = C.CDLL(path)
    i32, d, vp = C.c_int32, C.c_double, C.c_void_p
    P = C.POINTER
    sig = {
        "pyomgpu_version": (i32, []),
        "pyomgpu_last_error": (C.c_char_p, []),
        "pyomgpu_ctx_create": (i32, [P(Grid), P(vp)]),
        "pyomgpu_ctx_destroy": (None, [vp]),
        "pyomgpu_set_sync_timeout": (i32, [vp, d]),
        "pyomgpu_inject_barrier_stall": (i32, [vp, i32]),
        "pyomgpu_set_cg_kernel": (i32, [vp, i32]),
        "pyomgpu_set_batch_kernel": (i32, [vp, i32]),
        "pyomgpu_batch_schedule": (i32, [vp, i32, vp, vp, vp]),
        "pyomgpu_plan_batch": (i32, [i32, i32, vp, vp, i32, vp, vp, vp, vp]),
        "pyomgpu_plan_cut": (i32, [i32, i32, i32, C.c_int64, i32, i32, i32, vp, vp]),
        "pyomgpu_resident_layout": (i32, [vp, P(i32), P(i32), P(i32)]),
        "pyomgpu_resident_layout32": (i32, [vp, P(i32), P(i32), P(i32)]),
        "pyomgpu_set_psin_solve": (i32, [vp, C.c_double, i32]),
        "pyomgpu_momentum_tendencies": (i32, [vp, P(Momentum), vp]),
        "pyomgpu_vertical_velocity": (i32, [vp, P(Momentum), i32, vp]),
        "pyomgpu_resident_trace": (i32, [vp, vp, vp, C.c_double, i32, i32, P(C.c_uint64), P(i32), P(SolveInfo), vp]),
        "pyomgpu_autotune": (i32, [vp, i32, P(i32), P(i32), P(i32), P(d), vp]),
        "pyomgpu_isleperim": (i32, [vp, i32, i32, i32, i32, i32, i32, vp, P(i32), vp]),
        "pyomgpu_island_boundaries": (i32, [i32, i32, i32, vp, i32, i32, i32, P(i32), P(i32), vp, vp, vp]),
        "pyomgpu_island_boundaries_gpu": (i32, [i32, i32, i32, vp, i32, i32, i32, P(i32), P(i32), vp, vp, vp, vp]),
        "pyomgpu_streamfunction_init": (i32, [vp, vp, i32, i32, i32, d, i32, vp]),
        "pyomgpu_island_sizes": (i32, [vp, P(i32), P(i32)]),
        "pyomgpu_get_islands": (i32, [vp, vp, vp, vp, vp, vp, vp, vp]),
        "pyomgpu_set_islands": (i32, [vp, P(Islands), vp, vp, vp]),
        "pyomgpu_congrad_streamfunction": (i32, [vp, vp, vp, d, i32, P(SolveInfo), vp]),
        "pyomgpu_congrad_streamfunction_noalloc": (i32, [P(Grid), vp, vp, i32, vp, vp, d, i32, P(SolveInfo), vp]),
        "pyomgpu_congrad_streamfunction_batch": (i32, [P(vp), i32, P(vp), P(vp), d, i32, d, P(SolveInfo), vp]),
        "pyomgpu_congrad_surf_press": (i32, [vp, vp, vp, d, i32, P(SolveInfo), vp]),
        "pyomgpu_solve_rtol": (i32, [vp, vp, vp, d, i32, i32, P(SolveInfo), vp]),
        "pyomgpu_apply_op": (i32, [vp, i32, vp, vp, vp]),
        "pyomgpu_get_inv_diag": (i32, [vp, vp, vp]),
        "pyomgpu_line_integral": (i32, [vp, i32, vp, vp, P(d), vp]),
        "pyomgpu_solve_streamfunction": (i32, [vp, P(State), P(SolveInfo), vp]),
        "pyomgpu_solve_pressure": (i32, [vp, P(State), P(SolveInfo), vp]),
        "pyomgpu_solve_streamfunction_begin": (i32, [vp, P(State), vp, vp]),
        "pyomgpu_solve_streamfunction_end": (i32, [vp, P(State), vp]),
        "pyomgpu_conv3x3_bf16": (i32, [i32, i32, i32, i32, vp, vp, vp, i32, i32, vp, vp, vp, vp, i32, vp]),
        "pyomgpu_precond_num_params": (C.c_int64, []),
        "pyomgpu_precond_create": (i32, [vp, i32, P(vp)]),
        "pyomgpu_precond_destroy": (None, [vp]),
        "pyomgpu_precond_rebind": (i32, [vp, vp]),
        "pyomgpu_precond_set_params": (i32, [vp, vp, C.c_int64]),
        "pyomgpu_precond_get_params": (i32, [vp, vp, C.c_int64]),
        "pyomgpu_precond_get_grads": (i32, [vp, vp, C.c_int64]),
        "pyomgpu_precond_apply": (i32, [vp, vp, vp, vp]),
        "pyomgpu_precond_train_step": (i32, [vp, vp, vp, C.c_float, P(C.c_float), vp]),
        "pyomgpu_unet_forward_backward": (i32, [vp, vp, vp, vp, vp]),
        "pyomgpu_solve_fcg": (i32, [vp, vp, vp, vp, d, i32, P(SolveInfo), vp]),
        "pyomgpu_nh_create": (i32, [P(Grid3D), P(vp)]),
        "pyomgpu_nh_destroy": (None, [vp]),
        "pyomgpu_nh_set_sync_timeout": (i32, [vp, d]),
        "pyomgpu_nh_inject_barrier_stall": (i32, [vp, i32]),
        "pyomgpu_nh_set_grid": (i32, [vp, i32]),
        "pyomgpu_nh_set_brick": (i32, [vp, i32, i32]),
        "pyomgpu_nh_set_stages": (i32, [vp, i32]),
        "pyomgpu_nh_set_variant": (i32, [vp, i32]),
        "pyomgpu_apply_op_3d": (i32, [vp, vp, vp, vp]),
        "pyomgpu_congrad_non_hydro": (i32, [vp, vp, vp, d, i32, P(SolveInfo), vp]),
        "pyomgpu_solve_non_hydrostatic": (i32, [vp, P(State3D), P(SolveInfo), vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    return load().pyomgpu_last_error().decode(errors="replace")


def check(rc: int, allow=(OK,)):
    """Raise on hard errors (negative codes) and on solver statuses not in ``allow``."""
    if rc in allow:
        return rc
    raise PyOMGPUError(rc, last_error())
