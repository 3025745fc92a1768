"""Model state holder mirroring the pyOM2 Fortran module variables used by the
external-mode (barotropic) solve.

pyOM2 keeps its state in the Fortran module ``main_module``
(for_src/main/main_module.f90) and f2py exposes every array to Python as an
F-contiguous numpy view with the Fortran shape (py_src/pyOM.py:39).  This class
carries the same names, shapes and memory order so that the solver entry points
in :mod:`pyom2_b200.external` (streamfunction and surface-pressure solves) and
:mod:`pyom2_b200.non_hydrostatic` can be used on either an f2py module object or
on this stand-in.

Index conventions (py_src/pyOM.py:234-252): Fortran index ``i`` in
``is_pe-onx .. ie_pe+onx`` is Python index ``i + onx - is_pe``; time level
``t`` (1-based ``taum1/tau/taup1``) is Python index ``t - 1``.

Constants follow main_module.f90:13-19,52,189: pyOM2 declares them as
``real*8`` parameters initialised with default-real (single precision)
literals, so ``pi``, ``grav``, ``AB_eps`` and ``congr_epsilon`` carry the
float32 rounding of their decimal value.  The solver's stopping decisions
depend on ``congr_epsilon`` bit-for-bit, so the same rounding is kept here.
"""
from __future__ import annotations

import numpy as np

ONX = 2


def f32(x: float) -> float:
    """Value of a Fortran default-real literal stored into a real*8."""
    return float(np.float32(x))


PI_F = f32(3.14159265358979323846264338327950588)   # main_module.f90:13
RADIUS = f32(6370.0e3)                               # main_module.f90:14
DEGTOM = RADIUS / 180.0 * PI_F                       # main_module.f90:15
RHO_0 = f32(1024.0)                                  # main_module.f90:18
GRAV = f32(9.81)                                     # main_module.f90:19
AB_EPS = f32(0.1)                                    # main_module.f90:52
CONGR_EPSILON = f32(1e-12)                           # main_module.f90:189
CONGR_MAX_ITERATIONS = 1000                          # main_module.f90:190
CONGR_EPSILON_NON_HYDRO = f32(1e-12)                 # main_module.f90:222, default-real literal
CONGR_MAX_ITTS_NON_HYDRO = 1000                      # main_module.f90:223


def zeros_f(*shape, dtype=np.float64):
    return np.zeros(shape, dtype=dtype, order="F")


class ModelState:
    """Subset of ``main_module`` that the external-mode solve reads or writes.

    Arrays are allocated with the Fortran extents of main_module.f90:227-349
    for a serial run (``is_pe=1, ie_pe=nx, js_pe=1, je_pe=ny``,
    parallel_none.f90:16-19).
    """

    def __init__(self, nx: int, ny: int, nz: int, *, enable_cyclic_x=False,
                 enable_cyclic_y=False, coord_degree=True):
        self.nx, self.ny, self.nz, self.onx = int(nx), int(ny), int(nz), ONX
        self.is_pe, self.ie_pe, self.js_pe, self.je_pe = 1, self.nx, 1, self.ny
        self.enable_cyclic_x = bool(enable_cyclic_x)
        self.enable_cyclic_y = bool(enable_cyclic_y)
        self.coord_degree = bool(coord_degree)
        self.enable_free_surface = False
        self.enable_streamfunction = True
        self.enable_congrad_verbose = False
        self.dt_mom = 3600.0
        self.AB_eps = AB_EPS
        self.grav = GRAV
        self.rho_0 = RHO_0
        self.congr_epsilon = CONGR_EPSILON
        self.congr_max_iterations = CONGR_MAX_ITERATIONS
        self.congr_itts = 0
        self.congr_epsilon_non_hydro = CONGR_EPSILON_NON_HYDRO
        self.congr_max_itts_non_hydro = CONGR_MAX_ITTS_NON_HYDRO
        self.congr_itts_non_hydro = 0
        self.taum1, self.tau, self.taup1 = 1, 2, 3
        self.itt = 0
        X, Y = self.nx + 2 * ONX, self.ny + 2 * ONX
        nz = self.nz
        self.x_origin = 0.0
        self.y_origin = 0.0
        # 1-D grid (main_module.f90:234-241)
        for name, n in (("dxt", X), ("dxu", X), ("xt", X), ("xu", X),
                        ("dyt", Y), ("dyu", Y), ("yt", Y), ("yu", Y)):
            setattr(self, name, np.zeros(n))
        self.cost = np.ones(Y)
        self.cosu = np.ones(Y)
        self.dzt = np.zeros(nz)
        self.dzw = np.zeros(nz)
        self.zt = np.zeros(nz)
        self.zw = np.zeros(nz)
        # 2-D fields
        self.kbot = zeros_f(X, Y, dtype=np.int32)
        for name in ("ht", "hu", "hv", "hur", "hvr"):
            setattr(self, name, zeros_f(X, Y))
        # 3-D masks
        for name in ("maskT", "maskU", "maskV", "maskZ", "maskW"):
            setattr(self, name, zeros_f(X, Y, nz))
        # dynamics (main_module.f90:298-311)
        for name in ("u", "v", "du", "dv", "rho"):
            setattr(self, name, zeros_f(X, Y, nz, 3))
        for name in ("du_mix", "dv_mix", "p_hydro"):
            setattr(self, name, zeros_f(X, Y, nz))
        self.p_non_hydro = zeros_f(X, Y, nz, 3)          # main_module.f90:337
        self.w = zeros_f(X, Y, nz, 3)                    # main_module.f90:298-311
        self.dw = zeros_f(X, Y, nz, 3)
        self.dw_mix = zeros_f(X, Y, nz)
        self.psi = zeros_f(X, Y, 3)
        self.dpsi = zeros_f(X, Y, 3)
        # momentum inputs (main_module.f90:113-114,109-112,160-161,210): metric and
        # box areas of calc_grid, Coriolis frequency, wind stress, vertical viscosity
        self.tantr = np.zeros(Y)
        for name in ("area_t", "area_u", "area_v", "area_z", "coriolis_t", "surface_taux", "surface_tauy"):
            setattr(self, name, zeros_f(X, Y))
        self.kappaM = zeros_f(X, Y, nz)
        # physics switches and parameters of momentum (main_module.f90:196-203), the reference's defaults
        self.enable_hor_friction = False
        self.enable_hor_friction_cos_scaling = False
        self.hor_friction_cosPower = 3
        self.enable_bottom_friction = False
        self.enable_implicit_vert_friction = False
        self.A_h = 0.0
        self.r_bot = 0.0
        # island variables, allocated by streamfunction_init (streamfct_init.f90:87-93)
        self.nisle = 0
        self.boundary = None
        self.line_dir = None
        self.nr_boundary = None
        self.psin = None
        self.dpsin = None
        self.line_psin = None

    # --- index helpers, py_src/pyOM.py:234-252 ---------------------------------
    def if2py(self, i):
        return i + self.onx - self.is_pe

    def jf2py(self, j):
        return j + self.onx - self.js_pe

    @property
    def shape2d(self):
        return (self.nx + 2 * ONX, self.ny + 2 * ONX)

    def allocate_islands(self, nisle: int, max_boundary: int):
        X, Y = self.shape2d
        self.nisle = int(nisle)
        self.boundary = zeros_f(nisle, max_boundary, 2, dtype=np.int32)
        self.line_dir = zeros_f(nisle, max_boundary, 2, dtype=np.int32)
        self.nr_boundary = np.zeros(nisle, dtype=np.int32)
        self.psin = zeros_f(X, Y, nisle)
        self.dpsin = zeros_f(nisle, 3)
        self.line_psin = zeros_f(nisle, nisle)

    def copy(self) -> "ModelState":
        import copy
        return copy.deepcopy(self)
