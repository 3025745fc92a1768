"""Cases of the golden vectors made from the reference's own Fortran source
(tests/golden/make_ref_golden.py) and checked against the oracle
(tests/test_oracle_vs_reference_source.py): the seeded inputs, the loading
of a model state into the translated reference program, and the state
recipe of the time-step cases.  Test infrastructure only."""
import hashlib

import numpy as np

from pyom2_b200 import synth


def small_cyclic(seed=13, nx=96, ny=48, masses=6):
    return synth._global_like(nx, ny, -80.0, 80.0, seed, n_land_masses=masses, mask_sigma=4.0, depth_sigma=4.0,
                              name="small")


CASES = {
    "c0": lambda: synth.config0(),       # 40 x 40, closed, one interior island
    "cyclic96": lambda: small_cyclic(),  # 96 x 48, cyclic in x, five islands
}

# non-hydrostatic pressure solves (Cartesian tanks with a shelf and a rough
# slope, first guess and forcing seeded): closed 3-D, and a cyclic x-z slice
NH_CASES = {
    "nh_closed": lambda: synth.nonhydro_tank(20, 10, 8, 11, dx=0.5, first_guess=True),
    "nh_slice": lambda: synth.nonhydro_tank(24, 1, 10, 12, cyclic_x=True, dx=0.5, first_guess=True),
}

# momentum tendencies + solve_streamfunction (momentum.f90:4-168): a small
# re-entrant channel (config 4's recipe: 60S-30S, cyclic in x, one ridge)
MOMENTUM_CASE = ("channel", lambda: synth.config4(1004, nx=32, ny=24, nz=6))

# the cell widths the cases' set_grid step hands to calc_grid: degrees where
# coord_degree is set (pyOM2 converts them to metres there), metres otherwise;
# dzt is in metres
GRID_WIDTHS = {"c0": (2.0, 2.0), "cyclic96": (360.0 / 96, 160.0 / 48), "nh_closed": (0.5, 0.5),
               "nh_slice": (0.5, 0.5), "channel": (64.0 / 32, 30.0 / 24)}

# one-step cases of solve_pressure: (case, free surface, max iterations)
PRESSURE = [("c0", True, None), ("c0", False, 300), ("cyclic96", True, None)]

# grid inputs pyOM2's set_grid / set_topography hand to calc_grid / calc_topo
GRID_IN = ("dxt", "dyt", "dzt")
# what calc_grid / calc_topo derive (main_module names)
GRID_OUT = ("dxt", "dxu", "xt", "xu", "dyt", "dyu", "yt", "yu", "cost", "cosu", "zt", "zw", "dzw",
            "ht", "hu", "hv", "hur", "hvr", "maskT", "maskU", "maskV", "maskW", "maskZ")


def random_state(M, seed):
    """The prognostic state of the time-step cases (velocities, tendencies,
    density, streamfunction and island values), seeded."""
    rng = np.random.default_rng(seed)
    X, Y = M.shape2d
    nz = M.nz
    M.dt_mom = 1200.0
    for n in ("u", "v", "du", "dv"):
        getattr(M, n)[...] = rng.standard_normal((X, Y, nz, 3)) * 1e-3 * M.maskU[..., None]
    M.rho[...] = (rng.standard_normal((X, Y, nz, 3)) * 0.1 + 1.0) * M.maskT[..., None]
    M.du_mix[...] = rng.standard_normal((X, Y, nz)) * 1e-6 * M.maskU
    M.dv_mix[...] = rng.standard_normal((X, Y, nz)) * 1e-6 * M.maskV
    M.dpsi[...] = rng.standard_normal((X, Y, 3)) * 1e2
    M.psi[...] = rng.standard_normal((X, Y, 3)) * 1e4
    if M.dpsin is not None:
        M.dpsin[...] = rng.standard_normal(M.dpsin.shape) * 10


def digest(a):
    """SHA-256 of an array's values in Fortran order (bit-exact fingerprint)."""
    a = np.asarray(a)
    return hashlib.sha256(np.ascontiguousarray(a.reshape(-1, order="F")).tobytes()).hexdigest()


STEP_OUT_2D = ("dpsi", "psi")
STEP_OUT_3D = ("u", "v", "du", "dv", "p_hydro")


# parameters of the momentum case: the reference's channel set-up
# (py_config/acc2.py:41-49: harmonic friction with cos scaling, linear bottom
# friction, implicit vertical friction), with a given vertical viscosity in
# place of the TKE closure
MOMENTUM_PARAMS = dict(enable_hor_friction=True, enable_hor_friction_cos_scaling=True, hor_friction_cosPower=1,
                       enable_bottom_friction=True, r_bot=1e-5, enable_implicit_vert_friction=True, dt_mom=1800.0)
OMEGA = np.float64(np.float32(np.pi)) / 43082.0  # main_module.f90:16 (pi a default real)


def momentum_state(M, seed):
    """The inputs of the momentum case: smooth masked u, v at the three time
    levels with cyclic halos, Coriolis frequency 2 omega sin(lat), a zonal
    wind stress of 0.1 N/m^2 / rho_0 with a sin^2 profile across the channel,
    a seeded positive vertical viscosity around 1e-4 m^2/s, and the
    reference's A_h = (2 degtom)^3 2e-11 scaled to this grid; seeded."""
    from pyom2_b200.model import DEGTOM
    rng = np.random.default_rng(seed)
    X, Y = M.shape2d
    nz = M.nz
    for k, v in MOMENTUM_PARAMS.items():
        setattr(M, k, v)
    M.A_h = (2 * DEGTOM) ** 3 * 2e-11
    shape3 = (X, Y, nz)
    for lev in range(3):
        for name, mask in (("u", M.maskU), ("v", M.maskV)):
            f = synth.smooth_field(rng, shape3, (3.0, 3.0, 1.5), (True, False, False))
            f = np.asfortranarray(f * (0.05 / np.sqrt(np.mean(f ** 2))) * mask)
            synth.setcyclic_xy(M, f)
            getattr(M, name)[..., lev] = f
    M.coriolis_t[...] = (2 * OMEGA * np.sin(M.yt / 180.0 * np.pi))[None, :]
    y0, y1 = M.yu[2], M.yu[M.ny + 1]
    prof = np.sin(np.pi * (M.yt - y0) / (y1 - y0)) ** 2
    M.surface_taux[...] = M.maskU[:, :, -1] * (1e-4 * prof)[None, :]
    M.surface_tauy[...] = 0.0
    M.kappaM[...] = 1e-4 * (1.0 + 0.5 * rng.uniform(size=shape3))
    M.du[...] = 0.0
    M.dv[...] = 0.0


MOMENTUM_OUT_3D = ("du", "dv", "du_mix", "dv_mix")
