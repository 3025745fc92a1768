"""Golden vectors from the reference's own Fortran source.

This image has no Fortran compiler, so pyOM2's routines are run through the
Fortran-subset translator oracle/f90sub.py: the reference files below are
read from the reference checkout (REF, default /root/reference, only where
this script runs), translated to Python and executed with Fortran's
arithmetic and control flow.  For every case of tests/golden/ref_cases.py it
records what the reference computes:

* calc_grid / calc_topo (for_src/main/numerics.f90:34-168,187-261) from the
  case's dxt, dyt, dzt, origins and kbot;
* streamfunction_init (for_src/external/streamfct_init.f90:7-304: island
  labelling, perimeter tracing, the psin solves, line_psin);
* congrad_streamfunction (solve_streamfct.f90:153-327) from a zero first
  guess with the reference stop;
* two time steps of solve_streamfunction (solve_streamfct.f90:10-120) from a
  seeded prognostic state;
* one step of solve_pressure (for_src/external/solve_pressure.f90:10-82)
  with a free surface and with a rigid lid;
* congrad_non_hydro (for_src/non_hydrostatic/non_hydrostatic.f90:146-242)
  from a seeded first guess and one step of solve_non_hydrostatic (:5-63) on
  a closed tank and a cyclic x-z slice;
* one call of momentum (for_src/main/momentum.f90:4-168: Coriolis and metric
  terms, wind stress, momentum_advection, implicit vertical friction,
  harmonic and linear bottom friction, then solve_streamfunction) on a small
  re-entrant channel, with w(tau) from vertical_velocity_tau.

LAPACK's DGESV (called by solve_streamfunction, solve_streamfct.f90:81) is
not part of the reference; scipy's LAPACK dgesv stands in for the system
library the reference links.  The open-boundary hooks (set_obc_*) are not
loaded: open boundaries are off in every case, where they do nothing.

Output: tests/golden/ref_f90_<case>.npz, ref_f90_pressure.npz,
ref_f90_nh.npz and ref_f90_momentum.npz.  Arrays of
at most 60000 values are stored whole, larger ones as a SHA-256 digest of
their bytes, their L2 norm and a strided sample.

Run: python tests/golden/make_ref_golden.py   (a few minutes)
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from oracle import f90sub  # noqa: E402
from ref_cases import (CASES, GRID_OUT, GRID_WIDTHS, MOMENTUM_CASE, MOMENTUM_OUT_3D, NH_CASES, PRESSURE,  # noqa: E402
                       STEP_OUT_2D, STEP_OUT_3D, digest, momentum_state, random_state)

REF = os.environ.get("PYOM2_REFERENCE", "/root/reference")
SOURCES = ["for_src/main/main_module.f90", "for_src/parallel/parallel_none.f90", "for_src/main/numerics.f90",
           "for_src/external/island_module.f90", "for_src/external/streamfct_init.f90",
           "for_src/external/solve_streamfct.f90", "for_src/external/solve_pressure.f90",
           "for_src/non_hydrostatic/non_hydrostatic.f90"]
WHOLE = 60000


def _dgesv(prog, n, nrhs, A, lda, ipiv, B, ldb, info):
    import scipy.linalg.lapack as lapack
    n = int(n)
    lu, piv, x, inf = lapack.dgesv(np.array(A.a[:n, :n]), np.array(B.a[:n]).reshape(n, -1))
    A.a[:n, :n] = lu
    ipiv.a[:n] = piv + 1
    B.a[:n] = x.reshape(B.a[:n].shape)
    return (n, nrhs, None, lda, None, None, ldb, int(inf))


def _nothing(prog, *args):
    return tuple([None] * len(args))


def _panic(prog, *args):
    raise f90sub.HaltStop("panic_snap")


EXTERNALS = {"dgesv": _dgesv, "set_obc_streamfct": _nothing, "set_obc_topo": _nothing, "panic_snap": _panic,
             "set_obc_boundary_xyz": _nothing}


def program():
    return f90sub.translate([os.path.join(REF, p) for p in SOURCES], EXTERNALS)


# momentum (momentum.f90) and the modules it uses; the timers of timing_module
# (tic/toc) do nothing here, and the routines of features that are off in the
# momentum case are not loaded (a call would stop the generator)
MOMENTUM_SOURCES = ["for_src/isoneutral/isoneutral_module.f90", "for_src/idemix/idemix_module.f90",
                    "for_src/rossmix/rossmix_module.f90", "for_src/rossmix2/rossmix2_module.f90",
                    "for_src/etc/py_stuff.f90", "for_src/main/momentum.f90", "for_src/main/momentum_advection.f90",
                    "for_src/main/harmonic_friction.f90", "for_src/main/bottom_friction.f90",
                    "for_src/main/vertical_friction.f90", "for_src/main/vertical_velocity.f90"]


def _not_loaded(name):
    def f(prog, *args):
        raise f90sub.F90Error(f"{name} is not loaded: its feature is off in these cases")
    return f


def momentum_program():
    prog = f90sub.Program()
    prog.add_source("module timing_module\nend module timing_module\n", "timing_module (timers only)")
    for p in SOURCES[:1] + MOMENTUM_SOURCES + SOURCES[1:]:
        with open(os.path.join(REF, p)) as fh:
            prog.add_source(fh.read(), p.split("/")[-1])
    ext = dict(EXTERNALS)
    ext.update({"tic": _nothing, "toc": _nothing, "set_obc_momentum": _nothing})
    for n in ("isoneutral_friction", "idemix_friction", "idemix_friction_lee", "rossmix_friction",
              "rossmix2_friction", "biharmonic_friction", "momentum_sources_with_euler",
              "momentum_sources_with_ab"):
        ext[n] = _not_loaded(n)
    prog.externals.update(ext)
    prog.compile()
    return prog


def put(out, key, a):
    a = np.array(a)  # a copy: the program's arrays change in later steps
    if a.size <= WHOLE:
        out[key] = a
    else:
        out[key + "__digest"] = np.array(digest(a))
        out[key + "__norm"] = np.array(float(np.linalg.norm(a.astype(np.float64))))
        flat = a.reshape(-1, order="F")
        out[key + "__sample"] = flat[:: max(1, flat.size // 500)]


def setup_model(prog, M, widths, hydrostatic=True):
    """main_module of the translated reference: sizes and switches of M,
    pe_decomposition, allocate_main_module, then calc_grid and calc_topo
    from the case's cell widths (dxt, dyt), M's dzt, origins and kbot
    (pyOM2's set_grid / set_topography step)."""
    S = prog.state["main_module"]
    S["nx"], S["ny"], S["nz"] = M.nx, M.ny, M.nz
    prog.set("main_module", "enable_hydrostatic", hydrostatic)  # the non-hydrostatic arrays exist without it
    prog.call("pe_decomposition")
    prog.call("allocate_main_module")
    for n in ("enable_cyclic_x", "enable_cyclic_y", "coord_degree"):
        prog.set("main_module", n, bool(getattr(M, n)))
    prog.set("main_module", "x_origin", M.x_origin)
    prog.set("main_module", "y_origin", M.y_origin)
    S["dxt"].a[2:M.nx + 2] = widths[0]
    S["dyt"].a[2:M.ny + 2] = widths[1]
    S["dzt"].a[...] = M.dzt
    prog.call("calc_grid")
    S["kbot"].a[...] = M.kbot
    prog.call("calc_topo")
    prog.set("main_module", "congr_epsilon", M.congr_epsilon)
    prog.set("main_module", "congr_max_iterations", M.congr_max_iterations)
    prog.set("main_module", "congr_epsilon_non_hydro", M.congr_epsilon_non_hydro)
    prog.set("main_module", "congr_max_itts_non_hydro", M.congr_max_itts_non_hydro)


def grid_outputs(prog, out):
    S = prog.state["main_module"]
    for n in GRID_OUT:
        put(out, "grid_" + n, S[n.lower()].a)


def load_state(prog, M):
    S = prog.state["main_module"]
    for n in ("u", "v", "du", "dv", "rho", "du_mix", "dv_mix", "dpsi", "psi"):
        S[n.lower()].a[...] = getattr(M, n)
    if M.dpsin is not None and S["dpsin"] is not None:
        S["dpsin"].a[...] = M.dpsin
    prog.set("main_module", "dt_mom", M.dt_mom)
    for n in ("taum1", "tau", "taup1"):
        prog.set("main_module", n, getattr(M, n))


def rotate(prog):
    S = prog.state["main_module"]
    S["taum1"], S["tau"], S["taup1"] = S["tau"], S["taup1"], S["taum1"]


def case(name):
    t0 = time.time()
    W = CASES[name]()
    M = W.M
    out = {"forc__digest": np.array(digest(W.forc)), "kbot__digest": np.array(digest(M.kbot))}
    prog = program()
    setup_model(prog, M, GRID_WIDTHS[name])
    grid_outputs(prog, out)
    S = prog.state["main_module"]
    # streamfunction_init: islands, psin, line_psin
    prog.call("streamfunction_init")
    out["nisle"] = np.array(S["nisle"])
    for n in ("boundary", "line_dir", "nr_boundary", "psin", "line_psin"):
        put(out, n, S[n].a)
    out["init_itts"] = np.array(S["congr_itts"])
    # congrad_streamfunction from zero with the reference stop
    X, Y = M.shape2d
    forc = f90sub.FArray(np.asfortranarray(W.forc.copy()), (-1, -1))
    sol = f90sub.FArray(np.zeros((X, Y), order="F"), (-1, -1))
    r = prog.call("congrad_streamfunction", -1, M.nx + 2, -1, M.ny + 2, forc, 0, sol, False)
    put(out, "sol", sol.a)
    out["sol_iterations"] = np.array(r[5])
    out["sol_converged"] = np.array(bool(r[7]))
    # two steps of solve_streamfunction from the seeded state
    random_state(M, 4)
    M.allocate_islands(int(S["nisle"]), S["boundary"].a.shape[1])
    random_state(M, 4)  # dpsin exists now: the same recipe fills it
    load_state(prog, M)
    for step in range(2):
        prog.call("solve_streamfunction")
        tp1 = S["taup1"] - 1
        out[f"step{step}_itts"] = np.array(S["congr_itts"])
        for n in STEP_OUT_2D:
            put(out, f"step{step}_{n}", S[n].a[:, :, tp1])
        put(out, f"step{step}_dpsin", S["dpsin"].a)
        for n in STEP_OUT_3D:
            put(out, f"step{step}_{n}", S[n].a)
        rotate(prog)
    np.savez_compressed(os.path.join(HERE, f"ref_f90_{name}.npz"), **out)
    print(f"{name}: nisle {int(S['nisle'])}, congrad {r[5]} iterations, steps {int(out['step0_itts'])}/"
          f"{int(out['step1_itts'])}, {time.time() - t0:.0f} s", flush=True)


def pressure():
    out = {}
    for name, free, max_it in PRESSURE:
        t0 = time.time()
        W = CASES[name]()
        M = W.M
        M.enable_free_surface = free
        if max_it is not None:
            M.congr_max_iterations = max_it
        random_state(M, 5)
        prog = program()
        setup_model(prog, M, GRID_WIDTHS[name])
        load_state(prog, M)
        prog.set("main_module", "enable_free_surface", free)
        S = prog.state["main_module"]
        prog.call("solve_pressure")
        key = f"{name}_{'free' if free else 'rigid'}"
        tp1 = S["taup1"] - 1
        out[key + "_itts"] = np.array(S["congr_itts"])
        put(out, key + "_psi", S["psi"].a[:, :, tp1])
        for n in ("u", "v"):
            put(out, f"{key}_{n}", S[n].a)
        print(f"pressure {key}: {int(S['congr_itts'])} iterations, {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "ref_f90_pressure.npz"), **out)


def nonhydro():
    from pyom2_b200 import synth
    out = {}
    for name, make in NH_CASES.items():
        t0 = time.time()
        W = make()
        M = W.M
        prog = program()
        setup_model(prog, M, GRID_WIDTHS[name], hydrostatic=False)
        grid_outputs_nh = {}
        grid_outputs(prog, grid_outputs_nh)
        for k, v in grid_outputs_nh.items():
            out[f"{name}_{k}"] = v
        S = prog.state["main_module"]
        nz = M.nz
        tp1 = S["taup1"] - 1
        S["p_non_hydro"].a[:, :, :, tp1] = W.p0
        forc = f90sub.FArray(np.asfortranarray(W.forc.copy()), (-1, -1, 1))
        r = prog.call("congrad_non_hydro", -1, M.nx + 2, -1, M.ny + 2, nz, forc, 0)
        out[f"{name}_cg_iterations"] = np.array(r[6])
        put(out, f"{name}_cg_p", S["p_non_hydro"].a[:, :, :, tp1])
        # one step of solve_non_hydrostatic from the seeded state (a fresh program:
        # congrad_non_hydro keeps its operator from the first call, as the reference does)
        synth.nonhydro_state(W, 21)
        prog = program()
        setup_model(prog, M, GRID_WIDTHS[name], hydrostatic=False)
        S = prog.state["main_module"]
        for n in ("u", "v", "w", "dw", "dw_mix", "p_non_hydro"):
            S[n].a[...] = getattr(M, n)
        prog.set("main_module", "dt_mom", M.dt_mom)
        prog.set("main_module", "itt", int(M.itt))
        prog.call("solve_non_hydrostatic")
        out[f"{name}_step_itts"] = np.array(S["congr_itts_non_hydro"])
        for n in ("u", "v", "w", "p_non_hydro"):
            put(out, f"{name}_step_{n}", S[n].a)
        print(f"{name}: congrad_non_hydro {r[6]} iterations, step {int(S['congr_itts_non_hydro'])}, "
              f"{time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "ref_f90_nh.npz"), **out)


def momentum_case():
    """momentum (momentum.f90:4-168: tendencies, then solve_streamfunction) on
    the channel of MOMENTUM_CASE, one step from the seeded state, after
    streamfunction_init and vertical_velocity_tau for w(tau)."""
    t0 = time.time()
    name, make = MOMENTUM_CASE
    W = make()
    M = W.M
    momentum_state(M, 31)
    prog = momentum_program()
    setup_model(prog, M, GRID_WIDTHS[name])
    S = prog.state["main_module"]
    out = {"kbot__digest": np.array(digest(M.kbot))}
    for n in GRID_OUT + ("tantr", "area_t", "area_u", "area_v"):
        put(out, "grid_" + n, S[n.lower()].a)
    prog.set("main_module", "enable_streamfunction", True)
    prog.call("streamfunction_init")
    for n in ("enable_hor_friction", "enable_hor_friction_cos_scaling", "hor_friction_cosPower",
              "enable_bottom_friction", "enable_implicit_vert_friction", "A_h", "r_bot", "dt_mom"):
        prog.set("main_module", n.lower(), getattr(M, n))
    prog.set("main_module", "enable_conserve_energy", False)
    for n in ("u", "v", "coriolis_t", "surface_taux", "surface_tauy", "kappaM", "du", "dv"):
        S[n.lower()].a[...] = getattr(M, n)
    for n in ("taum1", "tau", "taup1"):
        prog.set("main_module", n, getattr(M, n))
    prog.call("vertical_velocity_tau", int(S["tau"]))
    put(out, "w_tau", S["w"].a[:, :, :, S["tau"] - 1])
    prog.call("momentum")
    tau, tp1 = S["tau"] - 1, S["taup1"] - 1
    for n in MOMENTUM_OUT_3D:
        a = S[n].a
        put(out, n, a[:, :, :, tau] if a.ndim == 4 else a)
    out["itts"] = np.array(S["congr_itts"])
    for n in ("psi", "dpsi"):
        put(out, n, S[n].a[:, :, tp1])
    put(out, "dpsin", S["dpsin"].a)
    for n in ("u", "v"):
        put(out, n + "_taup1", S[n].a[:, :, :, tp1])
    np.savez_compressed(os.path.join(HERE, "ref_f90_momentum.npz"), **out)
    print(f"momentum {name}: nisle {int(S['nisle'])}, solve {int(S['congr_itts'])} iterations, "
          f"{time.time() - t0:.0f} s", flush=True)


def main():
    for name in (sys.argv[1:] or list(CASES) + ["pressure", "nh", "momentum"]):
        if name == "pressure":
            pressure()
        elif name == "nh":
            nonhydro()
        elif name == "momentum":
            momentum_case()
        else:
            case(name)


if __name__ == "__main__":
    main()
