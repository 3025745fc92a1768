"""Config 4: a time-evolving sequence of streamfunction solves over an
ensemble of channel runs.

pyOM2's time step calls ``momentum`` (for_src/main/momentum.f90:4), which
builds the momentum tendencies ``du, dv`` at ``tau`` (Coriolis, metric terms,
the surface wind stress ``surface_taux/dzt(nz)`` at momentum.f90:86-93,
advection, friction) and then ``solve_streamfunction`` (momentum.f90:159).
:class:`ChannelEnsemble` runs the model's own momentum tendencies on the GPU
(pyomgpu_momentum_tendencies: Coriolis and metric terms, wind stress,
advection, implicit vertical, harmonic and bottom friction with the
reference's channel set-up, :func:`channel_physics`), or, with physics =
"synthetic", a stated sequence: per ensemble member,

* du(:,:,:,tau) = maskU * (sum_q a_q(t) Bu_q) plus, on the top level, the
  zonal wind stress 0.1 N/m^2 / rho_0 (1e-4 m^2/s^2) with a sin^2 profile
  across the channel, divided by dzt(nz) (momentum.f90:89);
* dv(:,:,:,tau) = maskV * (sum_q b_q(t) Bv_q);
* rho(:,:,:,tau) = a linear background stratification plus
  maskT * (sum_q c_q(t) Br_q), whose rms (0.0205 kg/m^3) is that of 0.1 K
  temperature noise under a linear equation of state (alpha = 2e-4 /K);

Bu, Bv, Br are seeded smooth fields (correlation 8 x 8 x 3 cells) shared by
the members, and the coefficients follow seeded AR(1) processes in time, one
per member (correlation 0.98 per step), so consecutive right-hand sides are
close and the reference's first guess 2 dpsi(tau) - dpsi(taum1)
(solve_streamfct.f90:56) is a warm start.

Each step runs ``pyomgpu_solve_streamfunction_begin`` for every member, one
of the solvers below on the members' forcings, and
``pyomgpu_solve_streamfunction_end`` for every member:

===========  ==========================================================================
"ref"        congrad_streamfunction per member (the reference algorithm and stop)
"batch_ref"  all members in one launch of the work-queue kernel, the reference's stop
"batch"      all members in one launch of the work-queue kernel (FP64 PCG, rtol stop)
"pcg64"      pyomgpu_solve_rtol FP64 per member (rtol stop)
"mixed32"    pyomgpu_solve_rtol FP32 with FP64 refinement per member (rtol stop)
"fcg"        the learned flexible CG per member (rtol stop, Jacobi-PCG fallback)
===========  ==========================================================================
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np

from . import _abi, synth
from .external import ExternalMode, _stream

TAUX = 1e-4          # 0.1 N/m^2 / rho_0, m^2/s^2
RHO_NOISE = 1024.0 * 2e-4 * 0.1


class TendencySequence:
    """Seeded synthetic du, dv, rho at ``tau`` for each member and step."""

    def __init__(self, M, members: int, seed: int, nbasis: int = 6, ar: float = 0.98, du_rms: float = 2e-7):
        self.M, self.members, self.nbasis, self.ar = M, int(members), int(nbasis), float(ar)
        rng = np.random.default_rng(np.random.PCG64(seed))
        shape3 = M.shape2d + (M.nz,)
        cyc = (M.enable_cyclic_x, M.enable_cyclic_y, False)

        def basis(mask, rms):
            out = []
            for _ in range(self.nbasis):
                f = synth.smooth_field(rng, shape3, (8.0, 8.0, 3.0), cyc)
                f *= rms / (np.sqrt(np.mean(f ** 2)) + 1e-300)
                f = np.asfortranarray(f * mask)
                synth.setcyclic_xy(M, f)
                out.append(f)
            return np.stack(out)

        self.Bu = basis(M.maskU, du_rms)
        self.Bv = basis(M.maskV, du_rms)
        self.Br = basis(M.maskT, RHO_NOISE)
        y0, y1 = M.yu[2], M.yu[M.ny + 1]
        prof = np.sin(np.pi * (M.yt - y0) / (y1 - y0)) ** 2
        self.wind = np.zeros(shape3, order="F")
        self.wind[:, :, -1] = M.maskU[:, :, -1] * (TAUX * prof)[None, :] / M.dzt[-1]
        self.rho_back = np.asfortranarray(M.maskT * (1024.0 + 2.0 * (-M.zt / 4000.0))[None, None, :])
        self.coef = rng.standard_normal((self.members, 3, self.nbasis))
        self._rng = rng
        self.t = 0
        self._dev = None

    def advance(self):
        xi = self._rng.standard_normal(self.coef.shape)
        self.coef = self.ar * self.coef + np.sqrt(1.0 - self.ar ** 2) * xi
        self.t += 1

    def host_fields(self, m):
        """du, dv, rho (Fortran-ordered numpy) of member m at the current step."""
        a = self.coef[m]
        du = np.asfortranarray(np.tensordot(a[0], self.Bu, axes=1) + self.wind)
        dv = np.asfortranarray(np.tensordot(a[1], self.Bv, axes=1))
        rho = np.asfortranarray(self.rho_back + np.tensordot(a[2], self.Br, axes=1))
        return du, dv, rho

    def device_fields(self, m, out_du, out_dv, out_rho):
        """Write member m's fields into device tensors (the transposed,
        C-ordered views of Fortran arrays, as external._to_device_f makes)."""
        import torch
        if self._dev is None:
            T = lambda a: torch.from_numpy(np.ascontiguousarray(a.reshape(a.shape[0], -1, order="F"))).cuda()
            self._dev = (T(self.Bu), T(self.Bv), T(self.Br),
                         torch.from_numpy(np.ascontiguousarray(self.wind.T)).cuda(),
                         torch.from_numpy(np.ascontiguousarray(self.rho_back.T)).cuda())
        Bu, Bv, Br, wind, rb = self._dev
        a = torch.from_numpy(self.coef[m]).cuda()
        out_du.copy_((a[0] @ Bu).view(out_du.shape) + wind)
        out_dv.copy_((a[1] @ Bv).view(out_dv.shape))
        out_rho.copy_((a[2] @ Br).view(out_rho.shape) + rb)


KAPPA_M = 1e-4  # vertical viscosity (m^2/s): kappaM_0 of a set-up without the TKE closure


def channel_physics(M):
    """The momentum set-up of the channel (the reference's channel set-up,
    py_config/acc2.py:41-49,95, without its closures): Coriolis frequency
    2 omega sin(lat); harmonic friction with cos scaling (power 1) and
    A_h = (dx degtom)^3 2e-11 for the zonal cell width dx in degrees; linear
    bottom friction r_bot = 1e-5 /s; implicit vertical friction with a
    constant kappaM = KAPPA_M; zonal wind stress 0.1 N/m^2 / rho_0 with a sin^2
    profile across the channel."""
    from .model import DEGTOM
    omega = float(np.float32(np.pi)) / 43082.0  # main_module.f90:16, pi a default real
    M.coriolis_t[...] = (2 * omega * np.sin(M.yt / 180.0 * np.pi))[None, :]
    dx_deg = float(M.dxt[2]) / DEGTOM
    M.enable_hor_friction = True
    M.enable_hor_friction_cos_scaling = True
    M.hor_friction_cosPower = 1
    M.A_h = (dx_deg * DEGTOM) ** 3 * 2e-11
    M.enable_bottom_friction = True
    M.r_bot = 1e-5
    M.enable_implicit_vert_friction = True
    M.kappaM[...] = KAPPA_M
    y0, y1 = M.yu[2], M.yu[M.ny + 1]
    prof = np.sin(np.pi * (M.yt - y0) / (y1 - y0)) ** 2
    M.surface_taux[...] = M.maskU[:, :, -1] * (TAUX * prof)[None, :]
    M.surface_tauy[...] = 0.0


class ChannelEnsemble:
    """``members`` copies of the config-4 channel, stepped together on the GPU.

    physics = "momentum": every step runs the model's own momentum tendencies
    (pyomgpu_momentum_tendencies with :func:`channel_physics`), the
    external-mode solve, and the end of the reference's step (cyclic halos of
    u, v and vertical_velocity); the members differ by their seeded density
    perturbation (0.1 K of temperature noise), which stays fixed (the tracer
    equations are outside this path).  physics = "synthetic": the stated
    tendency sequence of :class:`TendencySequence`."""

    def __init__(self, W, members: int = 8, seed: int = 1004, limits=None, physics: str = "momentum"):
        import torch
        self.W, self.M, self.members = W, W.M, int(members)
        M = self.M
        limits = limits or dict(maxipp=10**6, maxq=10**6)
        self.ems = []
        for _ in range(self.members):
            E = ExternalMode(M)
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", RuntimeWarning)
                E.streamfunction_init(**limits)
            self.ems.append(E)
        self.nisle = int(M.nisle)
        X, Y, nz = M.nx + 4, M.ny + 4, M.nz
        dev = torch.device("cuda")
        z = lambda *s: torch.zeros(tuple(reversed(s)), dtype=torch.float64, device=dev)
        H = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).to(dev)
        self.physics = physics
        if physics not in ("momentum", "synthetic"):
            raise ValueError(physics)
        self.shared = {"dzt": H(M.dzt), "dzw": H(M.dzw), "maskT": H(M.maskT), "maskU": H(M.maskU),
                       "maskV": H(M.maskV)}
        if physics == "momentum":
            channel_physics(M)
            for n in ("tantr", "maskW", "coriolis_t", "area_t", "area_u", "area_v", "surface_taux",
                      "surface_tauy", "kappaM"):
                self.shared[n] = H(getattr(M, n))
            self.kbot = torch.from_numpy(np.ascontiguousarray(np.asarray(M.kbot, dtype=np.int32).T)).to(dev)
        self.D = []
        for _ in range(self.members):
            d = {n: z(X, Y, nz, 3) for n in ("u", "v", "du", "dv", "rho")}
            d.update({n: z(X, Y, nz) for n in ("du_mix", "dv_mix", "p_hydro")})
            d.update({"psi": z(X, Y, 3), "dpsi": z(X, Y, 3), "dpsin": z(max(1, self.nisle), 3),
                      "forc": z(X, Y)})
            if physics == "momentum":
                d["w"] = z(X, Y, nz, 3)
            self.D.append(d)
        self.seq = TendencySequence(M, self.members, seed + 7)
        if physics == "momentum":  # each member's density: background plus its own fixed perturbation
            for m in range(self.members):
                rho = self.seq.host_fields(m)[2]
                for lev in range(3):
                    self.D[m]["rho"][lev].copy_(torch.from_numpy(np.ascontiguousarray(rho.T)))
        self.taum1, self.tau, self.taup1 = 1, 2, 3
        self.itt = 0
        self._L = _abi.load()
        self.pc = None

    def _state(self, m):
        M, d = self.M, self.D[m]
        s = _abi.State()
        s.nz = M.nz
        s.taum1, s.tau, s.taup1 = self.taum1, self.tau, self.taup1
        s.congr_max_iterations = int(M.congr_max_iterations)
        s.dt_mom, s.AB_eps, s.grav, s.rho_0 = float(M.dt_mom), float(M.AB_eps), float(M.grav), float(M.rho_0)
        s.congr_epsilon = float(M.congr_epsilon)
        for n, t in list(self.shared.items()) + [(k, v) for k, v in d.items() if k != "forc"]:
            setattr(s, n, t.data_ptr())
        return s

    def _momentum(self, m):
        M, d = self.M, self.D[m]
        p = _abi.Momentum()
        p.nz, p.taum1, p.tau, p.taup1 = M.nz, self.taum1, self.tau, self.taup1
        p.coord_degree = int(bool(M.coord_degree))
        p.enable_hor_friction = int(M.enable_hor_friction)
        p.enable_hor_friction_cos_scaling = int(M.enable_hor_friction_cos_scaling)
        p.hor_friction_cospower = int(M.hor_friction_cosPower)
        p.enable_bottom_friction = int(M.enable_bottom_friction)
        p.enable_implicit_vert_friction = int(M.enable_implicit_vert_friction)
        p.dt_mom, p.A_h, p.r_bot = float(M.dt_mom), float(M.A_h), float(M.r_bot)
        for n, t in self.shared.items():
            if hasattr(p, n):
                setattr(p, n, t.data_ptr())
        p.kbot = self.kbot.data_ptr()
        for n in ("u", "v", "w", "du", "dv", "du_mix", "dv_mix"):
            setattr(p, n, d[n].data_ptr())
        return p

    def dpsi_taup1(self, m):
        """Fortran-ordered (nx+4, ny+4) view of dpsi(:,:,taup1) of member m."""
        return self.D[m]["dpsi"][self.taup1 - 1].T

    def step(self, method: str = "ref", rtol: float = 1e-10, host_inputs=None):
        """One time step of every member; returns per-member solve infos.
        ``host_inputs`` (list of (du, dv, rho) numpy arrays per member)
        replaces the device-generated sequence (used by the parity tests)."""
        st = _stream()
        states = []
        moms = []
        if self.physics == "synthetic":
            self.seq.advance()
        for m in range(self.members):
            d = self.D[m]
            lv = self.tau - 1
            if self.physics == "momentum" and host_inputs is None:
                # momentum.f90:4-152: du, dv at tau, du_mix, dv_mix; rho stays the member's
                p = self._momentum(m)
                moms.append(p)
                _abi.check(self._L.pyomgpu_momentum_tendencies(self.ems[m]._ctx, C.byref(p), st))
            elif host_inputs is None:
                self.seq.device_fields(m, d["du"][lv], d["dv"][lv], d["rho"][lv])
            else:
                import torch
                for n, a in zip(("du", "dv", "rho"), host_inputs[m]):
                    d[n][lv].copy_(torch.from_numpy(np.ascontiguousarray(a.T)))
            s = self._state(m)
            states.append(s)
            _abi.check(self._L.pyomgpu_solve_streamfunction_begin(self.ems[m]._ctx, C.byref(s),
                                                                  C.c_void_p(d["forc"].data_ptr()), st))
        infos = self._solve(method, rtol, states)
        for m in range(self.members):
            _abi.check(self._L.pyomgpu_solve_streamfunction_end(self.ems[m]._ctx, C.byref(states[m]), st))
            if moms:  # the end of the reference's step (main.f90:114-117,147)
                _abi.check(self._L.pyomgpu_vertical_velocity(self.ems[m]._ctx, C.byref(moms[m]), self.taup1, st))
        self.taum1, self.tau, self.taup1 = self.tau, self.taup1, self.taum1
        self.itt += 1
        return infos

    def _solve(self, method, rtol, states):
        from .external import congrad_streamfunction_batch
        forcs = [self.D[m]["forc"].T for m in range(self.members)]
        sols = [self.dpsi_taup1(m) for m in range(self.members)]
        if method == "batch":
            return congrad_streamfunction_batch(self.ems, forcs, sols, eps=0.0, max_it=10**6, rtol=rtol)
        if method == "batch_ref":
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", RuntimeWarning)
                return congrad_streamfunction_batch(self.ems, forcs, sols, eps=float(self.M.congr_epsilon),
                                                    max_it=int(self.M.congr_max_iterations), rtol=0.0)
        out = []
        for m, E in enumerate(self.ems):
            if method == "ref":
                with warnings.catch_warnings():
                    warnings.simplefilter("ignore", RuntimeWarning)
                    it, conv, info = E.congrad_streamfunction(forcs[m], sols[m])
                out.append(info)
            elif method in ("pcg64", "mixed32"):
                prec = _abi.PREC_F64 if method == "pcg64" else _abi.PREC_F32
                out.append(E.solve_rtol(forcs[m], sols[m], rtol=rtol, precision=prec))
            elif method == "fcg":
                from . import learned
                if self.pc is None:
                    p = learned.load_params()
                    self.pc = [learned.LearnedPreconditioner(Em, params=p) for Em in self.ems]
                out.append(learned.solve_fcg(E, self.pc[m], forcs[m], sols[m], rtol=rtol))
            else:
                raise ValueError(method)
        return out

    def host_state(self, m, names=("u", "v", "psi", "dpsi", "dpsin", "p_hydro")):
        """Member m's arrays as Fortran-ordered numpy (current time labels)."""
        return {n: np.asfortranarray(self.D[m][n].cpu().numpy().T) for n in names}

    def close(self):
        for pc in self.pc or []:
            pc.close()
        for E in self.ems:
            E.close()
