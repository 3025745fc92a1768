"""Learned preconditioner: a U-Net run by the library's tcgen05 kernels inside
flexible CG (``pyomgpu_precond_*`` / ``pyomgpu_solve_fcg`` of the C ABI).

The reference has no learned component; its only preconditioner is Jacobi
(``make_inv_sfc``, solve_streamfct.f90:381-422), which stays the fallback of
:func:`solve_fcg`; every answer is accepted or rejected by its FP64 true
residual.

Training data are (residual, error) pairs produced by the plain solver
itself: for a right-hand side b, ``x*`` is the FP64 Jacobi-PCG solution to a
tight residual, and restarted PCG runs from randomly perturbed guesses give an
iterate x with residual r = b - A x and error e = x* - x.  The loss is the
relative energy-norm error of the network output against the scaled error
(see precond.cu).  Everything runs on the GPU; PyTorch only holds
device buffers.
"""
from __future__ import annotations

import ctypes as C
import os
import warnings

import numpy as np

from . import _abi, synth
from ._abi import PyOMGPUError
from .external import ExternalMode, _ptr, _stream

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "unet_c1_family.npz")

# (cin, cout) of the 12 convolutions, as in csrc/unet.cu
LAYERS = [(16, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 64), (64, 64), (64, 64), (64, 32),
          (32, 16), (16, 16)]


def num_params() -> int:
    return int(_abi.load().pyomgpu_precond_num_params())


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, zero biases; the output layer starts
    small and only its channel 0 is ever used (the others stay zero)."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    ws, bs = [], []
    for l, (ci, co) in enumerate(LAYERS):
        w = rng.standard_normal((co, ci, 3, 3)) * np.sqrt(2.0 / (9 * ci))
        if l == len(LAYERS) - 1:
            w *= 0.1
            w[1:] = 0.0
        ws.append(w.astype(np.float32).ravel())
        bs.append(np.zeros(co, dtype=np.float32))
    p = np.concatenate(ws + bs)
    assert p.size == num_params()
    return p


def load_params(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    with np.load(path) as z:
        return np.asarray(z["params"], dtype=np.float32)


class LearnedPreconditioner:
    """The network for one grid (an :class:`ExternalMode` with islands set)."""

    def __init__(self, em: ExternalMode, params=None, training=False, seed=0):
        L = _abi.load()
        self.em, self._L = em, L
        h = C.c_void_p()
        _abi.check(L.pyomgpu_precond_create(em._ctx, int(bool(training)), C.byref(h)))
        self._h = h
        self.n = num_params()
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if getattr(self, "_h", None):
            self._L.pyomgpu_precond_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def rebind(self, em: ExternalMode):
        """Move the network to another grid of the same size."""
        _abi.check(self._L.pyomgpu_precond_rebind(self._h, em._ctx))
        self.em = em

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n:
            raise PyOMGPUError(_abi.EINVAL, f"expected {self.n} parameters, got {p.size}")
        _abi.check(self._L.pyomgpu_precond_set_params(self._h, C.c_void_p(p.ctypes.data), self.n))

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n, dtype=np.float32)
        _abi.check(self._L.pyomgpu_precond_get_params(self._h, C.c_void_p(p.ctypes.data), self.n))
        return p

    def get_grads(self) -> np.ndarray:
        g = np.zeros(self.n, dtype=np.float32)
        _abi.check(self._L.pyomgpu_precond_get_grads(self._h, C.c_void_p(g.ctypes.data), self.n))
        return g

    def apply(self, r):
        """z = M(r) for a Fortran-ordered float64 CUDA tensor r."""
        from .external import _torch_like
        z = _torch_like(r)
        _abi.check(self._L.pyomgpu_precond_apply(self._h, _ptr(r, self.em.shape), _ptr(z, self.em.shape, True),
                                                 _stream()))
        return z

    def train_step(self, r, e, lr):
        loss = C.c_float()
        _abi.check(self._L.pyomgpu_precond_train_step(self._h, _ptr(r, self.em.shape), _ptr(e, self.em.shape),
                                                      float(lr), C.byref(loss), _stream()))
        return float(loss.value)

    def forward_backward(self, x0_bits, gz=None):
        """Network alone: x0 planar bf16 bits uint16 [2][Hp][Wp][8] -> z f32 [Hp][Wp]."""
        x0 = np.ascontiguousarray(x0_bits, dtype=np.uint16)
        Hp, Wp = x0.shape[1], x0.shape[2]
        z = np.zeros((Hp, Wp), dtype=np.float32)
        gzp = None
        if gz is not None:
            gzc = np.ascontiguousarray(gz, dtype=np.float32)
            gzp = C.c_void_p(gzc.ctypes.data)
        _abi.check(self._L.pyomgpu_unet_forward_backward(self._h, C.c_void_p(x0.ctypes.data), gzp,
                                                         C.c_void_p(z.ctypes.data), _stream()))
        return z


def solve_fcg(em: ExternalMode, pc: LearnedPreconditioner, forc, sol, rtol=1e-10, max_it=100000):
    """Flexible CG with the network to FP64 relative residual ``rtol`` (in
    place on ``sol``); Jacobi-PCG takes over if FCG stalls."""
    info = _abi.SolveInfo()
    rc = _abi.load().pyomgpu_solve_fcg(em._ctx, pc._h, _ptr(forc, em.shape), _ptr(sol, em.shape, True),
                                       float(rtol), int(max_it), C.byref(info), _stream())
    _abi.check(rc, allow=(_abi.OK, _abi.MAXITER, _abi.DIVERGED))
    return info.as_dict()


# ---------------------------------------------------------------------------
# training on pairs generated by the plain solver
def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().T


def rhs_basis(W, count, seed):
    """Seeded right-hand sides of the workload's recipe (smooth curl forcing,
    solve_streamfct.f90:39-53) with correlation lengths of 2-24 cells."""
    rng = np.random.default_rng(np.random.PCG64(seed))
    out = []
    for k in range(count):
        sigma = float(np.exp(rng.uniform(np.log(2.0), np.log(24.0))))
        fpx, fpy = synth.random_fp(W.M, rng, sigma=sigma, rms=1e-7)
        out.append(synth.forcing_from_fp(W.M, fpx, fpy))
    return out


def random_field(shape_f, sigma, gen):
    """Smooth Gaussian random field (Fortran-ordered CUDA tensor of shape
    ``shape_f``) with correlation length ``sigma`` cells, unit rms."""
    import torch
    nx4, ny4 = shape_f
    w = torch.randn((ny4, nx4), generator=gen, device="cuda", dtype=torch.float64)
    F = torch.fft.rfft2(w)
    ky = torch.fft.fftfreq(ny4, device="cuda", dtype=torch.float64)[:, None]
    kx = torch.fft.rfftfreq(nx4, device="cuda", dtype=torch.float64)[None, :]
    F *= torch.exp(-2.0 * (np.pi * sigma) ** 2 * (kx * kx + ky * ky))
    f = torch.fft.irfft2(F, s=(ny4, nx4))
    f /= f.pow(2).mean().sqrt().clamp_min(1e-300)
    return f.T  # Fortran view


def pair_stream(W, em: ExternalMode, basis, seed, pairs_per_rhs=24, restart_range=(0, 40)):
    """Endless stream of training pairs (r, e).  A right-hand side b is a
    random combination of ``basis``; its tight solution x* comes from
    Jacobi-PCG.  Each pair starts the plain solver from x* plus a smooth
    random perturbation (random correlation length 1-96 cells) and runs a
    random number of restarted PCG iterations; the iterate x gives r = b - A x
    and e = x* - x."""
    import torch
    rng = np.random.default_rng(np.random.PCG64(seed))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(int(seed) * 7919 + 1)
    B = [_dev(b) for b in basis]
    mask = _dev((em.make_inv_sfc() != 0).astype(np.float64))
    while True:
        c = rng.standard_normal(len(B))
        b = sum(float(ck) * Bk for ck, Bk in zip(c, B))
        b = b.T.contiguous().T  # Fortran order
        xs = torch.zeros_like(b).T.contiguous().T
        em.solve_rtol(b, xs, rtol=1e-12, precision=_abi.PREC_F64)
        xs_rms = float(xs[mask > 0].pow(2).mean().sqrt())
        for _ in range(pairs_per_rhs):
            sigma = float(np.exp(rng.uniform(np.log(1.0), np.log(96.0))))
            amp = xs_rms * float(np.exp(rng.uniform(np.log(1e-3), np.log(1.0))))
            d = random_field(em.shape, sigma, gen) * mask * amp
            x = (xs + d).T.contiguous().T
            m = int(rng.integers(restart_range[0], restart_range[1] + 1))
            if m > 0:
                with warnings.catch_warnings():
                    warnings.simplefilter("ignore", RuntimeWarning)
                    em.congrad_streamfunction(b, x, eps=0.0, max_it=m)
            r = ((b - em.apply_op(x)) * mask).T.contiguous().T
            e = (xs - x).T.contiguous().T
            yield r, e


def generate_and_train(pc: LearnedPreconditioner, W, em: ExternalMode, basis, steps, lr, seed, log=None,
                       pairs_per_rhs=24, restart_range=(0, 40), lr_final=None):
    """``steps`` Adam steps on fresh pairs from :func:`pair_stream`; with
    ``lr_final`` the learning rate decays geometrically from ``lr`` to it."""
    losses = []
    lr0 = lr
    stream = pair_stream(W, em, basis, seed, pairs_per_rhs, restart_range)
    for step in range(steps):
        r, e = next(stream)
        if lr_final is not None:
            lr = lr0 * (lr_final / lr0) ** (step / max(1, steps - 1))
        losses.append(pc.train_step(r, e, lr))
        if log and (step + 1) % 200 == 0:
            log(f"step {step + 1} loss(avg200) {np.mean(losses[-200:]):.4f}")
    return losses
