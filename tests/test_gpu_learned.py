"""GPU tests of the learned preconditioner: network values and gradients
against the FP64 CPU oracle (oracle/unet_oracle.py, with the GPU's bf16
storage points emulated), the training loss against a numpy evaluation with
the oracle operator, flexible CG to the 1e-10 true residual, training, and
an ablation: what the trained network gains over the untrained network and
over Jacobi-PCG on a held-out grid.

Tolerances: the GPU accumulates in FP32 and rounds activations and gradients
to bf16 at the same points as the oracle; rare round-to-nearest ties broken
the other way change single elements by one bf16 ulp (2**-8 relative), so
values agree to 1e-2 relative in L2 and gradients to 3e-2 per layer.
"""
import numpy as np
import pytest

from oracle import unet_oracle as U
from pyom2_b200 import _abi, learned, synth
from pyom2_b200.external import ExternalMode

pytestmark = pytest.mark.gpu
LIMITS = dict(maxipp=10**6, maxq=10**6)


def rel(a, b):
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / n if n > 0 else np.linalg.norm(a - b)


def grid(name):
    if name == "c0":
        return synth.config0()
    if name == "cyc96":
        return synth._global_like(96, 48, -80.0, 80.0, 13, n_land_masses=6, mask_sigma=4.0, depth_sigma=4.0,
                                  name="cyc96")
    if name == "cyc192":
        return synth._global_like(192, 96, -80.0, 80.0, 21, n_land_masses=8, mask_sigma=5.0, depth_sigma=5.0,
                                  name="cyc192")
    raise KeyError(name)


def setup(name):
    W = grid(name)
    E = ExternalMode(W.M)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(**LIMITS)
    return W, E


def test_network_values_and_gradients_match_oracle():
    W, E = setup("c0")
    pc = learned.LearnedPreconditioner(E, training=True, params=None, seed=3)
    rng = np.random.default_rng(5)
    p = learned.init_params(3)
    nw = sum(9 * a * b for a, b in learned.LAYERS)
    p[nw:] = rng.standard_normal(p.size - nw).astype(np.float32) * 0.1  # non-zero biases
    p[:nw] *= 1.5
    pc.set_params(p)
    Hp, Wp = 40, 40
    x0 = U.bf16_round(rng.standard_normal((16, Hp, Wp)))
    bits = U.bf16_bits(U.to_planar(x0))
    gz = rng.standard_normal((Hp, Wp)).astype(np.float32)
    z = pc.forward_backward(bits, gz)
    g = pc.get_grads()
    zo, A = U.unet_forward(p, x0, emulate=True)
    go = U.unet_backward(p, A, gz.astype(np.float64), emulate=True)
    assert rel(z, zo) < 1e-2, rel(z, zo)
    # per layer: weights then biases
    o = 0
    for l, (ci, co) in enumerate(learned.LAYERS):
        n = 9 * ci * co
        assert rel(g[o:o + n], go[o:o + n]) < 3e-2, (l, rel(g[o:o + n], go[o:o + n]))
        o += n
    for l, (ci, co) in enumerate(learned.LAYERS):
        assert rel(g[o:o + co], go[o:o + co]) < 3e-2, ("bias", l)
        o += co
    # the oracle's own FP64 gradients agree with the emulated ones to bf16 level
    zf, Af = U.unet_forward(p, x0, emulate=False)
    assert rel(zo, zf) < 5e-2
    pc.close()


def test_training_loss_matches_numpy(oracle_lib):
    W, E = setup("cyc96")
    import torch
    Mo = W.M.copy()
    O = oracle_lib.Oracle(Mo)
    O.streamfunction_init(**LIMITS)
    cf = O.make_coeff_streamfunction()
    pc = learned.LearnedPreconditioner(E, training=True, seed=1)
    rng = np.random.default_rng(2)
    Z = E.make_inv_sfc()
    mask = (Z != 0).astype(np.float64)
    r = np.asfortranarray(rng.standard_normal(W.M.shape2d) * mask)
    e = np.asfortranarray(rng.standard_normal(W.M.shape2d) * mask)
    rt, et = learned._dev(r), learned._dev(e)
    z = pc.apply(rt).cpu().numpy()
    loss = pc.train_step(rt, et, 0.0)
    M = W.M
    D = M.dxu[:, None] * M.dyu[None, :] * M.cosu[None, :]
    inner = (slice(2, M.nx + 2), slice(2, M.ny + 2))

    def S(u):
        return (D * O.apply_op(cf, np.asfortranarray(u)))[inner]

    m = mask > 0
    nu = m.sum()
    dbar = np.mean(1.0 / np.abs(Z[m]))
    # both fields enter the operator with their cyclic halo copies, as on the GPU
    zi = np.asfortranarray(np.where(m, z, 0.0))
    es = np.asfortranarray(e * dbar / np.sqrt(np.sum(r[m] ** 2) / nu))
    O.setcyclic_xy(zi)
    O.setcyclic_xy(es)
    a = np.sum(zi[inner] * S(es))
    b = np.sum(zi[inner] * S(zi))
    c = np.sum(es[inner] * S(es))
    want = (b - 2 * a + c) / c
    assert abs(loss - want) < 1e-6 * max(1.0, abs(want)), (loss, want)
    pc.close()


@pytest.mark.parametrize("name", ["c0", "cyc96"])
def test_fcg_reaches_1e10_and_matches_oracle(oracle_lib, name):
    import torch
    W, E = setup(name)
    pc = learned.LearnedPreconditioner(E, seed=7)  # untrained: FCG still converges (PCG takes over if needed)
    sol = np.zeros(W.M.shape2d, order="F")
    info = learned.solve_fcg(E, pc, W.forc, sol, rtol=2e-11)
    assert info["status"] == 0 and info["rel_residual"] <= 2e-11, info
    O = oracle_lib.Oracle(W.M.copy())
    O.streamfunction_init(**LIMITS)
    cf = O.make_coeff_streamfunction()
    Z = O.make_inv_sfc(cf)
    assert O.rel_residual(cf, Z, W.forc, sol) <= 3e-11
    so = np.zeros(W.M.shape2d, order="F")
    O.congrad_streamfunction(cf, W.forc, so, eps=0.0, max_it=100000, rtol=1e-14)
    O.setcyclic_xy(so)
    m = Z != 0
    assert np.linalg.norm((sol - so)[m]) / np.linalg.norm(so[m]) < 1e-10
    # device tensors in place give the same answer
    s_t = learned._dev(np.zeros(W.M.shape2d))
    learned.solve_fcg(E, pc, learned._dev(W.forc), s_t, rtol=2e-11)
    assert np.linalg.norm(s_t.cpu().numpy() - sol) <= 1e-9 * np.linalg.norm(sol)
    pc.close()


def test_training_reduces_loss():
    """Adam steps on solver-generated pairs of a grid of the training family
    (1440x720 recipe) lower the relative energy-norm loss on a fixed set of
    held-out pairs (the training loop runs end to end on the GPU: pair
    generation, forward, loss, backward, update).  Per-pair losses are noisy
    (random perturbation scales) and the gradient sums are not bit-for-bit
    reproducible, so the check is on the mean over 32 fixed pairs, with the
    learning rate annealed."""
    W = synth._global_like(1440, 720, -80.0, 80.0, 2002, n_land_masses=20, name="train_2002")
    E = ExternalMode(W.M)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(**LIMITS)
    basis = learned.rhs_basis(W, 2, seed=11)
    held = learned.pair_stream(W, E, basis, seed=99)
    held = [next(held) for _ in range(32)]
    pc = learned.LearnedPreconditioner(E, training=True, seed=0)
    before = np.mean([pc.train_step(r, e, 0.0) for r, e in held])
    losses = learned.generate_and_train(pc, W, E, basis, steps=800, lr=1e-3, lr_final=1e-4, seed=4)
    after = np.mean([pc.train_step(r, e, 0.0) for r, e in held])
    assert np.all(np.isfinite(losses))
    assert after < 0.85 * before, (before, after)
    pc.close()


def test_ablation_trained_network_gains():
    """What the trained network gains over the method without it, on a
    held-out grid of the family it was trained on (1440x720 recipe, a seed no
    training grid used): iterations to the 1e-10 true residual with the
    committed weights, with the untrained initial weights, and with
    Jacobi-PCG alone."""
    W = synth._global_like(1440, 720, -80.0, 80.0, 3001, n_land_masses=20, name="heldout_3001")
    E = ExternalMode(W.M)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(**LIMITS)

    def fcg(params):
        q = learned.LearnedPreconditioner(E, params=params)
        s = np.zeros(W.M.shape2d, order="F")
        info = learned.solve_fcg(E, q, W.forc, s, rtol=1e-10, max_it=20000)
        q.close()
        assert info["status"] == 0 and info["rel_residual"] <= 1e-10, info
        return info

    trained = fcg(learned.load_params())
    untrained = fcg(learned.init_params(0))
    s = np.zeros(W.M.shape2d, order="F")
    pcg = E.solve_rtol(W.forc, s, rtol=1e-10, precision=_abi.PREC_F64)
    print("ablation iterations: trained", trained["iterations"], "untrained", untrained["iterations"], "pcg",
          pcg["iterations"])
    assert trained["outer_iterations"] == 1  # converged without the Jacobi-PCG fallback
    assert trained["iterations"] < 0.8 * untrained["iterations"]
    assert trained["iterations"] < 0.8 * pcg["iterations"]


def test_fcg_on_config3_grid(oracle_lib):
    """Config 3: the network trained on the 1440x720 family drives flexible CG
    on the 2048x1024 grid to the FP64 true residual 1e-10; the answer agrees
    with Jacobi-PCG's to 1e-8 relative."""
    W = synth.config3()
    E = ExternalMode(W.M)
    import warnings
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        E.streamfunction_init(**LIMITS)
    pc = learned.LearnedPreconditioner(E, params=learned.load_params())
    s = np.zeros(W.M.shape2d, order="F")
    info = learned.solve_fcg(E, pc, W.forc, s, rtol=1e-10, max_it=20000)
    assert info["status"] == 0 and info["rel_residual"] <= 1e-10, info
    sp = np.zeros(W.M.shape2d, order="F")
    ip = E.solve_rtol(W.forc, sp, rtol=1e-10, precision=_abi.PREC_F64)
    m = E.make_inv_sfc() != 0
    assert np.linalg.norm((s - sp)[m]) <= 1e-8 * np.linalg.norm(sp[m])
    print("config 3 iterations: fcg", info["iterations"], "pcg", ip["iterations"])
    pc.close()
