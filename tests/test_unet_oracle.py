"""Known-answer checks that pin the CPU oracle of the learned preconditioner
(oracle/unet_oracle.py): convolution against a direct loop and against
torch's float64 conv2d, backward passes against central finite differences,
bf16 rounding against torch's bfloat16 conversion."""
import numpy as np
import torch

from oracle import unet_oracle as U


def test_conv_against_loop_and_torch():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((3, 5, 7))
    w = rng.standard_normal((4, 3, 3, 3))
    b = rng.standard_normal(4)
    y = U.conv3x3(x, w, b)
    ref = np.zeros_like(y)
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    for o in range(4):
        for i in range(5):
            for j in range(7):
                ref[o, i, j] = b[o] + np.sum(w[o] * xp[:, i:i + 3, j:j + 3])
    assert np.allclose(y, ref, rtol=1e-13, atol=1e-13)
    t = torch.nn.functional.conv2d(torch.from_numpy(x)[None], torch.from_numpy(w), torch.from_numpy(b), padding=1)
    assert np.allclose(y, t[0].numpy(), rtol=1e-13, atol=1e-13)


def test_conv_backward_finite_differences():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((2, 4, 6))
    w = rng.standard_normal((3, 2, 3, 3))
    g = rng.standard_normal((3, 4, 6))
    dx, dw, db = U.conv3x3_backward(x, w, g)
    f = lambda xx, ww: np.sum(g * U.conv3x3(xx, ww))
    h = 1e-6
    for idx in [(0, 0, 0), (1, 2, 3), (0, 3, 5)]:
        e = np.zeros_like(x)
        e[idx] = h
        assert abs((f(x + e, w) - f(x - e, w)) / (2 * h) - dx[idx]) < 1e-7
    for idx in [(0, 0, 0, 0), (2, 1, 2, 1), (1, 0, 1, 2)]:
        e = np.zeros_like(w)
        e[idx] = h
        assert abs((f(x, w + e) - f(x, w - e)) / (2 * h) - dw[idx]) < 1e-7
    assert np.allclose(db, g.sum(axis=(1, 2)))


def test_pool_up_adjoint():
    rng = np.random.default_rng(2)
    a = rng.standard_normal((2, 6, 8))
    c = rng.standard_normal((2, 3, 4))
    # <pool(a), c> = <a, pool^T(c)> and <up(c), a> = <c, up^T(a)>
    assert np.isclose(np.sum(U.pool2(a) * c), np.sum(a * U.pool2_backward(c)))
    assert np.isclose(np.sum(U.up2(c) * a), np.sum(c * U.up2_backward(a)))


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(3)
    v = (rng.standard_normal(10000) * 10.0 ** rng.integers(-8, 8, 10000)).astype(np.float32)
    t = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(U.bf16_round(v), t)
    assert np.array_equal(U.bits_to_f64(U.bf16_bits(v)), t)


def test_planar_roundtrip():
    x = np.arange(16 * 3 * 5, dtype=np.float64).reshape(16, 3, 5)
    p = U.to_planar(x)
    assert p.shape == (2, 3, 5, 8) and p[1, 2, 4, 3] == x[11, 2, 4]
    assert np.array_equal(U.from_planar(p), x)


def test_network_backward_finite_differences():
    """The oracle's U-Net gradient (pure FP64) against central differences."""
    rng = np.random.default_rng(4)
    n = U.num_params()
    p = rng.standard_normal(n) * 0.2
    x0 = rng.standard_normal((16, 16, 24))
    gz = rng.standard_normal((16, 24))
    z, A = U.unet_forward(p, x0, emulate=False)
    g = U.unet_backward(p, A, gz, emulate=False)
    f = lambda q: float(np.sum(gz * U.unet_forward(q, x0, emulate=False)[0]))
    h = 1e-6
    # one weight and one bias of several layers (offsets of the flat layout)
    offs, o = [], 0
    for ci, co, _, _ in U.LAYERS:
        offs.append(o + 9 * ci * co // 2)
        o += 9 * ci * co
    for ci, co, _, _ in U.LAYERS:
        offs.append(o + co // 2)
        o += co
    for k in offs[::3]:
        e = np.zeros(n)
        e[k] = h
        fd = (f(p + e) - f(p - e)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(fd)), (k, fd, g[k])
