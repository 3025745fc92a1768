"""GPU parity of the tcgen05 3x3 convolution (pyomgpu_conv3x3_bf16) against
the FP64 CPU oracle on the same bf16-rounded inputs and weights.

Tolerances: the GPU accumulates in FP32 (|rel| ~ 1e-6 of the sum of |terms|)
and rounds bf16 outputs to nearest even (half an ulp, 2**-9 relative), so
bf16 results must match the oracle rounded to bf16 within 2 bf16 ulps plus
a small absolute term scaled by the sum of |terms|; f32 results to 1e-5
of that scale.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import unet_oracle as U
from pyom2_b200 import _abi

pytestmark = pytest.mark.gpu

PAIRS = [(16, 16), (16, 32), (16, 64), (32, 16), (32, 32), (32, 64), (64, 16), (64, 32), (64, 64)]
SHAPES = [(8, 128), (12, 200), (6, 40), (36, 300)]


def dev_bits(a):
    return torch.from_numpy(U.bf16_bits(a).view(np.int16)).cuda()


def host_f64(t):
    return U.bits_to_f64(t.cpu().numpy().view(np.uint16))


def ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def run(cin, cout, H, W, x, w, b, relu=1, epi=0, gate=None, addend=None, pool=False, flip=0):
    L = _abi.load()
    xd = dev_bits(U.to_planar(x))
    wd = torch.from_numpy(np.ascontiguousarray(w, dtype=np.float32)).cuda()
    bd = None if b is None else torch.from_numpy(b.astype(np.float32)).cuda()
    if epi == 2:
        y = torch.zeros((H, W), dtype=torch.float32, device="cuda")
    elif epi == 1:
        y = torch.zeros((cout // 8, 2 * H, 2 * W, 8), dtype=torch.int16, device="cuda")
    else:
        y = torch.zeros((cout // 8, H, W, 8), dtype=torch.int16, device="cuda")
    gd = None if gate is None else dev_bits(U.to_planar(gate))
    ad = None if addend is None else dev_bits(U.to_planar(addend))
    pd = torch.zeros((cout // 8, H // 2, W // 2, 8), dtype=torch.int16, device="cuda") if pool else None
    rc = L.pyomgpu_conv3x3_bf16(cin, cout, H, W, ptr(xd), ptr(wd), ptr(bd), relu, epi, ptr(gd), ptr(ad), ptr(y),
                                ptr(pd), flip, None)
    _abi.check(rc)
    torch.cuda.synchronize()
    if epi == 2:
        return y.cpu().numpy().astype(np.float64), None
    out = U.from_planar(host_f64(y))
    return out, (None if pd is None else U.from_planar(host_f64(pd)))


def close_bf16(got, want, scale):
    err = np.abs(got - U.bf16_round(want))
    tol = 2.0 * 2.0 ** -8 * np.abs(want) + 1e-5 * scale
    assert np.all(err <= tol), (err.max(), np.argmax(err / tol))


def inputs(cin, cout, H, W, seed):
    rng = np.random.default_rng(seed)
    x = U.bf16_round(rng.standard_normal((cin, H, W)))
    w = U.bf16_round(rng.standard_normal((cout, cin, 3, 3)) / np.sqrt(9 * cin))
    b = rng.standard_normal(cout) * 0.1
    return x, w, b


@pytest.mark.parametrize("cin,cout", PAIRS)
def test_conv_plain_relu(cin, cout):
    for k, (H, W) in enumerate(SHAPES):
        x, w, b = inputs(cin, cout, H, W, 10 * cin + cout + k)
        got, _ = run(cin, cout, H, W, x, w, b, relu=1)
        want = U.relu(U.conv3x3(x, w, b.astype(np.float32).astype(np.float64)))
        scale = U.conv3x3(np.abs(x), np.abs(w)).max()
        close_bf16(got, want, scale)


@pytest.mark.parametrize("cin,cout", [(16, 16), (32, 64), (64, 64)])
def test_conv_f32_output(cin, cout):
    H, W = 12, 200
    x, w, b = inputs(cin, cout, H, W, 7)
    got, _ = run(cin, cout, H, W, x, w, b, relu=0, epi=2)
    bb = b.astype(np.float32).astype(np.float64)
    want = U.conv3x3(x, w, bb)[0]
    scale = U.conv3x3(np.abs(x), np.abs(w)).max()
    assert np.abs(got - want).max() <= 1e-5 * scale


@pytest.mark.parametrize("cin,cout", [(16, 32), (64, 16)])
def test_conv_gate_addend_pool(cin, cout):
    H, W = 8, 260
    x, w, b = inputs(cin, cout, H, W, 3)
    rng = np.random.default_rng(4)
    gate = U.bf16_round(rng.standard_normal((cout, H, W)))
    add = U.bf16_round(rng.standard_normal((cout, H, W)))
    got, pooled = run(cin, cout, H, W, x, w, b, relu=1, gate=gate, addend=add, pool=True)
    bb = b.astype(np.float32).astype(np.float64)
    want = np.where(gate > 0, U.relu(U.conv3x3(x, w, bb) + add), 0.0)
    scale = U.conv3x3(np.abs(x), np.abs(w)).max() + 3
    close_bf16(got, want, scale)
    # the pool averages the stored (bf16) outputs
    close_bf16(pooled, U.pool2(got), scale)


@pytest.mark.parametrize("cin,cout", [(64, 64), (32, 16)])
def test_conv_up_skip(cin, cout):
    H, W = 6, 70
    x, w, b = inputs(cin, cout, H, W, 5)
    skip = U.bf16_round(np.random.default_rng(6).standard_normal((cout, 2 * H, 2 * W)))
    got, _ = run(cin, cout, H, W, x, w, b, relu=1, epi=1, addend=skip)
    bb = b.astype(np.float32).astype(np.float64)
    want = U.relu(U.up2(U.conv3x3(x, w, bb)) + skip)
    scale = U.conv3x3(np.abs(x), np.abs(w)).max() + 3
    close_bf16(got, want, scale)


@pytest.mark.parametrize("cin,cout", [(16, 32), (64, 64), (32, 16)])
def test_conv_backward_data(cin, cout):
    """flip = 1 computes dx of the forward layer w: [cin][cout][3][3]."""
    H, W = 10, 150
    rng = np.random.default_rng(8)
    g = U.bf16_round(rng.standard_normal((cin, H, W)))
    wf = U.bf16_round(rng.standard_normal((cin, cout, 3, 3)) / np.sqrt(9 * cin))  # forward: cout -> cin
    xdummy = np.zeros((cout, H, W))
    dx, _, _ = U.conv3x3_backward(xdummy, wf, g)
    got, _ = run(cin, cout, H, W, g, wf, None, relu=0, flip=1)
    scale = U.conv3x3(np.abs(g), np.abs(np.transpose(wf, (1, 0, 2, 3)))).max()
    close_bf16(got, dx, scale)
