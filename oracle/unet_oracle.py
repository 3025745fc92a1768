"""CPU FP64 restatement of the learned preconditioner's network -- TEST
INFRASTRUCTURE ONLY.  Nothing in the product imports this module; the tests
use it as the checker of the GPU kernels (forward values and gradients).

The reference has no learned part, so this oracle is pinned by its own
known-answer checks instead (tests/test_unet_oracle.py): the convolution
against a direct loop and against torch's float64 conv2d on the CPU, the
backward pass against central finite differences.

Conventions match the GPU side (pyom2_b200/csrc/conv_tc.cuh):
* images are [C][H][W] float64 here; the GPU stores "channel-group planar"
  bf16 [C/8][H][W][8] (``to_planar`` / ``from_planar``);
* a 3x3 convolution is a cross-correlation with zero padding 1 and weights
  [Cout][Cin][3][3] (PyTorch order);
* 2x2 average pooling, nearest 2x upsampling.
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------------------
# bf16 helpers
def bf16_round(a):
    """Round float values to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a):
    """bfloat16 bit patterns (uint16) of float values (nearest even)."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def bits_to_f64(b):
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def to_planar(x):
    """[C][H][W] -> [C/8][H][W][8]."""
    C, H, W = x.shape
    return np.ascontiguousarray(x.reshape(C // 8, 8, H, W).transpose(0, 2, 3, 1))


def from_planar(p):
    """[C/8][H][W][8] -> [C][H][W]."""
    G, H, W, _ = p.shape
    return np.ascontiguousarray(p.transpose(0, 3, 1, 2).reshape(G * 8, H, W))


# ---------------------------------------------------------------------------
# layers
def conv3x3(x, w, b=None):
    """Cross-correlation, zero padding 1: out[o,y,x] = sum_c,ky,kx w[o,c,ky,kx] x[c,y+ky-1,x+kx-1]."""
    C, H, W = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    out = np.zeros((w.shape[0], H, W))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("oc,chw->ohw", w[:, :, ky, kx], xp[:, ky:ky + H, kx:kx + W], optimize=True)
    if b is not None:
        out += b[:, None, None]
    return out


def conv3x3_backward(x, w, g):
    """Gradients of conv3x3 for output gradient g: (dx, dw, db)."""
    C, H, W = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    gp = np.pad(g, ((0, 0), (1, 1), (1, 1)))
    dw = np.zeros_like(w)
    dx = np.zeros_like(x)
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("ohw,chw->oc", g, xp[:, ky:ky + H, kx:kx + W], optimize=True)
            # x[c, y', x'] feeds out[o, y'-ky+1, x'-kx+1]
            dx += np.einsum("oc,ohw->chw", w[:, :, ky, kx], gp[:, 2 - ky:2 - ky + H, 2 - kx:2 - kx + W],
                            optimize=True)
    return dx, dw, g.sum(axis=(1, 2))


def pool2(x):
    C, H, W = x.shape
    return x.reshape(C, H // 2, 2, W // 2, 2).mean(axis=(2, 4))


def pool2_backward(g):
    return np.repeat(np.repeat(g, 2, axis=1), 2, axis=2) * 0.25


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up2_backward(g):
    C, H, W = g.shape
    return g.reshape(C, H // 2, 2, W // 2, 2).sum(axis=(2, 4))


def relu(x):
    return np.maximum(x, 0.0)


# ---------------------------------------------------------------------------
# the network (pyom2_b200/csrc/unet.cuh): (cin, cout, level, epilogue)
LAYERS = [(16, 16, 0, "plain"), (16, 16, 0, "plain"), (16, 32, 1, "plain"), (32, 32, 1, "plain"),
          (32, 64, 2, "plain"), (64, 64, 2, "plain"), (64, 64, 3, "plain"), (64, 64, 3, "plain"),
          (64, 64, 3, "up"), (64, 32, 2, "up"), (32, 16, 1, "up"), (16, 16, 0, "f32")]


def split_params(params):
    """Flat f32 vector -> [(w [cout][cin][3][3], b [cout])] per layer."""
    params = np.asarray(params, dtype=np.float64)
    ws, o = [], 0
    for ci, co, _, _ in LAYERS:
        ws.append(params[o:o + 9 * ci * co].reshape(co, ci, 3, 3))
        o += 9 * ci * co
    out = []
    for (ci, co, _, _), w in zip(LAYERS, ws):
        out.append((w, params[o:o + co]))
        o += co
    return out


def num_params():
    return sum(9 * ci * co + co for ci, co, _, _ in LAYERS)


def _r(a, emulate):
    """The rounding of a stored bf16 activation (through f32, as on the GPU)."""
    return bf16_round(a) if emulate else a


def unet_forward(params, x0, emulate=True):
    """x0 [16][H][W] -> (z [H][W], activations).  With emulate, weights and
    every stored activation are rounded to bf16 where the GPU stores them."""
    L = split_params(params)
    wq = [(bf16_round(w) if emulate else w, np.float32(b).astype(np.float64) if emulate else b) for w, b in L]
    A = {"X0": x0}

    def cv(l, x):
        w, b = wq[l]
        return conv3x3(x, w, b)

    A["A1"] = _r(relu(cv(0, x0)), emulate)
    A["S1"] = _r(relu(cv(1, A["A1"])), emulate)
    A["P1"] = _r(pool2(A["S1"]), emulate)
    A["A2"] = _r(relu(cv(2, A["P1"])), emulate)
    A["S2"] = _r(relu(cv(3, A["A2"])), emulate)
    A["P2"] = _r(pool2(A["S2"]), emulate)
    A["A3"] = _r(relu(cv(4, A["P2"])), emulate)
    A["S3"] = _r(relu(cv(5, A["A3"])), emulate)
    A["P3"] = _r(pool2(A["S3"]), emulate)
    A["A4"] = _r(relu(cv(6, A["P3"])), emulate)
    A["B4"] = _r(relu(cv(7, A["A4"])), emulate)
    A["U3"] = _r(relu(up2(cv(8, A["B4"])) + A["S3"]), emulate)
    A["U2"] = _r(relu(up2(cv(9, A["U3"])) + A["S2"]), emulate)
    A["U1"] = _r(relu(up2(cv(10, A["U2"])) + A["S1"]), emulate)
    z = cv(11, A["U1"])[0]
    return z, A


def unet_backward(params, A, gz, emulate=True):
    """Parameter gradients of sum(gz * z) (flat, the layout of the params)."""
    L = split_params(params)
    wq = [bf16_round(w) if emulate else w for w, _ in L]
    dW = [None] * len(LAYERS)
    dB = [None] * len(LAYERS)

    def back(l, x, g, gate=None, need_dx=True):
        dx, dw, db = conv3x3_backward(x, wq[l], g)
        dW[l], dB[l] = dw, db
        if not need_dx:
            return None
        if gate is not None:
            dx = np.where(gate > 0, dx, 0.0)
        return _r(dx, emulate)

    gO = np.zeros((16,) + gz.shape)
    gO[0] = _r(gz, emulate)
    gU1 = back(11, A["U1"], gO, A["U1"])
    gv10 = _r(up2_backward(gU1), emulate)
    gU2 = back(10, A["U2"], gv10, A["U2"])
    gv9 = _r(up2_backward(gU2), emulate)
    gU3 = back(9, A["U3"], gv9, A["U3"])
    gv8 = _r(up2_backward(gU3), emulate)
    gB4 = back(8, A["B4"], gv8, A["B4"])
    gA4 = back(7, A["A4"], gB4, A["A4"])
    gP3 = back(6, A["P3"], gA4, None)
    gS3 = _r(np.where(A["S3"] > 0, gU3 + pool2_backward(gP3), 0.0), emulate)
    gA3 = back(5, A["A3"], gS3, A["A3"])
    gP2 = back(4, A["P2"], gA3, None)
    gS2 = _r(np.where(A["S2"] > 0, gU2 + pool2_backward(gP2), 0.0), emulate)
    gA2 = back(3, A["A2"], gS2, A["A2"])
    gP1 = back(2, A["P1"], gA2, None)
    gS1 = _r(np.where(A["S1"] > 0, gU1 + pool2_backward(gP1), 0.0), emulate)
    gA1 = back(1, A["A1"], gS1, A["A1"])
    back(0, A["X0"], gA1, need_dx=False)
    return np.concatenate([d.ravel() for d in dW] + [b.ravel() for b in dB])
