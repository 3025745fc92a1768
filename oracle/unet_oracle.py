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
