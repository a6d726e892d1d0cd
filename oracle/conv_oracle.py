"""CPU restatement of the learned corrector's convolution layers (numpy,
float64).  TEST INFRASTRUCTURE ONLY: the checker of the tcgen05 convolution
kernels (forward, input gradient, weight gradient) in tests/; never imported
by the package.

Conventions of csrc/pfag_corrector.cu: an activation is [B][H+2][W+2][C]
with a zero halo (the convolution's zero padding), weights are
[Cout][9][Cin] with tap t = (dy+1)*3 + (dx+1), i.e.
    y[b, y, x, co] = bias[co] + sum_{t, ci} w[co, t, ci] x[b, y+dy, x+dx, ci].
The reference has no learned part, so there is no reference code to pin this
against; the module is pinned by central finite differences of its own
forward pass (tests/test_conv_oracle.py).
"""
from __future__ import annotations

import math

import numpy as np

TAPS = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def bf16(a) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even) and return as float64."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def pad(x: np.ndarray) -> np.ndarray:
    """[B][H][W][C] -> [B][H+2][W+2][C] with a zero halo."""
    return np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))


def conv_fwd(xp: np.ndarray, w: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Pre-activation on the interior: [B][H][W][Cout] from the padded input."""
    B, Hp, Wp, _ = xp.shape
    H, W = Hp - 2, Wp - 2
    out = np.zeros((B, H, W, w.shape[0])) + b
    for t, (dy, dx) in enumerate(TAPS):
        out += np.einsum("bhwc,oc->bhwo", xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :], w[:, t, :])
    return out


def conv_dgrad(dz: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Input gradient on the interior [B][H][W][Cin] from dz [B][H][W][Cout]."""
    dzp = pad(dz)
    B, H, W, _ = dz.shape
    out = np.zeros((B, H, W, w.shape[2]))
    for t, (dy, dx) in enumerate(TAPS):
        out += np.einsum("bhwo,oc->bhwc", dzp[:, 1 - dy:1 - dy + H, 1 - dx:1 - dx + W, :], w[:, t, :])
    return out


def conv_wgrad(xp: np.ndarray, dz: np.ndarray):
    """dW [Cout][9][Cin] and db [Cout] from the padded input and dz [B][H][W][Cout]."""
    B, H, W, co = dz.shape
    dw = np.zeros((co, 9, xp.shape[3]))
    for t, (dy, dx) in enumerate(TAPS):
        dw[:, t, :] = np.einsum("bhwo,bhwc->oc", dz, xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W, :])
    return dw, dz.sum(axis=(0, 1, 2))


def gelu(x):
    return 0.5 * x * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + np.vectorize(math.erf)(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2 * math.pi)
