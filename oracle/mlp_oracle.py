"""CPU restatement of the learned initialiser's arithmetic (numpy, FP64).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA initialiser's forward pass,
loss and gradients (milne-eddington_b200/csrc/me_mlp.cu).  Only tests/ may
import it; no product path does.

The reference has no learned component, so nothing here restates reference
code.  The network is 4 layers: Z_l = A_{l-1} W_l^T + b_l, A_l = GELU(Z_l) for
l < 3 (GELU(z) = z Phi(z), the exact erf form), Y = A_2 W_3^T + b_3; loss =
mean over rows and the first `nout` outputs of (Y - T)^2.  Parameters are
flattened layer by layer as W [dout][din] then b [dout], the layout of
me_mlp_get_params.

`bf16=True` rounds the same tensors the device rounds to bfloat16 (round to
nearest even): the input rows, every weight matrix, the hidden activations,
dY, every dZ and, for the bias gradient, the same dZ; the products are then
summed in FP64 instead of the device's FP32, so the two agree to about 1e-6
relative apart from rare ties at a rounding boundary.  The finite-difference
check in the tests pins this file's backward pass against its own forward pass.
"""
from __future__ import annotations

import math

import numpy as np

HIDDEN = 256
NOUT = 10
NOUT_PAD = 32


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Rounds float values to the nearest bfloat16 (ties to even), returned as FP64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    cdf = 0.5 * (1.0 + _erf(z / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)
    return cdf + z * pdf


def shapes(nin_pad: int):
    """(dout, din) of the four layers."""
    return [(HIDDEN, nin_pad), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (NOUT_PAD, HIDDEN)]


def unflatten(params: np.ndarray, nin_pad: int):
    out, off = [], 0
    for dout, din in shapes(nin_pad):
        W = params[off:off + dout * din].reshape(dout, din).astype(np.float64)
        off += dout * din
        b = params[off:off + dout].astype(np.float64)
        off += dout
        out.append((W, b))
    assert off == params.size
    return out


def flatten(layers) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers])


def forward(params: np.ndarray, x: np.ndarray, nin_pad: int, bf16: bool = False):
    """Returns Y [rows][32] and the per-layer (A_prev, Z) cache."""
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unflatten(params, nin_pad)
    a = rnd(x)
    cache = []
    for l, (W, b) in enumerate(layers):
        z = a @ rnd(W).T + b
        cache.append((a, z))
        if l < len(layers) - 1:
            a = rnd(gelu(z))
        else:
            a = z
    return a, cache


def loss_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray, nin_pad: int,
              bf16: bool = False):
    """Mean squared error over rows x the first 10 outputs, and its gradient."""
    rnd = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unflatten(params, nin_pad)
    y, cache = forward(params, x, nin_pad, bf16)
    rows = x.shape[0]
    d = y[:, :NOUT] - t
    loss = float(np.mean(d * d))
    dy = np.zeros_like(y)
    dy[:, :NOUT] = 2.0 * d / (rows * NOUT)
    dz = rnd(dy)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        a_prev, _ = cache[l]
        W, _ = layers[l]
        gW = dz.T @ a_prev
        gb = dz.sum(axis=0)
        grads[l] = (gW, gb)
        if l == 0:
            break
        da = dz @ rnd(W)
        dz = rnd(da * gelu_grad(cache[l - 1][1]))
    return loss, flatten(grads)


def adam(params, m, v, g, t, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma and Ba 2015, with bias correction); returns new arrays."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** t)
    vh = v / (1 - b2 ** t)
    return params - lr * mh / (np.sqrt(vh) + eps), m, v
