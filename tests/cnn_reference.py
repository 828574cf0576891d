"""CPU FP64 restatement of the learned-preconditioner network (checker of the tensor-core
kernels): 4 layers of 3x3x3 convolution, 16 channels, ReLU after layers 1-3, zero padding.

Parameter layout (as the device library): per layer W[27 taps][16 out][16 in] then b[16],
tap = 9*(dk+1) + 3*(dj+1) + (di+1).  Arrays are (nK, nJ, nI, C), i fastest.

`bf16=True` rounds weights, the input and every stored activation / back-propagated
gradient to bfloat16 (round to nearest even) at the points where the device stores bf16.
"""
from __future__ import annotations

import numpy as np

C = 16
LAYER = 27 * 16 * 16 + 16
TAPS = [(dk, dj, di) for dk in (-1, 0, 1) for dj in (-1, 0, 1) for di in (-1, 0, 1)]


def bf16(a):
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    out = []
    for l in range(4):
        blk = params[l * LAYER:(l + 1) * LAYER]
        W = blk[:27 * 256].reshape(27, 16, 16).astype(np.float64)
        b = blk[27 * 256:].astype(np.float64)
        out.append((W, b))
    return out


def shift(x, dk, dj, di):
    """y[k,j,i] = x[k+dk, j+dj, i+di] with zeros outside."""
    nK, nJ, nI = x.shape[:3]
    y = np.zeros_like(x)
    ks, ke = max(0, -dk), min(nK, nK - dk)
    js, je = max(0, -dj), min(nJ, nJ - dj)
    is_, ie = max(0, -di), min(nI, nI - di)
    y[ks:ke, js:je, is_:ie] = x[ks + dk:ke + dk, js + dj:je + dj, is_ + di:ie + di]
    return y


def conv(x, W, b=None):
    out = np.zeros(x.shape[:3] + (W.shape[1],))
    for t, (dk, dj, di) in enumerate(TAPS):
        out += shift(x, dk, dj, di) @ W[t].T
    if b is not None:
        out += b
    return out


def conv_T(g, W):
    """Adjoint of conv: x_grad[c] = sum_t W[t]^T g[c - off(t)]."""
    out = np.zeros(g.shape[:3] + (W.shape[2],))
    for t, (dk, dj, di) in enumerate(TAPS):
        out += shift(g, -dk, -dj, -di) @ W[t]
    return out


def forward(params, x2, shape, bf=True, extra_const=None):
    """extra_const: value of a constant input channel 2 (the level channel), if any."""
    nI, nJ, nK = shape
    layers = unpack(params)
    rnd = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    x = np.zeros((nK, nJ, nI, C))
    x[..., :2] = rnd(x2.reshape(nK, nJ, nI, 2))
    if extra_const is not None:
        x[..., 2] = rnd(np.full((nK, nJ, nI), extra_const))
    acts = [x]
    for l in range(3):
        W, b = layers[l]
        z = conv(acts[-1], rnd(W), b)
        acts.append(rnd(np.maximum(z, 0.0)))
    W, b = layers[3]
    y = conv(acts[-1], rnd(W), b)[..., 0]
    return y.reshape(-1), acts


def grad(params, x2, dy, shape, bf=True):
    """d(sum dy * y)/d(params), back-propagated as the device does (bf16 gradients between layers)."""
    nI, nJ, nK = shape
    layers = unpack(params)
    rnd = bf16 if bf else (lambda a: np.asarray(a, dtype=np.float64))
    y, acts = forward(params, x2, shape, bf)
    g = np.zeros((nK, nJ, nI, C))
    g[..., 0] = rnd(dy.reshape(nK, nJ, nI))
    dparams = np.zeros(4 * LAYER)
    for l in range(3, -1, -1):
        x = acts[l]
        dW = np.zeros((27, 16, 16))
        for t, (dk, dj, di) in enumerate(TAPS):
            xs = shift(x, dk, dj, di).reshape(-1, C)
            dW[t] = g.reshape(-1, C).T @ xs
        db = g.reshape(-1, C).sum(0)
        dparams[l * LAYER:l * LAYER + 27 * 256] = dW.reshape(-1)
        dparams[l * LAYER + 27 * 256:(l + 1) * LAYER] = db
        if l == 0:
            break
        W, _ = layers[l]
        gx = conv_T(g, rnd(W))
        g = rnd(np.where(acts[l] > 0, gx, 0.0))
    return y, dparams


def random_params(seed, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(4 * LAYER, dtype=np.float32)
    for l in range(4):
        cin = 2 if l == 0 else 16
        W = np.zeros((27, 16, 16), dtype=np.float32)
        W[:, :, :cin] = rng.standard_normal((27, 16, cin)) * scale / np.sqrt(27 * cin)
        if l == 3:
            W[:, 1:, :] = 0.0
        p[l * LAYER:l * LAYER + 27 * 256] = W.reshape(-1)
        p[l * LAYER + 27 * 256:(l + 1) * LAYER] = rng.uniform(-0.1, 0.1, 16) * (l < 3)
    return p
