"""TEST INFRASTRUCTURE ONLY — FP64 numpy restatement of the learned-guess
network (105 -> 256 -> 256 -> 256 -> 37, exact-erf GELU on the hidden layers,
mean-squared-error loss) used to check the library's forward and backward
kernels.  The weights are rounded to BF16 (round to nearest even) exactly as
the library stores them for its products; the biases stay FP32."""
from __future__ import annotations

import math

import numpy as np

LAYERS = [(105, 256), (256, 256), (256, 256), (256, 37)]


def bf16(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def quantize(W: np.ndarray) -> np.ndarray:
    """The weights as the products use them: FP32 master copy rounded to BF16."""
    return bf16(W.astype(np.float32))


def unpack(params: np.ndarray):
    out, o = [], 0
    for ni, no in LAYERS:
        W = params[o:o + ni * no].reshape(no, ni)
        o += ni * no
        b = params[o:o + no]
        o += no
        out.append((W, b))
    return out


_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1 + _erf(z / math.sqrt(2)))


def gelu_grad(z):
    return 0.5 * (1 + _erf(z / math.sqrt(2))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def loss_and_grad(params: np.ndarray, x: np.ndarray, y: np.ndarray):
    layers = unpack(params.astype(np.float64))
    Wq = [quantize(W) for W, _ in layers]
    bs = [b.astype(np.float64) for _, b in layers]
    acts, pres = [x.astype(np.float64)], []
    h = acts[0]
    for l, (W, b) in enumerate(zip(Wq, bs)):
        z = h @ W.T + b
        pres.append(z)
        h = gelu(z) if l < len(LAYERS) - 1 else z
        acts.append(h)
    B, out = y.shape
    d = h - y.astype(np.float64)
    loss = float(np.mean(d * d))
    g = 2 * d / (B * out)
    grads = []
    for l in range(len(LAYERS) - 1, -1, -1):
        if l < len(LAYERS) - 1:
            g = g * gelu_grad(pres[l])
        dW = g.T @ acts[l]
        db = g.sum(0)
        grads.append((dW, db))
        g = g @ Wq[l]
    grads.reverse()
    flat = np.concatenate([np.r_[dW.ravel(), db] for dW, db in grads])
    return loss, flat
