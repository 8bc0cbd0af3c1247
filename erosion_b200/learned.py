"""The learned initial guess from Python: training sets from the solver's own
erosion runs, and training, through the C ABI (erosion_lw_*).

An erosion run solves twice per RK2 step (the state, then the half-step
state); each solve's warm start is the previous solve's density with every
body's rigid part carried to the new nodes (`reanchor`, the same arithmetic
as the library's k_warm_reanchor).  The network (learned.cu) predicts, per
body, the encoding of the increment of the density over that warm start from
the body's geometry features and the encoding of the previous solve's
increment; with warm_start = 2 the candidate guess is the warm start plus
that prediction.  A training row is therefore, for consecutive solves
i-2, i-1, i with unchanged body count,

    X = [geometry features of solve i (68) | encoding of d_{i-1} on solve i-1's nodes (37)]
    Y = encoding of d_i on solve i's nodes (37)

with d_i = x_i - reanchor(x_{i-1}) the increment of solve i over its warm
start.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PI64, check, ptr

PF = ctypes.POINTER(ctypes.c_float)


def dims() -> tuple[int, int, int]:
    g, i, o = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    _lib.load().erosion_lw_dims(ctypes.byref(g), ctypes.byref(i), ctypes.byref(o))
    return g.value, i.value, o.value


def _fp(a):
    return a.ctypes.data_as(PF)


def features(params, n, M, nout, xx, yy) -> np.ndarray:
    ng, _, _ = dims()
    f = np.zeros((M, ng), np.float32)
    check(_lib.load().erosion_lw_features(ctypes.byref(params), n, M, nout, ptr(xx), ptr(yy), _fp(f)))
    return f


def encode(params, n, M, nout, xx, yy, den) -> np.ndarray:
    _, _, no = dims()
    t = np.zeros((M, no), np.float32)
    den = np.ascontiguousarray(den, dtype=np.float64)
    check(_lib.load().erosion_lw_encode(ctypes.byref(params), n, M, nout, ptr(xx), ptr(yy), ptr(den), _fp(t)))
    return t


def getxy(n, M, th, ln, xs, ys):
    xx, yy = np.zeros(M * n), np.zeros(M * n)
    check(_lib.load().erosion_getxy(n, M, ptr(th), ptr(ln), ptr(xs), ptr(ys), ptr(xx), ptr(yy)))
    return xx, yy


def reanchor(n, nout, xo, yo, xn, yn, den):
    """The previous solve's density carried to new nodes: per body, the rigid
    part (node means t1, t2 of the two components; rotation coefficient t3
    about the node mean, least squares on (-(y - yc), x - xc)) is evaluated
    at the new nodes about their own mean, the remainder stays attached to
    the node index; wall and stokeslet/rotlet entries unchanged."""
    den = np.asarray(den, dtype=np.float64)
    out = den.copy()
    M = len(xo) // n
    xo, yo = np.asarray(xo).reshape(M, n), np.asarray(yo).reshape(M, n)
    xn, yn = np.asarray(xn).reshape(M, n), np.asarray(yn).reshape(M, n)
    for b in range(M):
        off = 2 * nout + 2 * n * b
        sx, sy = den[off:off + n], den[off + n:off + 2 * n]
        fx, fy = -(yo[b] - yo[b].mean()), xo[b] - xo[b].mean()
        gx, gy = -(yn[b] - yn[b].mean()), xn[b] - xn[b].mean()
        dd = (fx * fx + fy * fy).sum()
        t3 = (fx * sx + fy * sy).sum() / dd if dd > 0 else 0.0
        out[off:off + n] = sx + t3 * (gx - fx)
        out[off + n:off + 2 * n] = sy + t3 * (gy - fy)
    return out


def trajectory(params, sp, n, nout, th, ln, xs, ys, steps: int):
    """Runs `steps` RK2 erosion steps (erosion_rk2_step, host arrays, updated
    in place) and returns every solve in order, two per step: (xx, yy,
    density, M) of the nodes and density of each stage, with None for the
    solves of a step in which a body was deleted."""
    L = _lib.load()
    M = len(ln)
    nb = np.array([M], np.int64)
    t = np.zeros(1)
    dele = np.zeros(M, np.int64)
    out = []
    for _ in range(steps):
        Mk = int(nb[0])
        rc = L.erosion_rk2_step(ctypes.byref(params), ctypes.byref(sp), n, nb.ctypes.data_as(PI64), nout, ptr(th),
                                ptr(ln), ptr(xs), ptr(ys), ptr(t), dele.ctypes.data_as(PI64))
        check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
        if int(nb[0]) != Mk:
            out += [None, None]
            continue
        for stage in (0, 1):
            den = np.zeros(2 * nout + 2 * n * Mk + 3 * Mk)
            xx, yy = np.zeros(n * Mk), np.zeros(n * Mk)
            check(L.erosion_get_step_density(stage, ptr(den), den.size))
            check(L.erosion_get_step_nodes(stage, ptr(xx), ptr(yy), xx.size))
            out.append((xx, yy, den, Mk))
    return out


def training_rows(params, n, nout, traj):
    """(X, Y) rows of consecutive solve triples of a trajectory (see the
    module docstring); triples that cross a body deletion are skipped."""
    X, Y = [], []
    inc = [None] * len(traj)
    for i in range(1, len(traj)):
        a, b = traj[i - 1], traj[i]
        if a is None or b is None or a[3] != b[3]:
            continue
        inc[i] = b[2] - reanchor(n, nout, a[0], a[1], b[0], b[1], a[2])
    for i in range(2, len(traj)):
        if inc[i] is None or inc[i - 1] is None:
            continue
        xx, yy, _, M = traj[i]
        px, py = traj[i - 1][0], traj[i - 1][1]
        f = features(params, n, M, nout, xx, yy)
        hist = encode(params, n, M, nout, px, py, inc[i - 1])
        targ = encode(params, n, M, nout, xx, yy, inc[i])
        X.append(np.concatenate([f, hist], 1))
        Y.append(targ)
    if not X:
        _, ni, no = dims()
        return np.zeros((0, ni), np.float32), np.zeros((0, no), np.float32)
    return np.ascontiguousarray(np.concatenate(X)), np.ascontiguousarray(np.concatenate(Y))


def train(X, Y, epochs=300, batch=64, lr=1e-3, seed=3) -> float:
    """Trains the library's network from scratch on the rows; returns the
    last epoch's mean squared error of the standardised targets."""
    loss = ctypes.c_double()
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    check(_lib.load().erosion_lw_train(_fp(X), _fp(Y), len(X), epochs, batch, lr, seed, ctypes.byref(loss)))
    return loss.value


def areas(n, th, ln, xs, ys):
    """Body areas of a theta-L state as getareas computes them
    (PostProcess.jl:36-58): the two one-dimensional divergence-theorem
    estimates -sum (x - xsm) n_x ds and -sum (y - ysm) n_y ds with the
    inward normal (-sin th, cos th) and ds = L/n, clipped at zero and
    averaged."""
    M = len(ln)
    xx, yy = getxy(n, M, th[: M * n], ln[:M], xs[:M], ys[:M])
    x = xx.reshape(M, n) - xs[:M, None]
    y = yy.reshape(M, n) - ys[:M, None]
    t = th[: M * n].reshape(M, n)
    nx, ny = -np.sin(t), np.cos(t)
    ds = ln[:M] / n
    ax = np.maximum(-(x * nx).sum(1) * ds, 0.0)
    ay = np.maximum(-(y * ny).sum(1) * ds, 0.0)
    return 0.5 * (ax + ay)
