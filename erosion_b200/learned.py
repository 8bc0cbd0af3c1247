"""The learned initial guess from Python: training sets from the solver's own
erosion runs, and training, through the C ABI (erosion_lw_*).

The network (learned.cu) predicts, per body, the encoding of the density's
increment over one time step from the body's geometry features and the
encoding of its previous increment; the guess of an erosion step with
warm_start = 2 is the previous step's density plus that prediction.  A
training row is therefore

    X = [geometry features of step k (68) | encoding of x_{k-1} - x_{k-2} (37)]
    Y = encoding of x_k - x_{k-1} (37)

with x_k the density solved in the first stage of step k (on the state the
step starts from), all on the geometry of step k.
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


def trajectory(params, sp, n, nout, th, ln, xs, ys, steps: int):
    """Runs `steps` RK2 erosion steps (erosion_rk2_step, host arrays, updated
    in place) and returns per step the state's node coordinates and the
    density solved in its first stage: a list of (xx, yy, density, M), with
    None where a body was deleted during the step."""
    L = _lib.load()
    M = len(ln)
    nb = np.array([M], np.int64)
    t = np.zeros(1)
    dele = np.zeros(M, np.int64)
    out = []
    for _ in range(steps):
        Mk = int(nb[0])
        xx, yy = getxy(n, Mk, th[: Mk * n], ln[:Mk], xs[:Mk], ys[:Mk])
        rc = L.erosion_rk2_step(ctypes.byref(params), ctypes.byref(sp), n, nb.ctypes.data_as(PI64), nout, ptr(th),
                                ptr(ln), ptr(xs), ptr(ys), ptr(t), dele.ctypes.data_as(PI64))
        check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
        if int(nb[0]) != Mk:
            out.append(None)
            continue
        den = np.zeros(2 * nout + 2 * n * Mk + 3 * Mk)
        check(L.erosion_get_step_density(0, ptr(den), den.size))
        out.append((xx, yy, den, Mk))
    return out


def training_rows(params, n, nout, traj):
    """(X, Y) rows of consecutive triples of a trajectory (see the module
    docstring); triples that cross a body deletion are skipped."""
    X, Y = [], []
    for k in range(2, len(traj)):
        a, b, c = traj[k - 2], traj[k - 1], traj[k]
        if a is None or b is None or c is None or not (a[3] == b[3] == c[3]):
            continue
        xx, yy, den, M = c
        f = features(params, n, M, nout, xx, yy)
        hist = encode(params, n, M, nout, xx, yy, b[2] - a[2])
        targ = encode(params, n, M, nout, xx, yy, den - b[2])
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
