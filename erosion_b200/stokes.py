"""Numpy-level wrappers of the C ABI (host arrays in, host arrays out).

Each function takes a :class:`erosion_b200.geometry.Geometry` (or the raw
``n, M, nout, xx, yy`` through :func:`as_geometry`) and keyword overrides of
``erosion_params``.  Errors raise :class:`erosion_b200._lib.ErosionError`.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PD, PI64, check, ptr


def params_for(g, **kw) -> _lib.ErosionParams:
    base = {"wall": tuple(g.wall), "ibc": int(g.ibc)}
    base.update(kw)
    return _lib.default_params(**base)


def _xy(g):
    xx = np.ascontiguousarray(g.xx, dtype=np.float64)
    yy = np.ascontiguousarray(g.yy, dtype=np.float64)
    if xx.size == 0:
        xx = np.zeros(1)
        yy = np.zeros(1)
    return xx, yy


def solve(g, x0=None, allow=(_lib.EROSION_OK,), **kw):
    """GMRES solve; returns (density, iterations, stats)."""
    L = _lib.load()
    p = params_for(g, **kw)
    den = np.zeros(g.ntot) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    nits = np.zeros(1, np.int64)
    xx, yy = _xy(g)
    rc = L.erosion_solve(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy), ptr(den), nits.ctypes.data_as(PI64))
    check(rc, allow)
    return den, int(nits[0]), _lib.solve_stats()


def matvec(g, den, **kw):
    L = _lib.load()
    p = params_for(g, **kw)
    den = np.ascontiguousarray(den, dtype=np.float64)
    vel = np.zeros(g.ntot)
    xx, yy = _xy(g)
    check(L.erosion_matvec(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy), ptr(den), ptr(vel)))
    return vel


def rhs(g, **kw):
    L = _lib.load()
    p = params_for(g, **kw)
    out = np.zeros(g.ntot)
    xx, yy = _xy(g)
    check(L.erosion_rhs(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy), ptr(out)))
    return out


def geometry(g, **kw) -> dict:
    L = _lib.load()
    p = params_for(g, **kw)
    nb, M, no = g.n * g.M, g.M, g.nout
    a = {k: np.zeros(max(nb, 1)) for k in ("px", "py", "cur", "speed")}
    a.update({k: np.zeros(max(M, 1)) for k in ("cx", "cy")})
    a.update({k: np.zeros(no) for k in ("xo", "yo", "px0", "py0", "cur0", "speed0")})
    xx, yy = _xy(g)
    check(L.erosion_geometry(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy),
                             *[ptr(a[k]) for k in ("px", "py", "cur", "speed", "cx", "cy", "xo", "yo",
                                                   "px0", "py0", "cur0", "speed0")]))
    for k in ("px", "py", "cur", "speed"):
        a[k] = a[k][:nb]
    for k in ("cx", "cy"):
        a[k] = a[k][:M]
    return a


def shear_stress(g, den, **kw):
    """Returns (tau, E) with E of shape (3, n*M) = E11, E12, E22."""
    L = _lib.load()
    p = params_for(g, **kw)
    den = np.ascontiguousarray(den, dtype=np.float64)
    tau = np.zeros(max(g.n * g.M, 1))
    E = np.zeros(max(3 * g.n * g.M, 1))
    xx, yy = _xy(g)
    check(L.erosion_shear_stress(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy), ptr(den), ptr(tau), ptr(E)))
    nb = g.n * g.M
    return tau[:nb], E[:3 * nb].reshape(3, nb)


def qoi_targets(g, den, xt, yt, **kw):
    L = _lib.load()
    p = params_for(g, **kw)
    den = np.ascontiguousarray(den, dtype=np.float64)
    xt = np.ascontiguousarray(xt, dtype=np.float64)
    yt = np.ascontiguousarray(yt, dtype=np.float64)
    out = [np.zeros(len(xt)) for _ in range(4)]
    xx, yy = _xy(g)
    check(L.erosion_qoi_targets(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy), ptr(den), len(xt), ptr(xt),
                                ptr(yt), *[ptr(o) for o in out]))
    return out


def pressure(g, den, **kw):
    """Pressure on the body boundaries (computepressure_ semantics)."""
    L = _lib.load()
    p = params_for(g, **kw)
    den = np.ascontiguousarray(den, dtype=np.float64)
    out = np.zeros(g.n * g.M)
    xx, yy = _xy(g)
    check(L.erosion_pressure(ctypes.byref(p), g.n, g.M, g.nout, ptr(xx), ptr(yy), ptr(den), ptr(out)))
    return out


def near_info(M: int):
    L = _lib.load()
    lw = np.zeros(1, np.int64)
    wb = np.zeros(max(M, 1), np.int64)
    npairs = np.zeros(1, np.int64)
    k = L.erosion_near_info(lw.ctypes.data_as(PI64), wb.ctypes.data_as(PI64), npairs.ctypes.data_as(PI64))
    return int(lw[0]), wb[:k].tolist(), int(npairs[0])


def solve_batch(geoms, x0=None, allow=(_lib.EROSION_OK,), **kw):
    """Ensemble solve of independent geometries (one erosion_solve_batch call;
    all share the parameters, the wall shape and the boundary data of the
    first).  Returns (list of densities, iterations per geometry, batch stats)."""
    L = _lib.load()
    p = params_for(geoms[0], **kw)
    nb = len(geoms)
    npts = np.array([g.n for g in geoms], np.int64)
    nbods = np.array([g.M for g in geoms], np.int64)
    nout = np.array([g.nout for g in geoms], np.int64)
    xx = np.ascontiguousarray(np.concatenate([g.xx for g in geoms] + [np.zeros(1)]))
    yy = np.ascontiguousarray(np.concatenate([g.yy for g in geoms] + [np.zeros(1)]))
    sizes = [g.ntot for g in geoms]
    den = np.zeros(sum(sizes)) if x0 is None else np.ascontiguousarray(np.concatenate(x0), dtype=np.float64)
    nits = np.zeros(nb, np.int64)
    rc = L.erosion_solve_batch(ctypes.byref(p), nb, npts.ctypes.data_as(PI64), nbods.ctypes.data_as(PI64),
                               nout.ctypes.data_as(PI64), ptr(xx), ptr(yy), ptr(den), nits.ctypes.data_as(PI64))
    check(rc, allow)
    st = _lib.BatchStats()
    L.erosion_get_batch_stats(ctypes.byref(st))
    out, o = [], 0
    for n in sizes:
        out.append(den[o:o + n].copy())
        o += n
    return out, nits, st.as_dict()
