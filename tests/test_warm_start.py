"""The warm start of an erosion step's solves: the previous solve's density
with every body's rigid part carried to the new nodes (learned.reanchor on
the host, k_warm_reanchor in the library)."""
import ctypes

import numpy as np
import pytest

from erosion_b200 import _lib, geometry as G, learned, stokes


def _nodes(n, M, seed, shift=0.0, scale=1.0):
    rng = np.random.default_rng(seed)
    t = 2 * np.pi * (np.arange(n) + 0.5 + shift) / n
    cx, cy, r = rng.uniform(-0.5, 0.5, M), rng.uniform(-0.3, 0.3, M), rng.uniform(0.03, 0.08, M)
    x = cx[:, None] + scale * r[:, None] * np.cos(t)
    y = cy[:, None] + scale * r[:, None] * np.sin(t)
    return x.ravel(), y.ravel()


def test_rigid_density_is_carried_exactly():
    """A density that is a rigid motion on every body on the old nodes maps to
    the same rigid motion on the new nodes (nodes slid by a third of a spacing
    and shrunk by 1%); wall and stokeslet/rotlet entries are untouched."""
    n, M, nout = 64, 5, 32
    xo, yo = _nodes(n, M, 1)
    xn, yn = _nodes(n, M, 1, shift=0.33, scale=0.99)
    rng = np.random.default_rng(2)
    t = rng.standard_normal((M, 3)) * np.array([1.0, 1.0, 1e5])
    den = rng.standard_normal(2 * nout + 2 * n * M + 3 * M)

    def rigid(x, y):
        d = den.copy()
        x, y = x.reshape(M, n), y.reshape(M, n)
        for b in range(M):
            off = 2 * nout + 2 * n * b
            d[off:off + n] = t[b, 0] - t[b, 2] * (y[b] - y[b].mean())
            d[off + n:off + 2 * n] = t[b, 1] + t[b, 2] * (x[b] - x[b].mean())
        return d

    out = learned.reanchor(n, nout, xo, yo, xn, yn, rigid(xo, yo))
    want = rigid(xn, yn)
    assert np.abs(out - want).max() < 1e-9 * np.abs(want).max()
    assert np.array_equal(out[:2 * nout], den[:2 * nout])
    assert np.array_equal(out[2 * nout + 2 * n * M:], den[2 * nout + 2 * n * M:])


def test_remainder_stays_on_the_node_index():
    n, M, nout = 32, 3, 16
    xo, yo = _nodes(n, M, 3)
    xn, yn = _nodes(n, M, 3, shift=0.2)
    den = np.random.default_rng(4).standard_normal(2 * nout + 2 * n * M + 3 * M)
    a = learned.reanchor(n, nout, xo, yo, xn, yn, den)
    b = learned.reanchor(n, nout, xo, yo, xo, yo, den)
    assert np.array_equal(b, den)      # same nodes: unchanged
    assert not np.array_equal(a, den)  # moved nodes: the rotation part moves


@pytest.mark.gpu
def test_library_warm_start_matches_host_reanchor(lib):
    """Step 2's first solve starts from step 1's second-stage density carried
    to its nodes: the library's recorded initial residual equals the host
    restatement's, and is far below the index-aligned density's."""
    g = G.workload("c1", seed=0)
    th, ln, xs, ys = [a.copy() for a in G.to_thetalen(g)]
    p = stokes.params_for(g, precision=1, precond=1)
    sp = _lib.StepParams()
    lib.erosion_default_step_params(ctypes.byref(sp), g.n)
    sp.dt, sp.fixpdrop, sp.warm_start = 1e-5, 0, 1
    nb = np.array([g.M], np.int64)
    t = np.zeros(1)
    dele = np.zeros(g.M, np.int64)

    def step():
        rc = lib.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sp), g.n, nb.ctypes.data_as(_lib.PI64), g.nout,
                                  _lib.ptr(th), _lib.ptr(ln), _lib.ptr(xs), _lib.ptr(ys), t.ctypes.data_as(_lib.PD),
                                  dele.ctypes.data_as(_lib.PI64))
        assert rc == 0 and int(nb[0]) == g.M
        st = _lib.StepStats()
        lib.erosion_get_step_stats(ctypes.byref(st))
        return st.as_dict()

    def stage(k):
        den = np.zeros(g.ntot)
        xx, yy = np.zeros(g.n * g.M), np.zeros(g.n * g.M)
        _lib.check(lib.erosion_get_step_density(k, _lib.ptr(den), den.size))
        _lib.check(lib.erosion_get_step_nodes(k, _lib.ptr(xx), _lib.ptr(yy), xx.size))
        return xx, yy, den

    step()
    xo, yo, do = stage(1)
    st = step()
    xn, yn, _ = stage(0)
    gn = G.Geometry(g.n, g.nout, xn, yn, g.wall, g.ibc, g.radii, g.centers)
    b = stokes.rhs(gn)
    guess = learned.reanchor(g.n, g.nout, xo, yo, xn, yn, do)
    r_host = np.linalg.norm(b - stokes.matvec(gn, guess, precision=0)) / np.linalg.norm(b)
    r_raw = np.linalg.norm(b - stokes.matvec(gn, do, precision=0)) / np.linalg.norm(b)
    print(f"warm start residual: carried {r_host:.3e} (library {st['guess_residual'][0]:.3e}), "
          f"index-aligned {r_raw:.3e}")
    assert st["guess_used"][0] == 1
    assert abs(st["guess_residual"][0] - r_host) <= 1e-6 * r_host
    assert r_host < 0.1 * r_raw
