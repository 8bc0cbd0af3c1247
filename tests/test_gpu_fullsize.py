"""Parity at the configured sizes, where the oracle is too slow for a full
comparison: one FP64 operator application of the 100-body channel against the
oracle, and size-independent properties of the CUDA path on the 100- and
400-body channels — linearity, and the half-turn symmetry of the channel
(every body rotated by pi about the origin; the wall maps to itself with its
node k going to node k + nouter/2).  Under that rotation a density sigma maps
to T sigma: wall components shifted by nouter/2 and negated, body components
negated, stokeslet strengths negated, rotlet strengths kept; the rotated
operator satisfies A' (T sigma) = T (A sigma), and the solution of the rotated
problem with the same (even) wall data is -T x."""
import numpy as np
import pytest

from erosion_b200 import geometry as G, stokes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def half_turn(g):
    return G.Geometry(g.n, g.nout, -g.xx, -g.yy, g.wall, g.ibc, g.radii, -g.centers)


def T(g, v):
    nout, nb, M = g.nout, g.n * g.M, g.M
    out = np.empty_like(v)
    wx, wy = v[:nout], v[nout:2 * nout]
    out[:nout] = -np.roll(wx, nout // 2)
    out[nout:2 * nout] = -np.roll(wy, nout // 2)
    out[2 * nout:2 * nout + 2 * nb] = -v[2 * nout:2 * nout + 2 * nb]
    c = v[2 * nout + 2 * nb:].reshape(M, 3).copy()
    c[:, :2] *= -1
    out[2 * nout + 2 * nb:] = c.reshape(-1)
    return out


@pytest.fixture(scope="module")
def c2():
    return G.workload("c2")


def test_fp64_operator_matches_oracle_at_c2(lib, oracle, c2):
    den = np.random.default_rng(2).standard_normal(c2.ntot)
    a = stokes.matvec(c2, den, precision=0)
    b = oracle.matvec(c2, den, mode=1)
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-11


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_operator_linearity(lib, name):
    g = G.workload(name)
    rng = np.random.default_rng(4)
    x, y = rng.standard_normal(g.ntot), rng.standard_normal(g.ntot)
    for prec, tol in ((0, 1e-12), (1, 1e-6)):
        ax, ay = stokes.matvec(g, x, precision=prec), stokes.matvec(g, y, precision=prec)
        axy = stokes.matvec(g, 0.3 * x - 1.7 * y, precision=prec)
        assert rel(axy, 0.3 * ax - 1.7 * ay) < tol, prec


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_operator_half_turn(lib, name):
    g = G.workload(name)
    h = half_turn(g)
    x = np.random.default_rng(6).standard_normal(g.ntot)
    a = stokes.matvec(h, T(g, x), precision=0)
    b = T(g, stokes.matvec(g, x, precision=0))
    assert rel(a, b) < 1e-12


def test_mixed_solve_half_turn_c2(lib, c2):
    h = half_turn(c2)
    x, _, st = stokes.solve(c2, precision=1, precond=1)
    y, _, sh = stokes.solve(h, precision=1, precond=1)
    assert rel(y, -T(c2, x)) < 1e-6
    assert st["true_residual"] <= 2e-8 and sh["true_residual"] <= 2e-8
