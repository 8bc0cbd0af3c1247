"""Failure handling: bad inputs and numerical breakdowns come back as status
codes through the C ABI; none of them faults the GPU (every case is rejected
on the host or ends in a bounded loop)."""
import numpy as np
import pytest

from erosion_b200 import _lib, geometry as G, stokes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return G.workload("ref-small")


def status_of(fn):
    try:
        fn()
    except _lib.ErosionError as e:
        return e.code
    return _lib.EROSION_OK


def test_odd_npts_rejected(lib):
    g = G.custom(63, 256, [0.2], [[0, 0]])
    assert status_of(lambda: stokes.solve(g)) == _lib.EROSION_BAD_INPUT


def test_tiny_wall_rejected(lib):
    g = G.custom(64, 4, [0.2], [[0, 0]])
    assert status_of(lambda: stokes.solve(g)) == _lib.EROSION_BAD_INPUT


def test_nan_geometry_rejected(lib, small):
    g = G.Geometry(small.n, small.nout, small.xx.copy(), small.yy.copy(), small.wall, small.ibc, small.radii,
                   small.centers)
    g.xx[5] = np.nan
    assert status_of(lambda: stokes.solve(g)) == _lib.EROSION_BAD_INPUT


def test_body_through_wall_rejected(lib):
    g = G.custom(64, 256, [0.3], [[0.0, 0.85]])
    assert status_of(lambda: stokes.solve(g)) == _lib.EROSION_BAD_INPUT


def test_nan_initial_guess_is_breakdown(lib, small):
    x0 = np.zeros(small.ntot)
    x0[3] = np.nan
    assert status_of(lambda: stokes.solve(small, x0=x0)) == _lib.EROSION_BREAKDOWN


def test_maxl_one_reports_maxiter(lib, small):
    den, nits, st = stokes.solve(small, maxl=1, allow=(_lib.EROSION_MAXITER,))
    assert nits == 1
    assert _lib.last_error()[0] == _lib.EROSION_MAXITER
    assert np.isfinite(den).all()


def test_zero_rhs_returns_zero_density(lib, small):
    x0 = np.ones(small.ntot)
    with pytest.raises(_lib.ErosionError) as e:
        stokes.solve(small, x0=x0, rhs_mode=2)
    assert e.value.code == _lib.EROSION_BAD_INPUT


def test_deleted_body_shrinks_problem(lib, oracle, small):
    """TimeStepping.jl:103-126 deletes vanishing bodies; the next solve simply
    has one body fewer."""
    g2 = G.custom(small.n, small.nout, small.radii[:2], small.centers[:2])
    den, nits, st = stokes.solve(g2, tol=1e-12)
    ref, nits_o, ierr, err = oracle.solve(g2, tol=1e-12)
    assert np.linalg.norm(den - ref) / np.linalg.norm(ref) < 1e-10


def test_library_usable_after_errors(lib, small):
    den, nits, st = stokes.solve(small)
    assert st["est_residual"] <= 1e-8
