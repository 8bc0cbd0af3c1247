"""Ensemble solve (erosion_solve_batch): independent geometries of uneven
sizes solved together give what erosion_solve gives for each of them.

Tolerances: FP64 at tol 1e-12, density within 1e-10 of the single solve
(relative, max norm) and iterations within 2 (the batched Givens step runs on
the device, whose fused multiply-adds round differently from the host's);
mixed precision at tol 1e-8, density within 1e-6 of the FP64 tight solution
(the accuracy the 1e-8 stopping point allows)."""
import numpy as np
import pytest

from erosion_b200 import geometry as G, stokes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def ens():
    a = G.ensemble(3, seed=11, bodies=(2, 6), npts=(64, 128), porosity=(0.85, 0.95), nout=256)
    b = G.ensemble(2, seed=12, bodies=(1, 4), npts=(64, 128), porosity=(0.85, 0.95), nout=512)
    return a + b


@pytest.mark.parametrize("precond", [1, 0])
def test_fp64_batch_matches_single_solves(lib, ens, precond):
    tol = 1e-12 if precond else 1e-10
    dens, nits, st = stokes.solve_batch(ens, tol=tol, precond=precond)
    for g, d, k in zip(ens, dens, nits):
        ref, kref, _ = stokes.solve(g, tol=tol, precond=precond)
        assert rel(d, ref) < (1e-10 if precond else 1e-8)
        assert abs(int(k) - kref) <= 2, (k, kref)
    assert st["geometries"] == len(ens)
    assert st["rounds"] >= max(nits)
    assert st["graph_captures"] < st["rounds"]
    assert st["iterations"] == sum(nits)


def test_mixed_batch_reaches_fp64_answer(lib, ens):
    dens, nits, st = stokes.solve_batch(ens, precision=1, precond=1)
    for g, d in zip(ens, dens):
        ref, _, _ = stokes.solve(g, tol=1e-12, precond=1)
        assert rel(d, ref) < 1e-6
    assert st["max_true_residual"] <= 2e-8
    assert st["pairs32_total"] > 0 and st["pairs64_total"] > 0


def test_batch_with_initial_guess(lib, ens):
    rng = np.random.default_rng(3)
    x0 = [rng.standard_normal(g.ntot) * 1e-3 for g in ens]
    dens, nits, _ = stokes.solve_batch(ens, x0=x0, tol=1e-12, precond=1)
    for g, d, x in zip(ens, dens, x0):
        ref, _, _ = stokes.solve(g, x0=x, tol=1e-12, precond=1)
        assert rel(d, ref) < 1e-10


def test_single_geometry_batch(lib):
    g = G.workload("ref-small")
    dens, nits, st = stokes.solve_batch([g], tol=1e-12)
    ref, kref, _ = stokes.solve(g, tol=1e-12)
    assert rel(dens[0], ref) < 1e-10
    assert abs(int(nits[0]) - kref) <= 2


def test_batch_with_an_empty_channel_and_uneven_walls(lib):
    empty = G.custom(64, 256, [], [], wall=G.CHANNEL_WALL, ibc=0)
    ens = [G.ensemble(1, seed=21, bodies=(3, 3), npts=(64,), porosity=(0.9, 0.9), nout=512)[0], empty]
    dens, nits, st = stokes.solve_batch(ens, tol=1e-12, precond=1)
    for g, d in zip(ens, dens):
        ref, _, _ = stokes.solve(g, tol=1e-12, precond=1)
        assert rel(d, ref) < 1e-10


def test_batch_reports_bad_input_and_stays_usable(lib):
    from erosion_b200 import _lib
    good = G.ensemble(1, seed=31, bodies=(2, 2), npts=(64,), porosity=(0.9, 0.9), nout=256)[0]
    bad = G.Geometry(63, 256, good.xx[:63 * 2].copy(), good.yy[:63 * 2].copy(), good.wall, good.ibc,
                     good.radii, good.centers)
    with pytest.raises(_lib.ErosionError) as e:
        stokes.solve_batch([good, bad], tol=1e-10)
    assert e.value.code == _lib.EROSION_BAD_INPUT
    dens, nits, _ = stokes.solve_batch([good], tol=1e-10)
    assert nits[0] > 0 and np.isfinite(dens[0]).all()


def test_batch_iteration_cap(lib, ens):
    from erosion_b200 import _lib
    dens, nits, st = stokes.solve_batch(ens, tol=1e-14, maxl=5, precond=1,
                                        allow=(_lib.EROSION_OK, _lib.EROSION_MAXITER))
    assert (nits <= 5).all()
    assert _lib.load().erosion_last_status() == _lib.EROSION_MAXITER


def test_batch_members_with_different_block_sizes(lib):
    """Members whose preconditioner blocks need different shared-memory
    sizes (128, 256 and 512 nodes per body: blocks of 259, 515 and 1027) are
    set up concurrently on host threads; each launch must still get the
    shared memory it asks for."""
    ens = [G.ensemble(1, seed=40 + k, bodies=(2, 3), npts=(n,), porosity=(0.9, 0.9), nout=256)[0]
           for k, n in enumerate((128, 512, 256, 512, 128, 256))]
    dens, nits, st = stokes.solve_batch(ens, tol=1e-10, precond=1)
    for g, d in zip(ens, dens):
        ref, _, _ = stokes.solve(g, tol=1e-10, precond=1)
        assert rel(d, ref) < 1e-8
