"""Mixed precision: the FP32 far field (FP64 accumulation) inside FP64 iterative
refinement reaches the same 1e-8 relative residual as the FP64 path, and its
density and shear stress agree with the FP64 oracle within the tolerances the
1e-8 stopping point allows (1e-6 density, 1e-7 shear stress, relative)."""
import numpy as np
import pytest

from erosion_b200 import geometry as G
from erosion_b200 import stokes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", ["ref-small", "c1"])
def test_fp32_operator_error_small(lib, name):
    g = G.workload(name, seed=2)
    den = np.random.default_rng(5).standard_normal(g.ntot)
    a = stokes.matvec(g, den, precision=1)
    b = stokes.matvec(g, den, precision=0)
    e = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert e < 1e-5, e


@pytest.mark.parametrize("name", ["ref-small", "c1"])
def test_mixed_solve_reaches_fp64_tolerance(lib, oracle, name):
    g = G.workload(name, seed=2)
    den, nits, st = stokes.solve(g, precision=1)
    assert st["true_residual"] <= 1e-8
    assert st["matvecs_fp32"] > 0
    ref, _, _, _ = oracle.solve(g, tol=1e-13)
    assert np.linalg.norm(den - ref) / np.linalg.norm(ref) < 1e-6
    tau, _ = stokes.shear_stress(g, den)
    tau_o, _ = oracle.shear_stress(g, ref)
    assert rel(tau, tau_o) < 1e-7


def test_relaxed_mixed_iterations_close_to_fp64(lib):
    """Relaxed GMRES (FP32 far field once the estimate is below 1e-3, one
    sweep to tol before refining) takes about the FP64 iteration count; the
    default (FP32 from the first iteration, 5-decade sweeps) trades some
    iterations for FP32 sums throughout and meets the same tolerance."""
    g = G.workload("c1", seed=4)
    _, n64, s64 = stokes.solve(g, precision=0)
    _, n32, s32 = stokes.solve(g, precision=1, relax_tol=1e-3, sweep_decades=0)
    assert n32 <= 1.3 * n64 + 10
    assert s32["matvecs_fp32"] > 0 and s32["true_residual"] <= 1e-8
    _, nd, sd = stokes.solve(g, precision=1)
    assert sd["true_residual"] <= 2e-8 and sd["far64f_launches"] == 0
    assert sd["matvecs_fp32"] >= 0.9 * sd["matvecs"]


@pytest.mark.parametrize("precision", [0, 1])
def test_block_preconditioner_same_answer_fewer_iterations(lib, oracle, precision):
    """Right preconditioning keeps the stopping test on ||b - A x||/||b||, so
    the density matches the oracle's to the tolerance the 1e-8 stopping point
    allows while GMRES needs fewer iterations."""
    g = G.workload("c1", seed=4)
    _, n0, _ = stokes.solve(g, precision=precision)
    den, n1, st = stokes.solve(g, precision=precision, precond=1, true_residual=1)
    assert st["true_residual"] <= 1e-8
    assert n1 < n0
    ref, _, _, _ = oracle.solve(g, tol=1e-13)
    assert np.linalg.norm(den - ref) / np.linalg.norm(ref) < 1e-6


def test_block_preconditioner_tight_parity(lib, oracle):
    g = G.workload("ref-small")
    den, nits, st = stokes.solve(g, precond=1, tol=1e-13)
    ref, _, _, _ = oracle.solve(g, tol=1e-13)
    assert np.linalg.norm(den - ref) / np.linalg.norm(ref) < 1e-10


@pytest.mark.parametrize("name", ["ref-small", "c1"])
def test_fp32_from_the_first_iteration_with_decade_sweeps(lib, oracle, name):
    """relax_tol = 1 (FP32 far field from the first iteration) with refinement
    sweeps of 3 decades each (sweep_decades = 3): every sweep restarts from the
    true FP64 residual, the FP64 far field runs only for those residuals, and
    the answer meets the same tolerance and the same oracle bounds."""
    g = G.workload(name, seed=2)
    den, nits, st = stokes.solve(g, precision=1, precond=1, relax_tol=1.0, sweep_decades=3)
    assert st["true_residual"] <= 1e-8
    assert st["sweeps"] >= 3
    assert st["far64f_launches"] == 0 and st["far_launches"] == st["sweeps"]   # the true residuals only
    ref, _, _, _ = oracle.solve(g, tol=1e-13)
    assert np.linalg.norm(den - ref) / np.linalg.norm(ref) < 1e-6
    tau, _ = stokes.shear_stress(g, den)
    tau_o, _ = oracle.shear_stress(g, ref)
    assert rel(tau, tau_o) < 1e-7


@pytest.mark.parametrize("precision", [0, 1])
def test_coarse_correction_same_answer_fewer_iterations(lib, oracle, precision):
    """precond = 2 (block Gauss-Seidel after a coarse correction on every
    body's rigid-motion densities and stokeslet/rotlet unknowns) reaches the
    same tolerance and the oracle's density in no more iterations than the
    block preconditioner alone."""
    g = G.workload("c1", seed=4)
    _, n1, _ = stokes.solve(g, precision=precision, precond=1)
    den, n2, st = stokes.solve(g, precision=precision, precond=2, true_residual=1)
    assert st["true_residual"] <= 2e-8 and st["precond_active"] == 1
    assert n2 <= n1
    ref, _, _, _ = oracle.solve(g, tol=1e-13)
    assert np.linalg.norm(den - ref) / np.linalg.norm(ref) < 1e-6
