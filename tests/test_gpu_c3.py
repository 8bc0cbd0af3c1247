"""Parity at the 400-body configuration (400 circles x 256 nodes, 4096 wall
nodes, channel [-1,1] x [-0.5,0.5]; N = 106,496 nodes, 214,192 unknowns).

The oracle is too slow for a full solve here (one FP64 operator application
takes seconds on the host, and the plain method needs thousands), so the
chain is:

* the FP64 operator against oracle.matvec on a random density (1e-11);
* the density reference: the GPU's preconditioned FP64 solve at tol 1e-12,
  tied to the oracle by the oracle's own residual of it, b - A_oracle x, which
  must sit at the FP64 rounding floor of this problem (its densities reach
  ~4e7 in the rigid modes of the smallest bodies, so ||b - A x|| cannot go
  below ~1e-8 ||b|| in FP64, whoever computes it);
* the mixed-precision solve at tol 1e-8 against that reference: density to
  1e-6, the pressure drop between the slices x = -0.9 and x = 0.9 (inside the
  channel; the reference's slices at x = +-2 lie outside this wall) to 1e-6;
* the shear stress on 8 sampled target bodies (all 400 source bodies and the
  wall) against oracle.shear_stress on the same density, and the mixed
  solve's shear stress against the reference density's, both to 1e-7 of
  max |tau|.  The oracle evaluates every (node, source body) pair by the
  barycentric formulas, whose fields carry the density's large rigid parts;
  on this density each such evaluation has an absolute rounding error near
  1e-8 (compared against the trapezoid rule on the rigid-free density, pair by
  pair, the two differ by that much at every distance), and 400 sources add
  up to a few 1e-8 of max |tau|.  The library evaluates the distant pairs by
  the trapezoid rule on the rigid-free density, so the comparison is bounded
  by the oracle's rounding, not by a difference of method.
"""
import numpy as np
import pytest

from erosion_b200 import geometry as G, stokes

pytestmark = pytest.mark.gpu

SAMPLE_BODIES = [0, 57, 113, 170, 226, 283, 339, 399]


def rel2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def c3():
    return G.workload("c3")


@pytest.fixture(scope="module")
def ref(lib, c3):
    den, it, st = stokes.solve(c3, tol=1e-12, precision=0, precond=1, true_residual=1, maxl=4000,
                               allow=(0, 1))
    return den, st


@pytest.fixture(scope="module")
def mixed(lib, c3):
    den, it, st = stokes.solve(c3, tol=1e-8, precision=1, precond=1, maxl=4000)
    return den, st


def pressure_drop(g, den):
    """Mean pressure at x = -0.9 minus that at x = +0.9 over 13 points across
    the channel (getpdrop's 13-point slices, DensityStress.jl:129-138, moved
    inside this wall)."""
    y = np.linspace(-0.4, 0.4, 13)
    xl, xr = np.full(13, -0.9), np.full(13, 0.9)
    pl = stokes.qoi_targets(g, den, xl, y)[2]
    pr = stokes.qoi_targets(g, den, xr, y)[2]
    return pl.mean() - pr.mean()


def test_fp64_operator_matches_oracle_at_c3(lib, oracle, c3):
    den = np.random.default_rng(8).standard_normal(c3.ntot)
    a = stokes.matvec(c3, den, precision=0)
    b = oracle.matvec(c3, den, mode=1)
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-11


def test_reference_density_is_an_oracle_solution(lib, oracle, c3, ref):
    den, st = ref
    assert st["precond_active"] == 1 and st["precond_singular_blocks"] == 0
    b = stokes.rhs(c3)
    r_oracle = np.linalg.norm(b - oracle.matvec(c3, den, mode=1)) / np.linalg.norm(b)
    r_gpu = np.linalg.norm(b - stokes.matvec(c3, den, precision=0)) / np.linalg.norm(b)
    # the FP64 rounding floor eps ||A|| ||x|| / ||b|| of this problem is ~1e-8
    assert r_oracle < 5e-8, r_oracle
    assert abs(r_oracle - r_gpu) < 0.1 * r_oracle + 1e-10


def test_mixed_solve_density_and_pressure_drop(lib, c3, ref, mixed):
    d_ref, _ = ref
    d_mix, st = mixed
    assert st["true_residual"] <= 2e-8
    assert st["matvecs_fp32"] > 0
    assert rel2(d_mix, d_ref) < 1e-6
    dp_ref = pressure_drop(c3, d_ref)
    dp_mix = pressure_drop(c3, d_mix)
    assert abs(dp_mix - dp_ref) < 1e-6 * abs(dp_ref)


def test_shear_stress_sampled_bodies_match_oracle(lib, oracle, c3, ref, mixed):
    d_ref, _ = ref
    tau, _ = stokes.shear_stress(c3, d_ref)
    tau_o, _ = oracle.shear_stress(c3, d_ref, bodies=SAMPLE_BODIES)
    n = c3.n
    idx = np.concatenate([np.arange(b * n, (b + 1) * n) for b in SAMPLE_BODIES])
    scale = np.abs(tau_o[idx]).max()
    err = np.abs(tau[idx] - tau_o[idx]).max() / scale
    print(f"sampled-body shear stress vs oracle: {err:.2e} of max |tau|")
    assert err < 1e-7
    # the mixed solve's stress against the FP64 reference's, every body
    tau_m, _ = stokes.shear_stress(c3, mixed[0])
    assert np.abs(tau_m - tau).max() / np.abs(tau).max() < 1e-7
