"""Parity at the 400-body configuration (400 circles x 256 nodes, 4096 wall
nodes, channel [-1,1] x [-0.5,0.5]; N = 106,496 nodes, 214,192 unknowns).

The oracle is too slow for a full solve here (one FP64 operator application
takes seconds on the host, and the plain method needs thousands), so the
chain is:

* the FP64 operator against oracle.matvec on a random density (1e-11);
* the density reference: the GPU's preconditioned FP64 solve at tol 1e-12
  (its own true residual at the FP64 floor, 5e-8).  Its densities reach
  ~6e5 in the rotation modes of the smallest bodies and ~7e3 on the wall
  (||x|| ~ 4e7 against ||b|| ~ 35).  A rigid-motion density is in the null
  space of a body's double-layer block (-1/2 I + D) and reaches the
  equations only through the stokeslet/rotlet rows, so FP64 evaluations of
  A x differ there by rounding proportional to the amplitude (measured with
  the oracle alone: a rotation density of amplitude 6e5 on one body gives
  1.7e-5 on that body's nodes, where the exact value is 0).  The oracle's
  residual of the reference density is ~6e-6 of ||b|| (half of it from the
  rigid parts' rounding, the rest from the large wall and rigid-free
  densities), which is the rounding of an operator on this ||x||: the test
  asserts the normwise backward error ||b - A_oracle x|| / (||A|| ||x|| +
  ||b||) below 1e-11, the operators' own agreement on a random density, and
  that both operators' values on the rigid parts P x (per body, the
  least-squares fit by two translations and a rotation), away from the rows
  where they are not exactly zero, are rounding-sized (2e-10 of max |P x|);
* the mixed-precision solve at tol 1e-8 against that reference: density to
  1e-6, the pressure drop between the slices x = -0.9 and x = 0.9 (inside the
  channel; the reference's slices at x = +-2 lie outside this wall) to 1e-6;
* the shear stress on 8 sampled target bodies (all 400 source bodies and the
  wall) against oracle.shear_stress.  A rigid motion has no strain, so the
  rigid parts P x contribute nothing to the exact shear stress; evaluated in
  FP64 they contribute rounding, which the oracle's barycentric sums over
  every (node, source body) pair bring to ~4e-7 of max |tau| on this density
  (measured: oracle.shear_stress(P x) on the sampled bodies).  So the test
  compares the library and the oracle on the rigid-free density x - P x to
  1e-7 of max |tau|, checks that the library's own value on P x stays below
  1e-6, and compares the mixed solve's shear stress with the reference
  density's to 1e-7.
"""
import numpy as np
import pytest

from erosion_b200 import geometry as G, stokes
from oracle.rigid import rigid_parts as _rigid_parts

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


def rigid_parts(g, den):
    return _rigid_parts(g.n, g.M, g.nout, g.xx, g.yy, den)


def test_reference_density_is_an_oracle_solution(lib, oracle, c3, ref):
    den, st = ref
    assert st["precond_active"] == 1 and st["precond_singular_blocks"] == 0
    assert st["true_residual"] < 5e-8
    b = stokes.rhs(c3)
    nb = np.linalg.norm(b)
    P = rigid_parts(c3, den)
    a_free = oracle.matvec(c3, den - P, mode=1)
    a_rig_o = oracle.matvec(c3, P, mode=1)
    a_rig_g = stokes.matvec(c3, P, precision=0)
    r = b - a_free - a_rig_o
    r_oracle = np.linalg.norm(r) / nb
    r_hybrid = np.linalg.norm(b - a_free - a_rig_g) / nb
    # normwise backward error ||b - A x|| / (||A|| ||x|| + ||b||) with respect
    # to the oracle's operator, ||A|| bounded below by ||A z|| / ||z|| on a
    # random z: the reference density solves a problem within this relative
    # distance of the oracle's
    z = np.random.default_rng(8).standard_normal(c3.ntot)
    norm_a = np.linalg.norm(stokes.matvec(c3, z, precision=0)) / np.linalg.norm(z)
    eta = np.linalg.norm(r) / (norm_a * np.linalg.norm(den) + nb)
    rows = 2 * c3.nout + 2 * c3.n * c3.M   # A (P x) is exactly zero above the stokeslet/rotlet rows
    floor_o = np.abs(a_rig_o[:rows]).max() / np.abs(P).max()
    floor_g = np.abs(a_rig_g[:rows]).max() / np.abs(P).max()
    print(f"oracle residual {r_oracle:.2e} (with the library's values on P x {r_hybrid:.2e}); "
          f"backward error {eta:.2e} (||A|| >= {norm_a:.3g}, ||x|| = {np.linalg.norm(den):.3g}); "
          f"rounding on P x: oracle {floor_o:.2e}, library {floor_g:.2e} of max |P x|")
    assert eta < 1e-11, eta
    assert floor_o < 2e-10 and floor_g < 2e-10
    # the stokeslet/rotlet rows of A (P x) are moments of P x, n-term sums of
    # terms up to max |P x|: both evaluate them to the rounding of such sums
    assert np.abs(a_rig_o[rows:] - a_rig_g[rows:]).max() < 1e-13 * c3.n * np.abs(P).max()


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
    P = rigid_parts(c3, d_ref)
    n = c3.n
    idx = np.concatenate([np.arange(b * n, (b + 1) * n) for b in SAMPLE_BODIES])
    tau_free, _ = stokes.shear_stress(c3, d_ref - P)
    tau_o, _ = oracle.shear_stress(c3, d_ref - P, bodies=SAMPLE_BODIES)
    scale = np.abs(tau_o[idx]).max()
    err = np.abs(tau_free[idx] - tau_o[idx]).max() / scale
    tau_rig, _ = stokes.shear_stress(c3, P)
    floor_g = np.abs(tau_rig).max() / scale
    tau, _ = stokes.shear_stress(c3, d_ref)
    err_full = np.abs(tau[idx] - tau_o[idx]).max() / scale
    print(f"sampled-body shear stress vs oracle on x - P x: {err:.2e}; library on P x: {floor_g:.2e}; "
          f"library on x vs oracle on x - P x: {err_full:.2e} (of max |tau|)")
    assert err < 1e-7
    assert floor_g < 1e-6
    assert err_full < 1e-6
    # the mixed solve's stress against the FP64 reference's, every body
    tau_m, _ = stokes.shear_stress(c3, mixed[0])
    assert np.abs(tau_m - tau).max() / np.abs(tau).max() < 1e-7
