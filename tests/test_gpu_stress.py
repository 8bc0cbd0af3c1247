"""GPU parity of the shear stress (computeShearStress) and the target
quantities (computeQoiTargets) against the CPU FP64 oracle, through the C ABI.
Tolerance: 1e-9 relative (max norm) for the shear stress and the deformation
tensor, 1e-10 for the target quantities."""
import numpy as np
import pytest

from erosion_b200 import geometry as G
from erosion_b200 import stokes

pytestmark = pytest.mark.gpu

TAU_RTOL = 1e-9
QOI_RTOL = 1e-10


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def small():
    return G.workload("ref-small")


@pytest.fixture(scope="module")
def small_den(oracle, small):
    den, nits, ierr, err = oracle.solve(small, tol=1e-12)
    return den


@pytest.mark.parametrize("ibary", [1, 0])
def test_shear_stress_matches_oracle(lib, oracle, small, small_den, ibary):
    tau, E = stokes.shear_stress(small, small_den, ibary=ibary)
    tau_o, E_o = oracle.shear_stress(small, small_den, ibary=ibary)
    assert rel(tau, tau_o) < TAU_RTOL
    for q in range(3):
        assert rel(E[q], E_o[q]) < TAU_RTOL


def test_shear_stress_random_density(lib, oracle, small):
    den = np.random.default_rng(7).standard_normal(small.ntot)
    tau, _ = stokes.shear_stress(small, den)
    tau_o, _ = oracle.shear_stress(small, den)
    assert rel(tau, tau_o) < TAU_RTOL


def test_shear_stress_channel_c1(lib, oracle):
    g = G.workload("c1", seed=1)
    den = np.random.default_rng(3).standard_normal(g.ntot)
    tau, _ = stokes.shear_stress(g, den)
    tau_o, _ = oracle.shear_stress(g, den)
    assert rel(tau, tau_o) < TAU_RTOL


def test_shear_stress_abi_entry(lib, oracle, small, small_den):
    """computeshearstress_ (the drop-in symbol, by-reference int64 args)."""
    import ctypes
    from erosion_b200._lib import PD, PI64
    tau = np.zeros(small.n * small.M)
    i = lambda v: ctypes.byref(ctypes.c_int64(v))
    # the drop-in uses the reference wall
    lib.computeshearstress_(i(small.n), i(small.M), i(small.nout), small.xx.ctypes.data_as(PD),
                            small.yy.ctypes.data_as(PD), small_den.ctypes.data_as(PD), i(1),
                            tau.ctypes.data_as(PD))
    tau_o, _ = oracle.shear_stress(small, small_den)
    assert rel(tau, tau_o) < TAU_RTOL


@pytest.mark.parametrize("ibary", [1, 0])
def test_qoi_targets_matches_oracle(lib, oracle, small, small_den, ibary):
    ylocs = -1 + (np.arange(13) + 0.5) * 2 / 13
    xt = np.r_[np.full(13, 2.0), np.full(13, -2.0), [-1.0, 0.6, 1.5]]   # last: inside, inside, fluid
    yt = np.r_[ylocs, ylocs, [0.1, 0.72, 0.3]]
    a = stokes.qoi_targets(small, small_den, xt, yt, ibary=ibary)
    b = oracle.qoi_targets(small, small_den, xt, yt, ibary=ibary)
    for q in range(4):
        assert rel(a[q], b[q]) < QOI_RTOL, q
    assert a[0][26] == 0.0 and a[0][27] == 0.0    # inside bodies are zeroed
    assert a[0][28] != 0.0


def test_pressure_drop_flux_consistency(lib, small):
    """DensityStress.jl:149-152: the flux through x = +-x0 must agree."""
    den, _, _ = stokes.solve(small, tol=1e-10)
    ylocs = -1 + (np.arange(13) + 0.5) * 2 / 13
    up = stokes.qoi_targets(small, den, np.full(13, 2.0), ylocs)[0]
    um = stokes.qoi_targets(small, den, np.full(13, -2.0), ylocs)[0]
    assert abs(up.mean() - um.mean()) / abs(0.5 * (up.mean() + um.mean())) < 1e-3


@pytest.mark.parametrize("name", ["ref-small", "c1"])
def test_boundary_pressure_matches_oracle(lib, oracle, name):
    g = G.workload(name)
    den = oracle.solve(g, tol=1e-12)[0]
    a = stokes.pressure(g, den)
    b = oracle.pressure(g, den)
    # the shear stress bound: close bodies (c1 gaps of 0.02) make the 1/rho^4
    # pairs amplify summation-order rounding to ~1e-10
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-9


def test_computepressure_abi_entry(lib, oracle, small, small_den):
    import ctypes
    from erosion_b200 import _lib
    i64 = lambda v: ctypes.byref(ctypes.c_int64(v))
    out = np.zeros(small.n * small.M)
    lib.computepressure_(i64(small.n), i64(small.M), i64(small.nout), _lib.ptr(small.xx), _lib.ptr(small.yy),
                         _lib.ptr(small_den), _lib.ptr(out))
    assert lib.erosion_last_status() == 0
    ref = oracle.pressure(small, small_den)
    assert np.abs(out - ref).max() / np.abs(ref).max() < 1e-10


def test_boundary_pressure_manufactured(lib):
    r = 0.2
    g = G.custom(64, 256, [r], [[0.0, 0.0]])
    den, _, _ = stokes.solve(g, tol=1e-13, rhs_mode=1)
    exact = (g.xx + 2 * g.yy) / (2 * np.pi * (g.xx ** 2 + g.yy ** 2))
    assert np.abs(stokes.pressure(g, den) - exact).max() < 1e-9 * np.abs(exact).max()


def smooth_density(g, kmax, seed):
    """Random density with Fourier content up to mode kmax on every curve
    (wall and bodies, both components) and random stokeslet/rotlet unknowns."""
    rng = np.random.default_rng(seed)
    den = np.zeros(g.ntot)

    def curve(npts):
        th = 2 * np.pi * np.arange(npts) / npts
        k = np.arange(kmax + 1)[:, None]
        a, b = rng.standard_normal((2, kmax + 1, 1)) / (1.0 + k)
        return (a * np.cos(k * th) + b * np.sin(k * th)).sum(0)

    no, n = g.nout, g.n
    den[:no], den[no:2 * no] = curve(no), curve(no)
    for b in range(g.M):
        off = 2 * no + 2 * n * b
        den[off:off + n], den[off + n:off + 2 * n] = curve(n), curve(n)
    den[2 * no + 2 * n * g.M:] = rng.standard_normal(3 * g.M)
    return den


@pytest.mark.parametrize("name,seed", [("c1", 2), ("c2", 0)])
def test_hybrid_stress_equals_all_barycentric(lib, name, seed):
    """The default shear stress (barycentric within 12 node spacings of a
    source curve, trapezoid rule beyond) against the reference's evaluation
    of every pair by the barycentric formulas, on a random density resolved
    by the nodes (Fourier content up to mode 24).  Beyond 12 spacings the two
    rules agree to rounding on such densities (measured with the oracle on
    the 100-body channel: 1e-12 of the pair's value).  On content near the
    Nyquist mode they do not: there the barycentric formulas, which
    differentiate the density spectrally, carry an error of ~1e-6 of the
    pair's value at every distance (measured: mode 120 of 256 at 50
    spacings), while the trapezoid rule's error at 12 spacings is ~1e-16."""
    g = G.workload(name, seed=seed)
    den = smooth_density(g, 24, 5)
    tau, E = stokes.shear_stress(g, den)
    tau_b, E_b = stokes.shear_stress(g, den, stress_all_bary=1)
    assert rel(tau, tau_b) < 1e-10
    for q in range(3):
        assert rel(E[q], E_b[q]) < 1e-10
