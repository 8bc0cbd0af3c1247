"""The CUDA path against the committed golden fixtures (tests/golden), through
the C ABI; no oracle build needed.  Tolerances as in the oracle parity tests:
operator 1e-11, density 1e-10, shear stress 1e-9, targets 1e-9, RK2 step
1e-10 (all relative in the max norm)."""
import ctypes
import os

import numpy as np
import pytest

from erosion_b200 import _lib, geometry as G, stokes, thetalen as TL

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def fx():
    f = dict(np.load(os.path.join(GOLDEN, "ref_small_operator.npz")))
    f["g"] = G.Geometry(int(f["n"]), int(f["nout"]), f["xx"], f["yy"], tuple(f["wall"]), int(f["ibc"]),
                        f["radii"], f["centers"])
    return f


@pytest.mark.parametrize("ibary,ifmm,key", [(0, 1, "matvec_trap"), (1, 1, "matvec_fmmbary"),
                                            (1, 0, "matvec_bary")])
def test_operator_matches_golden(lib, fx, ibary, ifmm, key):
    assert rel(stokes.matvec(fx["g"], fx["density_in"], ibary=ibary, ifmm=ifmm), fx[key]) < 1e-11


def test_drop_in_solver_matches_golden(lib, fx):
    """stokessolver_ exactly as the Julia caller drives it (zero guess, 1e-8)."""
    g = fx["g"]
    i64 = lambda v: ctypes.byref(ctypes.c_int64(v))
    den = np.zeros(g.ntot)
    nits = ctypes.c_int64()
    lib.stokessolver_(i64(g.n), i64(g.M), i64(g.nout), i64(1), i64(1), i64(g.ibc), i64(8000),
                      _lib.ptr(g.xx), _lib.ptr(g.yy), _lib.ptr(den), ctypes.byref(nits))
    assert lib.erosion_last_status() == 0
    assert abs(nits.value - int(fx["nits_1e8"])) <= 2
    assert rel(den, fx["density"]) < 1e-6


def test_tight_solve_and_stress_match_golden(lib, fx):
    g = fx["g"]
    den, nits, st = stokes.solve(g, tol=1e-12)
    assert rel(den, fx["density"]) < 1e-10
    tau, _ = stokes.shear_stress(g, fx["density"])
    assert rel(tau, fx["tau"]) < 1e-9
    tau0, _ = stokes.shear_stress(g, fx["density"], ibary=0)
    assert rel(tau0, fx["tau_trap"]) < 1e-9
    out = stokes.qoi_targets(g, fx["density"], fx["xt"], fx["yt"])
    for a, k in zip(out, ("utar", "vtar", "ptar", "vortar")):
        assert rel(a, fx[k]) < 1e-9, k
    assert rel(stokes.pressure(g, fx["density"]), fx["pressure"]) < 1e-10


def test_rk2_step_matches_golden(lib):
    f = np.load(os.path.join(GOLDEN, "ref_small_rk2.npz"))
    n, nout = int(f["n"]), int(f["nout"])
    params = TL.ParamSet(npts=n, nouter=nout, tol=1e-12, fixpdrop=False, dt=float(f["dt"]))
    assert params.epsilon == pytest.approx(float(f["epsilon"])) and params.sigma == pytest.approx(float(f["sigma"]))
    out, _ = TL.rungekutta2(TL.circs2thlenden(n, *f["bodies"].T), params)
    assert np.abs(np.array([b.theta for b in out.thlenvec]) - f["theta1"]).max() < 1e-10
    assert np.abs(np.array([b.len for b in out.thlenvec]) - f["len1"]).max() < 1e-10
    assert np.abs(np.array([b.xsm for b in out.thlenvec]) - f["xsm1"]).max() < 1e-10
    assert np.abs(np.array([b.ysm for b in out.thlenvec]) - f["ysm1"]).max() < 1e-10
