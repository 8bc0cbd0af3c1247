"""The device-side erosion step (erosion_rk2_step) against the numpy
restatement of TimeStepping.jl/SpectralMethods.jl/ThetaLen.jl driven by the
CPU oracle's solve and shear stress.  Both solves run to 1e-12 so that the
comparison measures the step, not the GMRES stopping point."""
import numpy as np
import pytest

from erosion_b200 import thetalen as TL
from oracle import thetalen_oracle as TO

pytestmark = pytest.mark.gpu


def bodies_small():
    return [(0.3, -1.0, 0.1), (0.25, -0.35, 0.0), (0.2, 0.6, 0.72)]


def test_getxy_matches_oracle(lib):
    rng = np.random.default_rng(0)
    n = 64
    th = 0.5 * np.pi + TL.getalpha(n) + 0.05 * np.sin(3 * TL.getalpha(n)) + 0.01 * rng.standard_normal(n)
    b = TL.ThetaLenType(th, 1.3, 0.2, -0.1)
    xx, yy = TL.getxy(b)
    xo, yo = TO.getxy(TO.Body(th, 1.3, 0.2, -0.1))
    assert np.abs(xx - xo).max() < 1e-13
    assert np.abs(yy - yo).max() < 1e-13


@pytest.mark.parametrize("fixpdrop", [0, 1])
def test_rk2_step_matches_oracle(lib, oracle, fixpdrop):
    n, nout = 64, 256
    params = TL.ParamSet(npts=n, nouter=nout, tol=1e-12, fixpdrop=bool(fixpdrop), dt=1e-3)
    thld = TL.circs2thlenden(n, *zip(*bodies_small()))
    out, st = TL.rungekutta2(thld, params)
    tor = TO.ThetaLenOracle(oracle, nout, params.wall, params.ibc, params.epsilon, params.sigma, params.dt,
                            tol=1e-12, fixpdrop=bool(fixpdrop))
    ob = tor.rungekutta2([TO.circ2thlen(n, r, x, y) for r, x, y in bodies_small()])
    assert len(out.thlenvec) == len(ob)
    for a, b in zip(out.thlenvec, ob):
        assert np.abs(a.theta - b.theta).max() < 1e-10
        assert abs(a.len - b.len) < 1e-10 * b.len
        assert abs(a.xsm - b.xsm) < 1e-10 and abs(a.ysm - b.ysm) < 1e-10
    assert out.tt == pytest.approx(params.dt)
    assert st["gmres_iterations"][0] > 0 and st["gmres_iterations"][1] > 0


def test_rk2_several_steps_stay_close(lib, oracle):
    n, nout = 64, 256
    params = TL.ParamSet(npts=n, nouter=nout, tol=1e-12, fixpdrop=False, dt=2e-3)
    thld = TL.circs2thlenden(n, *zip(*bodies_small()))
    tor = TO.ThetaLenOracle(oracle, nout, params.wall, params.ibc, params.epsilon, params.sigma, params.dt,
                            tol=1e-12)
    ob = [TO.circ2thlen(n, r, x, y) for r, x, y in bodies_small()]
    for _ in range(3):
        thld, st = TL.rungekutta2(thld, params)
        ob = tor.rungekutta2(ob)
    for a, b in zip(thld.thlenvec, ob):
        assert np.abs(a.theta - b.theta).max() < 1e-9
        assert abs(a.len - b.len) < 1e-9


def test_warm_start_same_answer(lib):
    """A previous-step initial guess changes the Krylov path, not the answer.
    (On this operator it saves few iterations: GMRES's linear phase
    dominates, which the oracle shows too.)"""
    n, nout = 64, 256
    base = dict(npts=n, nouter=nout, tol=1e-10, fixpdrop=False, dt=1e-3)
    cold = TL.ParamSet(**base)
    warm = TL.ParamSet(**base, warm_start=1)
    s0 = TL.circs2thlenden(n, *zip(*bodies_small()))
    a, _ = TL.rungekutta2(s0, cold)
    a, sta = TL.rungekutta2(a, cold)
    b, _ = TL.rungekutta2(s0, warm)
    b, stb = TL.rungekutta2(b, warm)
    for x, y in zip(a.thlenvec, b.thlenvec):
        assert np.abs(x.theta - y.theta).max() < 1e-7
    assert sum(stb["gmres_iterations"]) <= sum(sta["gmres_iterations"]) + 10
