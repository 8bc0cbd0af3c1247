"""drag (PostProcess.jl:131-162) through erosion_drag against the oracle's
restatement (oracle/thetalen_oracle.py: drag), on the same solved density:
totals, per-node shear stress, smoothed |tau| and pressure to 1e-9, for the
flow and the rotated flow."""
import numpy as np
import pytest

from erosion_b200 import geometry as G, thetalen as TL
from oracle import thetalen_oracle as TO

pytestmark = pytest.mark.gpu


def state_and_density(oracle, name, rotation):
    g = G.workload(name)
    params = TL.ParamSet(npts=g.n, nouter=g.nout, wall=g.wall, ibc=g.ibc, fixpdrop=False)
    thld = TL.circs2thlenden(g.n, g.radii, g.centers[:, 0], g.centers[:, 1])
    bodies = [TO.Body(b.theta.copy(), b.len, b.xsm, b.ysm) for b in thld.thlenvec]
    xs, ys = zip(*[TO.getxy(b) for b in bodies])
    xv, yv = np.concatenate(xs), np.concatenate(ys)
    if rotation:
        xv, yv = -yv, xv
    gg = G.Geometry(g.n, g.nout, np.ascontiguousarray(xv), np.ascontiguousarray(yv), g.wall, g.ibc, g.radii,
                    g.centers)
    den, _, _, _ = oracle.solve(gg, tol=1e-12)
    if rotation:
        thld.denrot = den
    else:
        thld.density = den
    return g, params, thld, bodies, den


@pytest.mark.parametrize("name,rotation", [("ref-small", False), ("ref-small", True), ("c1", False)])
def test_drag_matches_oracle(lib, oracle, name, rotation):
    g, params, thld, bodies, den = state_and_density(oracle, name, rotation)
    d = TL.drag(thld, params, rotation=rotation)
    (pdx, pdy, vdx, vdy), tau, atau, press = TO.drag(oracle, bodies, den, g.nout, g.wall, g.ibc, params.sigma,
                                                     rotation=rotation)
    want = np.array([pdx, pdy, vdx, vdy])
    got = np.array([d.pdragx, d.pdragy, d.vdragx, d.vdragy])
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-9
    for a, b in ((d.tau_all, tau), (d.atau_all, atau), (d.press_all, press)):
        assert a.shape == b.shape
        assert np.abs(a - b).max() / np.abs(b).max() < 1e-9
    assert d.umax == 1.0
