"""drag (PostProcess.jl:131-162) through erosion_drag against the oracle's
restatement (oracle/thetalen_oracle.py: drag), on the same solved density:
totals, per-node shear stress, smoothed |tau| and pressure, for the flow and
the rotated flow (the geometry turned by 90 degrees inside the same wall, so
the rotated case needs bodies whose turned positions stay inside it: the
3-body case below; the library rejects a body outside the wall).

With every shear-stress pair evaluated by the barycentric formulas, as the
reference does (stress_all_bary = 1), the totals agree to 1e-9 and the
per-node arrays to 1e-9 plus the two sides' rounding on the density's rigid
parts (oracle/rigid.py: a rigid-motion density has exactly zero shear stress
and pressure, so whatever an evaluation returns for it is rounding; on the
10-body channel's solved density, whose rigid parts reach ~3e3, that is
~1e-9 of max |tau|).  The default evaluation (trapezoid rule beyond 12 node spacings) differs from the
all-barycentric one by the barycentric formulas' own rounding and
resolution error, which on the 10-body channel's solved density reaches
1e-9 of the largest value (measured): 1e-8 there."""
import numpy as np
import pytest

from erosion_b200 import geometry as G, thetalen as TL
from erosion_b200 import stokes
from oracle import thetalen_oracle as TO
from oracle.rigid import rigid_parts

pytestmark = pytest.mark.gpu


def geometry(name):
    if name == "turnable":   # turned by 90 degrees, every body stays inside the wall
        return G.custom(64, 256, [0.2, 0.15, 0.12], [[-0.4, 0.2], [0.3, -0.3], [0.35, 0.4]])
    return G.workload(name)


def state_and_density(oracle, name, rotation, all_bary=1):
    g = geometry(name)
    params = TL.ParamSet(npts=g.n, nouter=g.nout, wall=g.wall, ibc=g.ibc, fixpdrop=False,
                         stress_all_bary=all_bary)
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
    return g, gg, params, thld, bodies, den


@pytest.mark.parametrize("name,rotation,all_bary", [("ref-small", False, 1), ("turnable", False, 1),
                                                    ("turnable", True, 1), ("c1", False, 1), ("c1", False, 0)])
def test_drag_matches_oracle(lib, oracle, name, rotation, all_bary):
    g, gg, params, thld, bodies, den = state_and_density(oracle, name, rotation, all_bary)
    tol = 1e-9 if all_bary else 1e-8
    P = rigid_parts(gg.n, gg.M, gg.nout, gg.xx, gg.yy, den)
    tau_scale = np.abs(oracle.shear_stress(gg, den)[0]).max()
    p_scale = np.abs(oracle.pressure(gg, den)).max()
    floor_tau = (np.abs(oracle.shear_stress(gg, P)[0]).max()
                 + np.abs(stokes.shear_stress(gg, P, stress_all_bary=all_bary)[0]).max()) / tau_scale
    floor_p = (np.abs(oracle.pressure(gg, P)).max() + np.abs(stokes.pressure(gg, P)).max()) / p_scale
    print(f"rounding on the rigid parts: shear stress {floor_tau:.2e}, pressure {floor_p:.2e}")
    d = TL.drag(thld, params, rotation=rotation)
    (pdx, pdy, vdx, vdy), tau, atau, press = TO.drag(oracle, bodies, den, g.nout, g.wall, g.ibc, params.sigma,
                                                     rotation=rotation)
    want = np.array([pdx, pdy, vdx, vdy])
    got = np.array([d.pdragx, d.pdragy, d.vdragx, d.vdragy])
    assert np.abs(got - want).max() / np.abs(want).max() < tol
    for a, b, fl in ((d.tau_all, tau, floor_tau), (d.atau_all, atau, floor_tau), (d.press_all, press, floor_p)):
        assert a.shape == b.shape
        assert np.abs(a - b).max() / np.abs(b).max() < tol + fl
    assert d.umax == 1.0
