"""Generates the golden fixtures in this folder from the CPU FP64 oracle.

The reference (Fortran solver + Julia driver) cannot be built or run without a
Fortran compiler and Julia, and its repository ships no stored densities,
stresses or iteration counts for any geometry.  These fixtures therefore hold
the oracle's outputs on small seeded geometries; they freeze the oracle (a
change to it shows up as a fixture mismatch in the CPU tests) and give the GPU
tests a committed target independent of a rebuilt oracle.  What pins the
oracle to the reference's mathematics is the set of known-answer and identity
tests in tests/test_oracle.py.

Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from erosion_b200 import geometry as G  # noqa: E402
from oracle import Oracle  # noqa: E402
from oracle import thetalen_oracle as TO  # noqa: E402

SMALL_BODIES = [(0.3, -1.0, 0.1), (0.25, -0.35, 0.0), (0.2, 0.6, 0.72)]


def qoi_points():
    """The 13-point slices at x = -2 and x = +2 of getpdrop (DensityStress.jl:129-138)."""
    ny = 13
    dy = 2.0 / ny
    y = -1 + 0.5 * dy + dy * np.arange(ny)
    return np.r_[np.full(ny, -2.0), np.full(ny, 2.0)], np.r_[y, y]


def make_operator_fixture(o: Oracle) -> dict:
    g = G.workload("ref-small")
    rng = np.random.default_rng(0)
    d = rng.standard_normal(g.ntot)
    out = dict(n=g.n, nout=g.nout, ibc=g.ibc, wall=np.array(g.wall), xx=g.xx, yy=g.yy, radii=g.radii,
               centers=g.centers, density_in=d,
               matvec_fmmbary=o.matvec(g, d, mode=1), matvec_bary=o.matvec(g, d, mode=2),
               matvec_trap=o.matvec(g, d, mode=0), rhs=o.rhs(g))
    den, nits, ierr, err = o.solve(g, tol=1e-12)
    assert ierr == 0
    den8, nits8, ierr8, _ = o.solve(g, tol=1e-8)
    tau, E = o.shear_stress(g, den)
    tau0, _ = o.shear_stress(g, den, ibary=0)
    xt, yt = qoi_points()
    u, v, p, w = o.qoi_targets(g, den, xt, yt)
    out.update(density=den, nits_tight=nits, nits_1e8=nits8, tau=tau, E=E, tau_trap=tau0, xt=xt, yt=yt,
               utar=u, vtar=v, ptar=p, vortar=w, pressure=o.pressure(g, den))
    return out


def make_thetalen_fixture(o: Oracle) -> dict:
    n, nout, dt = 64, 256, 1e-3
    eps, sig = 15.0 / n, 10.0 / n     # ParamSet defaults, ThetaLen.jl:23-24, 35-36
    tor = TO.ThetaLenOracle(o, nout, G.REFERENCE_WALL, 1, eps, sig, dt, tol=1e-12)
    b0 = [TO.circ2thlen(n, r, x, y) for r, x, y in SMALL_BODIES]
    b1 = tor.rungekutta2([TO.Body(b.theta.copy(), b.len, b.xsm, b.ysm) for b in b0])
    return dict(n=n, nout=nout, dt=dt, epsilon=eps, sigma=sig, bodies=np.array(SMALL_BODIES),
                theta1=np.array([b.theta for b in b1]), len1=np.array([b.len for b in b1]),
                xsm1=np.array([b.xsm for b in b1]), ysm1=np.array([b.ysm for b in b1]))


def main():
    o = Oracle()
    np.savez_compressed(os.path.join(HERE, "ref_small_operator.npz"), **make_operator_fixture(o))
    np.savez_compressed(os.path.join(HERE, "ref_small_rk2.npz"), **make_thetalen_fixture(o))
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
