"""TEST INFRASTRUCTURE ONLY — rigid-motion parts of a density (numpy).

A rigid-motion density on a body, sigma(x) = (t1, t2) + t3 (-(y - yc), x - xc),
is in the null space of the body's double-layer block (-1/2 I + D): its
exterior field is exactly zero, it carries no strain and no pressure, and it
reaches the reference's equations only through the stokeslet/rotlet rows
(stokesSolver.f: the completion flow built from the density's moments).  The
smallest bodies of a dense packing carry large rotation parts (1e5-1e6 on
radius-0.015 circles), so FP64 evaluations of the operator, the shear stress
or the pressure on such densities differ by rounding proportional to them.
Tests use this split to compare evaluations on the rigid-free density and to
measure each side's rounding on the rigid parts, whose exact value is zero.
"""
import numpy as np


def rigid_parts(n, M, nout, xx, yy, den):
    """Per body, the least-squares fit of its density by (1, 0), (0, 1) and
    (-(y - yc), x - xc) ((xc, yc) the node mean); zero on the wall and in the
    stokeslet/rotlet unknowns.  Layout: wall x, wall y, then per body its n x
    and n y entries, then 3 unknowns per body."""
    den = np.asarray(den, dtype=np.float64)
    x = np.asarray(xx, dtype=np.float64).reshape(M, n)
    y = np.asarray(yy, dtype=np.float64).reshape(M, n)
    P = np.zeros_like(den)
    one, zero = np.ones(n), np.zeros(n)
    for b in range(M):
        rx, ry = x[b] - x[b].mean(), y[b] - y[b].mean()
        modes = np.stack([np.r_[one, zero], np.r_[zero, one], np.r_[-ry, rx]], 1)
        off = 2 * nout + 2 * n * b
        c, *_ = np.linalg.lstsq(modes, den[off:off + 2 * n], rcond=None)
        P[off:off + 2 * n] = modes @ c
    return P
