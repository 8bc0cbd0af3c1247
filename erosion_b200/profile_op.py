"""One application of the boundary operator on a named workload, with the
far-field launch shapes pinned: the small, fixed sequence of launches a
kernel profiler captures.

    python -m erosion_b200.profile_op [--workload c3] [--precision 1]
                                      [--shape64 0] [--shape32 0] [--shape64f 0] [--reps 1]

precision: 0 accurate FP64 far field, 1 mixed (FP32 body sources, FP64 wall
sources), 2 the fast FP64 far field.  The density is seeded random.  With
pinned shapes the set-up launches no autotuner timing.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import _lib, geometry as G, stokes


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--precision", type=int, default=1)
    ap.add_argument("--shape64", type=int, default=0)
    ap.add_argument("--shape32", type=int, default=0)
    ap.add_argument("--shape64f", type=int, default=0)
    ap.add_argument("--reps", type=int, default=1)
    args = ap.parse_args(argv)
    L = _lib.load()
    for kind, sh in ((0, args.shape64), (1, args.shape32), (2, args.shape64f)):
        _lib.check(L.erosion_set_far_shape(kind, sh))
    g = G.workload(args.workload)
    den = np.random.default_rng(0).standard_normal(g.ntot)
    for _ in range(args.reps):
        v = stokes.matvec(g, den, precision=args.precision)
    print(f"{args.workload}: N = {g.N}, precision {args.precision}, |A x| = {np.linalg.norm(v):.6e}")


if __name__ == "__main__":
    main()
