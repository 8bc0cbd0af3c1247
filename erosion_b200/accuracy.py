"""Error of the mixed-precision solver against the FP64 solver over an
erosion run: per step, on the state the step starts from, the density, the
pressure drop and the per-body shear stress of the mixed solve (FP32 far field
inside FP64 refinement to tol; the first-stage solve of the erosion step
itself, as the bench runs it) against those of the FP64 solve to a tighter
tolerance, both with the block preconditioner.  Every --fp64-every steps it
also solves in FP64 to the mixed solve's tolerance (1e-8), whose errors
against the tight solve are what the stopping tolerance alone allows.

    python -m erosion_b200.accuracy [--workload c3] [--steps 50] [--dt 5e-7] [--fp64-every 5]

Prints one JSON line per step and a summary line.  The pressure drop is the
mean pressure over 13 points on x = -0.9 minus that on x = +0.9 (the
reference's getpdrop slices, DensityStress.jl:129-138, at x = +-2, lie
outside the [-1,1] x [-0.5,0.5] channel, so they are moved inside it).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import time

import numpy as np

from . import _lib, geometry as G, learned, stokes


def pressure_drop(g, den):
    y = np.linspace(-0.4, 0.4, 13)
    pl = stokes.qoi_targets(g, den, np.full(13, -0.9), y)[2]
    pr = stokes.qoi_targets(g, den, np.full(13, 0.9), y)[2]
    return float(pl.mean() - pr.mean())


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--dt", type=float, default=5e-7)
    ap.add_argument("--ref-tol", type=float, default=1e-10)
    ap.add_argument("--fp64-every", type=int, default=5,
                    help="every k-th step also solve in FP64 at the mixed solve's tol (1e-8): the error any "
                         "solver stopped at that tolerance has")
    args = ap.parse_args(argv)
    L = _lib.load()
    g0 = G.workload(args.workload, seed=args.seed)
    n, nout = g0.n, g0.nout
    th, ln, xs, ys = [a.copy() for a in G.to_thetalen(g0)]
    p = _lib.default_params(wall=tuple(g0.wall), ibc=g0.ibc, precision=1, precond=1)
    sp = _lib.StepParams()
    L.erosion_default_step_params(ctypes.byref(sp), n)
    sp.dt = args.dt
    sp.fixpdrop = 0
    sp.warm_start = 1
    nb = np.array([g0.M], np.int64)
    t = np.zeros(1)
    dele = np.zeros(g0.M, np.int64)
    x64 = None
    prev_xy = None
    worst = {"density": 0.0, "pressure_drop": 0.0, "shear_stress": 0.0}
    for k in range(args.steps):
        M = int(nb[0])
        xx, yy = learned.getxy(n, M, th[: M * n], ln[:M], xs[:M], ys[:M])
        g = G.Geometry(n, nout, xx, yy, g0.wall, g0.ibc, np.zeros(M), np.zeros((M, 2)))
        if x64 is not None and len(x64) != g.ntot:
            x64 = None
        if x64 is not None:   # the previous step's solution, rigid parts carried to the new nodes
            x64 = learned.reanchor(n, nout, prev_xy[0], prev_xy[1], xx, yy, x64)
        prev_xy = (xx, yy)
        t0 = time.perf_counter()
        x64, it64, s64 = stokes.solve(g, x0=x64, tol=args.ref_tol, precision=0, precond=1, maxl=4000,
                                      allow=(0, 1))
        # the step itself solves its first stage on this state with the mixed solver
        rc = L.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sp), n, nb.ctypes.data_as(_lib.PI64), nout,
                                _lib.ptr(th), _lib.ptr(ln), _lib.ptr(xs), _lib.ptr(ys), t.ctypes.data_as(_lib.PD),
                                dele.ctypes.data_as(_lib.PI64))
        _lib.check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
        st = _lib.StepStats()
        L.erosion_get_step_stats(ctypes.byref(st))
        st = st.as_dict()
        if int(nb[0]) != M:
            print(json.dumps({"step": k, "bodies_deleted": M - int(nb[0])}), flush=True)
            continue
        x32 = np.zeros(g.ntot)
        _lib.check(L.erosion_get_step_density(0, _lib.ptr(x32), x32.size))
        it32 = st["gmres_iterations"][0]
        tau64, _ = stokes.shear_stress(g, x64)
        tau32, _ = stokes.shear_stress(g, x32)
        dp64, dp32 = pressure_drop(g, x64), pressure_drop(g, x32)
        scale = np.abs(tau64).max()
        per_body = (np.abs(tau32 - tau64).reshape(M, n).max(1) / scale)
        rec = {"step": k, "bodies": M,
               "density_rel_err": float(np.linalg.norm(x32 - x64) / np.linalg.norm(x64)),
               "pressure_drop": dp64, "pressure_drop_rel_err": abs(dp32 - dp64) / abs(dp64),
               "shear_stress_max_rel_err": float(per_body.max()),
               "shear_stress_median_body_rel_err": float(np.median(per_body)),
               "iterations_fp64": it64, "iterations_mixed": it32, "fp64_true_residual": s64["true_residual"],
               "mixed_max_residual": st["max_residual"],
               "mixed_fp32_matvec_share": st["matvecs_fp32"][0] / max(st["matvecs"][0], 1),
               "seconds": time.perf_counter() - t0}
        if args.fp64_every > 0 and k % args.fp64_every == 0:
            x8, it8, s8 = stokes.solve(g, tol=1e-8, precision=0, precond=1, maxl=4000, allow=(0, 1))
            tau8, _ = stokes.shear_stress(g, x8)
            rec["fp64_tol1e-8"] = {
                "density_rel_err": float(np.linalg.norm(x8 - x64) / np.linalg.norm(x64)),
                "pressure_drop_rel_err": abs(pressure_drop(g, x8) - dp64) / abs(dp64),
                "shear_stress_max_rel_err": float((np.abs(tau8 - tau64).reshape(M, n).max(1) / scale).max()),
                "iterations": it8}
            worst["fp64_tol1e-8_shear_stress"] = max(worst.get("fp64_tol1e-8_shear_stress", 0.0),
                                                    rec["fp64_tol1e-8"]["shear_stress_max_rel_err"])
        worst["density"] = max(worst["density"], rec["density_rel_err"])
        worst["pressure_drop"] = max(worst["pressure_drop"], rec["pressure_drop_rel_err"])
        worst["shear_stress"] = max(worst["shear_stress"], rec["shear_stress_max_rel_err"])
        print(json.dumps(rec), flush=True)
    print(json.dumps({"summary": True, "workload": args.workload, "steps": args.steps, "dt": args.dt,
                      "reference": f"FP64 operator, block preconditioner, tol {args.ref_tol}",
                      "mixed": "FP32 far field inside FP64 refinement, block preconditioner, tol 1e-8",
                      "fp64_tol1e-8": "FP64 operator, block preconditioner, tol 1e-8, zero initial guess, every "
                                      f"{args.fp64_every}th step",
                      "max_over_steps": worst}), flush=True)


if __name__ == "__main__":
    main()
