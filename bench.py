#!/usr/bin/env python
"""Erosion steps per second on one B200 (per GPU replica under torchrun).

A step is one RK2 erosion step of the theta-L state (TimeStepping.jl:189-202):
two GMRES solves of the Stokes boundary integral equation to relative residual
1e-8, two wall shear-stress evaluations and the theta-L updates, all in
libstokes_b200.so on the GPU.  Synthetic seeded geometries of the named
workloads (erosion_b200.geometry.workload); fixed pressure drop off.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3]
                  [--impl ours|reference] [--precision 0|1] [--warm-start 0|1|2]

Prints one JSON line on rank 0.  `value` is device-timed (CUDA events on the
library's stream) with the state resident in HBM; `e2e` repeats the same K
steps from the same starting state through the host-array C-ABI entry point
(erosion_rk2_step), the host<->device copies inside the timed region.  L2 is
flushed (a 256 MiB write) before every timed step.  The body count is fixed
over the timed window: the step dt is chosen so that no body erodes away, and
should one be deleted all the same the state is restored to the window's
starting state before the next step (counted in `config.restores`).  The
far-field launch shapes are tuned during the warm-up and then frozen, so no
tuning runs inside a timed region.  `plain_fp64` is one step of the
reference's algorithm on the GPU (FP64 operator, no preconditioner, zero
initial guess) from the same starting state.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# dt: the workloads' stated steps (1e-3, 5e-4) delete every body within the
# first step under the reference's erosion law in this channel (|tau| ~ 20-100,
# dL/dt ~ -100..-3000 against L ~ 0.1-0.7), so the step is scaled down until
# every body survives the warm-up, the timed window and the comparison legs.
# The work of a step (two solves, two shear stresses, the theta-L arithmetic)
# does not depend on dt itself, but the GMRES iteration count depends on the
# state: the freshly packed bodies (gaps of 4 node spacings) take the most
# iterations, and they fall as erosion opens the gaps (400-body channel: 604
# iterations for the first solve, 474 four steps of dt = 1e-6 later).  A small
# dt keeps the timed window at the configured packing.
WORKLOADS = {
    "c1": dict(desc="10 circles x 128 nodes, 1024 wall nodes, channel [-1,1]x[-0.5,0.5], parabolic inflow",
               dt=1e-5, dt_config=1e-3),
    "c2": dict(desc="100 perturbed bodies x 256 nodes (25.6k body nodes), 2048 wall nodes, channel "
                    "[-1,1]x[-0.5,0.5], parabolic inflow", dt=2e-6, dt_config=5e-4),
    "c3": dict(desc="400 circles x 256 nodes (102k body nodes), 4096 wall nodes, channel [-1,1]x[-0.5,0.5], "
                    "parabolic inflow", dt=5e-7, dt_config=5e-4),
    "c5": dict(desc="200 circles x 256 nodes, 4096 wall nodes, channel [-1,1]x[-0.5,0.5]", dt=1e-6,
               dt_config=5e-4),
    # ensemble: a step is one ensemble solve (every geometry to 1e-8), not an erosion step
    "c4": dict(desc="ensemble of independent channel geometries, bodies U{20..200}, nodes per body "
                    "{128,256,512}, porosity U[0.5,0.8], 2048 wall nodes", dt=None, dt_config=None),
}
METRIC = "erosion steps/s at 1e-8 residual"

# DRAM bytes per node and far-field launch (dram__bytes_read.sum +
# dram__bytes_write.sum of one launch divided by the node count N) from the ncu
# captures of k_far32 and the fast k_far64 on the 400-body channel (N =
# 106,496; one operator application with pinned launch shapes).  A launch
# reads each source and target record once (N x 64 B) and each target's row
# of the near mask once (N x 4 B per 32 curves: 52 B at 401 curves).  The
# accurate k_far64 and the wall-source launch read the same records as the
# fast k_far64 and carry its figure.
TRAFFIC_BYTES_PER_NODE = {"k_far32": (11398144 + 16384) / 106496, "k_far64_fast": 10671360 / 106496,
                          "k_far64": 10671360 / 106496, "k_far64_wall_sources": 10671360 / 106496}


# Plain FP64 GMRES iterations per erosion step (unpreconditioned, zero initial
# guess: the reference's algorithm) on the seeded workloads, as the plain_fp64
# leg of this script measures them on the GPU.  Used only by the reference
# arm's model for workloads whose CPU solve cannot finish in minutes; on c1
# the reference arm runs the oracle's own GMRES instead.
PLAIN_ITERATIONS_PER_STEP = {"c2": 3165, "c3": 13436}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", type=int, default=1, help="0 FP64, 1 mixed (FP32 far field + FP64 refinement)")
    ap.add_argument("--precond", type=int, default=1, help="0 none (reference), 1 block Gauss-Seidel")
    ap.add_argument("--warm-start", type=int, default=1,
                    help="0 zero guess (the reference), 1 previous step's density, 2 also the learned guess")
    ap.add_argument("--dt", type=float, default=None, help="override the workload's step")
    ap.add_argument("--compare-plain", type=int, default=1,
                    help="also time one step of the plain FP64 unpreconditioned form")
    ap.add_argument("--e2e", type=int, default=1, help="time the host-array entry point over the same K steps")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ensemble", type=int, default=64, help="geometries of the c4 ensemble")
    ap.add_argument("--c5-steps", type=int, default=30,
                    help="c5: target number of steps for 50%% of the body area to erode (sets dt)")
    ap.add_argument("--c5-max-steps", type=int, default=60, help="c5: cap on the steps of each run")
    ap.add_argument("--train-steps", type=int, default=15,
                    help="c5: steps of the 400-body run whose first-stage densities train the network")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
class Clocks:
    """Samples nvidia-smi during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
def dist_setup(args):
    """One process per GPU (torchrun): NCCL with a GPU, gloo without one (the
    reference arm and the CPU tests).  The timeout is short so that ranks
    waiting for a failed one end with an error."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(x: float, dist, local: int = 0) -> float:
    """The maximum of x over the ranks (x itself on one process)."""
    if not dist:
        return x
    import torch
    dev = torch.device("cuda", local) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU side: the oracle port of the reference's path (the reference itself,
# Julia + Fortran, cannot be built on this image).
def cpu_operator_time(o, g, budget_s: float, max_apps: int = 20):
    """Seconds per FP64 operator application of the oracle on workload g
    (direct far field + barycentric near field, matvec_DLP_bary semantics with
    the fmmbary near rules), averaged over as many applications as fit in
    about budget_s (at least one)."""
    den = np.random.default_rng(0).standard_normal(g.ntot)
    t0 = time.perf_counter()
    o.matvec(g, den, mode=1)
    n = 1
    while time.perf_counter() - t0 < budget_s and n < max_apps:
        o.matvec(g, den, mode=1)
        n += 1
    return (time.perf_counter() - t0) / n, n


def cpu_stress_model(o, g, sizes=(2, 4)):
    """Seconds of the oracle's shear stress on workload g from two timed
    sub-problems (the full wall with the first m bodies, m in sizes): the
    reference's cost is a per-body wall part plus a per-ordered-pair part,
    T(m) = a m + b m (m - 1), fitted to the two samples and evaluated at M."""
    from erosion_b200 import geometry as G
    ts = []
    for m in sizes:
        m = min(m, g.M)
        sub = G.Geometry(g.n, g.nout, g.xx[:m * g.n].copy(), g.yy[:m * g.n].copy(), g.wall, g.ibc, g.radii[:m],
                         g.centers[:m])
        d = np.random.default_rng(1).standard_normal(sub.ntot)
        t0 = time.perf_counter()
        o.shear_stress(sub, d)
        ts.append((m, time.perf_counter() - t0))
    (m1, t1), (m2, t2) = ts
    if m1 == m2 or g.M <= m2:
        return t2 * g.M / max(m2, 1), ts
    A = np.array([[m1, m1 * (m1 - 1)], [m2, m2 * (m2 - 1)]], float)
    a, b = np.linalg.solve(A, np.array([t1, t2]))
    a, b = max(a, 0.0), max(b, 0.0)
    return a * g.M + b * g.M * (g.M - 1), ts


def cpu_rate(g, iters_per_step: float, budget_s: float, threads: int | None = None):
    """Erosion steps/s of the oracle port on the host cores from a bounded
    sample: FP64 operator applications of the workload and the two-point
    shear-stress model.  Step = iterations x operator + 2 x stress (+ the
    O(M n^2) theta-L arithmetic, negligible)."""
    from oracle import Oracle
    o = Oracle()
    if threads:
        o.threads(threads)
    nthreads = o.threads()
    t_mv, nmv = cpu_operator_time(o, g, 0.5 * budget_s)
    t_stress, ts = cpu_stress_model(o, g)
    t_step = iters_per_step * t_mv + 2 * t_stress
    sample = (f"{nmv} FP64 operator applications of the full workload ({t_mv:.3f} s each) and the shear stress "
              f"of the wall with the first {ts[0][0]} and {ts[1][0]} bodies ({ts[0][1]:.2f} s, {ts[1][1]:.2f} s; "
              f"a m + b m(m-1) fit gives {t_stress:.1f} s at {g.M} bodies); step = {iters_per_step:.0f} GMRES "
              f"iterations x operator + 2 stresses")
    return 1.0 / t_step, nthreads, sample, t_step


def cpu_step_c1(o, g):
    """One erosion step's solver work of the oracle at c1, run for real: two
    GMRES solves to 1e-8 from zero (the oracle's SLATEC-semantics GMRES) and
    two shear stresses.  Returns (seconds, GMRES iterations)."""
    t0 = time.perf_counter()
    it = 0
    for _ in range(2):
        den, nits, _, _ = o.solve(g, tol=1e-8)
        it += nits
        o.shear_stress(g, den)
    return time.perf_counter() - t0, it


def run_reference(args, world, rank):
    """The reference's own CPU path cannot be built here (Fortran + Julia);
    this arm times the oracle port of it on all host cores: a real step at c1,
    a model from timed samples at the larger workloads."""
    if rank != 0:
        return
    if args.workload != "c1" and args.workload not in PLAIN_ITERATIONS_PER_STEP:
        print(json.dumps({"impl": "reference", "unavailable": f"no measured plain GMRES iteration count for "
                                                              f"{args.workload} to scale the CPU operator sample by "
                                                              f"(the arm is defined for c1, c2 and c3)"}))
        return
    from erosion_b200 import geometry as G
    from oracle import Oracle
    g = G.workload(args.workload, seed=args.seed)
    o = Oracle()
    nth = o.threads()
    vals = []
    if args.workload == "c1":
        for i in range(args.warmup + args.steps):
            t, it = cpu_step_c1(o, g)
            if i >= args.warmup:
                vals.append(1.0 / t)
        cb = {"kind": "port", "cores": nth, "timed": True,
              "sample": f"two oracle GMRES solves to 1e-8 from zero ({it} iterations) and two shear stresses of the "
                        f"full workload per step"}
    else:
        iters = float(PLAIN_ITERATIONS_PER_STEP[args.workload])
        t_stress, ts = cpu_stress_model(o, g)
        per_step = max(2.0, 150.0 / max(args.steps + args.warmup, 1))
        for i in range(args.warmup + args.steps):
            t_mv, nmv = cpu_operator_time(o, g, per_step, max_apps=4)
            if i >= args.warmup:
                vals.append(1.0 / (iters * t_mv + 2 * t_stress))
        cb = {"kind": "port", "cores": nth, "timed": False,
              "model": "step = plain GMRES iterations x timed operator application + 2 x shear stress (a m + "
                       "b m(m-1) fit of two timed sub-problems)",
              "iterations_per_step": iters,
              "iterations_source": "plain FP64 GMRES iterations per step (unpreconditioned, zero guess) that this "
                                   "script's plain_fp64 GPU leg measures on the same seeded workload",
              "sample": f"{nmv} oracle FP64 operator applications of the full workload per step ({t_mv:.2f} s each); "
                        f"shear stress of the wall with {ts[0][0]} and {ts[1][0]} bodies ({ts[0][1]:.2f} s, "
                        f"{ts[1][1]:.2f} s)"}
    v = float(np.mean(vals))
    cb["value"] = v
    cb["unit"] = "steps/s"
    out = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"{args.workload}: {WORKLOADS[args.workload]['desc']}",
                      "bodies": g.M, "nodes_per_body": g.n, "wall_nodes": g.nout, "tol": 1e-8,
                      "parallelism": "host threads (OpenMP)"},
           "impl": "reference", "cpu_baseline": cb,
           "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ---------------------------------------------------------------------------
def run_ensemble(args, world, rank, local, dist):
    """The batching workload: one step = one solve of every geometry of an
    ensemble to 1e-8 (mixed precision, block preconditioner) through
    erosion_solve_batch, host arrays in and out.  Reported as GMRES solves/s
    beside the same geometries solved one erosion_solve call after another."""
    import torch
    from erosion_b200 import geometry as G, stokes
    E = G.ensemble(args.ensemble, seed=args.seed + rank)
    kw = dict(precision=args.precision, precond=args.precond)
    for _ in range(args.warmup):
        stokes.solve_batch(E, **kw)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    stats = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            _, nits, st = stokes.solve_batch(E, **kw)
            stats.append(st)
    torch.cuda.synchronize()
    ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps, dist, local)
    dev_ms = float(np.mean([s["ms_total"] for s in stats]))
    t1 = time.perf_counter()
    seq_dev = 0.0
    for g in E:
        _, _, s1 = stokes.solve(g, **kw)
        seq_dev += s1["ms_total"]
    seq_ms = (time.perf_counter() - t1) * 1e3
    st = stats[-1]
    if rank == 0:
        line = {"metric": "ensemble GMRES solves/s at 1e-8 residual", "value": world * len(E) / (ms * 1e-3),
                "unit": "solves/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32",
                "data": "synthetic",
                "config": {"workload": f"c4: {WORKLOADS['c4']['desc']}", "geometries": len(E),
                           "bodies": [g.M for g in E], "nodes_per_body": [g.n for g in E],
                           "precision": "mixed" if args.precision else "fp64", "precond": args.precond,
                           "step": "one solve of every geometry (wall clock of erosion_solve_batch, host arrays)"},
                "device_ms_per_step": dev_ms,
                "host_time_share": max(0.0, 1.0 - dev_ms / ms),
                "setup_host_ms": float(np.mean([s["setup_host_ms"] for s in stats])),
                "rounds": st["rounds"], "iterations": st["iterations"],
                "graph_captures": st["graph_captures"], "max_true_residual": st["max_true_residual"],
                "far_pairs_per_s": (st["pairs64_total"] + st["pairs32_total"]) / (dev_ms * 1e-3),
                "one_by_one": {"ms": seq_ms, "device_ms_in_solves": seq_dev,
                               "speedup_of_batch": seq_ms / ms},
                "e2e": {"value": world * len(E) / (ms * 1e-3), "unit": "solves/s",
                        "h2d_bytes_per_step": int(sum(16 * g.n * g.M + 8 * g.ntot for g in E)),
                        "d2h_bytes_per_step": int(sum(8 * g.ntot for g in E)),
                        "entry_point": "erosion_solve_batch (host arrays)"},
                "clocks": clk.summary()}
        print(json.dumps(line))


# ---------------------------------------------------------------------------
def run_learned(args, world, rank, local, dist):
    """The learned warm start (workload c5): trains the increment network on
    the solves of a 400-body run (c3 shapes, a different seed; both stages of
    every step, increments over their carried-over warm starts), then erodes
    a 200-body, 256-node channel until half of its body area is gone, once
    with the carried-over previous solve as the GMRES initial guess
    (warm_start = 1) and once with the learned guess (warm_start = 2), both
    mixed precision + block preconditioner to 1e-8.  dt is set from a first
    step so that the run takes about --c5-steps steps.  value = erosion steps/s
    of the learned run (device time of its steps); the line reports both runs'
    GMRES iterations and time per step."""
    import torch
    from erosion_b200 import _lib, geometry as G, learned
    L = _lib.load()
    stream = torch.cuda.ExternalStream(L.erosion_stream(), device=torch.device("cuda", local))
    g5 = G.workload("c5", seed=args.seed + rank)
    n, nout = g5.n, g5.nout
    p = _lib.default_params(wall=tuple(g5.wall), ibc=g5.ibc, precision=args.precision, precond=args.precond)

    def sparams(dt, ws):
        sp = _lib.StepParams()
        L.erosion_default_step_params(ctypes.byref(sp), n)
        sp.dt = dt
        sp.fixpdrop = 0
        sp.warm_start = ws
        return sp

    init = [a.copy() for a in G.to_thetalen(g5)]
    A0 = float(learned.areas(n, *init).sum())
    # dt from the area lost over one probe step
    th, ln, xs, ys = [a.copy() for a in init]
    nb = np.array([g5.M], np.int64)
    t = np.zeros(1)
    dele = np.zeros(g5.M, np.int64)
    dt0 = 1e-6
    _lib.check(L.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sparams(dt0, 0)), n, nb.ctypes.data_as(_lib.PI64),
                                  nout, _lib.ptr(th), _lib.ptr(ln), _lib.ptr(xs), _lib.ptr(ys),
                                  t.ctypes.data_as(_lib.PD), dele.ctypes.data_as(_lib.PI64)), (0, 1))
    rate = max((A0 - float(learned.areas(n, th[: int(nb[0]) * n], ln[: nb[0]], xs[: nb[0]], ys[: nb[0]]).sum()))
               / dt0, 1e-12)
    dt = 0.5 * A0 / rate / max(args.c5_steps, 1)
    # training set: the solves of a 400-body run at the same dt
    g3 = G.workload("c3", seed=args.seed + 1)
    t3 = [a.copy() for a in G.to_thetalen(g3)]
    t_train0 = time.perf_counter()
    traj = learned.trajectory(p, sparams(dt, 1), g3.n, g3.nout, *t3, args.train_steps)
    X, Y = learned.training_rows(p, g3.n, g3.nout, traj)
    loss0 = learned.train(X, Y, epochs=1)
    loss = learned.train(X, Y, epochs=300)
    t_train = time.perf_counter() - t_train0
    runs = {}
    for ws in (1, 2):
        th, ln, xs, ys = [a.copy() for a in init]
        nb = np.array([g5.M], np.int64)
        t = np.zeros(1)
        dele = np.zeros(g5.M, np.int64)
        sp = sparams(dt, ws)
        rec = {"iterations": [], "ms": [], "guess_used": [], "guess_residual": [], "bodies": [], "area_frac": [],
               "candidates_last_solve": []}
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        area = A0
        while area > 0.5 * A0 and len(rec["ms"]) < args.c5_max_steps and int(nb[0]) > 0:
            with torch.cuda.stream(stream):
                e0.record(stream)
                rc = L.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sp), n, nb.ctypes.data_as(_lib.PI64), nout,
                                        _lib.ptr(th), _lib.ptr(ln), _lib.ptr(xs), _lib.ptr(ys),
                                        t.ctypes.data_as(_lib.PD), dele.ctypes.data_as(_lib.PI64))
                e1.record(stream)
            torch.cuda.synchronize()
            _lib.check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
            st = _lib.StepStats()
            L.erosion_get_step_stats(ctypes.byref(st))
            d = st.as_dict()
            M = int(nb[0])
            area = float(learned.areas(n, th[: M * n], ln[:M], xs[:M], ys[:M]).sum()) if M else 0.0
            rec["iterations"].append(d["gmres_iterations"])
            rec["ms"].append(e0.elapsed_time(e1))
            rec["guess_used"].append(d["guess_used"])
            rec["guess_residual"].append(d["guess_residual"])
            # the step's second solve: residuals of its candidates (zero, warm start, learned; -1 not tried)
            rec["candidates_last_solve"].append(_lib.solve_stats()["guess_residual"])
            rec["bodies"].append(M)
            rec["area_frac"].append(area / A0)
        steps = len(rec["ms"])
        tot_ms = float(np.sum(rec["ms"]))
        its = [sum(i) for i in rec["iterations"]]
        runs[ws] = {"steps": steps, "steps_per_s": steps / (tot_ms * 1e-3), "ms_per_step": tot_ms / steps,
                    "gmres_iterations_per_step": float(np.mean(its)),
                    "gmres_iterations_per_step_after_2": float(np.mean(its[2:])) if steps > 2 else None,
                    "ms_per_solve": tot_ms / (2 * steps),
                    "final_area_frac": rec["area_frac"][-1], "bodies_end": rec["bodies"][-1], "record": rec}
    if rank == 0:
        prev, lrn = runs[1], runs[2]
        used = [u for pair in lrn["record"]["guess_used"] for u in pair]
        line = {"metric": "erosion steps/s at 1e-8 residual, 200-body run to 50% eroded area (learned vs "
                          "previous-step warm start)",
                "value": lrn["steps_per_s"], "unit": "steps/s", "n_gpus": world, "steps": lrn["steps"],
                "warmup": 0, "ms_per_step": lrn["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
                "config": {"workload": f"c5: {WORKLOADS['c5']['desc']}", "bodies": g5.M, "nodes_per_body": n,
                           "wall_nodes": nout, "dt": dt, "dt_rule": f"half the body area in about "
                                                                      f"{args.c5_steps} steps (from one probe step)",
                           "tol": 1e-8, "precision": "mixed" if args.precision else "fp64",
                           "precond": "block Gauss-Seidel" if args.precond else "none",
                           "training": {"rows": int(len(X)), "source": f"per-body increments of the two solves of each of "
                                                                       f"{args.train_steps} steps of a 400-body "
                                                                       f"run (c3 shapes, seed {args.seed + 1}), "
                                                                       f"over their carried-over warm starts",
                                        "epochs": 300, "mse_first_epoch": loss0, "mse_last_epoch": loss,
                                        "seconds": t_train}},
                "previous_step": {k: v for k, v in prev.items() if k != "record"},
                "learned": {k: v for k, v in lrn.items() if k != "record"},
                "learned_guess_used_stages": int(sum(u == 2 for u in used)), "stages": len(used),
                "gain": {"iterations_per_step": prev["gmres_iterations_per_step"] - lrn["gmres_iterations_per_step"],
                         "time_per_step_ratio": prev["ms_per_step"] / lrn["ms_per_step"]},
                "records": {"previous_step": prev["record"], "learned": lrn["record"]}}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
class Stepper:
    """The theta-L state of one workload on the device, stepped through
    erosion_rk2_step_device, with snapshot/restore of the starting state."""

    def __init__(self, L, g, dev, dt, warm_start):
        import torch
        from erosion_b200 import _lib, geometry as G
        self.L, self.g, self.torch, self._lib = L, g, torch, _lib
        th, ln, xs, ys = G.to_thetalen(g)
        self.n = g.n
        self.d = [torch.tensor(a, dtype=torch.float64, device=dev) for a in (th, ln, xs, ys)]
        self.nb = np.array([g.M], np.int64)
        self.tt = np.zeros(1)
        self.deleted = np.zeros(g.M, np.int64)
        self.sp = _lib.StepParams()
        L.erosion_default_step_params(ctypes.byref(self.sp), g.n)
        self.sp.dt = dt
        self.sp.fixpdrop = 0
        self.sp.warm_start = warm_start
        self.snap = None

    @property
    def M(self) -> int:
        return int(self.nb[0])

    def step(self, params, sp=None):
        _lib = self._lib
        sp = sp or self.sp
        th, ln, xs, ys = self.d
        rc = self.L.erosion_rk2_step_device(ctypes.byref(params), ctypes.byref(sp), self.n,
                                            self.nb.ctypes.data_as(_lib.PI64), self.g.nout, th.data_ptr(),
                                            ln.data_ptr(), xs.data_ptr(), ys.data_ptr(),
                                            self.tt.ctypes.data_as(_lib.PD), self.deleted.ctypes.data_as(_lib.PI64))
        _lib.check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
        st = _lib.StepStats()
        self.L.erosion_get_step_stats(ctypes.byref(st))
        return st.as_dict()

    def snapshot(self):
        self.snap = ([a.clone() for a in self.d], int(self.nb[0]), float(self.tt[0]))

    def restore(self):
        arrs, M, t = self.snap
        for a, s in zip(self.d, arrs):
            a.copy_(s)
        self.nb[0] = M
        self.tt[0] = t

    def host_state(self):
        """The snapshot as host arrays (the e2e leg's input)."""
        arrs, M, _ = self.snap
        n = self.n
        return (arrs[0][: M * n].cpu().numpy().copy(), arrs[1][:M].cpu().numpy().copy(),
                arrs[2][:M].cpu().numpy().copy(), arrs[3][:M].cpu().numpy().copy())


def kernel_roofline(s0, s1, N, curves, peak64, peak32, ms_timed):
    """Per far-field kernel: launches, time, pairs per launch, achieved
    TFLOP/s (20 flops per pair), fraction of the measured FMA peak of its pipe
    and the DRAM bytes per launch (ncu figure per node x N) beside the
    algorithmic bytes (64 B per node record plus the node's near-mask row,
    4 B per 32 curves)."""
    algorithmic = N * (64 + 4 * ((curves + 31) // 32))
    kernels = {}
    spec = (("k_far64", "ms_far", "far_launches", "far64_pairs", peak64),
            ("k_far64_fast", "ms_far64f", "far64f_launches", "far64_pairs", peak64),
            ("k_far64_wall_sources", "ms_farw", "farw_launches", "farw_pairs", peak64),
            ("k_far32", "ms_far32", "far32_launches", "far32_pairs", peak32))
    for name, kms, kn, kp, peak in spec:
        ms = s1[kms] - s0[kms]
        nl = s1[kn] - s0[kn]
        if nl <= 0:
            continue
        pairs = s1[kp]
        a = 20.0 * pairs / (ms / nl * 1e-3) / 1e12
        kernels[name] = {"launches": nl, "ms_total": ms, "ms_avg": ms / nl, "pairs_per_launch": pairs,
                         "achieved_tflops": a, "peak_tflops": peak, "frac": a / peak,
                         "share_of_timed": ms / ms_timed,
                         "traffic_bytes_per_launch": TRAFFIC_BYTES_PER_NODE[name] * N,
                         "algorithmic_bytes_per_launch": algorithmic}
    return kernels


def run_steps(args, world, rank, local, dist):
    import torch
    from erosion_b200 import _lib, geometry as G
    L = _lib.load()
    dev = torch.device("cuda", local)
    wl = WORKLOADS[args.workload]
    dt = args.dt if args.dt is not None else wl["dt"]
    g = G.workload(args.workload, seed=args.seed + rank)
    p = _lib.default_params(wall=tuple(g.wall), ibc=g.ibc, precision=args.precision, precond=args.precond)
    p_plain = _lib.default_params(wall=tuple(g.wall), ibc=g.ibc, precision=0, precond=0)
    S = Stepper(L, g, dev, dt, args.warm_start)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(L.erosion_stream(), device=dev)

    def solve_stats():
        s = _lib.SolveStats()
        L.erosion_get_solve_stats(ctypes.byref(s))
        return s.as_dict()

    M_start0 = S.M
    for _ in range(args.warmup):
        S.step(p)
    # freeze the launch shapes the warm-up tuned
    shapes = _lib.far_shapes()
    L.erosion_set_far_shape(0, shapes["fp64"]["index"])
    L.erosion_set_far_shape(1, shapes["fp32"]["index"])
    if "fp64_fast" in shapes:
        L.erosion_set_far_shape(2, shapes["fp64_fast"]["index"])
    S.snapshot()
    M0 = S.M
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    s0 = solve_stats()
    launches0 = L.erosion_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    per_step, restores, deleted = [], 0, 0
    with Clocks(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                flush.zero_()
                st = S.step(p)
                per_step.append(st)
                if S.M != M0:
                    deleted += M0 - S.M
                    S.restore()
                    restores += 1
            ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = L.erosion_launch_count() - launches0
    s1 = solve_stats()
    M_end = S.M
    ms = max_over_ranks(ms, dist, local)
    value = world * args.steps / (ms * 1e-3)
    N = g.nout + g.n * M0
    peak64 = L.erosion_peak_tflops(0)
    peak32_scalar = L.erosion_peak_tflops(1)
    peak32_packed = L.erosion_peak_tflops(2)
    peak32 = max(peak32_scalar, peak32_packed)
    kernels = kernel_roofline(s0, s1, N, M0 + 1, peak64, peak32, ms)
    dom = max(kernels, key=lambda k: kernels[k]["ms_total"]) if kernels else None
    roofline = {"bound": ("fp32" if dom == "k_far32" else "fp64") if dom else None,
                "achieved": kernels[dom]["achieved_tflops"] if dom else None,
                "peak": kernels[dom]["peak_tflops"] if dom else None, "unit": "TFLOP/s",
                "frac": kernels[dom]["frac"] if dom else None,
                "traffic": kernels[dom]["traffic_bytes_per_launch"] if dom else None, "kernel": dom,
                "algorithmic": "20 flops per source-target pair; pairs per launch: k_far64 (accurate FP64) and "
                               "k_far64_fast (the mixed solve's FP64 phase) = node pairs of distinct curves less the "
                               "barycentric near pairs (self-curve pairs run in k_self64); in the mixed operator's "
                               "FP32 phase k_far32 takes the body-source pairs and k_far64_wall_sources the "
                               "wall-source pairs",
                "peak_source": "of measured: FMA loop on this GPU (erosion_peak_tflops), vector pipe; FP32 = max of "
                               "scalar and packed two-lane FMA",
                "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum per launch of the ncu captures of "
                                  "k_far32 and the fast k_far64 on the 400-body channel, per node, times N",
                "peaks_measured_tflops": {"fp64": peak64, "fp32_scalar": peak32_scalar,
                                          "fp32_packed": peak32_packed},
                "launch_shapes": shapes, "kernels": kernels}
    mv = sum(sum(st["matvecs"]) for st in per_step)
    mv32 = sum(sum(st["matvecs_fp32"]) for st in per_step)

    # end to end: the same K steps from the same starting state through the
    # host-array entry point
    e2e = None
    if args.e2e:
        hth, hln, hxs, hys = S.host_state()
        Mh = np.array([M0], np.int64)
        tt = np.zeros(1)
        dl = np.zeros(M0, np.int64)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        h2d = d2h = 0
        t0 = time.perf_counter()
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                flush.zero_()
                Mc = int(Mh[0])
                h2d += (Mc * g.n + 3 * Mc) * 8
                rc = L.erosion_rk2_step(ctypes.byref(p), ctypes.byref(S.sp), g.n, Mh.ctypes.data_as(_lib.PI64),
                                        g.nout, _lib.ptr(hth), _lib.ptr(hln), _lib.ptr(hxs), _lib.ptr(hys),
                                        tt.ctypes.data_as(_lib.PD), dl.ctypes.data_as(_lib.PI64))
                _lib.check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
                d2h += (int(Mh[0]) * g.n + 3 * int(Mh[0])) * 8
            e1.record(stream)
        torch.cuda.synchronize()
        wall_e2e = time.perf_counter() - t0
        ems = max_over_ranks(e0.elapsed_time(e1), dist, local)
        e2e = {"value": world * args.steps / (ems * 1e-3), "unit": "steps/s", "steps": args.steps,
               "h2d_bytes_per_step": h2d // args.steps, "d2h_bytes_per_step": d2h // args.steps,
               "entry_point": "erosion_rk2_step (host arrays), same starting state and step count as value",
               "host_wall_s": wall_e2e, "bodies_end": int(Mh[0])}

    plain = None
    if args.compare_plain:
        S.restore()
        sp_plain = _lib.StepParams()
        ctypes.memmove(ctypes.byref(sp_plain), ctypes.byref(S.sp), ctypes.sizeof(sp_plain))
        sp_plain.warm_start = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sp0 = solve_stats()
        with torch.cuda.stream(stream):
            flush.zero_()
            e0.record(stream)
            stp = S.step(p_plain, sp_plain)
            e1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(e0.elapsed_time(e1), dist, local)
        sp1 = solve_stats()
        pv = world / (pms * 1e-3)
        plain = {"value": pv, "unit": "steps/s", "steps": 1,
                 "gmres_iterations_per_step": sum(stp["gmres_iterations"]),
                 "step_breakdown_ms": {k: stp[k] for k in ("ms_solve", "ms_stress", "ms_thetalen", "ms_total")},
                 "far64_ms": sp1["ms_far"] - sp0["ms_far"],
                 "form": "FP64 operator, no preconditioner, zero initial guess (the reference's algorithm), from "
                         "the timed window's starting state",
                 "speedup_of_value": value / pv,
                 "speedup_of_e2e": (e2e["value"] / pv) if e2e else None}
    L.erosion_set_far_shape(0, -1)
    L.erosion_set_far_shape(1, -1)

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            it_ref = plain["gmres_iterations_per_step"] if plain else PLAIN_ITERATIONS_PER_STEP.get(args.workload, 0)
            v, nth, sample, t_step = cpu_rate(g, it_ref, args.cpu_seconds)
            cpu = {"value": v, "unit": "steps/s", "cores": nth, "kind": "port", "sample": sample, "timed": False,
                   "iterations_source": "this run's plain_fp64 leg" if plain else "PLAIN_ITERATIONS_PER_STEP"}
        pairs_per_s = (s1["matvecs"] - s0["matvecs"]) * N * (N - 1) / (ms * 1e-3) * world
        iters = [sum(st["gmres_iterations"]) for st in per_step]
        out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "f64+f32",
               "data": "synthetic",
               "config": {"workload": f"{args.workload}: {wl['desc']}", "bodies": M_start0,
                          "bodies_start": M0, "bodies_end": M_end, "bodies_deleted_in_window": deleted,
                          "restores": restores, "nodes_per_body": g.n, "wall_nodes": g.nout,
                          "unknowns": 2 * N + 3 * M0, "dt": dt,
                          "dt_note": f"configured dt {wl['dt_config']} deletes every body within the first step at "
                                     f"this shear-stress scale; scaled so that every body survives the run",
                          "fixpdrop": 0, "tol": 1e-8,
                          "precision": "fp64" if args.precision == 0 else "mixed", "warm_start": args.warm_start,
                          "precond": "block Gauss-Seidel" if args.precond else "none",
                          "launch_shapes": "tuned in the warm-up, frozen for the timed regions",
                          "parallelism": "replicas" if world > 1 else "single GPU",
                          "l2": "flushed (256 MiB write) before every step"},
               "gmres_iterations_per_step": float(np.mean(iters)) if iters else 0.0,
               "gmres_iterations_per_solve": [i for st in per_step for i in st["gmres_iterations"]],
               "far_field_launches": {"total": mv, "fp32": mv32, "fp32_share": mv32 / mv if mv else None},
               "pair_interactions_per_s": pairs_per_s,
               "gmres_solves_per_s": 2 * value,
               "step_breakdown_ms": {k: float(np.mean([s[k] for s in per_step])) for k in
                                     ("ms_solve", "ms_stress", "ms_thetalen", "ms_total", "ms_setup",
                                      "ms_precond_setup")},
               "preconditioner": {"active_every_solve": all(a for st in per_step for a in st["precond_active"]),
                                  "singular_blocks_max": max(b for st in per_step
                                                             for b in st["precond_singular_blocks"]),
                                  "setup_ms_per_step": float(np.mean([s["ms_precond_setup"] for s in per_step]))},
               "guess_used": [u for st in per_step for u in st["guess_used"]],
               "plain_fp64": plain,
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
               "clocks": clk.summary()}
        print(json.dumps(out), flush=True)


def main(argv=None):
    args = parse(argv)
    world, rank, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
            return
        import torch
        from erosion_b200 import _lib, build
        build.build()
        _lib.load()
        torch.cuda.set_device(local)
        if args.workload == "c4":
            run_ensemble(args, world, rank, local, dist)
        elif args.workload == "c5":
            run_learned(args, world, rank, local, dist)
        else:
            run_steps(args, world, rank, local, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
