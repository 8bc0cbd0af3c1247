#!/usr/bin/env python
"""Erosion steps per second on one B200 (per GPU replica under torchrun).

A step is one RK2 erosion step of the theta-L state (TimeStepping.jl:189-202):
two GMRES solves of the Stokes boundary integral equation to relative residual
1e-8, two wall shear-stress evaluations and the theta-L updates, all in
libstokes_b200.so on the GPU.  Synthetic seeded geometries of the named
workloads (erosion_b200.geometry.workload); fixed pressure drop off.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2]
                  [--impl ours|reference] [--precision 0|1] [--warm-start 0|1]

Prints one JSON line on rank 0.  `value` is device-timed (CUDA events on the
library's stream) with the state resident in HBM; `e2e` goes through the
host-array C-ABI entry point with the host<->device copies inside the timed
region.  L2 is flushed (a 256 MiB write) before every timed step.
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
# dL/dt ~ -100..-600 against L ~ 0.2-0.7), so the step is scaled to 1e-5,
# which keeps every body through the timed window.  The per-step work (two
# solves, two shear stresses, the theta-L arithmetic) does not depend on dt.
WORKLOADS = {
    "c1": dict(desc="10 circles x 128 nodes, 1024 wall nodes, channel [-1,1]x[-0.5,0.5], parabolic inflow",
               dt=1e-5, dt_config=1e-3),
    "c2": dict(desc="100 perturbed bodies x 256 nodes (25.6k body nodes), 2048 wall nodes, channel "
                    "[-1,1]x[-0.5,0.5], parabolic inflow", dt=1e-5, dt_config=5e-4),
    "c3": dict(desc="400 circles x 256 nodes (102k body nodes), 4096 wall nodes, channel [-1,1]x[-0.5,0.5]",
               dt=1e-5, dt_config=5e-4),
    "c5": dict(desc="200 circles x 256 nodes, 4096 wall nodes, channel [-1,1]x[-0.5,0.5]", dt=1e-5,
               dt_config=5e-4),
    # ensemble: a step is one ensemble solve (every geometry to 1e-8), not an erosion step
    "c4": dict(desc="ensemble of independent channel geometries, bodies U{20..200}, nodes per body "
                    "{128,256,512}, porosity U[0.5,0.8], 2048 wall nodes", dt=None, dt_config=None),
}
METRIC = "erosion steps/s at 1e-8 residual"
ITER_FILE = os.path.join(ROOT, "profiles", "gmres_iterations.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "far_field_traffic.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", type=int, default=1, help="0 FP64, 1 mixed (FP32 far field + FP64 refinement)")
    ap.add_argument("--precond", type=int, default=1, help="0 none (reference), 1 block Gauss-Seidel")
    ap.add_argument("--warm-start", type=int, default=0)
    ap.add_argument("--compare-plain", type=int, default=1,
                    help="also time one step of the plain FP64 unpreconditioned form")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ensemble", type=int, default=64, help="geometries of the c4 ensemble")
    return ap.parse_args()


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


def cpu_rate(g, iters_per_step: float, budget_s: float, threads: int | None = None):
    """Erosion steps/s of the oracle port on the host cores, from a bounded
    sample: FP64 operator applications of the workload (mode: direct far field
    + barycentric near field) and the shear stress on a sub-problem of the
    first m bodies, scaled by M(M-1)/(m(m-1)).  Step = iterations x operator +
    2 x stress (+ the O(M n^2) theta-L arithmetic, negligible)."""
    from oracle import Oracle
    from erosion_b200 import geometry as G
    o = Oracle()
    if threads:
        o.threads(threads)
    nthreads = o.threads()
    den = np.random.default_rng(0).standard_normal(g.ntot)
    t0 = time.perf_counter()
    o.matvec(g, den, mode=1)
    t_mv = time.perf_counter() - t0
    nmv = 1
    while time.perf_counter() - t0 < 0.4 * budget_s and nmv < 20:
        o.matvec(g, den, mode=1)
        nmv += 1
    t_mv = (time.perf_counter() - t0) / nmv
    m = min(g.M, 12)
    sub = G.Geometry(g.n, g.nout, g.xx[:m * g.n].copy(), g.yy[:m * g.n].copy(), g.wall, g.ibc, g.radii[:m],
                     g.centers[:m])
    dsub = np.random.default_rng(1).standard_normal(sub.ntot)
    t1 = time.perf_counter()
    o.shear_stress(sub, dsub)
    t_st_sub = time.perf_counter() - t1
    scale = (g.M * (g.M - 1)) / max(m * (m - 1), 1)
    t_stress = t_st_sub * scale
    t_step = iters_per_step * t_mv + 2 * t_stress
    sample = (f"{nmv} FP64 operator applications of the full workload ({t_mv:.3f} s each) and one shear stress "
              f"of its first {m} bodies ({t_st_sub:.2f} s, scaled x{scale:.1f}); step = {iters_per_step:.0f} "
              f"GMRES iterations x operator + 2 stresses")
    return 1.0 / t_step, nthreads, sample, t_step


def load_iterations(workload: str):
    try:
        with open(ITER_FILE) as f:
            return json.load(f).get(workload)
    except Exception:
        return None


def run_reference(args, world, rank):
    """The reference's own CPU path cannot be built here (Fortran + Julia);
    this arm times the oracle port of it on all host cores."""
    if rank != 0:
        return
    if args.workload == "c4":
        print(json.dumps({"impl": "reference", "unavailable": "the reference arm is defined per geometry (c1-c3, "
                                                              "c5); the ensemble has no recorded plain iteration "
                                                              "counts to scale the CPU sample by"}))
        return
    from erosion_b200 import geometry as G
    g = G.workload(args.workload, seed=args.seed)
    rec = load_iterations(args.workload)
    if not rec:
        print(json.dumps({"impl": "reference", "unavailable": f"no recorded GMRES iteration count for "
                                                              f"{args.workload} in profiles/gmres_iterations.json"}))
        return
    iters = float(rec["iterations_per_step"])
    per_step_budget = max(4.0, 60.0 / max(args.steps + args.warmup, 1))
    vals = []
    for i in range(args.warmup + args.steps):
        v, nth, sample, t_step = cpu_rate(g, iters, per_step_budget)
        if i >= args.warmup:
            vals.append(v)
    v = float(np.mean(vals))
    out = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"{args.workload}: {WORKLOADS[args.workload]['desc']}",
                      "parallelism": "host threads (OpenMP)"},
           "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "steps/s", "cores": nth, "kind": "port", "sample": sample},
           "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_ensemble(args, world, rank, local, dist):
    """The batching workload: one step = one solve of every geometry of an
    ensemble to 1e-8 (mixed precision, block preconditioner) through
    erosion_solve_batch, host arrays in and out.  Reported as GMRES solves/s
    beside the same geometries solved one erosion_solve call after another."""
    import torch
    from erosion_b200 import _lib, geometry as G, stokes
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
                "device_ms_per_step": dev_ms, "rounds": st["rounds"], "iterations": st["iterations"],
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


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
        if dist:
            dist.destroy_process_group()
        return
    import torch
    from erosion_b200 import _lib, build, geometry as G
    build.build()
    L = _lib.load()
    torch.cuda.set_device(local)
    if args.workload == "c4":
        run_ensemble(args, world, rank, local, dist)
        if dist:
            dist.destroy_process_group()
        return
    dev = torch.device("cuda", local)

    wl = WORKLOADS[args.workload]
    g = G.workload(args.workload, seed=args.seed + rank)
    th, ln, xs, ys = G.to_thetalen(g)
    M0, n = g.M, g.n
    p = _lib.default_params(wall=tuple(g.wall), ibc=g.ibc, precision=args.precision, precond=args.precond)
    p_plain = _lib.default_params(wall=tuple(g.wall), ibc=g.ibc, precision=0, precond=0)
    sp = _lib.StepParams()
    L.erosion_default_step_params(ctypes.byref(sp), n)
    sp.dt = wl["dt"]
    sp.fixpdrop = 0
    sp.warm_start = args.warm_start

    d_th = torch.tensor(th, dtype=torch.float64, device=dev)
    d_ln = torch.tensor(ln, dtype=torch.float64, device=dev)
    d_xs = torch.tensor(xs, dtype=torch.float64, device=dev)
    d_ys = torch.tensor(ys, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(L.erosion_stream(), device=dev)
    nb = np.array([M0], np.int64)
    tt = np.zeros(1)
    deleted = np.zeros(M0, np.int64)
    PI64, PD = _lib.PI64, _lib.PD

    def step(params=None):
        params = params or p
        rc = L.erosion_rk2_step_device(ctypes.byref(params), ctypes.byref(sp), n, nb.ctypes.data_as(PI64), g.nout,
                                       d_th.data_ptr(), d_ln.data_ptr(), d_xs.data_ptr(), d_ys.data_ptr(),
                                       tt.ctypes.data_as(PD), deleted.ctypes.data_as(PI64))
        _lib.check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
        st = _lib.StepStats()
        L.erosion_get_step_stats(ctypes.byref(st))
        return st.as_dict()

    def solve_stats():
        s = _lib.SolveStats()
        L.erosion_get_solve_stats(ctypes.byref(s))
        return s.as_dict()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    s0 = solve_stats()
    launches0 = L.erosion_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    iters = []
    per_step = []
    with Clocks(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(args.steps):
                flush.zero_()
                st = step()
                iters.append(sum(st["gmres_iterations"]))
                per_step.append(st)
            ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = L.erosion_launch_count() - launches0
    s1 = solve_stats()
    ms = max_over_ranks(ms, dist, local)
    value = world * args.steps / (ms * 1e-3)

    # roofline of the dominant far-field kernel: FP64 (k_far64) or FP32
    # (k_far32), against the measured FMA peak of the pipe it runs on
    N = g.nout + n * int(nb[0])
    far64_ms = s1["ms_far"] - s0["ms_far"]
    far64_n = s1["far_launches"] - s0["far_launches"]
    far32_ms = s1["ms_far32"] - s0["ms_far32"]
    far32_n = s1["far32_launches"] - s0["far32_launches"]
    peak64 = L.erosion_peak_tflops(0)
    peak32_scalar = L.erosion_peak_tflops(1)
    peak32_packed = L.erosion_peak_tflops(2)
    peak32 = max(peak32_scalar, peak32_packed)   # the higher of scalar and two-lane FMA
    kernels = {}
    if far64_n:
        a = 20.0 * s1["far64_pairs"] / (far64_ms / far64_n * 1e-3) / 1e12
        kernels["k_far64"] = {"launches": far64_n, "ms_total": far64_ms, "ms_avg": far64_ms / far64_n,
                              "pairs_per_launch": s1["far64_pairs"], "achieved_tflops": a, "peak_tflops": peak64,
                              "frac": a / peak64, "share_of_timed": far64_ms / ms}
    farw_ms = s1["ms_farw"] - s0["ms_farw"]
    farw_n = s1["farw_launches"] - s0["farw_launches"]
    if farw_n:
        a = 20.0 * s1["farw_pairs"] / (farw_ms / farw_n * 1e-3) / 1e12
        kernels["k_far64_wall_sources"] = {"launches": farw_n, "ms_total": farw_ms, "ms_avg": farw_ms / farw_n,
                                           "pairs_per_launch": s1["farw_pairs"], "achieved_tflops": a,
                                           "peak_tflops": peak64, "frac": a / peak64, "share_of_timed": farw_ms / ms}
    if far32_n:
        pairs32 = s1["far32_pairs"]
        a = 20.0 * pairs32 / (far32_ms / far32_n * 1e-3) / 1e12
        kernels["k_far32"] = {"launches": far32_n, "ms_total": far32_ms, "ms_avg": far32_ms / far32_n,
                              "pairs_per_launch": pairs32, "achieved_tflops": a, "peak_tflops": peak32,
                              "frac": a / peak32, "share_of_timed": far32_ms / ms}
    dom = max(kernels, key=lambda k: kernels[k]["ms_total"]) if kernels else None
    traffic = None
    try:
        with open(TRAFFIC_FILE) as f:
            traffic = json.load(f).get(f"{args.workload}:{dom}") or json.load(open(TRAFFIC_FILE)).get(args.workload)
    except Exception:
        pass
    roofline = {"bound": "fp32" if dom == "k_far32" else "fp64", "achieved": kernels[dom]["achieved_tflops"] if dom else None,
                "peak": kernels[dom]["peak_tflops"] if dom else None, "unit": "TFLOP/s",
                "frac": kernels[dom]["frac"] if dom else None, "traffic": traffic, "kernel": dom,
                "algorithmic": "20 flops per source-target pair; pairs per launch: k_far64 = node pairs of distinct "
                               "curves less the barycentric near pairs (self-curve pairs run in k_self64); in the "
                               "mixed operator k_far32 takes the body-source pairs and k_far64_wall_sources the "
                               "wall-source pairs",
                "peak_source": "measured FMA loop on this GPU (erosion_peak_tflops), vector pipe; FP32 = max of "
                               "scalar and packed two-lane FMA",
                "peaks_measured_tflops": {"fp64": peak64, "fp32_scalar": peak32_scalar, "fp32_packed": peak32_packed},
                "launch_shapes": _lib.far_shapes(),
                "kernels": kernels}

    # end to end through the host-array entry point (state in host memory)
    e2e = None
    if args.e2e_steps > 0:
        hth = d_th[: int(nb[0]) * n].cpu().numpy().copy()
        hln = d_ln[: int(nb[0])].cpu().numpy().copy()
        hxs = d_xs[: int(nb[0])].cpu().numpy().copy()
        hys = d_ys[: int(nb[0])].cpu().numpy().copy()
        Mh = np.array([int(nb[0])], np.int64)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        h2d = d2h = 0
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.e2e_steps):
                flush.zero_()
                Mcur = int(Mh[0])
                h2d += (Mcur * n + 3 * Mcur) * 8
                rc = L.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sp), n, Mh.ctypes.data_as(PI64), g.nout,
                                        _lib.ptr(hth), _lib.ptr(hln), _lib.ptr(hxs), _lib.ptr(hys),
                                        tt.ctypes.data_as(PD), deleted.ctypes.data_as(PI64))
                _lib.check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
                d2h += (int(Mh[0]) * n + 3 * int(Mh[0])) * 8
            e1.record(stream)
        torch.cuda.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1), dist, local)
        e2e = {"value": world * args.e2e_steps / (ems * 1e-3), "unit": "steps/s",
               "h2d_bytes_per_step": h2d // args.e2e_steps, "d2h_bytes_per_step": d2h // args.e2e_steps,
               "entry_point": "erosion_rk2_step (host arrays)"}

    mean_iters = float(np.mean(iters)) if iters else 0.0
    plain = None
    if args.compare_plain:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sp0 = solve_stats()
        with torch.cuda.stream(stream):
            flush.zero_()
            e0.record(stream)
            stp = step(p_plain)
            e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1)
        sp1 = solve_stats()
        plain = {"value": 1.0 / (pms * 1e-3) * world, "unit": "steps/s", "steps": 1,
                 "gmres_iterations_per_step": sum(stp["gmres_iterations"]),
                 "step_breakdown_ms": {k: stp[k] for k in ("ms_solve", "ms_stress", "ms_thetalen", "ms_total")},
                 "far64_ms": sp1["ms_far"] - sp0["ms_far"],
                 "form": "FP64 operator, no preconditioner, zero initial guess (the reference's algorithm)",
                 "speedup_of_value": value / (1.0 / (pms * 1e-3) * world)}
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            it_ref = plain["gmres_iterations_per_step"] if plain else (load_iterations(args.workload) or {}).get(
                "iterations_per_step", mean_iters)
            v, nth, sample, t_step = cpu_rate(g, it_ref, args.cpu_seconds)
            cpu = {"value": v, "unit": "steps/s", "cores": nth, "kind": "port", "sample": sample}
        pairs_per_s = (s1["matvecs"] - s0["matvecs"]) * N * (N - 1) / (ms * 1e-3) * world
        out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "f64+f32",
               "data": "synthetic",
               "config": {"workload": f"{args.workload}: {wl['desc']}", "bodies": M0, "nodes_per_body": n,
                          "wall_nodes": g.nout, "unknowns": g.ntot, "dt": wl["dt"],
                          "dt_note": f"configured dt {wl['dt_config']} deletes every body in step 1 at this "
                                     f"shear-stress scale; scaled to keep the bodies", "fixpdrop": 0, "tol": 1e-8,
                          "precision": "fp64" if args.precision == 0 else "mixed", "warm_start": args.warm_start,
                          "precond": "block Gauss-Seidel" if args.precond else "none",
                          "parallelism": "replicas" if world > 1 else "single GPU",
                          "l2": "flushed (256 MiB write) before every step"},
               "gmres_iterations_per_step": mean_iters,
               "pair_interactions_per_s": pairs_per_s,
               "gmres_solves_per_s": 2 * value,
               "step_breakdown_ms": {k: float(np.mean([s[k] for s in per_step])) for k in
                                     ("ms_solve", "ms_stress", "ms_thetalen", "ms_total")},
               "plain_fp64": plain,
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
               "clocks": clk.summary()}
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
