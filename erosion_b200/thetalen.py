"""Host-side mirror of the reference's Julia interface for the erosion loop:
``ParamSet``/``ThetaLenType``/``ThLenDenType`` (ErosionPackage/src/ThetaLen.jl:13-51),
``getalpha``/``circ2thlen`` (ThetaLen.jl:113-116, Main.jl:30-35) and the calls
that reach the native library: ``getxy``/``getnxy`` (ThetaLen.jl:92-111),
``compute_density``/``compute_density_`` (DensityStress.jl:43-66),
``compute_stress`` (:191-210), ``compute_qoi_targets`` (:76-98),
``getpdrop``/``getumax``/``getnxyden`` (:129-185), ``getstress_``
(:23-36) and ``rungekutta2`` (TimeStepping.jl:189-202).

Julia's mutating ``name!`` functions are spelled ``name_`` here.  Every
numerical operation runs in libstokes_b200.so on the GPU; this module only
packs and unpacks arrays.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import numpy as np

from . import _lib
from ._lib import PD, PI64, check, ptr
from .geometry import CHANNEL_WALL, REFERENCE_WALL, Geometry


@dataclasses.dataclass
class ParamSet:
    """ThetaLen.jl:13-37 with the same defaults, plus the wall the Fortran
    hard-codes (stokesSolver.f:184-191) and the solve tolerance (:482)."""
    infolder: str = "input_geos/"
    label: str = "02-8"
    npts: int = 128
    ibary: int = 1
    ifmm: int = 1
    ibc: int = 1
    epsfac: float = 15.0
    sigfac: float = 10.0
    dt: float = 1e-3
    outstride: int = 4
    fixpdrop: bool = True
    fixarea: bool = False
    tfin: float = 1.0
    maxl: int = 8000
    nouter: int = 1024
    wall: tuple = REFERENCE_WALL
    tol: float = 1e-8
    precision: int = 0
    warm_start: int = 0
    stress_all_bary: int = 0   # 1: every shear-stress pair by the barycentric formulas, as the reference

    @property
    def epsilon(self) -> float:
        return self.epsfac / self.npts

    @property
    def sigma(self) -> float:
        return self.sigfac / self.npts

    def erosion_params(self) -> _lib.ErosionParams:
        return _lib.default_params(wall=tuple(self.wall), tol=self.tol, maxl=self.maxl, ibary=self.ibary,
                                   ifmm=self.ifmm, ibc=self.ibc, precision=self.precision,
                                   stress_all_bary=self.stress_all_bary)

    def step_params(self):
        sp = StepParams()
        _lib.load().erosion_default_step_params(ctypes.byref(sp), self.npts)
        sp.dt = self.dt
        sp.epsilon = self.epsilon
        sp.sigma = self.sigma
        sp.fixarea = int(self.fixarea)
        sp.fixpdrop = int(self.fixpdrop)
        sp.warm_start = int(self.warm_start)
        return sp


StepParams = _lib.StepParams
StepStats = _lib.StepStats


@dataclasses.dataclass
class ThetaLenType:
    theta: np.ndarray
    len: float
    xsm: float
    ysm: float
    matau: float = math.nan


@dataclasses.dataclass
class ThLenDenType:
    thlenvec: list
    tt: float = 0.0
    density: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    denrot: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))


def save_thldvec(path: str, thldvec: list, params: ParamSet | None = None) -> None:
    """The run output of Main.jl:130 (`jldsave(outfile; params, thldvec,
    cpu_hours)`) as a numpy .npz: for every saved state k, the time, each
    body's theta, L, xsm, ysm, matau, and the density and rotated density
    when present; the ParamSet fields as scalars."""
    out = {"nstates": np.array(len(thldvec))}
    for k, st in enumerate(thldvec):
        out[f"s{k}/tt"] = np.array(st.tt)
        out[f"s{k}/theta"] = np.array([b.theta for b in st.thlenvec]) if st.thlenvec else np.zeros((0, 0))
        for f in ("len", "xsm", "ysm", "matau"):
            out[f"s{k}/{f}"] = np.array([getattr(b, f) for b in st.thlenvec], float)
        out[f"s{k}/density"] = np.asarray(st.density, float)
        out[f"s{k}/denrot"] = np.asarray(st.denrot, float)
    if params is not None:
        for f in dataclasses.fields(params):
            v = getattr(params, f.name)
            out[f"params/{f.name}"] = np.array(v if not isinstance(v, tuple) else list(v))
    np.savez_compressed(path, **out)


def load_thldvec(path: str) -> tuple[list, dict]:
    """Inverse of save_thldvec: (list of ThLenDenType, dict of the saved ParamSet fields)."""
    with np.load(path) as d:
        states = []
        for k in range(int(d["nstates"])):
            th = d[f"s{k}/theta"]
            bodies = [ThetaLenType(th[i].copy(), float(d[f"s{k}/len"][i]), float(d[f"s{k}/xsm"][i]),
                                   float(d[f"s{k}/ysm"][i]), float(d[f"s{k}/matau"][i])) for i in range(len(th))]
            states.append(ThLenDenType(bodies, float(d[f"s{k}/tt"]), d[f"s{k}/density"].copy(),
                                       d[f"s{k}/denrot"].copy()))
        params = {k.split("/", 1)[1]: d[k][()] for k in d.files if k.startswith("params/")}
    return states, params


def new_thlenden(thlenvec) -> ThLenDenType:
    return ThLenDenType(list(thlenvec), 0.0)


def getalpha(npts: int) -> np.ndarray:
    d = 2 * np.pi / npts
    return 0.5 * d + d * np.arange(npts)


def circ2thlen(npts: int, rad: float, xc: float, yc: float) -> ThetaLenType:
    return ThetaLenType(0.5 * np.pi + getalpha(npts), 2 * np.pi * rad, xc, yc)


def circs2thlenden(npts: int, rvec, xc, yc) -> ThLenDenType:
    return new_thlenden([circ2thlen(npts, r, x, y) for r, x, y in zip(rvec, xc, yc)])


def circs2thlenden_file(params: ParamSet, path: str) -> ThLenDenType:
    """circs2thlenden(params) of Main.jl:37-45: the initial state from a JLD2
    circle file (rvec, xc, yc), read with erosion_b200.jld2."""
    from . import jld2
    rvec, xc, yc = jld2.circles(path)
    return circs2thlenden(params.npts, rvec, xc, yc)


def pack_state(thlenden: ThLenDenType):
    tl = thlenden.thlenvec
    th = np.ascontiguousarray(np.concatenate([b.theta for b in tl]), dtype=np.float64)
    ln = np.array([b.len for b in tl], dtype=np.float64)
    xs = np.array([b.xsm for b in tl], dtype=np.float64)
    ys = np.array([b.ysm for b in tl], dtype=np.float64)
    return th, ln, xs, ys


def getnxy(thlenden: ThLenDenType):
    """Node coordinates of every body, computed on the device."""
    M = len(thlenden.thlenvec)
    if M == 0:
        return 0, np.zeros(0), np.zeros(0)
    th, ln, xs, ys = pack_state(thlenden)
    n = len(thlenden.thlenvec[0].theta)
    xx = np.zeros(M * n)
    yy = np.zeros(M * n)
    check(_lib.load().erosion_getxy(n, M, ptr(th), ptr(ln), ptr(xs), ptr(ys), ptr(xx), ptr(yy)))
    return M, xx, yy


def getxy(thlen: ThetaLenType):
    _, xx, yy = getnxy(ThLenDenType([thlen]))
    return xx, yy


def xyrot(xv, yv):
    return -yv, xv


def _geom(nbods, xv, yv, params: ParamSet) -> Geometry:
    return Geometry(params.npts, params.nouter, np.ascontiguousarray(xv, dtype=np.float64),
                    np.ascontiguousarray(yv, dtype=np.float64), tuple(params.wall), params.ibc,
                    np.zeros(nbods), np.zeros((nbods, 2)))


def compute_density(xx, yy, nbods: int, params: ParamSet):
    """DensityStress.jl:43-54 through the drop-in solve."""
    from . import stokes
    g = _geom(nbods, xx, yy, params)
    den, nits, st = stokes.solve(g, **_solve_kw(params))
    return den


def _solve_kw(params: ParamSet) -> dict:
    return dict(tol=params.tol, maxl=params.maxl, ibary=params.ibary, ifmm=params.ifmm, precision=params.precision)


def compute_density_(thlenden: ThLenDenType, params: ParamSet, rotation: bool = False):
    """DensityStress.jl:58-66: solve once per state and cache the result."""
    cached = thlenden.denrot if rotation else thlenden.density
    if len(cached) > 0:
        return
    nbods, xv, yv = getnxy(thlenden)
    if rotation:
        xv, yv = xyrot(xv, yv)
    den = compute_density(xv, yv, nbods, params)
    if rotation:
        thlenden.denrot = den
    else:
        thlenden.density = den


def compute_qoi_targets(xx, yy, density, xtar, ytar, npts, nbods, nouter, ibary, params: ParamSet | None = None):
    from . import stokes
    params = params or ParamSet(npts=npts, nouter=nouter)
    g = _geom(nbods, xx, yy, params)
    return stokes.qoi_targets(g, density, xtar, ytar, ibary=ibary)


def getpdrop(thlenden: ThLenDenType, params: ParamSet, x0: float = 2.0, rotation: bool = False):
    """DensityStress.jl:129-154."""
    nypts = 13
    dy = 2 / nypts
    ylocs = -1 + 0.5 * dy + dy * np.arange(nypts)
    nbods, xv, yv, den = getnxyden(thlenden, params, False, rotation)
    up, _, pp, _ = compute_qoi_targets(xv, yv, den, np.full(nypts, x0), ylocs, params.npts, nbods, params.nouter,
                                       params.ibary, params)
    um, _, pm, _ = compute_qoi_targets(xv, yv, den, np.full(nypts, -x0), ylocs, params.npts, nbods, params.nouter,
                                       params.ibary, params)
    pdrop = np.mean(pm) - np.mean(pp)
    qavg = 0.5 * (np.mean(up) + np.mean(um))
    return pdrop, qavg


def getumax(thlenden, params: ParamSet, fixpdrop: bool, x0: float = 2.0) -> float:
    if not fixpdrop:
        return 1.0
    pdrop = getpdrop(thlenden, params)[0]
    return 4 * x0 / (pdrop + 1e-4)


def getnxyden(thlenden, params: ParamSet, fixpdrop: bool, rotation: bool):
    nbods, xv, yv = getnxy(thlenden)
    rescale = getumax(thlenden, params, fixpdrop)
    if rotation:
        xv, yv = xyrot(xv, yv)
        den = rescale * thlenden.denrot
    else:
        den = rescale * thlenden.density
    return nbods, xv, yv, den


def compute_stress(thlenden, params: ParamSet, fixpdrop: bool = False, rotation: bool = False):
    """DensityStress.jl:191-210; returns an (npts, nbods) array."""
    from . import stokes
    nbods, xv, yv, den = getnxyden(thlenden, params, fixpdrop, rotation)
    if nbods == 0:
        return np.zeros((params.npts, 0))
    g = _geom(nbods, xv, yv, params)
    tau, _ = stokes.shear_stress(g, den, ibary=params.ibary)
    return tau.reshape(nbods, params.npts).T


def rungekutta2(thld0: ThLenDenType, params: ParamSet) -> tuple[ThLenDenType, dict]:
    """One RK2 step (TimeStepping.jl:189-202) executed on the device through
    erosion_rk2_step.  Returns the new state and the step statistics."""
    L = _lib.load()
    M = len(thld0.thlenvec)
    n = params.npts
    th, ln, xs, ys = pack_state(thld0)
    nb = np.array([M], np.int64)
    t = np.array([thld0.tt], np.float64)
    deleted = np.zeros(max(M, 1), np.int64)
    p = params.erosion_params()
    sp = params.step_params()
    rc = L.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sp), n, nb.ctypes.data_as(PI64), params.nouter, ptr(th),
                            ptr(ln), ptr(xs), ptr(ys), ptr(t), deleted.ctypes.data_as(PI64))
    check(rc, (_lib.EROSION_OK, _lib.EROSION_MAXITER))
    st = StepStats()
    L.erosion_get_step_stats(ctypes.byref(st))
    Mn = int(nb[0])
    thl = [ThetaLenType(th[b * n:(b + 1) * n].copy(), float(ln[b]), float(xs[b]), float(ys[b]))
           for b in range(Mn)]
    out = new_thlenden(thl)
    out.tt = float(t[0])
    stats = st.as_dict()
    stats["deleted"] = deleted[:M - Mn].tolist()
    return out, stats


@dataclasses.dataclass
class DragData:
    """PostProcess.jl:126-129."""
    pdragx: float
    pdragy: float
    vdragx: float
    vdragy: float
    umax: float
    tau_all: np.ndarray     # (npts, nbods)
    atau_all: np.ndarray    # (npts, nbods)
    press_all: np.ndarray   # (npts, nbods)


def drag(thlenden: ThLenDenType, params: ParamSet, rotation: bool = False) -> DragData:
    """drag (PostProcess.jl:131-162) through erosion_drag: the pressure and
    viscous drag summed over all bodies (density solved and cached first, as
    compute_stress does), with the unsmoothed shear stress, its smoothed
    absolute value and the pressure on every node (umax = 1 in all of them;
    the reported umax follows params.fixpdrop as getumax does)."""
    compute_density_(thlenden, params, rotation=rotation)
    L = _lib.load()
    M = len(thlenden.thlenvec)
    n = params.npts
    th, ln, xs, ys = pack_state(thlenden)
    den = np.ascontiguousarray(thlenden.denrot if rotation else thlenden.density, dtype=np.float64)
    out = np.zeros(4)
    tau = np.zeros(M * n)
    atau = np.zeros(M * n)
    press = np.zeros(M * n)
    p = params.erosion_params()
    check(L.erosion_drag(ctypes.byref(p), n, M, params.nouter, ptr(th), ptr(ln), ptr(xs), ptr(ys), ptr(den),
                         1 if rotation else 0, params.sigma, ptr(out), None, ptr(tau), ptr(atau), ptr(press)))
    umax = getumax(thlenden, params, params.fixpdrop)
    shape = lambda a: a.reshape(M, n).T
    return DragData(float(out[0]), float(out[1]), float(out[2]), float(out[3]), umax, shape(tau), shape(atau),
                    shape(press))
