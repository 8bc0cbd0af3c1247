"""ctypes binding of oracle/stokes_oracle.cpp (test infrastructure only)."""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_int, c_int64

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle_stokes.so")
PD = POINTER(c_double)
PI64 = POINTER(c_int64)


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "stokes_oracle.cpp")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        env = dict(os.environ)
        env.pop("CXX", None)
        subprocess.run(["make", "-s", "-C", HERE, "-B" if force else "all"], check=True, env=env)
    return LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(PD)


def _wall(wall):
    return None if wall is None else np.ascontiguousarray(wall, dtype=np.float64)


class Oracle:
    """Thin wrapper with numpy in/out."""

    def __init__(self):
        build_oracle()
        L = ctypes.CDLL(LIB)
        L.oracle_stokessolver.restype = c_int64
        L.oracle_stokessolver.argtypes = [c_int64] * 7 + [PD, PD, PD, PI64, c_double, PD, c_int64, PD]
        L.oracle_matvec.argtypes = [c_int64] * 4 + [PD, PD, PD, PD, PD]
        L.oracle_far_field.argtypes = [c_int64] * 3 + [PD, PD, PD, PD, PD]
        L.oracle_rhs.argtypes = [c_int64] * 5 + [PD, PD, PD, PD]
        L.oracle_geometry.argtypes = [c_int64] * 3 + [PD] * 15
        L.oracle_shear_stress.argtypes = [c_int64] * 3 + [PD, PD, PD, c_int64, PD, PD, PD]
        L.oracle_shear_stress_bodies.argtypes = [c_int64] * 3 + [PD, PD, PD, c_int64, PD, ctypes.c_void_p, PD, PD]
        L.oracle_qoi_targets.argtypes = [c_int64] * 4 + [PD, PD, PD, c_int64, PD, PD, PD, PD, PD, PD, PD]
        L.oracle_pressure.argtypes = [c_int64] * 3 + [PD, PD, PD, PD, PD]
        L.oracle_near_wall.restype = c_int64
        L.oracle_near_wall.argtypes = [c_int64] * 3 + [PD, PD, PD, PI64, PI64]
        L.oracle_stokes_dlp.argtypes = [c_int64, c_int64, PD, PD, PD, PD, PD, PD, c_int64, PD, PD, c_int64, PD]
        L.oracle_bdval.argtypes = [c_int64, c_int64, PD, PD, PD, PD, PD, PD]
        L.oracle_fourier_diff.argtypes = [c_int64, PD, PD]
        L.oracle_num_threads.restype = c_int
        L.oracle_set_threads.argtypes = [c_int]
        self.L = L

    def threads(self, n: int | None = None) -> int:
        if n:
            self.L.oracle_set_threads(int(n))
        return self.L.oracle_num_threads()

    def solve(self, g, ibary=1, ifmm=1, maxl=8000, tol=1e-8, rhs_mode=0, x0=None, ibc=None):
        den = np.zeros(g.ntot) if x0 is None else np.array(x0, dtype=np.float64)
        nits = np.zeros(1, np.int64)
        err = np.zeros(1)
        ibc = g.ibc if ibc is None else ibc
        ierr = self.L.oracle_stokessolver(g.n, g.M, g.nout, ifmm, ibary, ibc, maxl, _p(g.xx), _p(g.yy), _p(den),
                                          nits.ctypes.data_as(PI64), tol, _p(_wall(g.wall)), rhs_mode, _p(err))
        return den, int(nits[0]), int(ierr), float(err[0])

    def matvec(self, g, den, mode=1):
        vel = np.zeros(g.ntot)
        den = np.ascontiguousarray(den, dtype=np.float64)
        self.L.oracle_matvec(g.n, g.M, g.nout, mode, _p(g.xx), _p(g.yy), _p(_wall(g.wall)), _p(den), _p(vel))
        return vel

    def far_field(self, g, den):
        vel = np.zeros(g.ntot)
        den = np.ascontiguousarray(den, dtype=np.float64)
        self.L.oracle_far_field(g.n, g.M, g.nout, _p(g.xx), _p(g.yy), _p(_wall(g.wall)), _p(den), _p(vel))
        return vel

    def rhs(self, g, rhs_mode=0, ibc=None):
        out = np.zeros(g.ntot)
        ibc = g.ibc if ibc is None else ibc
        self.L.oracle_rhs(g.n, g.M, g.nout, ibc, rhs_mode, _p(g.xx), _p(g.yy), _p(_wall(g.wall)), _p(out))
        return out

    def geometry(self, g):
        nb, M, no = g.n * g.M, g.M, g.nout
        a = {k: np.zeros(nb) for k in ("px", "py", "cur", "speed")}
        a.update({k: np.zeros(M) for k in ("cx", "cy")})
        a.update({k: np.zeros(no) for k in ("xo", "yo", "px0", "py0", "cur0", "speed0")})
        self.L.oracle_geometry(g.n, g.M, g.nout, _p(g.xx), _p(g.yy), _p(_wall(g.wall)),
                               *[_p(a[k]) for k in ("px", "py", "cur", "speed", "cx", "cy", "xo", "yo",
                                                    "px0", "py0", "cur0", "speed0")])
        return a

    def shear_stress(self, g, den, ibary=1, bodies=None):
        """(tau, E) on every body, or, with bodies (indices), on those target
        bodies only (from every source curve; the other entries are zero)."""
        tau = np.zeros(g.n * g.M)
        E = np.zeros(3 * g.n * g.M)
        den = np.ascontiguousarray(den, dtype=np.float64)
        if bodies is None:
            self.L.oracle_shear_stress(g.n, g.M, g.nout, _p(g.xx), _p(g.yy), _p(den), ibary, _p(_wall(g.wall)),
                                       _p(tau), _p(E))
        else:
            sel = np.zeros(max(g.M, 1), np.uint8)
            sel[np.asarray(bodies, int)] = 1
            self.L.oracle_shear_stress_bodies(g.n, g.M, g.nout, _p(g.xx), _p(g.yy), _p(den), ibary,
                                              _p(_wall(g.wall)), sel.ctypes.data_as(ctypes.c_void_p), _p(tau),
                                              _p(E))
        return tau, E.reshape(3, -1)

    def qoi_targets(self, g, den, xt, yt, ibary=1):
        xt = np.ascontiguousarray(xt, dtype=np.float64)
        yt = np.ascontiguousarray(yt, dtype=np.float64)
        out = [np.zeros(len(xt)) for _ in range(4)]
        den = np.ascontiguousarray(den, dtype=np.float64)
        self.L.oracle_qoi_targets(g.n, g.M, g.nout, ibary, _p(g.xx), _p(g.yy), _p(den), len(xt), _p(xt), _p(yt),
                                  _p(_wall(g.wall)), *[_p(o) for o in out])
        return out

    def pressure(self, g, den):
        p = np.zeros(g.n * g.M)
        den = np.ascontiguousarray(den, dtype=np.float64)
        self.L.oracle_pressure(g.n, g.M, g.nout, _p(g.xx), _p(g.yy), _p(den), _p(_wall(g.wall)), _p(p))
        return p

    def near_wall(self, g):
        lw = np.zeros(1, np.int64)
        wb = np.zeros(max(g.M, 1), np.int64)
        k = self.L.oracle_near_wall(g.n, g.M, g.nout, _p(g.xx), _p(g.yy), _p(_wall(g.wall)),
                                    lw.ctypes.data_as(PI64), wb.ctypes.data_as(PI64))
        return int(lw[0]), wb[:k].tolist()

    def stokes_dlp(self, exterior, xs, ys, dx, dy, nx, ny, xt, yt, nder=1):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (xs, ys, dx, dy, nx, ny, xt, yt)]
        out = np.zeros(6 * len(xt))
        self.L.oracle_stokes_dlp(int(exterior), len(xs), *[_p(a) for a in arrs[:6]], len(xt), _p(arrs[6]),
                                 _p(arrs[7]), nder, _p(out))
        return out.reshape(6, -1)

    def bdval(self, exterior, xs, ys, f):
        f = np.asarray(f, dtype=np.complex128)
        xs = np.ascontiguousarray(xs, dtype=np.float64)
        ys = np.ascontiguousarray(ys, dtype=np.float64)
        fr, fi = np.ascontiguousarray(f.real), np.ascontiguousarray(f.imag)
        br, bi = np.zeros(len(xs)), np.zeros(len(xs))
        self.L.oracle_bdval(int(exterior), len(xs), _p(xs), _p(ys), _p(fr), _p(fi), _p(br), _p(bi))
        return br + 1j * bi

    def fourier_diff(self, f):
        f = np.asarray(f, dtype=np.complex128)
        re, im = np.ascontiguousarray(f.real), np.ascontiguousarray(f.imag)
        self.L.oracle_fourier_diff(len(f), _p(re), _p(im))
        return re + 1j * im
