"""TEST INFRASTRUCTURE ONLY — CPU restatement (numpy FFT) of the reference's
theta-L time stepping, the oracle for the library's device-side RK2 step.

Follows ErosionPackage/src/SpectralMethods.jl:10-67 (fftshift conventions,
kvec with the highest mode zeroed or kept), ThetaLen.jl:92-116 (getxy,
getalpha), TimeStepping.jl:42-202 (tangvel, getderivs, delete_indices,
timestep!, rungekutta2) and DensityStress.jl:23-36 (getstress!), with the
solve and the shear stress taken from the C++ oracle.
"""
from __future__ import annotations

import dataclasses

import numpy as np


# --- SpectralMethods.jl ----------------------------------------------------
def kvec(nn: int, hmode: int = 0) -> np.ndarray:
    if nn % 2 == 0:
        nsm = nn // 2 - 1
        return np.r_[hmode * (nsm + 1), np.arange(-nsm, nsm + 1)].astype(float)
    nsm = (nn - 1) // 2
    return np.arange(-nsm, nsm + 1).astype(float)


def fftnice(fx):
    return np.fft.fftshift(np.fft.fft(fx))


def ifftnice(fh):
    return np.fft.ifft(np.fft.ifftshift(fh))


def specdiff(fx, intvlen=2 * np.pi):
    fh = fftnice(fx)
    kv = kvec(len(fx), 0)
    return np.real(ifftnice(2 * np.pi * 1j * kv * fh)) / intvlen


def specint(fx, intvlen=2 * np.pi):
    fh = fftnice(fx)
    kv = kvec(len(fx), 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        Fh = fh / (2 * np.pi * 1j * kv)
    Fh[kv == 0] = 0.0
    return np.real(ifftnice(Fh)) * intvlen


def expsmooth(fx, factor):
    fh = fftnice(fx)
    kv = kvec(len(fx), 1)
    fh = fh * np.exp(-factor * np.abs(kv) ** 2)
    return np.real(ifftnice(fh))


def gaussfilter(fx, sigma):
    return expsmooth(fx, 0.5 * sigma ** 2)


# --- ThetaLen.jl -------------------------------------------------------------
def getalpha(npts):
    d = 2 * np.pi / npts
    return 0.5 * d + d * np.arange(npts)


@dataclasses.dataclass
class Body:
    theta: np.ndarray
    len: float
    xsm: float
    ysm: float
    matau: float = np.nan


def getxy(b: Body):
    assert b.len > 0
    dx = b.len / (2 * np.pi) * (np.cos(b.theta) - np.mean(np.cos(b.theta)))
    dy = b.len / (2 * np.pi) * (np.sin(b.theta) - np.mean(np.sin(b.theta)))
    return specint(dx) + b.xsm, specint(dy) + b.ysm


def circ2thlen(npts, rad, xc, yc):
    return Body(0.5 * np.pi + getalpha(npts), 2 * np.pi * rad, xc, yc)


# --- TimeStepping.jl ------------------------------------------------------------
def tangvel(dtheta, vnorm):
    dthvn = dtheta * vnorm
    mdthvn = np.mean(dthvn)
    mterm = -2 * np.pi * mdthvn
    vtang = specint(dthvn - mdthvn)
    return vtang, mterm


def getderivs_body(b: Body, epsilon, fixarea, atau):
    ataueff = atau - fixarea * b.matau
    alpha = getalpha(len(b.theta))
    dtheta = specdiff(b.theta - alpha) + 1.0
    vnorm = ataueff + epsilon * b.matau * (dtheta - 1.0)
    vtang, mterm = tangvel(dtheta, vnorm)
    datau = specdiff(atau)
    nterm = 2 * np.pi / b.len * (datau + dtheta * vtang)
    xsmdot = np.mean(-vnorm * np.sin(b.theta) + vtang * np.cos(b.theta))
    ysmdot = np.mean(vnorm * np.cos(b.theta) + vtang * np.sin(b.theta))
    return mterm, nterm, xsmdot, ysmdot


class ThetaLenOracle:
    """rungekutta2 with getstress! from the C++ oracle (solve to `tol`)."""

    def __init__(self, oracle, nout, wall, ibc, epsilon, sigma, dt, fixarea=0, tol=1e-8, ibary=1, ifmm=1,
                 fixpdrop=False):
        self.o = oracle
        self.fixpdrop = fixpdrop
        self.nout, self.wall, self.ibc = nout, wall, ibc
        self.eps, self.sigma, self.dt, self.fixarea = epsilon, sigma, dt, fixarea
        self.tol, self.ibary, self.ifmm = tol, ibary, ifmm
        self.iterations = []

    def _geom(self, bodies):
        from erosion_b200.geometry import Geometry
        xs, ys = zip(*[getxy(b) for b in bodies])
        n = len(bodies[0].theta)
        return Geometry(n, self.nout, np.ascontiguousarray(np.concatenate(xs)),
                        np.ascontiguousarray(np.concatenate(ys)), self.wall, self.ibc,
                        np.zeros(len(bodies)), np.zeros((len(bodies), 2)))

    def getstress(self, bodies):
        g = self._geom(bodies)
        den, nits, ierr, err = self.o.solve(g, ibary=self.ibary, ifmm=self.ifmm, tol=self.tol)
        self.iterations.append(nits)
        if self.fixpdrop:   # getumax/getpdrop, DensityStress.jl:129-167
            nypts = 13
            dy = 2 / nypts
            ylocs = -1 + 0.5 * dy + dy * np.arange(nypts)
            pp = self.o.qoi_targets(g, den, np.full(nypts, 2.0), ylocs, ibary=self.ibary)[2]
            pm = self.o.qoi_targets(g, den, np.full(nypts, -2.0), ylocs, ibary=self.ibary)[2]
            pdrop = np.mean(pm) - np.mean(pp)
            den = den * (4 * 2.0 / (pdrop + 1e-4))
        tau, _ = self.o.shear_stress(g, den, ibary=self.ibary)
        stress = tau.reshape(len(bodies), -1)
        out = []
        for i, b in enumerate(bodies):
            a = gaussfilter(np.abs(stress[i]), self.sigma)
            b.matau = float(np.mean(a))
            out.append(a)
        return out

    def timestep(self, thld0, thld_d, dt1, dt2):
        atau = self.getstress(thld_d)
        dvec = [getderivs_body(b, self.eps, self.fixarea, a) for b, a in zip(thld_d, atau)]
        keep = []
        for i, (b, d) in enumerate(zip(thld0, dvec)):
            minlen = -np.sqrt(2) * d[0] * 1.0 * dt1
            if not (b.len <= minlen or d[0] > 10.0):
                keep.append(i)
        thld0[:] = [thld0[i] for i in keep]
        dvec = [dvec[i] for i in keep]
        if thld_d is not thld0:
            thld_d[:] = [thld_d[i] for i in keep]
        alpha = getalpha(len(thld0[0].theta)) if thld0 else None
        out = []
        for b0, bd, (mterm, nterm, xsd, ysd) in zip(thld0, thld_d, dvec):
            len1 = b0.len + dt1 * mterm
            assert len1 > 0
            zeta0 = 2 * np.pi / b0.len * b0.matau
            zetad = 2 * np.pi / bd.len * bd.matau
            fac1 = self.eps * dt1 * zetad
            fac2 = self.eps * dt2 * (2 * zetad - zeta0)
            th1 = expsmooth(b0.theta - alpha, fac1) + alpha
            th1 = th1 + dt1 * expsmooth(nterm, fac2)
            out.append(Body(th1, len1, b0.xsm + dt1 * xsd, b0.ysm + dt1 * ysd))
        return out

    def rungekutta2(self, thld0):
        dt = self.dt
        thld05 = self.timestep(thld0, thld0, 0.5 * dt, 0.5 * dt)
        thld1 = self.timestep(thld0, thld05, dt, 0.5 * dt)
        return thld1


# --- PostProcess.jl: getns, drag ------------------------------------------------
def getns(theta, rotation=False):
    """PostProcess.jl:23-33: CCW tangent (rotated for the rotated flow) and the
    inward normal."""
    if not rotation:
        sx, sy = np.cos(theta), np.sin(theta)
    else:
        sx, sy = -np.sin(theta), np.cos(theta)
    return sx, sy, -sy, sx


def drag(oracle, bodies, den, nout, wall, ibc, sigma, rotation=False):
    """drag (PostProcess.jl:131-162) for a solved density of the state
    `bodies` (of the rotated problem when rotation): the shear stress and the
    pressure on every node from the C++ oracle (computeShearStress,
    computePressure semantics, umax = 1), per body
    pdrag = sum p n ds, vdrag = sum tau s ds with ds = L/npts, summed in body
    order.  Returns (pdragx, pdragy, vdragx, vdragy), tau_all, atau_all,
    press_all (arrays (npts, nbods))."""
    from erosion_b200.geometry import Geometry
    xs, ys = zip(*[getxy(b) for b in bodies])
    xv, yv = np.concatenate(xs), np.concatenate(ys)
    if rotation:   # xyrot, DensityStress.jl:40
        xv, yv = -yv, xv
    n, M = len(bodies[0].theta), len(bodies)
    g = Geometry(n, nout, np.ascontiguousarray(xv), np.ascontiguousarray(yv), wall, ibc, np.zeros(M),
                 np.zeros((M, 2)))
    tau, _ = oracle.shear_stress(g, den)
    press = oracle.pressure(g, den)
    tau = tau.reshape(M, n)
    press = press.reshape(M, n)
    pdx = pdy = vdx = vdy = 0.0
    atau = np.zeros((M, n))
    for b in range(M):
        atau[b] = gaussfilter(np.abs(tau[b]), sigma)
        sx, sy, nx, ny = getns(bodies[b].theta, rotation)
        ds = bodies[b].len / n
        pdx += np.dot(press[b], nx) * ds
        pdy += np.dot(press[b], ny) * ds
        vdx += np.dot(tau[b], sx) * ds
        vdy += np.dot(tau[b], sy) * ds
    return (pdx, pdy, vdx, vdy), tau.T, atau.T, press.T
