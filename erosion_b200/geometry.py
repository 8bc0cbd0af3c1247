"""Seeded synthetic porous-channel geometries.

The reference reads circle packings (``rvec, xc, yc``) from JLD2 files
(ErosionPackage/src/Main.jl:37-45) and converts each circle to theta-L form
with ``circ2thlen`` (Main.jl:30-35): theta = pi/2 + alpha on the offset grid
alpha_j = (j + 1/2) 2 pi/n (ThetaLen.jl:113-116), L = 2 pi r.  Its node
coordinates then come from ``getxy`` (ThetaLen.jl:92-101).  This module
generates packings of the workload shapes with a seeded rejection sampler and
returns the same node layout the solver expects: body-major, node-minor,
counter-clockwise, equal arclength, starting at alpha_0 = pi/n.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

REFERENCE_WALL = (3.0, 1.0, 8.0)    # stokesSolver.f:184-191
CHANNEL_WALL = (1.0, 0.5, 8.0)      # [-1,1] x [-0.5,0.5] smoothed rectangle


@dataclasses.dataclass
class Geometry:
    n: int
    nout: int
    xx: np.ndarray          # (M*n,) body-major
    yy: np.ndarray
    wall: tuple             # (a, b, order)
    ibc: int
    radii: np.ndarray
    centers: np.ndarray     # (M, 2)

    @property
    def M(self) -> int:
        return len(self.radii)

    @property
    def ntot(self) -> int:
        return 2 * self.nout + 2 * self.n * self.M + 3 * self.M

    @property
    def N(self) -> int:
        return self.nout + self.n * self.M


def getalpha(n: int) -> np.ndarray:
    """ThetaLen.jl:113-116: alpha = 2 pi s/L on the offset grid."""
    d = 2 * np.pi / n
    return 0.5 * d + d * np.arange(n)


def circle_nodes(n: int, r: float, xc: float, yc: float) -> tuple[np.ndarray, np.ndarray]:
    """Nodes of circ2thlen + getxy for a circle: x = xc + r cos(alpha), y = yc + r sin(alpha)."""
    a = getalpha(n)
    return xc + r * np.cos(a), yc + r * np.sin(a)


def perturbed_nodes(n: int, r0: float, xc: float, yc: float, rng: np.random.Generator,
                    modes=(2, 8), amp: float = 0.02, dense: int = 16) -> tuple[np.ndarray, np.ndarray]:
    """A circle of radius r0 with a random Fourier perturbation of modes
    modes[0]..modes[1], scaled so that max |r(phi)/r0 - 1| = amp, resampled at
    n nodes equally spaced in arclength (the theta-L parametrisation)."""
    ks = np.arange(modes[0], modes[1] + 1)
    a = rng.uniform(-1, 1, len(ks))
    b = rng.uniform(-1, 1, len(ks))
    m = n * dense
    phi = 2 * np.pi * np.arange(m) / m
    pert = (a[:, None] * np.cos(ks[:, None] * phi) + b[:, None] * np.sin(ks[:, None] * phi)).sum(0)
    pert *= amp / np.abs(pert).max()
    r = r0 * (1 + pert)
    x = r * np.cos(phi)
    y = r * np.sin(phi)
    seg = np.hypot(np.diff(np.r_[x, x[0]]), np.diff(np.r_[y, y[0]]))
    s = np.r_[0.0, np.cumsum(seg)]
    L = s[-1]
    st = L * getalpha(n) / (2 * np.pi)
    xs = np.interp(st, s, np.r_[x, x[0]])
    ys = np.interp(st, s, np.r_[y, y[0]])
    return xc + xs, yc + ys


def _inside_wall(px, py, wall) -> np.ndarray:
    a, b, p = wall
    return (np.abs(px) / a) ** p + (np.abs(py) / b) ** p < 1.0


def pack(M: int, rmin: float, rmax: float, wall, gap_fn, rng: np.random.Generator,
         max_tries: int = 400000) -> tuple[np.ndarray, np.ndarray]:
    """Seeded random sequential placement of M discs inside the wall with
    clearance gap_fn(r) to the wall and gap_fn(r_i) + gap_fn(r_j) between
    discs (sampled from the superellipse's bounding box)."""
    a, b, _ = wall
    radii = rng.uniform(rmin, rmax, M)
    radii = np.sort(radii)[::-1]           # large first packs more reliably
    cs = np.zeros((M, 2))
    ring = np.linspace(0, 2 * np.pi, 64, endpoint=False)
    placed = 0
    tries = 0
    while placed < M:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could not place {M} bodies (placed {placed})")
        r = radii[placed]
        g = gap_fn(r)
        c = np.array([rng.uniform(-a, a), rng.uniform(-b, b)])
        R = r + g
        if not _inside_wall(c[0] + R * np.cos(ring), c[1] + R * np.sin(ring), wall).all():
            continue
        if placed:
            d = np.hypot(cs[:placed, 0] - c[0], cs[:placed, 1] - c[1])
            need = radii[:placed] + r + np.array([gap_fn(q) for q in radii[:placed]]) * 0.5 + g * 0.5
            if (d < need).any():
                continue
        cs[placed] = c
        placed += 1
    return radii, cs


def make_bodies(n: int, radii, centers, rng=None, perturb: bool = False):
    xs, ys = [], []
    for r, (cx, cy) in zip(radii, centers):
        if perturb:
            x, y = perturbed_nodes(n, r, cx, cy, rng)
        else:
            x, y = circle_nodes(n, r, cx, cy)
        xs.append(x)
        ys.append(y)
    if not xs:
        return np.zeros(0), np.zeros(0)
    return np.ascontiguousarray(np.concatenate(xs)), np.ascontiguousarray(np.concatenate(ys))


def workload(name: str, seed: int = 0) -> Geometry:
    """The named workloads:

    * ``c1``: 10 circles, r ~ U[0.05, 0.12], gap >= 0.02, 128 nodes each,
      1024 wall nodes, channel [-1,1]x[-0.5,0.5], parabolic wall data.
    * ``c2``: 100 bodies, r ~ U[0.03, 0.06] plus a Fourier perturbation of
      modes 2-8 with amplitude 2% of r, gap >= 4 h, 256 nodes each, 2048 wall
      nodes.
    * ``c3``: 400 bodies, r ~ U[0.015, 0.03], gap >= 4 h, 256 nodes, 4096
      wall nodes.
    * ``c5``: 200 bodies in the c3 style with 4096 wall nodes.
    * ``ref-small``: 3 circles in the reference's 3 x 1 wall, one of them
      near the wall, two close to each other (exercises every near rule).
    """
    rng = np.random.default_rng(seed)
    if name == "c1":
        n, nout, M, wall = 128, 1024, 10, CHANNEL_WALL
        radii, cs = pack(M, 0.05, 0.12, wall, lambda r: 0.02, rng)
        xx, yy = make_bodies(n, radii, cs)
        return Geometry(n, nout, xx, yy, wall, 0, radii, cs)
    if name in ("c2", "c3", "c5"):
        if name == "c2":
            n, nout, M, rlo, rhi, pert = 256, 2048, 100, 0.03, 0.06, True
        elif name == "c3":
            n, nout, M, rlo, rhi, pert = 256, 4096, 400, 0.015, 0.03, False
        else:
            n, nout, M, rlo, rhi, pert = 256, 4096, 200, 0.015, 0.03, False
        wall = CHANNEL_WALL
        h = lambda r: 2 * np.pi * r * (1.02 if pert else 1.0) / n
        radii, cs = pack(M, rlo, rhi, wall, lambda r: 4 * h(r), rng)
        xx, yy = make_bodies(n, radii, cs, rng, perturb=pert)
        return Geometry(n, nout, xx, yy, wall, 0, radii, cs)
    if name == "ref-small":
        n, nout = 64, 256
        radii = np.array([0.3, 0.25, 0.2])
        cs = np.array([[-1.0, 0.1], [-0.35, 0.0], [0.6, 0.72]])
        xx, yy = make_bodies(n, radii, cs)
        return Geometry(n, nout, xx, yy, REFERENCE_WALL, 1, radii, cs)
    raise KeyError(name)


def superellipse_area(wall) -> float:
    a, b, p = wall
    return 4 * a * b * math.gamma(1 + 1 / p) ** 2 / math.gamma(1 + 2 / p)


def lattice_pack(M: int, n: int, porosity: float, wall, rng: np.random.Generator, spread: float = 0.15):
    """M discs whose total area leaves the given porosity inside the wall,
    with clearance 4 h (h = node spacing 2 pi r / n) between discs and to the
    wall: radii r_i = rbar (1 + U[-spread, spread]) scaled to the area, centres
    on random sites of a hexagonal lattice of spacing 2 r_max + 4 h(r_max),
    jittered within the slack.  The porosity rises (radii shrink) until the
    lattice has M admissible sites."""
    area = superellipse_area(wall)
    rel = 1 + rng.uniform(-spread, spread, M)
    a, b, _ = wall
    ring = np.linspace(0, 2 * np.pi, 64, endpoint=False)
    phi = porosity
    for _ in range(200):
        scale = math.sqrt((1 - phi) * area / (math.pi * (rel ** 2).sum()))
        radii = scale * rel
        rmax = radii.max()
        gap = 4 * 2 * math.pi * rmax / n
        d = 2 * rmax + gap * 1.05
        xs = np.arange(-a, a + d, d)
        ys = np.arange(-b, b + d, d * math.sqrt(3) / 2)
        sites = [(x + (0.5 * d if j % 2 else 0.0), y) for j, y in enumerate(ys) for x in xs]
        R = rmax + gap
        ok = [(x, y) for x, y in sites if _inside_wall(x + R * np.cos(ring), y + R * np.sin(ring), wall).all()]
        if len(ok) >= M:
            pick = rng.choice(len(ok), M, replace=False)
            cs = np.array([ok[i] for i in pick])
            slack = 0.5 * (d - 2 * rmax - gap)
            cs = cs + rng.uniform(-slack, slack, cs.shape) * 0.5
            return radii, cs, phi
        phi = min(0.98, phi + 0.01)
    raise RuntimeError(f"could not place {M} bodies")


def ensemble(count: int, seed: int = 0, bodies=(20, 200), npts=(128, 256, 512), porosity=(0.5, 0.8),
             nout: int = 2048, wall=CHANNEL_WALL):
    """An ensemble of independent channel geometries with uneven sizes: body
    count U{bodies}, nodes per body drawn from npts, porosity U[porosity]
    (radii scaled to it, lattice_pack), parabolic wall data.  The default is
    the 64-geometry batching workload when count = 64."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        M = int(rng.integers(bodies[0], bodies[1] + 1))
        n = int(rng.choice(npts))
        phi = float(rng.uniform(*porosity))
        radii, cs, _ = lattice_pack(M, n, phi, wall, rng)
        xx, yy = make_bodies(n, radii, cs)
        out.append(Geometry(n, nout, xx, yy, tuple(wall), 0, radii, cs))
    return out


_INPUT_GEOS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                           "input_geos.npz")


def reference_inputs() -> list[str]:
    """Names of the reference's simulation input geometries (``01-3`` ...
    ``80-9``: body count and seed), extracted from its JLD2 files."""
    with np.load(_INPUT_GEOS) as d:
        return sorted({k.split("/")[0] for k in d.files})


def reference_input(name: str, npts: int = 128, nouter: int = 1024) -> Geometry:
    """One of the reference's input circle packings as circs2thlenden builds it
    (Main.jl:37-45 with the ParamSet defaults npts = 128, nouter = 1024, the
    3 x 1 wall and uniform wall data), from the extracted fixture
    (tests/golden/make_input_geos.py); erosion_b200.jld2.circles reads the
    original files directly."""
    with np.load(_INPUT_GEOS) as d:
        r, xc, yc = d[f"{name}/rvec"], d[f"{name}/xc"], d[f"{name}/yc"]
    cs = np.stack([xc, yc], 1)
    xx, yy = make_bodies(npts, r, cs)
    return Geometry(npts, nouter, xx, yy, REFERENCE_WALL, 1, np.asarray(r, float), cs)


def custom(n: int, nout: int, radii, centers, wall=REFERENCE_WALL, ibc: int = 1) -> Geometry:
    radii = np.asarray(radii, float)
    centers = np.asarray(centers, float).reshape(-1, 2)
    xx, yy = make_bodies(n, radii, centers)
    return Geometry(n, nout, xx, yy, tuple(wall), ibc, radii, centers)


def to_thetalen(g: Geometry):
    """theta-L state (theta [M*n], L [M], xsm [M], ysm [M]) of body-major nodes
    sampled at equal arclength on the offset grid: theta is the tangent angle
    (unwrapped, theta - alpha periodic), L the perimeter, (xsm, ysm) the
    surface mean (ThetaLen.jl:42-51)."""
    n, M = g.n, g.M
    x = g.xx.reshape(M, n)
    y = g.yy.reshape(M, n)
    k = np.fft.fftfreq(n, 1.0 / n)
    k[n // 2] = 0.0
    dx = np.real(np.fft.ifft(1j * k * np.fft.fft(x, axis=1), axis=1))
    dy = np.real(np.fft.ifft(1j * k * np.fft.fft(y, axis=1), axis=1))
    th = np.unwrap(np.arctan2(dy, dx), axis=1)
    L = np.mean(np.hypot(dx, dy), axis=1) * 2 * np.pi
    return (np.ascontiguousarray(th.reshape(-1)), np.ascontiguousarray(L), np.ascontiguousarray(x.mean(1)),
            np.ascontiguousarray(y.mean(1)))
