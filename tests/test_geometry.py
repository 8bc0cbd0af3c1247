"""The seeded synthetic geometries (CPU): every body node strictly inside the
wall, the configured clearances between bodies and to the wall, the
configured sizes, and determinism in the seed."""
import os

import numpy as np
import pytest

from erosion_b200 import geometry as G


def min_gap(g):
    """Smallest node-to-node distance between different bodies, and from any
    body node to the wall's superellipse level set (measured radially)."""
    n, M = g.n, g.M
    x = g.xx.reshape(M, n)
    y = g.yy.reshape(M, n)
    gap = np.inf
    for i in range(M):
        for j in range(i + 1, M):
            if np.hypot(*(g.centers[i] - g.centers[j])) > 3 * (g.radii[i] + g.radii[j]) + 0.1:
                continue
            d = np.hypot(x[i][:, None] - x[j][None, :], y[i][:, None] - y[j][None, :]).min()
            gap = min(gap, d)
    return gap


def inside(g):
    a, b, p = g.wall
    return ((np.abs(g.xx) / a) ** p + (np.abs(g.yy) / b) ** p < 1).all()


@pytest.mark.parametrize("name,M,n,nout", [("c1", 10, 128, 1024), ("c2", 100, 256, 2048)])
def test_workloads(name, M, n, nout):
    g = G.workload(name)
    assert (g.M, g.n, g.nout) == (M, n, nout)
    assert inside(g)
    h = 2 * np.pi * g.radii.max() / n
    assert min_gap(g) > (0.02 if name == "c1" else 2 * h)
    g2 = G.workload(name)
    assert np.array_equal(g.xx, g2.xx)


def test_ensemble_shapes_and_clearance():
    E = G.ensemble(6, seed=5)
    assert len(E) == 6
    for g in E:
        assert 20 <= g.M <= 200 and g.n in (128, 256, 512) and g.nout == 2048
        assert inside(g)
        h = 2 * np.pi * g.radii.max() / g.n
        assert min_gap(g) > 2 * h
        solid = np.pi * (g.radii ** 2).sum() / G.superellipse_area(g.wall)
        assert 0.02 <= solid <= 0.5 + 1e-9


def test_lattice_pack_reaches_target_porosity():
    rng = np.random.default_rng(0)
    radii, cs, phi = G.lattice_pack(60, 256, 0.6, G.CHANNEL_WALL, rng)
    assert phi == pytest.approx(0.6)
    assert np.pi * (radii ** 2).sum() / G.superellipse_area(G.CHANNEL_WALL) == pytest.approx(0.4, rel=1e-9)


def test_reference_input_geometries_load():
    names = G.reference_inputs()
    assert len(names) == 31 and "02-8" in names and "100-3" in names
    for name in names:
        g = G.reference_input(name)
        assert g.M == int(name.split("-")[0])
        assert (g.n, g.nout, g.wall) == (128, 1024, G.REFERENCE_WALL)
        assert inside(g)


@pytest.mark.skipif(not os.path.isdir("/root/reference/simulations/input_geos"),
                    reason="the reference repository is not checked out here")
def test_jld2_reader_matches_fixture():
    from erosion_b200 import jld2
    for name in ("01-3", "20-11", "100-9"):
        r, xc, yc = jld2.circles(f"/root/reference/simulations/input_geos/{name}.jld2")
        g = G.reference_input(name)
        assert np.array_equal(r, g.radii) and np.array_equal(xc, g.centers[:, 0])


def test_state_file_round_trip(tmp_path):
    from erosion_b200 import thetalen as TL
    params = TL.ParamSet(npts=64, nouter=256)
    st = TL.circs2thlenden(64, [0.3, 0.2], [-1.0, 0.5], [0.1, -0.2])
    st.tt = 0.25
    st.density = np.arange(5.0)
    st.thlenvec[0].matau = 1.5
    path = tmp_path / "run.npz"
    TL.save_thldvec(str(path), [st, TL.circs2thlenden(64, [0.25], [0.0], [0.0])], params)
    back, p = TL.load_thldvec(str(path))
    assert len(back) == 2 and back[0].tt == 0.25
    assert np.array_equal(back[0].thlenvec[1].theta, st.thlenvec[1].theta)
    assert back[0].thlenvec[0].matau == 1.5 and np.array_equal(back[0].density, st.density)
    assert int(p["npts"]) == 64 and tuple(p["wall"]) == G.REFERENCE_WALL
