"""erosion_matvec_noalloc, the operator form for callers that cannot allocate
GPU memory (for example a solver running inside a runtime that owns all
device memory, or one whose device memory is reserved up front): it must give
what erosion_matvec gives with ibary = 0 and precision = 0 (1e-11 relative,
the operator tolerance of the other parity tests) on consecutive calls that
reuse its fixed scratch array, allocate no device memory, and reject sizes
beyond that array.

This file is collected last on purpose; it passes alone in a fresh process
and after the other tests."""
import ctypes

import numpy as np
import pytest

from erosion_b200 import _lib, geometry as G, stokes

pytestmark = pytest.mark.gpu

MATVEC_RTOL = 1e-11


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def call_noalloc(lib, g, d_xx, d_yy, d_den, d_vel, stream, **kw):
    p = stokes.params_for(g, ibary=0, **kw)
    return lib.erosion_matvec_noalloc(ctypes.byref(p), g.n, g.M, g.nout, d_xx.data_ptr(), d_yy.data_ptr(),
                                      d_den.data_ptr(), d_vel.data_ptr(), stream.cuda_stream)


def device_inputs(torch, g, den):
    dev = torch.device("cuda", 0)
    return (torch.tensor(g.xx, dtype=torch.float64, device=dev), torch.tensor(g.yy, dtype=torch.float64, device=dev),
            torch.tensor(den, dtype=torch.float64, device=dev), torch.full((g.ntot,), np.nan, dtype=torch.float64,
                                                                           device=dev))


def test_noalloc_matches_matvec_on_consecutive_calls(lib):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream()
    cases = [(G.workload("c1", seed=3), 1), (G.workload("ref-small"), 2), (G.workload("c1", seed=3), 3)]
    for g, seed in cases:    # larger, smaller, larger again: stale scratch must not leak into a result
        den = np.random.default_rng(seed).standard_normal(g.ntot)
        want = stokes.matvec(g, den, ibary=0, precision=0)
        d_xx, d_yy, d_den, d_vel = device_inputs(torch, g, den)
        for _ in range(2):
            d_vel.fill_(float("nan"))
            assert call_noalloc(lib, g, d_xx, d_yy, d_den, d_vel, stream) == _lib.EROSION_OK
            torch.cuda.synchronize()
            got = d_vel.cpu().numpy()
            assert np.isfinite(got).all()
            assert rel(got, want) < MATVEC_RTOL


def test_noalloc_allocates_no_device_memory(lib):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream()
    g = G.workload("c1", seed=5)
    den = np.random.default_rng(7).standard_normal(g.ntot)
    d_xx, d_yy, d_den, d_vel = device_inputs(torch, g, den)
    assert call_noalloc(lib, g, d_xx, d_yy, d_den, d_vel, stream) == _lib.EROSION_OK   # per-device set-up
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert call_noalloc(lib, g, d_xx, d_yy, d_den, d_vel, stream) == _lib.EROSION_OK
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_rejects_what_does_not_fit(lib):
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream()
    g = G.workload("c2")            # its arrays serve as buffers; the sizes passed below do not fit
    den = np.zeros(g.ntot)
    d_xx, d_yy, d_den, d_vel = device_inputs(torch, g, den)
    p = stokes.params_for(g, ibary=0)
    too_many_bodies = lib.erosion_matvec_noalloc(ctypes.byref(p), g.n, 129, g.nout, d_xx.data_ptr(),
                                                 d_yy.data_ptr(), d_den.data_ptr(), d_vel.data_ptr(),
                                                 stream.cuda_stream)
    assert too_many_bodies == _lib.EROSION_BAD_INPUT
    assert b"128" in lib.erosion_last_error()
    too_many_nodes = lib.erosion_matvec_noalloc(ctypes.byref(p), 512, 64, 4096, d_xx.data_ptr(), d_yy.data_ptr(),
                                                d_den.data_ptr(), d_vel.data_ptr(), stream.cuda_stream)
    assert too_many_nodes == _lib.EROSION_BAD_INPUT
    assert b"32768" in lib.erosion_last_error()
    p1 = stokes.params_for(g, ibary=1)
    assert lib.erosion_matvec_noalloc(ctypes.byref(p1), g.n, g.M, g.nout, d_xx.data_ptr(), d_yy.data_ptr(),
                                      d_den.data_ptr(), d_vel.data_ptr(), stream.cuda_stream) == _lib.EROSION_BAD_INPUT


def test_noalloc_at_the_largest_channel_size_that_fits(lib):
    """c2 (27,648 nodes) fits the fixed array; the result still matches."""
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream()
    g = G.workload("c2")
    den = np.random.default_rng(11).standard_normal(g.ntot)
    want = stokes.matvec(g, den, ibary=0, precision=0)
    d_xx, d_yy, d_den, d_vel = device_inputs(torch, g, den)
    assert call_noalloc(lib, g, d_xx, d_yy, d_den, d_vel, stream) == _lib.EROSION_OK
    torch.cuda.synchronize()
    assert rel(d_vel.cpu().numpy(), want) < MATVEC_RTOL


def test_noalloc_wall_only_channel(lib):
    """nbods = 0: the wall alone (the body pointers may be null)."""
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream()
    g = G.custom(64, 1024, [], [], wall=G.CHANNEL_WALL, ibc=0)
    den = np.random.default_rng(13).standard_normal(g.ntot)
    want = stokes.matvec(g, den, ibary=0, precision=0)
    d_den = torch.tensor(den, dtype=torch.float64, device="cuda")
    d_vel = torch.full((g.ntot,), float("nan"), dtype=torch.float64, device="cuda")
    p = stokes.params_for(g, ibary=0)
    for _ in range(2):
        rc = lib.erosion_matvec_noalloc(ctypes.byref(p), g.n, 0, g.nout, None, None, d_den.data_ptr(),
                                        d_vel.data_ptr(), stream.cuda_stream)
        assert rc == _lib.EROSION_OK
        torch.cuda.synchronize()
        got = d_vel.cpu().numpy()
        assert np.isfinite(got).all() and rel(got, want) < MATVEC_RTOL


def test_noalloc_at_the_node_limit(lib):
    """The largest accepted layout: nouter = 4096 and npts = 512 with 56 bodies
    (4096 + 56 x 512 = 32,768 nodes), which leaves the least room for the
    split-K partial sums; then a small call again."""
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(17)
    n, nout, M = 512, 4096, 56
    radii, cs = G.pack(M, 0.03, 0.05, G.CHANNEL_WALL, lambda r: 4 * 2 * np.pi * r / n, rng)
    g = G.custom(n, nout, radii, cs, wall=G.CHANNEL_WALL, ibc=0)
    assert g.N == 32768
    small = G.workload("ref-small")
    for geo, seed in ((g, 19), (small, 23), (g, 29)):
        den = np.random.default_rng(seed).standard_normal(geo.ntot)
        want = stokes.matvec(geo, den, ibary=0, precision=0)
        d_xx, d_yy, d_den, d_vel = device_inputs(torch, geo, den)
        assert call_noalloc(lib, geo, d_xx, d_yy, d_den, d_vel, stream) == _lib.EROSION_OK
        torch.cuda.synchronize()
        got = d_vel.cpu().numpy()
        assert np.isfinite(got).all() and rel(got, want) < MATVEC_RTOL
