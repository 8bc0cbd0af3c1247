"""Far-field launch shapes: every candidate the autotuner may pick computes
the same operator (accurate FP64 shapes, either reciprocal, to 1e-11 of the
oracle; fast FP64 shapes to 1e-10;
FP32 shapes to 1e-5 of the FP64 operator and to 1e-6 of each other — the
split-K grouping of the tiles differs between shapes), and the autotuner
times every candidate on a problem large enough to tune."""
import numpy as np
import pytest

from erosion_b200 import _lib, geometry as G, stokes

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture
def auto_shapes(lib):
    yield
    for kind in (0, 1, 2):
        assert lib.erosion_set_far_shape(kind, -1) == 0


def test_every_shape_computes_the_same_operator(lib, oracle, auto_shapes):
    g = G.workload("c1", seed=4)
    den = np.random.default_rng(9).standard_normal(g.ntot)
    ref = oracle.matvec(g, den, mode=1)
    ref32 = None
    num = _lib.far_shapes()
    for i in range(len(num["fp64"]["tuned_ms"])):
        assert lib.erosion_set_far_shape(0, i) == 0
        assert rel(stokes.matvec(g, den, precision=0), ref) < 1e-11, i
        assert _lib.far_shapes()["fp64"]["index"] == i
    for i in range(len(num["fp64_fast"]["tuned_ms"])):   # the fast FP64 operator (reciprocal to ~1e-12)
        assert lib.erosion_set_far_shape(2, i) == 0
        assert rel(stokes.matvec(g, den, precision=2), ref) < 1e-10, i
        assert _lib.far_shapes()["fp64_fast"]["index"] == i
    for i in range(len(num["fp32"]["tuned_ms"])):
        assert lib.erosion_set_far_shape(1, i) == 0
        a = stokes.matvec(g, den, precision=1)
        assert np.linalg.norm(a - ref) / np.linalg.norm(ref) < 1e-5, i
        if ref32 is None:
            ref32 = a
        assert np.linalg.norm(a - ref32) / np.linalg.norm(ref32) < 1e-6, i
        assert _lib.far_shapes()["fp32"]["index"] == i


def test_unknown_shape_rejected(lib):
    assert lib.erosion_set_far_shape(1, 17) == _lib.EROSION_BAD_INPUT
    assert lib.erosion_set_far_shape(3, 0) == _lib.EROSION_BAD_INPUT
    assert lib.erosion_set_far_shape(-1, 0) == _lib.EROSION_BAD_INPUT


def test_autotuner_times_every_candidate(lib, auto_shapes):
    g = G.workload("c2")
    den = np.random.default_rng(1).standard_normal(g.ntot)
    stokes.matvec(g, den, precision=1)
    sh = _lib.far_shapes()
    for kind in ("fp64", "fp32", "fp64_fast"):
        ms = sh[kind]["tuned_ms"]
        assert all(v > 0 for v in ms.values()), (kind, ms)
        best = min(ms, key=ms.get)
        assert sh[kind]["shape"] == best
    print("far-field shapes:", sh)
