"""The learned initial guess: the backward kernels against the FP64 numpy
oracle, the density encoding, training on the solver's own densities, and
what the trained network gains over the previous-step initial guess."""
import ctypes

import numpy as np
import pytest

from erosion_b200 import _lib, geometry as G, learned, stokes
from oracle import mlp_oracle

pytestmark = pytest.mark.gpu

PF = ctypes.POINTER(ctypes.c_float)


def fptr(a):
    return a.ctypes.data_as(PF)


def test_gradients_match_cpu_oracle(lib):
    assert lib.erosion_lw_init(7) == 0
    npar = lib.erosion_lw_num_params()
    params = np.zeros(npar, np.float32)
    assert lib.erosion_lw_get_params(fptr(params)) == 0
    rng = np.random.default_rng(0)
    x = rng.standard_normal((8, mlp_oracle.LAYERS[0][0])).astype(np.float32)
    y = rng.standard_normal((8, mlp_oracle.LAYERS[-1][1])).astype(np.float32)
    loss = ctypes.c_double()
    grads = np.zeros(npar, np.float32)
    assert lib.erosion_lw_loss_grad(fptr(x), fptr(y), 8, ctypes.byref(loss), fptr(grads)) == 0
    l_ref, g_ref = mlp_oracle.loss_and_grad(params, x, y)
    assert abs(loss.value - l_ref) / l_ref < 1e-5
    assert np.linalg.norm(grads - g_ref) / np.linalg.norm(g_ref) < 1e-4
    # per layer as well
    o = 0
    for ni, no in mlp_oracle.LAYERS:
        k = ni * no + no
        a, b = grads[o:o + k], g_ref[o:o + k]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4
        o += k


def test_encode_decode_round_trip(lib):
    g = G.workload("c1", seed=11)
    den, _, _ = stokes.solve(g, precond=1)
    p = stokes.params_for(g)
    t = np.zeros((g.M, 37), np.float32)
    assert lib.erosion_lw_encode(ctypes.byref(p), g.n, g.M, g.nout, _lib.ptr(g.xx), _lib.ptr(g.yy), _lib.ptr(den),
                                 fptr(t)) == 0
    back = np.zeros(g.ntot)
    assert lib.erosion_lw_decode(ctypes.byref(p), g.n, g.M, g.nout, _lib.ptr(g.xx), _lib.ptr(g.yy), fptr(t),
                                 _lib.ptr(back)) == 0
    nb0 = 2 * g.nout
    body, rec = den[nb0:nb0 + 2 * g.n * g.M], back[nb0:nb0 + 2 * g.n * g.M]
    # modes -8..8 carry most of a smooth density; the rest is the truncation
    assert np.linalg.norm(rec - body) / np.linalg.norm(body) < 0.2
    assert np.allclose(back[-3 * g.M:], den[-3 * g.M:], rtol=1e-6, atol=1e-6 * np.abs(den[-3 * g.M:]).max())


def _state(seed):
    g = G.workload("c1", seed=seed)
    th, ln, xs, ys = G.to_thetalen(g)
    return g, th.copy(), ln.copy(), xs.copy(), ys.copy()


def _step_params(g, warm_start, dt=1e-5):
    sp = _lib.StepParams()
    _lib.load().erosion_default_step_params(ctypes.byref(sp), g.n)
    sp.dt = dt
    sp.fixpdrop = 0
    sp.warm_start = warm_start
    return sp


def test_training_and_learned_guess_gain(lib):
    """Trains the increment network on a 40-step erosion run of one ten-body
    channel (rows: geometry + previous increment -> next increment, from the
    solver's own densities), then runs a held-out channel for 12 steps with
    the previous-step guess (warm_start = 1) and with the learned guess
    (warm_start = 2: previous density plus the predicted increment, used
    only when its FP64 residual is smaller).  Both reach the tolerance; the
    learned candidate is evaluated every stage once it has a history, and the
    measured gain in initial residual and iterations is printed."""
    g, th, ln, xs, ys = _state(100)
    p = stokes.params_for(g, precision=1, precond=1)
    traj = learned.trajectory(p, _step_params(g, 1), g.n, g.nout, th, ln, xs, ys, 40)
    X, Y = learned.training_rows(p, g.n, g.nout, traj)
    assert X.shape[1] == learned.dims()[1] and len(X) >= 300
    loss0 = learned.train(X, Y, epochs=1)
    loss = learned.train(X, Y, epochs=300)
    assert loss < 0.5 * loss0
    runs = {}
    for ws in (1, 2):
        g2, th, ln, xs, ys = _state(200)
        sp = _step_params(g2, ws)
        nb = np.array([g2.M], np.int64)
        t = np.zeros(1)
        dele = np.zeros(g2.M, np.int64)
        its, res, used, cand = [], [], [], []
        for k in range(12):
            rc = lib.erosion_rk2_step(ctypes.byref(p), ctypes.byref(sp), g2.n, nb.ctypes.data_as(_lib.PI64), g2.nout,
                                      _lib.ptr(th), _lib.ptr(ln), _lib.ptr(xs), _lib.ptr(ys),
                                      t.ctypes.data_as(_lib.PD), dele.ctypes.data_as(_lib.PI64))
            assert rc == 0
            st = _lib.StepStats()
            lib.erosion_get_step_stats(ctypes.byref(st))
            d = st.as_dict()
            assert d["max_residual"] <= 2e-8
            if k >= 2:   # the learned candidate needs the previous increment
                its.append(sum(d["gmres_iterations"]))
                res.append(np.mean(d["guess_residual"]))
                used.append(d["guess_used"])
                cand.append(_lib.solve_stats()["guess_residual"][2])   # learned candidate, second solve
        runs[ws] = (np.mean(its), np.mean(res), used, cand)
    assert all(u in (1, 2) for pair in runs[2][2] for u in pair)
    print(f"training MSE {loss0:.3f} -> {loss:.3f}; initial residual previous-step {runs[1][1]:.3g} vs learned "
          f"{runs[2][1]:.3g}; iterations per step {runs[1][0]:.1f} vs {runs[2][0]:.1f}; learned used "
          f"{sum(u == 2 for pair in runs[2][2] for u in pair)} of {2 * len(runs[2][2])} stages; learned candidate "
          f"residual {np.mean(runs[2][3]):.3g}")
    assert runs[2][0] <= runs[1][0] + 2
