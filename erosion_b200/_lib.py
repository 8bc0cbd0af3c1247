"""ctypes binding of the C ABI in ``include/erosion_b200.h``.

The library ``libstokes_b200.so`` is built in-tree (``erosion_b200/build.py``).
There is no CPU fallback: every function here raises if the shared library is
missing, and the library itself reports EROSION_NO_DEVICE when no CUDA device
is visible.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libstokes_b200.so")

EROSION_OK = 0
EROSION_MAXITER = 1
EROSION_BREAKDOWN = 2
EROSION_BAD_INPUT = 3
EROSION_CUDA_ERROR = 4
EROSION_NO_DEVICE = 5

STATUS_NAMES = {
    EROSION_OK: "ok",
    EROSION_MAXITER: "maxiter",
    EROSION_BREAKDOWN: "breakdown",
    EROSION_BAD_INPUT: "bad_input",
    EROSION_CUDA_ERROR: "cuda_error",
    EROSION_NO_DEVICE: "no_device",
}

PD = POINTER(c_double)
PI64 = POINTER(c_int64)
PF32 = POINTER(ctypes.c_float)


class ErosionParams(ctypes.Structure):
    """Mirror of ``erosion_params``."""

    _fields_ = [
        ("wall_a", c_double),
        ("wall_b", c_double),
        ("wall_order", c_double),
        ("tol", c_double),
        ("maxl", c_int64),
        ("ibary", c_int32),
        ("ifmm", c_int32),
        ("ibc", c_int32),
        ("precision", c_int32),
        ("rhs_mode", c_int32),
        ("true_residual", c_int32),
        ("precond", c_int32),
        ("learned_guess", c_int32),
        ("fast_fp64", c_int32),
        ("precond_refresh", c_int32),
        ("stress_all_bary", c_int32),
        ("sweep_decades", c_int32),
        ("relax_tol", c_double),
    ]


class SolveStats(ctypes.Structure):
    """Mirror of ``erosion_solve_stats``."""

    _fields_ = [
        ("iterations", c_int64),
        ("matvecs", c_int64),
        ("matvecs_fp32", c_int64),
        ("sweeps", c_int64),
        ("est_residual", c_double),
        ("true_residual", c_double),
        ("ms_total", c_double),
        ("ms_far", c_double),
        ("far_launches", c_int64),
        ("near_pairs", c_int64),
        ("ms_far32", c_double),
        ("far32_launches", c_int64),
        ("far32_pairs", c_int64),
        ("true_residual_checks", c_double),
        ("sweep_residual", c_double * 8),
        ("sweep_iterations", c_int64 * 8),
        ("floor_accepted", c_int64),
        ("guess_used", c_int64),
        ("guess_residual", c_double * 3),
        ("far64_pairs", c_int64),
        ("ms_farw", c_double),
        ("farw_launches", c_int64),
        ("farw_pairs", c_int64),
        ("precond_active", c_int64),
        ("precond_singular_blocks", c_int64),
        ("ms_setup", c_double),
        ("ms_precond_setup", c_double),
        ("ms_far64f", c_double),
        ("far64f_launches", c_int64),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["sweep_residual"] = list(self.sweep_residual)[: max(self.sweeps, 0)]
        d["sweep_iterations"] = list(self.sweep_iterations)[: max(self.sweeps, 0)]
        d["guess_residual"] = list(self.guess_residual)
        return d


class BatchStats(ctypes.Structure):
    """Mirror of ``erosion_batch_stats``."""

    _fields_ = [("geometries", c_int64), ("rounds", c_int64), ("iterations", c_int64), ("graph_captures", c_int64),
                ("ms_total", c_double), ("pairs64_per_round", c_double), ("pairs32_per_round", c_double),
                ("pairs64_total", c_double), ("pairs32_total", c_double), ("max_true_residual", c_double),
                ("shape64", c_int64), ("shape32", c_int64), ("tune_ms", ctypes.c_float * 8),
                ("setup_host_ms", c_double)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["tune_ms"] = list(self.tune_ms)
        return d


class StepParams(ctypes.Structure):
    """Mirror of ``erosion_step_params``."""

    _fields_ = [("dt", c_double), ("epsilon", c_double), ("sigma", c_double),
                ("fixarea", c_int32), ("fixpdrop", c_int32), ("warm_start", c_int32),
                ("reserved", c_int32 * 5)]


class StepStats(ctypes.Structure):
    """Mirror of ``erosion_step_stats``."""

    _fields_ = [("gmres_iterations", c_int64 * 2), ("bodies_deleted", c_int64),
                ("ms_solve", c_double), ("ms_stress", c_double), ("ms_thetalen", c_double),
                ("ms_total", c_double), ("max_residual", c_double), ("matau", c_double * 2),
                ("guess_used", c_int64 * 2), ("guess_residual", c_double * 2),
                ("ms_setup", c_double), ("ms_precond_setup", c_double), ("precond_active", c_int64 * 2),
                ("precond_singular_blocks", c_int64 * 2), ("matvecs", c_int64 * 2), ("matvecs_fp32", c_int64 * 2)]

    def as_dict(self) -> dict:
        return {"gmres_iterations": list(self.gmres_iterations), "bodies_deleted": self.bodies_deleted,
                "ms_solve": self.ms_solve, "ms_stress": self.ms_stress, "ms_thetalen": self.ms_thetalen,
                "ms_total": self.ms_total, "max_residual": self.max_residual, "matau": list(self.matau),
                "guess_used": list(self.guess_used), "guess_residual": list(self.guess_residual),
                "ms_setup": self.ms_setup, "ms_precond_setup": self.ms_precond_setup,
                "precond_active": list(self.precond_active),
                "precond_singular_blocks": list(self.precond_singular_blocks),
                "matvecs": list(self.matvecs), "matvecs_fp32": list(self.matvecs_fp32)}


# Every entry point declared in include/erosion_b200.h, with its signature.
SIGNATURES = {
    "stokessolver_": (None, [PI64] * 7 + [PD, PD, PD, PI64]),
    "computeshearstress_": (None, [PI64, PI64, PI64, PD, PD, PD, PI64, PD]),
    "computeqoitargets_": (None, [PI64, PI64, PI64, PI64, PD, PD, PD, PI64, PD, PD, PD, PD, PD, PD]),
    "erosion_last_status": (c_int, []),
    "erosion_last_error": (c_char_p, []),
    "erosion_default_params": (None, [POINTER(ErosionParams)]),
    "erosion_solve": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, PI64]),
    "erosion_solve_device": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, PI64]),
    "erosion_get_solve_stats": (None, [POINTER(SolveStats)]),
    "computepressure_": (None, [PI64, PI64, PI64, PD, PD, PD, PD]),
    "erosion_pressure": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, PD]),
    "erosion_solve_batch": (c_int, [POINTER(ErosionParams), c_int32, PI64, PI64, PI64, PD, PD, PD, PI64]),
    "erosion_get_batch_stats": (None, [POINTER(BatchStats)]),
    "erosion_matvec": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, PD]),
    "erosion_matvec_noalloc": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "erosion_rhs": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD]),
    "erosion_geometry": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD] + [PD] * 12),
    "erosion_shear_stress": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, PD, PD]),
    "erosion_shear_stress_device": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64,
                                            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "erosion_qoi_targets": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, c_int64,
                                    PD, PD, PD, PD, PD, PD]),
    "erosion_near_info": (c_int64, [PI64, PI64, PI64]),
    "erosion_default_step_params": (None, [POINTER(StepParams), c_int64]),
    "erosion_get_step_stats": (None, [POINTER(StepStats)]),
    "erosion_rk2_step": (c_int, [POINTER(ErosionParams), POINTER(StepParams), c_int64, PI64, c_int64,
                                 PD, PD, PD, PD, PD, PI64]),
    "erosion_rk2_step_device": (c_int, [POINTER(ErosionParams), POINTER(StepParams), c_int64, PI64, c_int64,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                        PD, PI64]),
    "erosion_getxy": (c_int, [c_int64, c_int64, PD, PD, PD, PD, PD, PD]),
    "erosion_drag": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, PD, PD, c_int32,
                             c_double, PD, PD, PD, PD, PD]),
    "erosion_stream": (ctypes.c_void_p, []),
    "erosion_get_step_density": (c_int, [c_int32, PD, c_int64]),
    "erosion_get_step_nodes": (c_int, [c_int32, PD, PD, c_int64]),
    "erosion_lw_dims": (c_int, [ctypes.POINTER(c_int32)] * 3),
    "erosion_lw_features": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PF32]),
    "erosion_lw_encode": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PD, PF32]),
    "erosion_lw_decode": (c_int, [POINTER(ErosionParams), c_int64, c_int64, c_int64, PD, PD, PF32, PD]),
    "erosion_lw_init": (c_int, [ctypes.c_uint64]),
    "erosion_lw_num_params": (c_int64, []),
    "erosion_lw_get_params": (c_int, [PF32]),
    "erosion_lw_set_params": (c_int, [PF32]),
    "erosion_lw_loss_grad": (c_int, [PF32, PF32, c_int64, PD, PF32]),
    "erosion_lw_train": (c_int, [PF32, PF32, c_int64, c_int64, c_int64, c_double, ctypes.c_uint64, PD]),
    "erosion_lw_predict": (c_int, [PF32, c_int64, PF32]),
    "erosion_launch_count": (c_int64, []),
    "erosion_peak_tflops": (c_double, [c_int32]),
    "erosion_set_far_shape": (c_int, [c_int32, c_int32]),
    "erosion_get_far_shapes": (c_int, [POINTER(c_int32), POINTER(c_int32), PF32, POINTER(c_int32)]),
    "erosion_release": (None, []),
}

_lib = None


class ErosionError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"{p} is missing: build it with `python -m erosion_b200.build` "
                          "(the CUDA library has no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        if not hasattr(lib, name):
            continue    # reported by missing_symbols(); calling it raises AttributeError
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def missing_symbols(lib: ctypes.CDLL | None = None) -> list[str]:
    lib = lib or load()
    return [n for n in SIGNATURES if not hasattr(lib, n)]


def ptr(a: np.ndarray) -> PD:
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(PD)


def default_params(**kw) -> ErosionParams:
    p = ErosionParams()
    load().erosion_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if k in ("wall",):
            p.wall_a, p.wall_b, p.wall_order = v
        else:
            setattr(p, k, v)
    return p


def last_error() -> tuple[int, str]:
    lib = load()
    return lib.erosion_last_status(), (lib.erosion_last_error() or b"").decode()


def check(rc: int, allow=(EROSION_OK,)) -> int:
    if rc not in allow:
        code, msg = last_error()
        raise ErosionError(rc, msg)
    return rc


def solve_stats() -> dict:
    s = SolveStats()
    load().erosion_get_solve_stats(ctypes.byref(s))
    return s.as_dict()


RCP_LABELS = {0: "div", 1: "f32est+2nr", 2: "f32est+1nr", 3: "f64est+2nr", 4: "f64est+1nr"}


def far_shapes() -> dict:
    """The far-field launch shapes in use and the autotuner's timings."""
    lib = load()
    shape = (c_int32 * 3)()
    desc = (c_int32 * 36)()
    ms = (ctypes.c_float * 24)()
    num = (c_int32 * 3)()
    lib.erosion_get_far_shapes(shape, desc, ms, num)
    out = {}
    for kind, name in ((0, "fp64"), (1, "fp32"), (2, "fp64_fast")):
        cands = [tuple(desc[12 * kind + 3 * i: 12 * kind + 3 * i + 3]) for i in range(num[kind])]
        if kind != 1:
            label = lambda c: f"{c[0]}x{c[1]}-{RCP_LABELS.get(c[2], c[2])}"
        else:
            label = lambda c: f"{c[0]}x{c[1]}-unroll{c[2] % 10}-{c[2] // 10}cta"
        out[name] = {"shape": label(cands[shape[kind]]), "index": shape[kind],
                     "tuned_ms": {label(c): round(ms[8 * kind + i], 4) for i, c in enumerate(cands)}}
    return out
