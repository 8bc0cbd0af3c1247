"""The C-ABI library builds, loads without a GPU and exports every symbol the
header declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from erosion_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "erosion_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", src, re.M)
    return sorted(set(n for n in names if n not in ("if", "while")))


def test_library_builds_and_loads():
    path = build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    assert lib is not None


def test_exports_every_header_symbol():
    lib = _lib.load()
    declared = header_functions()
    assert "stokessolver_" in declared and "computeshearstress_" in declared and "computeqoitargets_" in declared
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(header_functions()) == set(_lib.SIGNATURES)


def test_param_struct_layout():
    # erosion_params: 4 doubles, int64, 6 int32 flags, 6 reserved int32, 1 double
    assert ctypes.sizeof(_lib.ErosionParams) == 4 * 8 + 8 + 6 * 4 + 6 * 4 + 8
    p = _lib.default_params()
    assert (p.wall_a, p.wall_b, p.wall_order, p.tol, p.maxl) == (3.0, 1.0, 8.0, 1e-8, 8000)
    assert (p.ibary, p.ifmm, p.ibc, p.precision) == (1, 1, 1, 0)


def test_no_device_is_an_error_not_a_fallback():
    """Without a GPU the library reports EROSION_NO_DEVICE (never a CPU result)."""
    import numpy as np
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is visible")
    from erosion_b200 import geometry as G, stokes
    g = G.workload("ref-small")
    with pytest.raises(_lib.ErosionError) as e:
        stokes.matvec(g, np.zeros(g.ntot))
    assert e.value.code == _lib.EROSION_NO_DEVICE


@pytest.mark.parametrize("cname,pyname", [("erosion_params", "ErosionParams"), ("erosion_solve_stats", "SolveStats"),
                                          ("erosion_batch_stats", "BatchStats"),
                                          ("erosion_step_params", "StepParams"),
                                          ("erosion_step_stats", "StepStats")])
def test_struct_mirrors_match_the_header(tmp_path, cname, pyname):
    """Every ctypes mirror has the size and field offsets the C compiler gives
    the header's struct (the ABI a Julia or C caller sees)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    py = getattr(_lib, pyname)
    fields = [f[0] for f in py._fields_]
    src = tmp_path / "layout.c"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "erosion_b200.h"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({cname}));']
    lines += [f'  printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == ctypes.sizeof(py)
    assert out[1:] == [getattr(py, f).offset for f in fields]
