"""Builds the in-tree CUDA library ``erosion_b200/libstokes_b200.so`` for sm_100a.

    python -m erosion_b200.build [--force]

nvcc cross-compiles without a GPU.  Every ``csrc/*.cu`` file is compiled into
one shared library with a C ABI (``include/erosion_b200.h``); the CUDA runtime
is linked statically so the library needs only the driver at run time.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "libstokes_b200.so")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def deps() -> list[str]:
    return sources() + sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))) + [
        os.path.join(INCLUDE, "erosion_b200.h")]


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in deps())


COMPILE_FLAGS = [*ARCH_FLAGS, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"]


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object file (in parallel: the kernels of
    each file have internal linkage, so no relocatable device code is needed)
    and links the shared library."""
    if not force and up_to_date():
        return OUT
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = nvcc_path()
    jobs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        jobs.append((obj, [nvcc, *COMPILE_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", "-o", obj, src]))
    if verbose:
        for _, cmd in jobs:
            print(" ".join(cmd))
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(lambda j: subprocess.run(j[1], capture_output=True, text=True), jobs))
    for (obj, cmd), r in zip(jobs, results):
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    link = [nvcc, *ARCH_FLAGS, "-shared", "-o", OUT + ".tmp", *[o for o, _ in jobs]]
    if verbose:
        print(" ".join(link))
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
