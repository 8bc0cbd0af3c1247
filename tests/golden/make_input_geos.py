"""Extracts the reference's simulation input geometries (circle packings,
``simulations/input_geos/*.jld2`` of quaife/erosion) into
``input_geos.npz`` with the package's JLD2 reader, so that tests and users on
machines without the reference repository can run the reference's own
geometries.  Keys: ``<name>/rvec``, ``<name>/xc``, ``<name>/yc``,
``<name>/areafrac``, ``<name>/seed``.

Run from the repository root with the reference checked out:
    python tests/golden/make_input_geos.py /path/to/erosion
"""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from erosion_b200 import jld2  # noqa: E402


def main(ref_root: str):
    out = {}
    for f in sorted(glob.glob(os.path.join(ref_root, "simulations", "input_geos", "*.jld2"))):
        name = os.path.basename(f)[:-5]
        d = jld2.read(f)
        for k in ("rvec", "xc", "yc", "areafrac", "seed"):
            out[f"{name}/{k}"] = np.asarray(d[k])
    np.savez_compressed(os.path.join(HERE, "input_geos.npz"), **out)
    print(len(out) // 5, "geometries")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
