"""B200-native Stokes boundary-integral path of quaife/erosion.

The compute lives in ``libstokes_b200.so`` (hand-written sm_100a CUDA behind a
C ABI, ``include/erosion_b200.h``).  This package holds its ctypes binding,
the host-side mirror of the reference's Julia interface, the synthetic
workload generator and the build helper.
"""
from . import geometry  # noqa: F401
