"""CPU FP64 oracle of the Stokes boundary-integral path (test infrastructure).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline arm of
``bench.py`` use this package, and only as the checker or the timed CPU
baseline; the shipped library never loads it.
"""
from .binding import Oracle, build_oracle  # noqa: F401
