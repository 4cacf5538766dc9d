"""lagbound_b200: the augmented-Lagrangian inner loop of lagbound ("Atris") as hand-written CUDA kernels for B200
(sm_100a) behind a C ABI (include/lagbound_b200.h), with host-side objects in Python.

Importing the package loads the native library; there is no CPU fallback.
"""
from ._capi import LBError, lib  # noqa: F401  (fails loudly when the native library is missing)
from .problem import Context, Problem  # noqa: F401

__all__ = ["Context", "Problem", "LBError"]
