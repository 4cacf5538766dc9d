"""lagbound_b200: the augmented-Lagrangian inner loop of lagbound ("Atris") as hand-written CUDA kernels for B200
(sm_100a) behind a C ABI (include/lagbound_b200.h), with host-side objects in Python.

The native library is loaded on first use (creating a Context); there is no CPU fallback: without the library every
entry point raises ImportError.
"""
from ._capi import LBError, get_lib  # noqa: F401
from .problem import BatchedProblem, Context, Problem  # noqa: F401

__all__ = ["Context", "Problem", "BatchedProblem", "LBError"]
