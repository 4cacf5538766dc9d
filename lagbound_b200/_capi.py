"""ctypes binding of the C ABI in include/lagbound_b200.h (the library built by lagbound_b200/build.py).

There is no CPU fallback: if the shared library is missing or cannot be loaded, importing this module raises.
"""
import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liblagbound_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "lagbound_b200.h")

LB_OK = 0
LB_ERR = {-1: "LB_ERR_INVALID", -2: "LB_ERR_CUDA", -3: "LB_ERR_NOMEM", -4: "LB_ERR_STATE", -5: "LB_ERR_TIMEOUT",
          -6: "LB_ERR_NUMERIC"}
LB_F64, LB_F32, LB_BF16 = 0, 1, 2
LB_EVAL_GRAD, LB_EVAL_FIXED, LB_EVAL_TIMING = 1, 2, 4
PHASES = ("aggregates", "pair", "vcs", "tri", "rows", "final")


class LBError(RuntimeError):
    def __init__(self, code, fn, msg):
        super().__init__(f"{fn} failed with {LB_ERR.get(code, code)}: {msg}")
        self.code = code


class EvalOut(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("primal", ctypes.c_double), ("quadA", ctypes.c_double),
                ("zz", ctypes.c_double), ("level_tot", ctypes.c_double), ("tri_tot", ctypes.c_double),
                ("vcs_tot", ctypes.c_double), ("gmin", ctypes.c_double), ("nviol", ctypes.c_int64),
                ("vcs_nviol", ctypes.c_int64), ("lam_sum", ctypes.c_double), ("reserved", ctypes.c_double * 5)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int32
_D = ctypes.c_double
_INT = ctypes.c_int

SIGNATURES = {
    "lb_version": (ctypes.c_char_p, []),
    "lb_last_error": (ctypes.c_char_p, []),
    "lb_ctx_create": (_INT, [_INT, ctypes.POINTER(_P)]),
    "lb_ctx_create_on_stream": (_INT, [_INT, _P, ctypes.POINTER(_P)]),
    "lb_ctx_destroy": (_INT, [_P]),
    "lb_ctx_synchronize": (_INT, [_P]),
    "lb_ctx_set_cache": (_INT, [_P, _INT, _D]),
    "lb_gather_probe": (_INT, [_P, _I64, _I32, _I64, _I32, ctypes.POINTER(ctypes.c_float)]),
    "lb_ctx_timer": (_INT, [_P, _INT, ctypes.POINTER(ctypes.c_float)]),
    "lb_problem_create": (_INT, [_P, _I64, _P, _P, _P, _P, _D, _D, _I32, _INT, ctypes.POINTER(_P)]),
    "lb_problem_create_ordered": (_INT, [_P, _I64, _P, _P, _P, _P, _D, _D, _I32, _INT, _P, ctypes.POINTER(_P)]),
    "lb_problem_destroy": (_INT, [_P]),
    "lb_problem_info": (_INT, [_P, ctypes.POINTER(_I32), ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
    "lb_set_V": (_INT, [_P, _P]),
    "lb_get_V": (_INT, [_P, _P]),
    "lb_set_V_raw": (_INT, [_P, _P, _INT]),
    "lb_pair_level_add": (_INT, [_P, _I32, _P, _D, ctypes.POINTER(_I32)]),
    "lb_pair_level_set_sigma": (_INT, [_P, _I32, _P]),
    "lb_pair_level_get_sigma": (_INT, [_P, _I32, _P]),
    "lb_set_pair_weight": (_INT, [_P, _D, _D]),
    "lb_vcs_level_add": (_INT, [_P, _I32, _P, _D, ctypes.POINTER(_I32)]),
    "lb_vcs_set_ws": (_INT, [_P, _I32, _I64, _P, _P, _P, _P]),
    "lb_vcs_get_ws": (_INT, [_P, _I32, _P, _P]),
    "lb_tri_set": (_INT, [_P, _I64, _P, _P]),
    "lb_tri_get_lam": (_INT, [_P, _P]),
    "lb_eval": (_INT, [_P, _D, _D, _INT, ctypes.POINTER(EvalOut)]),
    "lb_eval_async": (_INT, [_P, _D, _D, _INT]),
    "lb_eval_fetch": (_INT, [_P, ctypes.POINTER(EvalOut)]),
    "lb_eval_host": (_INT, [_P, _P, _D, _D, _INT, ctypes.POINTER(EvalOut)]),
    "lb_get_G": (_INT, [_P, _P]),
    "lb_set_V_device": (_INT, [_P, _P]),
    "lb_set_V_device_async": (_INT, [_P, _P]),
    "lb_lobpcg": (_INT, [_P, _I32, _P, _P, _P, _P, _I32, _P, ctypes.POINTER(_I32)]),
    "lb_get_G_device": (_INT, [_P, _P]),
    "lb_get_G_device_async": (_INT, [_P, _P]),
    "lb_get_pair_pp": (_INT, [_P, _I32, _P]),
    "lb_get_tri_pt": (_INT, [_P, _P, _P]),
    "lb_get_vcs_ppv": (_INT, [_P, _I32, _P, _P, _P]),
    "lb_multiplier_update": (_INT, [_P]),
    "lb_sweeps": (_INT, [_P, _I32, _D, _D, _D, _I32, _P, _D]),
    "lb_outer_loop": (_INT, [_P, _I32, _P, _I32, _D, _D, _D, _I32, _D, _I32, ctypes.POINTER(_I64)]),
    "lb_separate": (_INT, [_P, _D, _I32, _I32, _I32, _I32, _D, _I64, _I64, _I32, _I32, _I32, ctypes.POINTER(_I64),
                           ctypes.POINTER(_I64)]),
    "lb_separate_get": (_INT, [_P, _I32, _P, _P]),
    "lb_vcs_separate": (_INT, [_P, _I32, _I64, _D, _I32, ctypes.POINTER(_I64), _P]),
    "lb_vcs_separate_get": (_INT, [_P, _P, _P, _P]),
    "lb_vcs_sig_stats": (_INT, [_P, _I32, ctypes.POINTER(_D), ctypes.POINTER(_I64)]),
    "lb_vcs_grow": (_INT, [_P, _I32, _I64, _D, _I32, _I32, _I64, _P, _P]),
    "lb_tri_pool_round": (_INT, [_P, _D, _I32, _I32, _I32, _I32, _D, _I32, _I32, _I64, _I64, _I64, _P]),
    "lb_tri_get": (_INT, [_P, _P]),
    "lb_problem_create_batched": (_INT, [_P, _I32, _P, _I64, _P, _P, _P, _P, _P, _P, _I32, _INT, _P,
                                         ctypes.POINTER(_P)]),
    "lb_eval_graphs": (_INT, [_P, _P]),
    "lb_ctx_capture_begin": (_INT, [_P]),
    "lb_ctx_capture_end": (_INT, [_P, ctypes.POINTER(_P)]),
    "lb_cuda_graph_launch": (_INT, [_P]),
    "lb_cuda_graph_kernels": (_INT, [_P, ctypes.POINTER(_I64)]),
    "lb_cuda_graph_destroy": (_INT, [_P]),
    "lb_tri_count": (_INT, [_P, ctypes.POINTER(_I64)]),
    "lb_vcs_get_structure": (_INT, [_P, _I32, _P, _P]),
    "lb_vcs_nnz": (_INT, [_P, _I32, ctypes.POINTER(_I64)]),
    "lb_timing_collect": (_INT, [_P, _P, ctypes.POINTER(_I64)]),
    "lb_launch_count": (_INT, [_P, ctypes.POINTER(_I64)]),
    "lb_set_light_threshold": (_INT, [_P, _I32]),
    "lb_get_G_raw": (_INT, [_P, _P]),
    "lb_eval_host_pipelined": (_INT, [_P, _I32, _P, _P, _D, _D, _INT, _P]),
    "lb_nd_order": (_INT, [_I64, _P, _P, _P, _P]),
    "lb_chol_fill": (_INT, [_I64, _P, _P, _P, _I64, _P]),
    "lb_get_light_threshold": (_INT, [_P, ctypes.POINTER(_I32), _P]),
    "lb_bv_noalloc": (_INT, [_I64, _I64, _P, _P, _P, _P, _D, _D, _P, _INT, _I32, _P, _P, _P]),
    "lb_reduce_exact": (_INT, [_P, _I64, _I64, _P, ctypes.POINTER(_P)]),
    "lb_reduce_info": (_INT, [_P, _P]),
    "lb_reduce_get": (_INT, [_P, _P, _P, _P, _P]),
    "lb_reduce_labels": (_INT, [_P, _P, _P, _P]),
    "lb_reduce_destroy": (_INT, [_P]),
    "lb_simple_graph": (_INT, [_P, _I64, _P, _I64, ctypes.POINTER(_P)]),
    "lb_graph_info": (_INT, [_P, _P]),
    "lb_graph_get": (_INT, [_P, _P, _P, _P, _P]),
    "lb_graph_destroy": (_INT, [_P]),
    "lb_modularity_counts": (_INT, [_P, _I64, _I64, _P, _P, _P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)]),
}


def header_functions(path=HEADER):
    """Names of every function declared in the public header."""
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(lb_\w+)\s*\(", txt, flags=re.M)))


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"lagbound_b200 native library not built: {LIB_PATH} is missing "
                          "(run `python -m lagbound_b200.build`); there is no CPU fallback")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def get_lib():
    """The loaded native library (loaded on first use, so that the build step can import this package)."""
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def __getattr__(name):
    if name == "lib":
        return get_lib()
    raise AttributeError(name)


def check(rc, fn):
    if rc != LB_OK:
        raise LBError(rc, fn, get_lib().lb_last_error().decode(errors="replace"))


def call(fn, *args):
    check(getattr(get_lib(), fn)(*args), fn)


def ptr(a):
    """Data pointer of a C-contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return ctypes.c_void_p(a.ctypes.data)


def c(a, dt):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)
