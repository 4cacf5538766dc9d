"""The C-ABI library loads and exports every entry point declared in include/*.h (no GPU needed)."""
import ctypes
import glob
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    from lagbound_b200 import _capi as C
    lib = ctypes.CDLL(C.LIB_PATH)
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names += C.header_functions(h)
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the ctypes signature table covers the whole header
    assert set(C.SIGNATURES) >= set(C.header_functions()), set(C.header_functions()) - set(C.SIGNATURES)


def test_version_and_error_reporting_without_device():
    torch = pytest.importorskip("torch")
    from lagbound_b200 import _capi as C
    assert b"sm_100a" in C.lib.lb_version()
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; the no-device path is not exercised")
    h = ctypes.c_void_p()
    rc = C.lib.lb_ctx_create(0, ctypes.byref(h))
    assert rc != 0
    assert len(C.lib.lb_last_error()) > 0


def test_null_arguments_are_rejected_before_any_device_work():
    from lagbound_b200 import _capi as C
    rc = C.lib.lb_problem_create(None, 10, None, None, None, None, 1.0, 0.0, 8, 0, None)
    assert rc == -1 and b"null" in C.lib.lb_last_error()
    assert C.lib.lb_eval(None, 0.02, 1.0, 1, None) == -1


def test_new_entry_points_reject_null_handles_without_device_work():
    """The outer loop, the pipelined host evaluations, the native LOBPCG, the on-stream context and the asynchronous
    device copies refuse a null problem or null buffers on the host (LB_ERR_INVALID, message set)."""
    from lagbound_b200 import _capi as C
    lib = C.get_lib()
    perms = (ctypes.c_int64 * 4)(0, 1, 2, 3)
    assert lib.lb_outer_loop(None, 1, perms, 1, 0.02, 1.0, 0.0, 1, 1.0, 1, None) == -1
    assert b"null" in lib.lb_last_error()
    vp = (ctypes.c_void_p * 1)(None)
    assert lib.lb_eval_host_pipelined(None, 1, vp, None, 0.02, 1.0, 1, None) == -1
    assert b"null" in lib.lb_last_error()
    assert lib.lb_lobpcg(None, 4, None, None, None, None, 10, None, None) == -1
    assert b"null" in lib.lb_last_error()
    assert lib.lb_set_V_device_async(None, None) == -1
    assert lib.lb_get_G_device_async(None, None) == -1
    out = ctypes.c_void_p()
    assert lib.lb_ctx_create_on_stream(-1, None, ctypes.byref(out)) != 0
