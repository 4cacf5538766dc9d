"""lb_bv_noalloc, the entry point for callers that cannot allocate device memory (a host whose pool owns every
device byte, e.g. a serving loop admitting requests against an HBM budget): it works in a fixed static scratch
array, with the caller's device buffers for inputs and outputs.  Checked through the C ABI against the regular
evaluation (lb_eval, which allocates its scratch) on two calls in a row, at the tolerances of the other GPU tests.

This file sorts last so that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def _graph():
    from lagbound_b200 import synth
    g = synth.sbm(1500, 6, 0.05, 0.004, seed=4)
    # add a hub row (degree > 2048 is split across warps by lb_eval, not by lb_bv_noalloc)
    n = g.n
    hub_nb = np.arange(1, n)
    u = np.r_[np.repeat(np.arange(n), np.diff(g.indptr)), np.zeros(n - 1, np.int64)]
    v = np.r_[g.indices, hub_nb]
    return synth._csr_from_pairs(n, u, v)


@pytest.mark.parametrize("dtype,tol", [("f64", 1e-12), ("f32", 2e-5), ("bf16", 2e-5)])
def test_noalloc_matches_regular_evaluation_twice(torch_cuda, dtype, tol):
    torch = torch_cuda
    from lagbound_b200 import Context, Problem, synth
    from lagbound_b200 import _capi as C
    g = _graph()
    r = 13
    V = synth.random_V(g.n, r, seed=7)
    C0 = 3.0
    ctx = Context(0)
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, C0, r, dtype)
    p.set_V(V)
    ld = p.info()["ld"]
    Vr = p.get_V()                                    # V as stored in the regular path (rounded to dtype)
    ref = p.eval(grad=True, fixed=True)               # no levels or triangles: G = A V - d (d^T V)/L
    G_ref = p.G()
    tdt = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16}[dtype]
    gdt = torch.float64 if dtype == "f64" else torch.float32
    dev = torch.device("cuda:0")
    indptr = torch.from_numpy(g.indptr.astype(np.int64)).to(dev)
    indices = torch.from_numpy(g.indices.astype(np.int32)).to(dev)
    d = torch.from_numpy(g.d).to(dev)
    Vd = torch.zeros((g.n, ld), dtype=tdt, device=dev)
    Vd[:, :r] = torch.from_numpy(Vr).to(dev).to(tdt)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        G = torch.full((g.n, ld), float("nan"), dtype=gdt, device=dev)
        out = torch.full((4,), float("nan"), dtype=torch.float64, device=dev)
        rc = C.get_lib().lb_bv_noalloc(g.n, indptr.data_ptr(), indices.data_ptr(), None, d.data_ptr(), g.L, C0,
                                       Vd.data_ptr(), p.dtype, ld, G.data_ptr(), out.data_ptr(),
                                       ctypes.c_void_p(stream))
        assert rc == 0, C.get_lib().lb_last_error()
        torch.cuda.synchronize()
        Gh = G[:, :r].double().cpu().numpy()
        o = out.cpu().numpy()
        assert np.isfinite(Gh).all()
        assert np.linalg.norm(Gh - G_ref) / np.linalg.norm(G_ref) < tol, call
        assert o[0] == pytest.approx(ref["quadA"], rel=tol), call
        assert o[1] == pytest.approx(ref["zz"], rel=tol, abs=1e-9), call
        assert o[2] == pytest.approx(ref["primal"], rel=tol), call
        assert o[3] == 0.0
    p.close()
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(torch_cuda):
    from lagbound_b200 import _capi as C
    lib = C.get_lib()
    dummy = ctypes.c_void_p(16)           # never dereferenced: the size check comes first
    rc = lib.lb_bv_noalloc(10, dummy, dummy, None, dummy, 1.0, 0.0, dummy, C.LB_F32, 128, dummy, dummy, None)
    assert rc == -1 and b"at most 64" in lib.lb_last_error()
    rc = lib.lb_bv_noalloc(10, dummy, dummy, None, dummy, 1.0, 0.0, dummy, C.LB_F64, 3, dummy, dummy, None)
    assert rc == -1
