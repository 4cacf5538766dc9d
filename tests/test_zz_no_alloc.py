"""lb_bv_noalloc, the entry point for callers that cannot allocate device memory: a host whose own pool owns every
device byte (a serving loop admitting requests against an HBM budget, or a runtime that accounts for all device
memory) cannot let a library call cudaMalloc, which synchronises the device and escapes the pool's accounting.  The
entry point works in a fixed static scratch array, with the caller's device buffers for inputs and outputs.

Checked through the C ABI against the regular evaluation (lb_eval, which allocates its scratch) and against the
oracle, on two calls in a row, at the tolerances of the other GPU tests: a small graph with a hub row, a weighted
graph with more rows than the scratch has blocks (so blocks cover several rows and some blocks have none), the
widest row the scratch allows (ld = 64), invalid column indices and a malformed indptr (counted, never read past
the arrays), and arguments refused on the host before anything is launched.

This file sorts last so that a run stopping at the first failure has run every other test first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 2e-5, "bf16": 2e-5}


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def _hub_graph():
    from lagbound_b200 import synth
    g = synth.sbm(1500, 6, 0.05, 0.004, seed=4)
    # add a hub row (degree > 2048 is split across warps by lb_eval, not by lb_bv_noalloc)
    n = g.n
    hub_nb = np.arange(1, n)
    u = np.r_[np.repeat(np.arange(n), np.diff(g.indptr)), np.zeros(n - 1, np.int64)]
    v = np.r_[g.indices, hub_nb]
    return synth._csr_from_pairs(n, u, v)


def _weighted_graph():
    """n = 20,000 Chung-Lu graph (more than 8 x 1024 rows: the scratch's 1024 blocks each cover several rows and the
    last blocks cover none) with symmetric integer edge multiplicities 1..3 (FP32-exact)."""
    from lagbound_b200 import synth
    g = synth.chung_lu_communities(20_000, 10.0, 2.3, 500, 120, 0.25, seed=3)
    rows = np.repeat(np.arange(g.n), np.diff(g.indptr))
    a = np.minimum(rows, g.indices); b = np.maximum(rows, g.indices)
    w = ((a * 7919 + b * 104729) % 3 + 1).astype(np.float64)
    g.data = w
    g.d = np.bincount(rows, weights=w, minlength=g.n)
    g.L = float(w.sum())
    return g


class _Dev:
    """The caller-owned device buffers of one lb_bv_noalloc call (torch tensors)."""

    def __init__(self, torch, g, V, dtype, ld, weights=None, indices=None, indptr=None):
        dev = torch.device("cuda:0")
        tdt = {"f64": torch.float64, "f32": torch.float32, "bf16": torch.bfloat16}[dtype]
        self.gdt = torch.float64 if dtype == "f64" else torch.float32
        self.indptr = torch.from_numpy(np.asarray(g.indptr if indptr is None else indptr, np.int64)).to(dev)
        self.indices = torch.from_numpy(np.asarray(g.indices if indices is None else indices, np.int32)).to(dev)
        self.w = None if weights is None else torch.from_numpy(np.asarray(weights, np.float32)).to(dev)
        self.d = torch.from_numpy(np.asarray(g.d, np.float64)).to(dev)
        self.V = torch.zeros((g.n, ld), dtype=tdt, device=dev)
        self.V[:, :V.shape[1]] = torch.from_numpy(V).to(dev).to(tdt)
        self.n, self.ld, self.dev, self.torch = g.n, ld, dev, torch

    def call(self, lib, dtype_code, nnz, L, C0):
        torch = self.torch
        G = torch.full((self.n, self.ld), float("nan"), dtype=self.gdt, device=self.dev)
        out = torch.full((5,), float("nan"), dtype=torch.float64, device=self.dev)
        stream = torch.cuda.current_stream().cuda_stream
        rc = lib.lb_bv_noalloc(self.n, int(nnz), self.indptr.data_ptr(), self.indices.data_ptr(),
                               None if self.w is None else self.w.data_ptr(), self.d.data_ptr(), float(L), float(C0),
                               self.V.data_ptr(), dtype_code, self.ld, G.data_ptr(), out.data_ptr(),
                               ctypes.c_void_p(stream))
        assert rc == 0, lib.lb_last_error()
        torch.cuda.synchronize()
        return G.double().cpu().numpy(), out.cpu().numpy()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _check_against_regular(torch, g, r, dtype, weights=None, C0=3.0):
    """lb_bv_noalloc twice vs lb_eval (fixed multipliers, no levels or triangles: G = A V - d (d^T V)/L) and vs the
    oracle's A V - d (d^T V)/L, all at the V the regular path stores (rounded to dtype)."""
    from lagbound_b200 import Context, Problem, synth
    from lagbound_b200 import _capi as C
    from oracle import oracle as O
    tol = TOL[dtype]
    V = synth.random_V(g.n, r, seed=7)
    ctx = Context(0)
    p = Problem(ctx, g.n, g.indptr, g.indices, weights, g.d, g.L, C0, r, dtype)
    p.set_V(V)
    ld = p.info()["ld"]
    Vr = p.get_V()
    ref = p.eval(grad=True, fixed=True)
    G_ref = p.G()
    inst = O.Instance(g.n, g.indptr, g.indices, np.ones(g.nnz) if weights is None else weights, g.d, g.L, C0)
    G_orc = O.apply_C(inst, Vr)
    bufs = _Dev(torch, g, Vr, dtype, ld, weights=weights)
    for call in range(2):
        Gh, o = bufs.call(C.get_lib(), p.dtype, g.nnz, g.L, C0)
        assert np.isfinite(Gh).all()
        assert np.all(Gh[:, r:] == 0.0), call
        Gh = Gh[:, :r]
        assert _rel(Gh, G_ref) < tol, call
        assert _rel(Gh, G_orc) < tol, call
        assert o[0] == pytest.approx(ref["quadA"], rel=tol), call
        assert o[1] == pytest.approx(ref["zz"], rel=tol, abs=1e-9), call
        assert o[2] == pytest.approx(ref["primal"], rel=tol), call
        assert o[3] == 0.0 and o[4] == 0.0, call
    p.close()
    ctx.close()


@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_noalloc_matches_regular_evaluation_twice(torch_cuda, dtype):
    _check_against_regular(torch_cuda, _hub_graph(), 13, dtype)


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_noalloc_weighted_more_rows_than_blocks(torch_cuda, dtype):
    g = _weighted_graph()
    assert g.n > 8 * 1024
    _check_against_regular(torch_cuda, g, 32, dtype, weights=g.data)


@pytest.mark.parametrize("dtype", ["f32", "bf16"])
def test_noalloc_widest_row(torch_cuda, dtype):
    # ld = 64 elements: the widest row the scratch holds
    _check_against_regular(torch_cuda, _hub_graph(), 64, dtype)


def test_noalloc_counts_bad_columns_and_clamps_rows(torch_cuda):
    """Three column indices outside [0, n) are skipped and counted (out[3] = 3); indptr[n] past nnz clamps the last
    row's range to nnz (out[4] = 1).  G equals the graph's with those three entries dropped."""
    torch = torch_cuda
    from lagbound_b200 import synth
    from lagbound_b200 import _capi as C
    from oracle import oracle as O
    g = _hub_graph()
    r, C0 = 16, 0.5
    V = synth.random_V(g.n, r, seed=11)
    bad_at = np.array([5, g.nnz // 2, g.nnz - 3])
    indices = g.indices.astype(np.int32).copy()
    indices[bad_at] = [g.n, -1, g.n + 100]
    indptr = g.indptr.copy()
    indptr[-1] = g.nnz + 1000
    data = np.ones(g.nnz)
    data[bad_at] = 0.0
    G_orc = O.apply_C(O.Instance(g.n, g.indptr, g.indices, data, g.d, g.L, C0), V)
    A_V_V = float(np.einsum("ij,ij->", O.spmm(O.Instance(g.n, g.indptr, g.indices, data, g.d, g.L, C0), V), V))
    bufs = _Dev(torch, g, V, "f64", 16, indices=indices, indptr=indptr)
    for call in range(2):
        Gh, o = bufs.call(C.get_lib(), C.LB_F64, g.nnz, g.L, C0)
        assert _rel(Gh[:, :r], G_orc) < 1e-12, call
        assert o[0] == pytest.approx(A_V_V, rel=1e-12), call
        assert o[3] == 3.0 and o[4] == 1.0, call


def test_noalloc_refuses_misaligned_and_oversize_arguments(torch_cuda):
    """Checked on the host before any launch: the pointers below are never dereferenced."""
    from lagbound_b200 import _capi as C
    lib = C.get_lib()
    a = ctypes.c_void_p(1 << 20)                # 16-byte aligned stand-ins
    odd = ctypes.c_void_p((1 << 20) + 8)        # 8-byte aligned, not 16
    args = lambda V=a, G=a, ip=a, dt=C.LB_F32, ld=32: (10, 20, ip, a, None, a, 1.0, 0.0, V, dt, ld, G, a, None)
    rc = lib.lb_bv_noalloc(*args(V=odd))
    assert rc == -1 and b"16-byte aligned" in lib.lb_last_error()
    rc = lib.lb_bv_noalloc(*args(G=odd))
    assert rc == -1 and b"16-byte aligned" in lib.lb_last_error()
    rc = lib.lb_bv_noalloc(*args(ip=ctypes.c_void_p((1 << 20) + 4)))
    assert rc == -1 and b"8-byte aligned" in lib.lb_last_error()
    rc = lib.lb_bv_noalloc(*args(ld=128))
    assert rc == -1 and b"at most 64" in lib.lb_last_error()
    rc = lib.lb_bv_noalloc(*args(dt=C.LB_F64, ld=3))
    assert rc == -1
    rc = lib.lb_bv_noalloc(10, -1, a, a, None, a, 1.0, 0.0, a, C.LB_F32, 32, a, a, None)
    assert rc == -1 and b"nnz" in lib.lb_last_error()
