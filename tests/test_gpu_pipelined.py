"""lb_eval_host_pipelined: evaluations from host buffers with the V uploads and G downloads overlapped (three
streams, two staging slots each way) return exactly what the call-by-call sequence lb_eval_host + lb_get_G_raw
returns, step by step: same scalars and bit-identical G.

Cases: BF16 V with r = 13 (rows padded to 16) in a community order (the permuted raw-copy kernels) and triangles,
five steps over three V arrays (a buffer appears at several steps, so slots are reused while earlier copies are in
flight), pinned host buffers; FP32 and FP64 V with r = 32 in the natural order, pageable buffers; evaluations
without the gradient and without G buffers; arguments refused on the host.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RHO, TRI_W = 0.02, 1.0


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def _raw(torch, V, dtype, pinned):
    t = torch.from_numpy(V)
    t = {"bf16": t.to(torch.bfloat16).view(torch.int16), "f32": t.to(torch.float32), "f64": t}[dtype].contiguous()
    return (t.pin_memory() if pinned else t.clone()).numpy()


def _gbuf(torch, n, r, dtype, pinned):
    t = torch.empty((n, r), dtype=torch.float64 if dtype == "f64" else torch.float32)
    return (t.pin_memory() if pinned else t).numpy()


@pytest.mark.parametrize("dtype,r,ordered,pinned", [("bf16", 13, True, True), ("f32", 32, False, False),
                                                     ("f64", 32, False, False)])
def test_pipelined_equals_call_by_call(torch_cuda, dtype, r, ordered, pinned):
    torch = torch_cuda
    from lagbound_b200 import Context, Problem, synth
    from lagbound_b200.problem import locality_order
    g = synth.chung_lu_communities(50_000, 12.0, 2.3, 3000, 400, 0.25, seed=8)
    TI = synth.wedge_triples(g, 60_000, seed=3)
    lam = synth.tri_multipliers(len(TI), seed=3)
    ctx = Context(0)
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, r, dtype,
                order=locality_order(g.labels) if ordered else None)
    p.set_triangles(TI, lam)
    Vs = [_raw(torch, synth.random_V(g.n, r, seed=s), dtype, pinned) for s in (1, 2, 3)]
    seq = [0, 1, 2, 0, 1]
    # call by call
    ref = []
    for k in seq:
        o = p.eval_host(Vs[k], RHO, TRI_W)
        G = _gbuf(torch, g.n, r, dtype, False)
        p.G_raw(G)
        ref.append((o, G.copy()))
    Gs = [_gbuf(torch, g.n, r, dtype, pinned) for _ in range(2)]
    for rep in range(2):                                  # twice: the second call reuses the pipeline's buffers
        # two G buffers used alternately (each written again two steps later)
        res = p.eval_host_pipelined([Vs[k] for k in seq], [Gs[m % 2] for m in range(len(seq))], RHO, TRI_W)
        for m in range(len(seq)):
            assert res[m]["value"] == ref[m][0]["value"], (rep, m)
            assert res[m]["quadA"] == ref[m][0]["quadA"] and res[m]["tri_tot"] == ref[m][0]["tri_tot"]
        # the last two steps' G are what the two buffers hold
        assert np.array_equal(Gs[(len(seq) - 1) % 2], ref[-1][1])
        assert np.array_equal(Gs[(len(seq) - 2) % 2], ref[-2][1])
    # every step's G, each into its own buffer
    Gall = [_gbuf(torch, g.n, r, dtype, pinned) for _ in seq]
    p.eval_host_pipelined([Vs[k] for k in seq], Gall, RHO, TRI_W)
    for m in range(len(seq)):
        assert np.array_equal(Gall[m], ref[m][1]), m
    # no gradient, no G buffers
    res = p.eval_host_pipelined([Vs[k] for k in seq], None, RHO, TRI_W, grad=False)
    assert [o["value"] for o in res] == [o["value"] for o, _ in ref]
    p.close()
    ctx.close()


def test_pipelined_refuses_bad_arguments(torch_cuda):
    from lagbound_b200 import Context, Problem, synth
    from lagbound_b200._capi import LBError
    g = synth.sbm(2000, 8, 0.08, 0.002, seed=0)
    ctx = Context(0)
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, 16, "f32")
    V = synth.random_V(g.n, 16, seed=1).astype(np.float32)
    G = np.empty((g.n, 16), np.float32)
    with pytest.raises(AssertionError):
        p.eval_host_pipelined([V], [G], RHO, TRI_W, grad=False)     # G buffers need the gradient
    import ctypes
    from lagbound_b200 import _capi as C
    vp = (ctypes.c_void_p * 1)(None)
    with pytest.raises(LBError):
        C.call("lb_eval_host_pipelined", p.h, 1, vp, None, RHO, TRI_W, C.LB_EVAL_GRAD, None)
    assert p.eval_host_pipelined([], None, RHO, TRI_W) == []
    p.close()
    ctx.close()
