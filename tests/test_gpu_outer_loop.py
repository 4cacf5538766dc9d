"""lb_outer_loop: AL outer iterations (sweep, evaluation, multiplier update) in one native call, replayed as a CUDA
graph of two iterations, against the same iterations made call by call (lb_sweeps + lb_eval + lb_multiplier_update)
with the same row orders.  The sweeps' FP64 atomics make runs differ in the last bits, so the states are compared at
1e-9 (FP64), 1e-6 (FP32: G accumulates in FP32) and the value at 1e-4 (BF16, whose rounding of V can flip on such a
difference).

Instance: a Chung-Lu + communities graph (n = 20,000) in community order with a pair level on the communities and
20,000 wedge triples; 9 iterations (one direct, four graph replays of two) with 9 row orders, and 3 iterations (too
few for a graph: all direct) with 2 row orders used cyclically.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
RHO, TRI_W = 0.02, 1.0


@pytest.fixture(scope="module")
def inst():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lagbound_b200 import Context, synth
    g = synth.chung_lu_communities(20_000, 12.0, 2.3, 500, 150, 0.25, seed=3)
    TI = synth.wedge_triples(g, 20_000, seed=2)
    lam = synth.tri_multipliers(len(TI), seed=2)
    lab = np.unique(g.labels, return_inverse=True)[1].astype(np.int64)
    rng = np.random.default_rng(5)
    perms = np.stack([rng.permutation(g.n) for _ in range(9)])
    ctx = Context(0)
    yield dict(g=g, TI=TI, lam=lam, lab=lab, perms=perms, V=synth.random_V(g.n, 16, seed=4), ctx=ctx)
    ctx.close()


def _problem(c, dtype):
    from lagbound_b200 import Problem
    from lagbound_b200.problem import locality_order
    g = c["g"]
    p = Problem(c["ctx"], g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, 16, dtype, order=locality_order(c["lab"]))
    p.set_V(c["V"])
    p.add_pair_level(c["lab"], int(c["lab"].max()) + 1, 0.03)
    p.set_triangles(c["TI"], c["lam"])
    return p


def _state(p):
    out = p.eval(RHO, TRI_W, grad=True)
    return dict(V=p.get_V(), sig=p.get_pair_sigma(0), lam=p.get_lam(), value=out["value"], G=p.G())


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _run(c, dtype, mode, perms, iters, nbatch=64):
    p = _problem(c, dtype)
    kern = 0
    if mode == "calls":
        for k in range(iters):
            p.sweeps(perms[k % len(perms)][None], RHO, RHO * TRI_W, 0.0, nbatch, 1.0)
            p.eval(RHO, TRI_W, grad=False)
            p.multiplier_update()
    else:
        kern = p.outer_loop(perms, RHO, TRI_W, 0.0, nbatch, 1.0, iters=iters, graph=(mode == "graph"))
    st = _state(p)
    p.close()
    return st, kern


@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_outer_loop_graph_matches_calls(inst, dtype):
    ref, _ = _run(inst, dtype, "calls", inst["perms"], 9)
    st, kern = _run(inst, dtype, "graph", inst["perms"], 9)
    direct, kern0 = _run(inst, dtype, "direct", inst["perms"], 9)
    assert kern > 100 and kern0 == 0
    if dtype == "bf16":
        for s in (st, direct):
            assert s["value"] == pytest.approx(ref["value"], rel=1e-4)
            assert _rel(s["lam"], ref["lam"]) < 1e-2
        return
    tol = {"f64": 1e-9, "f32": 1e-6}[dtype]      # FP32: G's accumulation rounds at 6e-8
    for s in (st, direct):
        assert s["value"] == pytest.approx(ref["value"], rel=tol)
        for k in ("V", "sig", "lam", "G"):
            assert _rel(s[k], ref[k]) < tol, k
    # the iterations did move the state
    assert _rel(ref["V"], inst["V"]) > 1e-3


def test_outer_loop_short_and_cyclic_orders(inst):
    perms = inst["perms"][:2]
    ref, _ = _run(inst, "f64", "calls", perms, 3)
    st, kern = _run(inst, "f64", "graph", perms, 3)
    assert kern == 0                       # three iterations: no graph
    assert st["value"] == pytest.approx(ref["value"], rel=1e-9)
    assert _rel(st["V"], ref["V"]) < 1e-9


def test_outer_loop_refuses_bad_orders(inst):
    from lagbound_b200._capi import LBError
    p = _problem(inst, "f32")
    bad = inst["perms"][:1].copy()
    bad[0, 0] = bad[0, 1]
    with pytest.raises(LBError):
        p.outer_loop(bad, RHO, TRI_W)
    p.close()
