"""Batched problems (several graphs in one block-diagonal CSR, evaluated in the same launches): every graph's value,
primal, quadA, |d^T V|^2, triangle term and gradient rows agree with the graph evaluated alone and with the FP64
oracle; results are identical from run to run; inputs that would couple two graphs are refused."""
import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import rel

pytestmark = pytest.mark.gpu
RHO, TW = 0.02, 1.0


@pytest.fixture(scope="module")
def ctx():
    from lagbound_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _graphs(seed=0, count=7):
    from lagbound_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(300), np.log(8000))))
        if k % 2 == 0:
            g = synth.sbm(n, max(2, n // 200), min(0.5, 12.0 / 200), 2.0 / n, seed=seed + k)
        else:
            g = synth.chung_lu_communities(n, float(rng.uniform(5, 30)), 2.3, max(50, n // 10), max(2, n // 120), 0.25,
                                           seed=seed + k)
        out.append(g)
    return out


def _triangles(graphs, offsets, per_node=3, seed=5):
    from lagbound_b200 import synth
    TI, lam = [], []
    for k, g in enumerate(graphs):
        t = synth.wedge_triples(g, per_node * g.n, seed=seed + k)
        TI.append(t + offsets[k]); lam.append(synth.tri_multipliers(len(t), seed=seed + k))
    return np.concatenate(TI), np.concatenate(lam)


@pytest.mark.parametrize("dtype", ["f64", "f32", "bf16"])
def test_batched_matches_graphs_alone_and_oracle(ctx, dtype):
    from lagbound_b200 import BatchedProblem, Problem, synth
    graphs = _graphs(1)
    r = 16
    orders = None if dtype == "f64" else [np.random.default_rng(k).permutation(g.n) for k, g in enumerate(graphs)]
    bp = BatchedProblem(ctx, graphs, r, dtype, orders=orders)
    V = synth.random_V(bp.n, r, seed=3)
    bp.set_V(V)
    TI, lam = _triangles(graphs, bp.offsets)
    bp.set_triangles(TI, lam)
    bp.set_light_threshold(256)
    tot = bp.eval(RHO, TW, grad=True)
    per = bp.eval_graphs()
    Gb = bp.G()
    Vs = bp.get_V()
    tv = 1e-12 if dtype == "f64" else 1e-6
    for k, g in enumerate(graphs):
        a, b = bp.offsets[k], bp.offsets[k + 1]
        sel = (TI[:, 1] >= a) & (TI[:, 1] < b)
        p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, r, dtype,
                    order=None if orders is None else orders[k])
        p.set_V(V[a:b])
        p.set_triangles(TI[sel] - a, lam[sel])
        p.set_light_threshold(256)
        e = p.eval(RHO, TW, grad=True)
        # FP64 rows agree to rounding; FP32 accumulation follows the rows' edge offsets in the CSR (tile alignment),
        # which the concatenation shifts, so the reduced forms agree to FP32 rounding
        ta, tg = (1e-12, 1e-12) if dtype == "f64" else (1e-6, 2e-5)
        for key in ("value", "primal", "quadA", "zz", "tri_tot"):
            assert per[key][k] == pytest.approx(e[key], rel=ta, abs=ta * max(1.0, abs(e["primal"]))), (k, key)
        assert rel(Gb[a:b], p.G()) < tg, k
        p.close()
        inst = O.Instance(g.n, g.indptr, g.indices, g.data, g.d, g.L, g.C0)
        ref = O.evaluate(inst, Vs[a:b], [], TI[sel] - a, lam[sel], [], RHO, TW, 1.0)
        scale = max(abs(ref["value"]), 1.0)
        assert abs(per["value"][k] - ref["value"]) / scale < tv, k
        assert abs(per["primal"][k] - ref["primal"]) / scale < tv, k
        assert rel(Gb[a:b], ref["G"]) < (1e-11 if dtype == "f64" else 2e-5), k
    assert tot["value"] == pytest.approx(per["value"].sum(), rel=1e-12)
    assert tot["quadA"] == pytest.approx(per["quadA"].sum(), rel=1e-12)
    bp.close()


def test_evaluations_are_reproducible(ctx):
    """The row terms are summed per row and then in a fixed order: repeated evaluations agree bit for bit."""
    from lagbound_b200 import BatchedProblem, Problem, synth
    graphs = _graphs(2, count=4)
    bp = BatchedProblem(ctx, graphs, 32, "f32")
    bp.set_V(synth.random_V(bp.n, 32, seed=4))
    TI, lam = _triangles(graphs, bp.offsets, seed=9)
    bp.set_triangles(TI, lam)
    runs = [(bp.eval(RHO, TW, grad=True), bp.eval_graphs(), bp.G()) for _ in range(3)]
    for e, per, G in runs[1:]:
        assert e == runs[0][0]
        assert all(np.array_equal(per[k], runs[0][1][k]) for k in per)
        assert np.array_equal(G, runs[0][2])
    bp.close()
    g = graphs[1]
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, 32, "bf16")
    p.set_V(synth.random_V(g.n, 32, seed=6))
    first = p.eval(RHO, TW, grad=True)
    for _ in range(3):
        assert p.eval(RHO, TW, grad=True) == first
    p.close()


def test_batched_refuses_coupled_inputs(ctx):
    from lagbound_b200 import BatchedProblem, LBError, synth
    graphs = _graphs(3, count=3)
    bp = BatchedProblem(ctx, graphs, 8, "f32")
    o = bp.offsets
    with pytest.raises(LBError, match="spans two graphs"):
        bp.set_triangles(np.array([[0, 1, int(o[1])]]), np.ones(1))
    with pytest.raises(LBError, match="grouped by graph"):
        t1 = synth.wedge_triples(graphs[1], 5, seed=1) + o[1]
        t0 = synth.wedge_triples(graphs[0], 5, seed=1)
        bp.set_triangles(np.vstack([t1, t0]), np.ones(10))
    with pytest.raises(LBError, match="not supported on batched"):
        bp.add_pair_level(np.zeros(bp.n, np.int64), 1, 1.0)
    with pytest.raises(LBError, match="not supported on batched"):
        bp.sweeps(np.arange(bp.n)[None], RHO, RHO, 0.0, 4)
    bp.close()
    # an edge joining two graphs
    g0, g1 = graphs[0], graphs[1]

    class Joined:
        pass
    bad = Joined()
    bad.n = g0.n
    bad.indptr = g0.indptr.copy()
    bad.indices = g0.indices.copy()
    bad.indices[0] = g0.n + 1                     # points into the next graph
    bad.d, bad.L, bad.C0, bad.data = g0.d, g0.L, g0.C0, g0.data
    with pytest.raises(LBError, match="block diagonal"):
        BatchedProblem(ctx, [bad, g1], 8, "f32")


def test_captured_step_matches_direct_evaluations(ctx):
    """A CUDA graph of one batched step (one evaluation per rank group) replays to the same results as direct
    evaluations, bit for bit, and reads V as it is at replay time."""
    from lagbound_b200 import BatchedProblem, synth
    graphs = _graphs(4, count=6)
    groups = [graphs[0::2], graphs[1::2]]
    probs = []
    for k, grp in enumerate(groups):
        bp = BatchedProblem(ctx, grp, 8 * (k + 1), "f32")
        bp.set_V(synth.random_V(bp.n, 8 * (k + 1), seed=k))
        TI, lam = _triangles(grp, bp.offsets, seed=20 + k)
        bp.set_triangles(TI, lam)
        bp.eval(RHO, TW, grad=True)                   # first evaluation: autotune and allocations
        probs.append(bp)
    with ctx.capture() as g:
        for bp in probs:
            bp.eval_async(RHO, TW, grad=True)
    assert g.kernels >= 2 * 5
    for seed in (7, 8):
        for k, bp in enumerate(probs):
            bp.set_V(synth.random_V(bp.n, bp.r, seed=seed + 10 * k))
        g.launch()
        ctx.synchronize()
        replay = [(bp.eval_fetch(), bp.eval_graphs(), bp.G()) for bp in probs]
        direct = [(bp.eval(RHO, TW, grad=True), bp.eval_graphs(), bp.G()) for bp in probs]
        for (e1, p1, G1), (e2, p2, G2) in zip(replay, direct):
            assert e1 == e2
            assert all(np.array_equal(p1[k], p2[k]) for k in p1)
            assert np.array_equal(G1, G2)
    g.close()
    for bp in probs:
        bp.close()
