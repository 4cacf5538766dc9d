"""Continuous batching of bound requests (lagbound_b200.serving): each request's bound is the same alone and in the
mix (within 1e-4, the sweeps' atomics order being the only difference), admission respects the slots and the HBM
budget, and a request larger than the budget is refused."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(arrivals, **kw):
    from lagbound_b200 import synth
    from lagbound_b200.serving import BoundRequest
    out = []
    for k, t in enumerate(arrivals):
        n = [1200, 3000, 2000, 4000][k % 4]
        g = synth.chung_lu_communities(n, 12.0 + 4 * k, 2.3, n // 10, max(2, n // 150), 0.25, seed=40 + k)
        out.append(BoundRequest.from_graph(k, g, r=16, dtype="f32", outers=12, tri_every=4, eig_iters=60,
                                           arrival=t, **kw))
    return out


def _modularity(req):
    lab = np.unique(req.labels, return_inverse=True)[1]
    rows = np.repeat(np.arange(req.n), np.diff(req.indptr))
    inside = float((lab[rows] == lab[req.indices]).sum())
    vol = np.bincount(lab, weights=req.d)
    return inside / req.L - float((vol ** 2).sum()) / req.L ** 2


def test_bounds_alone_and_in_the_mix():
    from lagbound_b200.serving import BoundServer, latency_stats
    reqs = _requests([0.0, 0.05, 0.1, 0.15])
    alone = {}
    for q in reqs:
        res = BoundServer(0, slots=1).run([dataclasses.replace(q, arrival=0.0)])
        alone[q.rid] = res[0].ub
    mixed = BoundServer(0, slots=4).run(reqs)
    assert sorted(r.rid for r in mixed) == [0, 1, 2, 3]
    # the requests overlapped: some request was admitted before another finished
    done = {r.rid: r.done for r in mixed}
    assert any(r.admitted < min(done[o] for o in done if o != r.rid) for r in mixed)
    for r in mixed:
        assert abs(r.ub - alone[r.rid]) < 1e-4, (r.rid, r.ub, alone[r.rid])
        assert r.ub >= _modularity(reqs[r.rid]) - 1e-6 and r.ub < 1.0
    st = latency_stats(mixed)
    assert st["p99_s"] >= st["p50_s"] > 0 and st["requests"] == 4


def test_admission_by_memory_and_refusal():
    from lagbound_b200.serving import BoundServer
    reqs = _requests([0.0, 0.0, 0.0])
    needs = sorted(q.device_bytes() for q in reqs)
    need = needs[-1]
    budget = needs[0] + needs[1] - 1                # any one request fits, no two do
    assert budget >= need
    res = BoundServer(0, slots=3, hbm_budget=budget).run(reqs)
    res.sort(key=lambda r: r.admitted)
    for a, b in zip(res, res[1:]):               # one at a time: each admitted after the previous one finished
        assert b.admitted >= a.done - 1e-3
    with pytest.raises(RuntimeError, match="needs"):
        BoundServer(0, slots=2, hbm_budget=0.5 * need).run(_requests([0.0]))
