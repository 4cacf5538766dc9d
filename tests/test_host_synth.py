"""The synthetic instance generators stand in for the benchmark graphs: check the batched shape's ranges (graph
sizes, ranks, mean degrees) and the simple-graph invariants of what they return."""
import numpy as np


def test_batch_graphs_follow_the_batched_shape():
    from lagbound_b200 import synth
    out = synth.batch_graphs(8, seed=3)
    assert len(out) == 8
    for k, (g, r) in enumerate(out):
        assert r in (8, 16, 32)
        assert 400 <= g.n <= 50_000                      # isolated vertices dropped from n in [500, 50000]
        deg = np.diff(g.indptr)
        assert deg.min() >= 1 and 3.0 <= deg.mean() <= 42.0
        rows = np.repeat(np.arange(g.n), deg)
        assert np.all(rows != g.indices)                # no self-loops
        key = rows * g.n + g.indices
        assert len(np.unique(key)) == len(key)          # no duplicate edges
        assert np.all(np.diff(g.indices[g.indptr[0]:g.indptr[1]]) > 0)
        assert g.L == float(len(g.indices)) and g.labels is not None and len(g.labels) == g.n
