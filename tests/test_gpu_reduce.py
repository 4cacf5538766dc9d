"""GPU exact reduction, simple-graph construction and exact modularity against the reference's golden outputs and
the oracle: bit-exact integers (keys, weights, volumes, group numbers, union counts, restricted labels) and equal
Fractions."""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

from oracle import oracle as O
from _fixtures import GOLDEN, reduce_names, graph_names

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from lagbound_b200 import Context
    c = Context(0)
    yield c
    c.close()


def _same_reduction(g, r):
    assert g.n == r["n"]
    assert np.array_equal(g.keys, r["keys"]) and np.array_equal(g.weights, r["weights"])
    assert np.array_equal(g.vol, r["vol"]) and np.array_equal(g.group_of, r["group_of"])
    assert g.L_orig == r["L_orig"] and g.inside_edges == r["leaf_edges"]
    assert g.leaf_unions == r["leaf_unions"] and g.twin_unions == r["twin_unions"]


@pytest.mark.parametrize("name", reduce_names())
def test_reduction_matches_reference(ctx, name):
    from lagbound_b200.reduce import reduce_exact
    z = np.load(os.path.join(GOLDEN, f"reduce_{name}.npz"))
    g = reduce_exact(ctx, int(z["n"]), z["keys"])
    _same_reduction(g, dict(n=int(z["rn"]), keys=z["rkeys"], weights=z["rweights"], vol=z["rvol"],
                            group_of=z["group_of"], L_orig=int(z["L_orig"]), leaf_edges=int(z["leaf_edges"]),
                            leaf_unions=int(z["leaf_unions"]), twin_unions=int(z["twin_unions"])))
    r = O.reduce_exact(int(z["n"]), z["keys"])
    for i in range(2):
        lr, Qorig, Qo, Qr = g.restrict_labels(z[f"lab{i}"])
        assert np.array_equal(lr, z[f"lr{i}"])
        assert Qo == Qr
        assert (Qorig, Qo, Qr) == O.restrict_labels(r, int(z["n"]), z["keys"], z[f"lab{i}"])[1:]
        assert np.array_equal(np.round([float(Qorig), float(Qo), float(Qr)], 6) + 0.0, z[f"q{i}"] + 0.0)
    g.close()


def leaves_twins_graph(n0, seed):
    """Sparse random graph plus stars of leaves, isolated edges and true-twin classes of sizes 2-5."""
    rng = np.random.default_rng(seed)
    e = set()
    while len(e) < 3 * n0:
        a, b = (int(x) for x in rng.integers(0, n0, 2))
        if a != b:
            e.add((min(a, b), max(a, b)))
    adj = {}
    for a, b in e:
        adj.setdefault(a, set()).add(b); adj.setdefault(b, set()).add(a)
    nxt = n0
    for hub in rng.choice(n0, n0 // 10, replace=False):             # leaves, 1-3 per hub
        for _ in range(int(rng.integers(1, 4))):
            e.add((int(hub), nxt)); nxt += 1
    for a in rng.choice(n0, n0 // 10, replace=False):               # true twins of existing vertices
        cls = [int(a)]
        for _ in range(int(rng.integers(1, 5))):
            t = nxt; nxt += 1
            for b in adj.get(int(a), ()):
                e.add((min(b, t), max(b, t)))
            for c in cls:
                e.add((c, t))
            cls.append(t)
    for _ in range(n0 // 50):                                         # isolated edges
        e.add((nxt, nxt + 1)); nxt += 2
    e = np.array(sorted(e), np.int64)
    # shuffle vertex names so that groups do not follow creation order
    perm = rng.permutation(nxt)
    a, b = perm[e[:, 0]], perm[e[:, 1]]
    keys = np.unique(np.minimum(a, b) * nxt + np.maximum(a, b))
    return nxt, keys


@pytest.mark.parametrize("n0,seed", [(300, 1), (5000, 2), (40000, 3)])
def test_reduction_matches_oracle(ctx, n0, seed):
    from lagbound_b200.reduce import reduce_exact
    n, keys = leaves_twins_graph(n0, seed)
    g = reduce_exact(ctx, n, keys)
    r = O.reduce_exact(n, keys)
    assert r["leaf_unions"] > 0 and r["twin_unions"] > 0
    _same_reduction(g, r)
    lab = np.random.default_rng(seed).integers(0, 17, n)
    lr, Qorig, Qo, Qr = g.restrict_labels(lab)
    lr_o, Qorig_o, Qo_o, Qr_o = O.restrict_labels(r, n, keys, lab)
    assert np.array_equal(lr, lr_o) and (Qorig, Qo, Qr) == (Qorig_o, Qo_o, Qr_o) and Qo == Qr
    g.close()


def test_reduction_keys_in_either_order(ctx):
    """The reference reads keys.npy as u * n + v without requiring u < v."""
    from lagbound_b200.reduce import reduce_exact
    n, keys = leaves_twins_graph(2000, 7)
    u, v = keys // n, keys % n
    flip = np.random.default_rng(0).random(len(keys)) < 0.5
    keys2 = np.where(flip, v * n + u, keys)
    g = reduce_exact(ctx, n, keys2)
    _same_reduction(g, O.reduce_exact(n, keys2))
    g.close()


def test_reduction_of_c2_shape_matches_oracle(ctx):
    """Chung-Lu with communities at n = 300,000 (mean degree 13, min degree 1: many leaves)."""
    from lagbound_b200 import synth
    from lagbound_b200.reduce import reduce_exact
    gr = synth.config_graph("c2", seed=0)
    n = gr.n
    rows = np.repeat(np.arange(n), np.diff(gr.indptr))
    up = rows < gr.indices
    keys = rows[up] * n + gr.indices[up]
    g = reduce_exact(ctx, n, keys)
    r = O.reduce_exact(n, keys)
    _same_reduction(g, r)
    # size-independent identities
    assert int(g.vol.sum()) == g.L_orig and int(g.weights.sum()) + g.inside_edges == len(keys)
    assert np.all(np.diff(g.keys) > 0)
    g.close()


def test_reduction_without_edges_and_invalid_input(ctx):
    from lagbound_b200 import LBError
    from lagbound_b200.reduce import reduce_exact
    g = reduce_exact(ctx, 5, np.zeros(0, np.int64))
    assert g.n == 5 and g.m == 0 and np.array_equal(g.group_of, np.arange(5)) and g.inside_edges == 0
    g.close()
    with pytest.raises(LBError):
        reduce_exact(ctx, 4, np.array([1, 1], np.int64))            # the same edge twice
    with pytest.raises(LBError):
        reduce_exact(ctx, 4, np.array([5], np.int64))               # self-loop 1-1
    with pytest.raises(LBError):
        reduce_exact(ctx, 4, np.array([16], np.int64))              # outside [0, n^2)


def test_modularity_matches_reference(ctx):
    from lagbound_b200.reduce import modularity
    for rec in json.load(open(os.path.join(GOLDEN, "modularity.json"))):
        q = modularity(ctx, rec["n"], rec["u"], rec["v"], rec["labels"], exact=True)
        assert q == Fraction(int(rec["num"]), int(rec["den"]))
        assert modularity(ctx, rec["n"], rec["u"], rec["v"], rec["labels"]) == float(q)


def test_modularity_large_matches_oracle(ctx):
    from lagbound_b200.reduce import modularity
    rng = np.random.default_rng(4)
    n, m = 200_000, 1_500_000
    u = rng.integers(0, n, m); v = rng.integers(0, n, m)
    keep = u != v; u, v = u[keep], v[keep]
    lab = rng.integers(-5, 3000, n) * 7          # arbitrary integer labels are compacted like the reference
    d = np.bincount(np.r_[u, v], minlength=n)
    assert modularity(ctx, n, u, v, lab, exact=True) == O.modularity_exact(len(u), u, v, d, lab)


@pytest.mark.parametrize("name", graph_names())
def test_simple_graph_matches_reference(ctx, name):
    from lagbound_b200.reduce import simple_graph
    z = np.load(os.path.join(GOLDEN, f"graph_{name}.npz"))
    nn = int(z["n_names"])
    g = simple_graph(ctx, z["pairs"], None if nn < 0 else list(range(nn)))
    assert g.n == int(z["n"]) and np.array_equal(g.u, z["u"]) and np.array_equal(g.v, z["v"])
    assert np.array_equal(np.asarray(g.labels, np.int64), z["labels"])
    assert np.array_equal(np.asarray(g.isolated, np.int64).reshape(-1), z["isolated"])


def test_simple_graph_large_matches_oracle(ctx):
    from lagbound_b200.reduce import simple_graph
    rng = np.random.default_rng(9)
    pairs = rng.integers(-10**9, 10**9, (400_000, 2)) // 1000
    pairs[::11, 1] = pairs[::11, 0]
    pairs = np.r_[pairs, pairs[:50_000, ::-1]]
    g = simple_graph(ctx, pairs)
    n, u, v, kept, iso, loops = O.simple_graph(pairs)
    assert g.n == n and np.array_equal(g.u, u) and np.array_equal(g.v, v) and g.self_loops == loops
    assert np.array_equal(np.asarray(g.labels), kept) and np.array_equal(np.asarray(g.isolated, np.int64), iso)


def test_simple_graph_errors(ctx):
    from lagbound_b200.reduce import simple_graph
    with pytest.raises(ValueError):
        simple_graph(ctx, np.zeros((0, 2), np.int64))
    with pytest.raises(ValueError):
        simple_graph(ctx, np.array([[3, 3], [4, 4]]))
