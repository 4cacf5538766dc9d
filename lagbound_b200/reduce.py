"""Exact graph reduction and exact modularity on the GPU (host side of lb_reduce_* / lb_modularity_counts).

reduce_exact() returns what src/lagbound/_core/reduce_exact.py:12-46 writes (graph.json n/m, keys, weights, vol,
group_of, meta.json), ReducedGraph.restrict_labels() what its label loop (51-62) writes and asserts, modularity()
follows src/lagbound/modularity.py:21-33.  Run as a script it is a drop-in for reduce_exact.py:

    python -m lagbound_b200.reduce <tag> [label files ...]

reading data/<tag>/{graph.json, keys.npy} and writing data/<tag>__rx/ with the same files and printed lines.
"""
from __future__ import annotations

import ctypes
import json
import os
import sys
from fractions import Fraction

import numpy as np

from . import _capi as C
from .problem import Context


class ReducedGraph:
    """Device-resident result of one exact reduction (lb_reduction handle)."""

    def __init__(self, ctx: Context, n, keys):
        self.ctx = ctx
        keys = C.c(keys, np.int64)
        h = ctypes.c_void_p()
        C.call("lb_reduce_exact", ctx.h, int(n), len(keys), C.ptr(keys), ctypes.byref(h))
        self.h = h
        info = np.zeros(7, np.int64)
        C.call("lb_reduce_info", self.h, C.ptr(info))
        self.n, self.m, self.L_orig, self.inside_edges, self.leaf_unions, self.twin_unions, self.n_orig = \
            (int(x) for x in info)
        self.keys = np.empty(self.m, np.int64)
        self.weights = np.empty(self.m, np.float64)
        self.vol = np.empty(self.n, np.int64)
        self.group_of = np.empty(self.n_orig, np.int64)
        C.call("lb_reduce_get", self.h, C.ptr(self.keys), C.ptr(self.weights), C.ptr(self.vol), C.ptr(self.group_of))

    def as_dict(self):
        """The oracle's / reference's result fields."""
        return dict(n=self.n, keys=self.keys, weights=self.weights, vol=self.vol, group_of=self.group_of,
                    L_orig=self.L_orig, leaf_edges=self.inside_edges, leaf_unions=self.leaf_unions,
                    twin_unions=self.twin_unions)

    def meta(self, m_orig):
        """meta.json of reduce_exact.py:42-43."""
        return {"L_orig": self.L_orig, "leaf_edges": self.inside_edges, "inside_edges": self.inside_edges,
                "n_orig": self.n_orig, "m_orig": int(m_orig), "leaf_unions": self.leaf_unions,
                "twin_unions": self.twin_unions}

    def restrict_labels(self, lab):
        """reduce_exact.py:51-62: the label of each group (its first member's), and the exact modularities
        (original, rules enforced, reduced) as Fractions; the last two must agree."""
        lab = C.c(lab, np.int64)
        if len(lab) != self.n_orig:
            raise ValueError(f"label file has {len(lab)} entries, graph has {self.n_orig} nodes")
        lr = np.empty(self.n, np.int64)
        cnt = np.zeros(6, np.int64)
        C.call("lb_reduce_labels", self.h, C.ptr(lab), C.ptr(lr), C.ptr(cnt))
        L = self.L_orig
        ein, s2, ein_r, s2_r, ein_o, s2_o = (int(x) for x in cnt)
        Qo = Fraction(2 * ein, L) - Fraction(s2, L * L)
        Qr = Fraction(2 * self.inside_edges + 2 * ein_r, L) - Fraction(s2_r, L * L)
        Qorig = Fraction(2 * ein_o, L) - Fraction(s2_o, L * L)
        return lr, Qorig, Qo, Qr

    def close(self):
        if getattr(self, "h", None):
            C.get_lib().lb_reduce_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reduce_exact(ctx: Context, n, keys) -> ReducedGraph:
    return ReducedGraph(ctx, n, keys)


class SimpleGraph:
    """The simple undirected graph of integer node pairs (graph.py:71-100 _from_pairs on the GPU): n, m, u < v in
    key order, labels (names of the kept nodes) and isolated (names set aside), as the reference's Graph holds."""

    def __init__(self, ctx: Context, pairs, names=None):
        pairs = np.asarray(pairs)
        if pairs.size == 0:
            raise ValueError("the graph has no edges")
        if pairs.ndim != 2 or pairs.shape[1] != 2:
            raise ValueError("edges must have shape (m, 2)")
        p = C.c(pairs, np.int64)
        h = ctypes.c_void_p()
        C.call("lb_simple_graph", ctx.h, len(p), C.ptr(p), -1 if names is None else len(names), ctypes.byref(h))
        try:
            info = np.zeros(5, np.int64)
            C.call("lb_graph_info", h, C.ptr(info))
            self.n, m, niso, self.self_loops, _ = (int(x) for x in info)
            self.u = np.empty(m, np.int64); self.v = np.empty(m, np.int64)
            kept = np.empty(self.n, np.int64); iso = np.empty(niso, np.int64)
            C.call("lb_graph_get", h, C.ptr(self.u), C.ptr(self.v), C.ptr(kept), C.ptr(iso))
        finally:
            C.get_lib().lb_graph_destroy(h)
        if self.n == 0:
            raise ValueError("the graph has no edges after removing self-loops")
        if names is None:
            self.labels, self.isolated = kept.tolist(), iso.tolist()
        else:
            self.labels = [names[i] for i in kept]; self.isolated = [names[i] for i in iso]

    @property
    def m(self):
        return len(self.u)

    @property
    def keys(self):
        """keys.npy of the stage scripts' data directory: u * n + v, ascending."""
        return self.u * self.n + self.v

    @property
    def degrees(self):
        return np.bincount(np.r_[self.u, self.v], minlength=self.n).astype(np.int64)


def simple_graph(ctx: Context, pairs, names=None) -> SimpleGraph:
    return SimpleGraph(ctx, pairs, names)


def modularity_counts(ctx: Context, n, u, v, labels):
    """(inside, sum of squared volumes) of a membership array over 0..n-1 (labels compacted as the reference's
    np.unique(return_inverse=True) does, so any integer labels are accepted)."""
    lab = np.unique(np.asarray(labels), return_inverse=True)[1].astype(np.int64)
    u = C.c(u, np.int64); v = C.c(v, np.int64)
    if len(lab) != int(n):
        raise ValueError(f"partition has {len(lab)} entries, graph has {n} nodes")
    ins = ctypes.c_int64(); s2 = ctypes.c_int64()
    C.call("lb_modularity_counts", ctx.h, int(n), len(u), C.ptr(u), C.ptr(v), C.ptr(lab), ctypes.byref(ins),
           ctypes.byref(s2))
    return int(ins.value), int(s2.value)


def modularity(ctx: Context, n, u, v, partition, exact=False):
    """modularity.py:21-33: Q = inside/m - sum_c vol_c^2 / (4 m^2); a Fraction when exact."""
    m = len(u)
    ins, s2 = modularity_counts(ctx, n, u, v, partition)
    q = Fraction(ins, m) - Fraction(s2, 4 * m * m)
    return q if exact else float(q)


def main(argv):
    """The command line of reduce_exact.py (usage: <tag> [label files ...])."""
    tag = argv[0]
    D = f"data/{tag}/"; Dz = f"data/{tag}__rx/"
    os.makedirs(Dz, exist_ok=True)
    n = json.load(open(D + "graph.json"))["n"]
    keys = np.load(D + "keys.npy")
    m = len(keys)
    ctx = Context(0)
    r = reduce_exact(ctx, n, keys)
    assert int(r.vol.sum()) == r.L_orig and int(r.weights.sum()) + r.inside_edges == m
    json.dump({"n": r.n, "m": r.m}, open(Dz + "graph.json", "w"))
    np.save(Dz + "keys.npy", r.keys)
    np.save(Dz + "weights.npy", r.weights)
    np.save(Dz + "vol.npy", r.vol)
    np.save(Dz + "group_of.npy", r.group_of)
    json.dump(r.meta(m), open(Dz + "meta.json", "w"))
    wmax = r.weights.max() if r.m else 0
    print(f"{tag}: n {n} -> {r.n} (leaf edges {r.leaf_unions}, twin pairs {r.twin_unions}), m {m} -> {r.m} weighted "
          f"(max w {wmax}), inside edges {r.inside_edges}, C0/L {2 * r.inside_edges / r.L_orig:.6f}")
    for f in argv[1:]:
        lr, Qorig, Qo, Qr = r.restrict_labels(np.load(f).astype(np.int64))
        assert Qo == Qr, (float(Qo), float(Qr))
        np.save(Dz + os.path.basename(f), lr)
        print(f"  {os.path.basename(f)}: original Q {float(Qorig):.6f}; with rules enforced {float(Qo):.6f} == "
              f"reduced {float(Qr):.6f} OK")
    r.close()
    ctx.close()


if __name__ == "__main__":
    main(sys.argv[1:])
