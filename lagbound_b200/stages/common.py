"""Shared pieces of the drop-in stage scripts: the DATA_DIR instance files and the log prefix."""
from __future__ import annotations

import json
import os
import resource
import sys
import time

import numpy as np


def data_dir():
    D = os.environ.get("DATA_DIR", "data/")
    return D if D.endswith("/") else D + "/"


def load_instance(tag, D=None):
    """DATA_DIR/<tag>/{graph.json, keys.npy[, weights.npy, vol.npy, meta.json]} as the stage scripts read them
    (alm_vcs.py:1103-1117, est_dual_vcs.py:171-180): symmetric CSR with ascending columns, edge weights (None when
    absent: unit), volumes d (degrees, or vol.npy of a reduced instance), L = 2 m (or L_orig) and C0 = 2 leaf_edges."""
    D = data_dir() if D is None else D
    n = int(json.load(open(D + tag + "/graph.json"))["n"])
    keys = np.load(D + tag + "/keys.npy").astype(np.int64)
    u = keys // n
    v = keys % n
    m = len(keys)
    L = 2 * m
    wpath = D + tag + "/weights.npy"
    w = np.load(wpath).astype(np.float64) if os.path.exists(wpath) else None
    rows = np.concatenate([u, v])
    cols = np.concatenate([v, u])
    order = np.argsort(rows * n + cols, kind="stable")
    indices = cols[order]
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=indptr[1:])
    data = None if w is None else np.concatenate([w, w])[order]
    d = np.bincount(rows, minlength=n).astype(np.float64)
    C0 = 0.0
    if os.path.exists(D + tag + "/vol.npy"):
        meta = json.load(open(D + tag + "/meta.json"))
        d = np.load(D + tag + "/vol.npy").astype(np.float64)
        L = int(meta["L_orig"])
        C0 = 2.0 * meta["leaf_edges"]
        assert int(d.sum()) == L
    if data is not None and np.all(data == 1.0):
        data = None
    return dict(n=n, m=m, L=L, C0=C0, d=d, indptr=indptr, indices=indices, weights=data)


class Logger:
    """The stage scripts' log prefix: elapsed seconds and peak resident set size (MB)."""

    def __init__(self, decimals=0):
        self.t0 = time.time()
        self.fmt = "{:8.%df}s" % decimals

    def rss(self):
        return resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / (2 ** 20 if sys.platform == "darwin" else 2 ** 10)

    def __call__(self, *s):
        print(f"[{self.fmt.format(time.time() - self.t0)} {self.rss():6.0f}MB]", *s, flush=True)
