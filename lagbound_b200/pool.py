"""Triangle pool maintenance of the solver's main loop (host side; the separation itself runs on the GPU).

The pool holds normalised triples (min(a, c), b = centre, max(a, c)) with multipliers lam.  At a separation round
(alm_vcs.py:1735-1756) triangles with lam = 0 are purged, the new candidates of the one-edge-arm family keep the
best tri1_add by value and join the edge-arm family with its values raised by 10 (so that both budgets are kept),
candidates already pooled or repeated are dropped, and the best min(tri_add + tri1_add, room) join with lam = 0.
The sorts below use numpy's default (introsort) ordering, as the reference does: which of two equal values is kept
depends on it.
"""
from __future__ import annotations

import numpy as np


def tri_keys(TI, n):
    """(a n + b) n + c in int64 arithmetic (wrapping as the reference's numpy arithmetic does for n^3 > 2^63)."""
    TI = np.asarray(TI, np.int64).reshape(-1, 3)
    with np.errstate(over="ignore"):
        return (TI[:, 0] * n + TI[:, 1]) * n + TI[:, 2]


def purge(TI, lam):
    """Drop triangles whose multiplier is zero (alm_vcs.py:1738)."""
    keep = np.asarray(lam) > 0
    return np.asarray(TI, np.int64).reshape(-1, 3)[keep], np.asarray(lam, np.float64)[keep]


def merge(n, TI, lam, new0, val0, new1, val1, tri_add, tri1_add, room):
    """Merge separated candidates into the (purged) pool; returns (TI, lam, number added)."""
    new = np.asarray(new0, np.int64).reshape(-1, 3)
    val = np.asarray(val0, np.float64)
    if tri1_add:
        new1 = np.asarray(new1, np.int64).reshape(-1, 3)
        if len(new1):
            best1 = np.argsort(-np.asarray(val1, np.float64))[:tri1_add]
            new = np.vstack([new, new1[best1]])
            val = np.concatenate([val + 10.0, np.asarray(val1, np.float64)[best1]])
    if not len(new):
        return TI, lam, 0
    kn = tri_keys(new, n)
    pooled = np.sort(tri_keys(TI, n))
    at = np.searchsorted(pooled, kn)
    fresh = np.ones(len(kn), bool)
    inside = at < len(pooled)
    fresh[inside] = pooled[at[inside]] != kn[inside]
    new, val, kn = new[fresh], val[fresh], kn[fresh]
    first = np.unique(kn, return_index=True)[1]
    new, val = new[first], val[first]
    best = np.argsort(-val)[:min(tri_add + tri1_add, room)]
    new = new[best]
    return np.vstack([TI, new]), np.concatenate([lam, np.zeros(len(new))]), len(new)


def normalise(TI, lam, n):
    """Checkpoint triangles to (min(a, c), b, max(a, c)), duplicates merged by summing lam (alm_vcs.py:1188-1191)."""
    TI = np.asarray(TI, np.int64).reshape(-1, 3)
    lam = np.asarray(lam, np.float64)
    if not len(TI):
        return TI, lam, False
    TI = np.stack([np.minimum(TI[:, 0], TI[:, 2]), TI[:, 1], np.maximum(TI[:, 0], TI[:, 2])], 1)
    _, first, inv = np.unique(tri_keys(TI, n), return_index=True, return_inverse=True)
    if len(first) < len(TI):
        return TI[first], np.bincount(inv, weights=lam), True
    return TI, lam, False
