"""Host side of the VCS working set between separations (vcsops.py:388-430 update_ws): the working set is a
row-CSR (ptr int64, col int32 ascending in each row) with sig FP64 and age uint8 per entry."""
from __future__ import annotations

import numpy as np


def merge_working_set(n, P, ptr, col, sig, age, keep, new_rows, new_cols):
    """Entries with keep False are dropped; the new entries (disjoint from the kept ones) join with sig 0 and age 0;
    every row stays sorted by cluster.  Returns (ptr, col, sig, age)."""
    ptr = np.asarray(ptr, np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ptr))
    keep = np.asarray(keep, bool)
    r = np.concatenate([rows[keep], np.asarray(new_rows, np.int64)])
    c = np.concatenate([np.asarray(col, np.int64)[keep], np.asarray(new_cols, np.int64)])
    key = r * int(P) + c
    o = np.argsort(key, kind="stable")
    if len(key) > 1 and np.any(key[o][1:] == key[o][:-1]):
        raise ValueError("new working-set entries overlap the kept ones")
    s = np.concatenate([np.asarray(sig, np.float64)[keep], np.zeros(len(new_rows))])[o]
    a = np.concatenate([np.asarray(age, np.uint8)[keep], np.zeros(len(new_rows), np.uint8)])[o]
    nptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(r, minlength=n), out=nptr[1:])
    return nptr, c[o].astype(np.int32), s, a
