"""Host side of the VCS working set between separations (vcsops.py:388-430 update_ws): the working set is a
row-CSR (ptr int64, col int32 ascending in each row) with sig FP64 and age uint8 per entry."""
from __future__ import annotations

import numpy as np


def merge_working_set(n, P, ptr, col, sig, age, keep, new_rows, new_cols):
    """Entries with keep False are dropped; the new entries (disjoint from the kept ones) join with sig 0 and age 0;
    every row stays sorted by cluster.  Returns (ptr, col, sig, age).  The kept entries are already in (row,
    cluster) order, so the new ones are placed by a binary search and one linear insertion."""
    ptr = np.asarray(ptr, np.int64)
    keep = np.asarray(keep, bool)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(ptr))
    kept_rows = rows[keep]
    kept_keys = kept_rows * int(P) + np.asarray(col, np.int64)[keep]
    new_rows = np.asarray(new_rows, np.int64)
    new_cols = np.asarray(new_cols, np.int64)
    new_keys = new_rows * int(P) + new_cols
    o = np.argsort(new_keys, kind="stable")
    new_keys, new_rows, new_cols = new_keys[o], new_rows[o], new_cols[o]
    at = np.searchsorted(kept_keys, new_keys)
    clash = at < len(kept_keys)
    if np.any(kept_keys[at[clash]] == new_keys[clash]) or np.any(new_keys[1:] == new_keys[:-1]):
        raise ValueError("new working-set entries repeat or overlap the kept ones")
    col_out = np.insert(np.asarray(col, np.int32)[keep], at, new_cols.astype(np.int32))
    sig_out = np.insert(np.asarray(sig, np.float64)[keep], at, 0.0)
    age_out = np.insert(np.asarray(age, np.uint8)[keep], at, 0)
    nptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(kept_rows, minlength=n) + np.bincount(new_rows, minlength=n), out=nptr[1:])
    return nptr, col_out.astype(np.int32), sig_out, age_out.astype(np.uint8)
