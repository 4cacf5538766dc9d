"""The nested-dissection ordering (lb_nd_order) that stands in for pymetis in the reference's certificate and
verifier (src/lagbound/_core/certify_lifted_vc.py:247-251, verify_cert.py:353-356): a valid permutation and its
inverse, deterministic, robust to self loops, duplicates, isolated vertices and disconnected graphs, and a factor
fill well below reverse Cuthill-McKee (the ordering the verifier falls back to) on meshes and power-law graphs.  The
fill is counted symbolically (lb_chol_fill) and checked against SciPy's dense Cholesky pattern on a small graph."""
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

from lagbound_b200 import _capi as C

DROPIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "lagbound_b200", "dropin")


def nd(A):
    A = A.tocsr()
    ip = A.indptr.astype(np.int64); ix = A.indices.astype(np.int64)
    n = A.shape[0]
    perm = np.empty(n, np.int64); iperm = np.empty(n, np.int64)
    C.call("lb_nd_order", n, C.ptr(ip), C.ptr(ix), C.ptr(perm), C.ptr(iperm))
    return perm, iperm


def fill(A, perm):
    A = A.tocsr()
    ip = A.indptr.astype(np.int64); ix = A.indices.astype(np.int64); pm = np.ascontiguousarray(perm, np.int64)
    out = np.zeros(1, np.int64)
    C.call("lb_chol_fill", A.shape[0], C.ptr(ip), C.ptr(ix), C.ptr(pm), 0, C.ptr(out))
    return int(out[0])


def sym(n, u, v):
    return sp.csr_matrix((np.ones(2 * len(u)), (np.r_[u, v], np.r_[v, u])), shape=(n, n))


def grid(k):
    idx = np.arange(k * k).reshape(k, k)
    return sym(k * k, np.r_[idx[:, :-1].ravel(), idx[:-1, :].ravel()], np.r_[idx[:, 1:].ravel(), idx[1:, :].ravel()])


def check_perm(perm, iperm, n):
    assert np.array_equal(np.sort(perm), np.arange(n))
    assert np.array_equal(iperm[perm], np.arange(n))


def test_fill_count_matches_dense_cholesky_pattern():
    rng = np.random.default_rng(3)
    n = 60
    u = rng.integers(0, n, 150); v = rng.integers(0, n, 150)
    A = sym(n, u[u != v], v[u != v])
    perm = rng.permutation(n)
    B = A[perm][:, perm].toarray() != 0
    M = B * 1.0 + np.eye(n) * (n + 1.0)            # diagonally dominant with A's pattern: no cancellation in L
    L = np.linalg.cholesky(M)
    assert fill(A, perm) == int((np.abs(L) > 0).sum())


@pytest.mark.parametrize("k", [30, 120])
def test_grid_fill_far_below_rcm(k):
    A = grid(k)
    perm, iperm = nd(A)
    check_perm(perm, iperm, k * k)
    f_nd = fill(A, perm)
    f_rcm = fill(A, reverse_cuthill_mckee(A, symmetric_mode=True))
    assert f_nd < (0.6 if k > 50 else 0.9) * f_rcm, (f_nd, f_rcm)


def test_power_law_fill_below_rcm_and_deterministic():
    from lagbound_b200 import synth
    g = synth.chung_lu_communities(20_000, 13.0, 2.1, 1500, 200, 0.3, seed=2)
    A = sp.csr_matrix((np.ones(g.nnz), g.indices, g.indptr), shape=(g.n, g.n))
    perm, iperm = nd(A)
    check_perm(perm, iperm, g.n)
    assert np.array_equal(perm, nd(A)[0])
    assert fill(A, perm) < 0.6 * fill(A, reverse_cuthill_mckee(A, symmetric_mode=True))


def test_degenerate_inputs():
    for n in (0, 1, 2):
        perm, iperm = nd(sp.csr_matrix((n, n)))
        check_perm(perm, iperm, n)
    # self loops, duplicate entries, an unsymmetric pattern, isolated vertices and several components
    rows = np.array([0, 0, 0, 1, 3, 3, 5, 6, 7, 8, 8])
    cols = np.array([0, 1, 1, 2, 4, 3, 6, 7, 5, 9, 9])
    A = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(12, 12))
    A.sum_duplicates()
    perm, iperm = nd(A)
    check_perm(perm, iperm, 12)
    # a clique and a star: no useful separator
    for B in (sp.csr_matrix(np.ones((300, 300)) - np.eye(300)),
              sym(2000, np.zeros(1999, np.int64), np.arange(1, 2000))):
        perm, iperm = nd(B)
        check_perm(perm, iperm, B.shape[0])


def test_invalid_index_is_refused():
    ip = np.array([0, 1, 2], np.int64); ix = np.array([1, 5], np.int64)
    perm = np.empty(2, np.int64)
    with pytest.raises(C.LBError, match="outside"):
        C.call("lb_nd_order", 2, C.ptr(ip), C.ptr(ix), C.ptr(perm), None)


def test_pymetis_dropin_module():
    sys.path.insert(0, DROPIN)
    try:
        import pymetis
        assert os.path.dirname(os.path.dirname(pymetis.__file__)) == DROPIN
        A = grid(40)
        perm, iperm = pymetis.nested_dissection(pymetis.CSRAdjacency(A.indptr, A.indices))
        check_perm(np.asarray(perm), np.asarray(iperm), 1600)
        assert np.array_equal(perm, nd(A)[0])
    finally:
        sys.path.remove(DROPIN)
        sys.modules.pop("pymetis", None)
