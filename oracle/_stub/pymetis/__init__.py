"""Test infrastructure: stand-in for the pymetis package (absent here) used by the reference's certificate and
verifier scripts only to choose an elimination order.  Any order is valid for them; this one is reverse
Cuthill-McKee from SciPy."""
import numpy as np


class CSRAdjacency:
    def __init__(self, indptr, indices):
        self.indptr = np.asarray(indptr, np.int64)
        self.indices = np.asarray(indices, np.int64)


def nested_dissection(adjacency):
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    n = len(adjacency.indptr) - 1
    A = sp.csr_matrix((np.ones(len(adjacency.indices)), adjacency.indices, adjacency.indptr), shape=(n, n))
    perm = np.asarray(reverse_cuthill_mckee(A, symmetric_mode=True), np.int64)
    iperm = np.empty(n, np.int64)
    iperm[perm] = np.arange(n)
    return perm, iperm
