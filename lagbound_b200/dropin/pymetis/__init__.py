"""pymetis-compatible ordering for the reference's certificate and verifier.

The reference imports pymetis only for `pymetis.nested_dissection(pymetis.CSRAdjacency(indptr, indices))[0]`
(src/lagbound/_core/certify_lifted_vc.py:247-251, verify_cert.py:353-356) and accepts any symmetric ordering.  With
this directory on PYTHONPATH (lagbound_b200.stages.install() adds it to the certificate and verifier stages when no
pymetis is installed), those calls run this library's nested dissection (lb_nd_order: multilevel bisection, vertex
separators, minimum-degree leaves; native host code).
"""
import os
import sys

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
if _ROOT not in sys.path:
    sys.path.append(_ROOT)


class CSRAdjacency:
    """Adjacency in CSR form (as pymetis.CSRAdjacency: row offsets and column indices)."""

    def __init__(self, adj_starts, adjacent):
        self.adj_starts = np.ascontiguousarray(adj_starts, np.int64)
        self.adjacent = np.ascontiguousarray(adjacent, np.int64)


def nested_dissection(adjacency=None, options=None):
    """(perm, iperm) of a fill-reducing nested-dissection ordering: perm[k] is the vertex eliminated k-th, iperm its
    inverse (as pymetis.nested_dissection)."""
    from lagbound_b200 import _capi as C
    ip = adjacency.adj_starts
    ix = adjacency.adjacent
    n = len(ip) - 1
    perm = np.empty(max(n, 0), np.int64)
    iperm = np.empty(max(n, 0), np.int64)
    C.call("lb_nd_order", n, C.ptr(ip), C.ptr(ix), C.ptr(perm), C.ptr(iperm))
    return perm, iperm
