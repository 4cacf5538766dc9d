"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: the CPU oracle of the augmented-Lagrangian inner loop.

A restatement of the reference (Yahiahu/Lagbound) algorithm for this path: the FP64 kernels live in oracle.c
(loaded here through ctypes from oracle/liboracle.so, built by oracle/Makefile) and are composed here in the order of
the reference's driver code. Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this module; the
product package never does.

Pinned against golden fixtures produced by the reference itself (tests/golden/make_golden.py): see
tests/test_oracle_golden.py.

Citations are paths inside the reference project.
"""
from __future__ import annotations

import ctypes
import os
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_I = ctypes.c_int64
_D = ctypes.c_double
_lib = None


def build():
    """Compile oracle.c (gcc, -ffp-contract=off so per-row arithmetic matches the reference's Numba kernels)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "orc_spmm": (None, [_I, _I, _i64p, _i64p, _f64p, _f64p, _f64p]),
            "orc_quadA": (_D, [_I, _I, _i64p, _i64p, _f64p, _f64p, _f64p]),
            "orc_cluster_sums": (None, [_I, _I, _i64p, _f64p, _f64p, _I, _f64p]),
            "orc_dTV": (None, [_I, _I, _f64p, _f64p, _f64p]),
            "orc_pair_H": (None, [_I, _I, _f64p, _f64p, _f64p]),
            "orc_level_aug": (_D, [_I, _f64p, _f64p, _f64p, _D, _D, _f64p, ctypes.POINTER(_I)]),
            "orc_tri_aug": (_D, [_I, _I, _i64p, _f64p, _f64p, _D, _f64p, _f64p, ctypes.POINTER(_D)]),
            "orc_incidence": (None, [_I, _I, _i64p, _i64p, _i64p]),
            "orc_tri_apply": (None, [_I, _I, _i64p, _f64p, _i64p, _i64p, _f64p, _f64p]),
            "orc_vcs_aug": (None, [_I, _I, _f64p, _f64p, _i64p, _f64p, _i64p, _i32p, _f64p, _f64p, _D, _D, _f64p,
                                   _u8p, _f64p, ctypes.c_int, _f64p, _i64p]),
            "orc_vcs_apply": (None, [_I, _I, _I, _f64p, _f64p, _i64p, _i64p, _i32p, _f64p, _i64p, _f64p, _f64p,
                                     _f64p]),
            "orc_vcs_sigt": (None, [_I, _I, _f64p, _f64p, _i64p, _f64p, _i64p, _i32p, _f64p, _f64p, _D, _D, _f64p]),
            "orc_vcs_zinit": (None, [_I, _I, _I, _f64p, _f64p, _i64p, _i32p, _f64p, _f64p, _f64p]),
            "orc_vcs_pre": (None, [_I, _i64p, _I, _f64p, _f64p, _i64p, _f64p, _f64p, _i64p, _i32p, _f64p, _f64p,
                                   _i64p, _f64p, _f64p, _f64p, _D, _D, _D, _f64p, _f64p]),
            "orc_acc_rows": (None, [_I, _i64p, _I, _f64p, _f64p, _I, _I, _i64p, _i64p, _f64p]),
            "orc_vcs_post": (None, [_I, _i64p, _I, _f64p, _f64p, _f64p, _i64p, _f64p, _i64p, _i32p, _f64p, _f64p,
                                    _f64p, _D, _D, _f64p, _f64p]),
            "orc_pair_rows": (None, [_I, _i64p, _I, _I, _f64p, _f64p, _f64p, _f64p, _D, _D, _f64p, _f64p]),
            "orc_kq": (None, [_I, _f64p, _f64p, _f64p, _D, _f64p, _D, _f64p]),
            "orc_batch_step": (None, [_I, _i64p, _I, _I, _f64p, _f64p, _i64p, _i64p, _f64p, _f64p, _f64p, _D, _I,
                                      _i64p, _i64p, _f64p, _f64p, _f64p, _i64p, _i64p, _i64p, _f64p, _D, _D,
                                      ctypes.c_int, _f64p, _f64p, _f64p]),
            "orc_sep_candidates": (_I, [ctypes.c_int, _I, _I, _i64p, _i64p, _f64p, _D, _I, _I, _I, _I, _D, _I, _i64p,
                                        _f64p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------------------------------------- problem containers
class PairLevelData:
    """One cluster-pair level (aggops.py:51-68 PairLevel; rq per alm_vcs.py:1181-1184)."""

    def __init__(self, lab, d, sig=None, w=1.0):
        self.lab = np.unique(lab, return_inverse=True)[1].astype(np.int64)
        self.P = int(self.lab.max()) + 1
        cnt = np.bincount(self.lab, minlength=self.P).astype(float)
        vol = np.maximum(np.bincount(self.lab, weights=d, minlength=self.P), 1.0)
        self.rq = cnt / vol ** 2
        self.dsq = np.bincount(self.lab, weights=d * d, minlength=self.P)
        self.sig = np.zeros((self.P, self.P)) if sig is None else _c(sig, np.float64)
        self.w = float(w)


class VCSLevelData:
    """One sparse vertex-cluster level (vcsops.py:31-71 VCSLevel): row-CSR working set with int32 columns."""

    def __init__(self, lab, d, ptr, col, sig):
        self.lab = np.unique(lab, return_inverse=True)[1].astype(np.int64)
        self.P = int(self.lab.max()) + 1
        n = len(lab)
        cnt = np.bincount(self.lab, minlength=self.P).astype(float)
        self.vol = np.maximum(np.bincount(self.lab, weights=d, minlength=self.P), 1.0)
        self.rq = cnt / self.vol ** 2
        self.ptr = _c(ptr, np.int64)
        self.col = _c(col, np.int32)
        self.sig = _c(sig, np.float64)
        own = np.full(n, -1, np.int64)             # vcsops.py:83-91 own_entry
        rows = np.repeat(np.arange(n), np.diff(self.ptr))
        hit = np.flatnonzero(self.col == self.lab[rows])
        own[rows[hit[::-1]]] = hit[::-1]           # first matching entry of each row
        self.own = own

    @property
    def nnz(self):
        return int(self.ptr[-1])


class Instance:
    """CSR instance as alm_vcs.py:1103-1117 builds it (int64 indptr/indices, FP64 data, volumes d, L, C0)."""

    def __init__(self, n, indptr, indices, data, d, L, C0=0.0):
        self.n = int(n)
        self.indptr = _c(indptr, np.int64)
        self.indices = _c(indices, np.int64)
        self.data = _c(data, np.float64)
        self.d = _c(d, np.float64)
        self.L = float(L)
        self.C0 = float(C0)

    @classmethod
    def from_keys(cls, n, keys, weights=None, vol=None, L_orig=None, C0=0.0):
        import scipy.sparse as sp
        u = keys // n; v = keys % n; m = len(keys); L = 2 * m
        d = np.bincount(np.r_[u, v], minlength=n).astype(float)
        W_ = np.ones(m) if weights is None else weights
        A = sp.csr_matrix((np.r_[W_, W_], (np.r_[u, v], np.r_[v, u])), shape=(n, n))
        A.sort_indices()
        if vol is not None:
            d = vol.astype(float); L = int(L_orig)
        return cls(n, A.indptr, A.indices, A.data, d, L, C0)


# ------------------------------------------------------------------------------------------- primitives
def spmm(inst, X):
    X = _c(X, np.float64); out = np.empty_like(X)
    lib().orc_spmm(inst.n, X.shape[1], inst.indptr, inst.indices, inst.data, X, out)
    return out


def cluster_sums(lab, d, V, P):
    V = _c(V, np.float64); out = np.zeros((P, V.shape[1]))
    lib().orc_cluster_sums(V.shape[0], V.shape[1], _c(lab, np.int64), _c(d, np.float64), V, P, out)
    return out


def incidence(n, TI):
    TI = _c(TI.reshape(-1, 3), np.int64)
    ptr = np.zeros(n + 1, np.int64); codes = np.empty(3 * len(TI), np.int64)
    lib().orc_incidence(n, len(TI), TI, ptr, codes)
    return ptr, codes


def tri_apply(n, TI, w, V, out):
    ptr, codes = incidence(n, TI)
    lib().orc_tri_apply(n, V.shape[1], _c(TI, np.int64), _c(w, np.float64), ptr, codes, _c(V, np.float64), out)


def vcs_apply(Lv, sig, X, d):
    X = _c(X, np.float64); n, k = X.shape; out = np.zeros_like(X)
    lib().orc_vcs_apply(n, k, Lv.P, X, _c(d, np.float64), Lv.lab, Lv.ptr, Lv.col, _c(sig, np.float64), Lv.own,
                        out, np.zeros((Lv.P, k)), np.zeros((Lv.P, k)))
    return out


def pair_H(Y, dsq):
    Y = _c(Y, np.float64); P, k = Y.shape; H = np.empty((P, P))
    lib().orc_pair_H(P, k, Y, _c(dsq, np.float64), H)
    return H


# ------------------------------------------------------------------------------------------- one evaluation
def evaluate(inst, V, plev=(), TI=None, lam=None, vlev=(), rho=0.02, tri_weight=1.0, wv=1.0, want_G=True):
    """One augmented-Lagrangian evaluation at fixed multipliers (alm_vcs.py:1496-1533 augmented()) plus the
    gradient G = C(y_eff) V at the effective multipliers (alm_vcs.py:1299-1312 CV with sig -> pp, lam -> pt,
    VCS sig -> ppv).  Returns a dict with value, primal, the per-term sums, effective multipliers and counts."""
    L_ = lib()
    V = _c(V, np.float64); n, k = V.shape
    TI = np.zeros((0, 3), np.int64) if TI is None else _c(TI, np.int64).reshape(-1, 3)
    lam = np.zeros(0) if lam is None else _c(lam, np.float64)
    z = np.zeros(k); L_.orc_dTV(n, k, inst.d, V, z)
    qA = L_.orc_quadA(n, k, inst.indptr, inst.indices, inst.data, V, np.empty(n))
    val0 = qA - float(z @ z) / inst.L
    val = val0
    out = dict(quadA=qA, zz=z, val0=val0)
    ltot, nviol, pps, Ys = [], [], [], []
    for Lv in plev:
        Y = cluster_sums(Lv.lab, inst.d, V, Lv.P); Ys.append(Y)
        H = pair_H(Y, Lv.dsq); pp = np.empty_like(H); nv = _I(0)
        tot = L_.orc_level_aug(Lv.P, H, Lv.sig, Lv.rq, Lv.w, rho, pp, ctypes.byref(nv))
        val -= tot; ltot.append(tot); nviol.append(nv.value); pps.append(pp)
    rt = rho * tri_weight
    T = len(TI); gt = np.empty(T); pt = np.empty(T); gmin = _D(np.inf); ttot = 0.0
    if T:
        ttot = L_.orc_tri_aug(T, k, TI, V, lam, rt, gt, pt, ctypes.byref(gmin)); val -= ttot
    vtot, vnv, ppvs, slks, stns = [], [], [], [], []
    for Lv in vlev:
        Yv = cluster_sums(Lv.lab, inst.d, V, Lv.P)
        ppv = np.empty(Lv.nnz); slk = np.empty(Lv.nnz, np.uint8); stn = np.empty(Lv.nnz)
        trow = np.empty(n); nrow = np.empty(n, np.int64)
        L_.orc_vcs_aug(n, k, V, inst.d, Lv.lab, Yv, Lv.ptr, Lv.col, Lv.sig, Lv.rq, wv, rho, ppv, slk, stn, 1, trow, nrow)
        tot = float(trow.sum()); val -= tot
        vtot.append(tot); vnv.append(int(nrow.sum())); ppvs.append(ppv); slks.append(slk); stns.append(stn)
    out.update(value=val + inst.C0, primal=val0 + inst.C0, level_tot=np.array(ltot), nviol=np.array(nviol, np.int64),
               tri_tot=ttot, gmin=gmin.value, gt=gt, pt=pt, vcs_tot=np.array(vtot), vcs_nviol=np.array(vnv, np.int64),
               pp=pps, ppv=ppvs, slack=slks, stn=stns, Y=Ys)
    if want_G:
        out["G"] = apply_C(inst, V, plev, pps, TI, pt, vlev, ppvs)
    return out


def apply_C(inst, X, plev=(), sigs=(), TI=None, w=None, vlev=(), vsigs=()):
    """C(y) X = A X - d (d^T X)/L + sum_l [d (sig_l Y_l)[lab] - diag(sig_l)[lab] d^2 X] + sum S_vc X + T(w) X
    (alm_vcs.py:1296-1312 CV; est_dual_vcs.py:227-242)."""
    X = _c(X, np.float64); n, k = X.shape
    out = spmm(inst, X)
    z = np.zeros(k); lib().orc_dTV(n, k, inst.d, X, z)
    out -= np.outer(inst.d, z) / inst.L
    d = inst.d
    for Lv, s in zip(plev, sigs):
        Y = cluster_sums(Lv.lab, d, X, Lv.P)
        out += d[:, None] * (s @ Y)[Lv.lab] - (np.diag(s)[Lv.lab] * d ** 2)[:, None] * X
    for Lv, s in zip(vlev, vsigs):
        out += vcs_apply(Lv, s, X, d)
    if TI is not None and len(TI):
        tri_apply(n, TI, w, X, out)
    return out


def candidate_value(inst, W, plev=(), TI=None, lam=None, vlev=(), mu_sum=0.0):
    """est_dual_vcs.py:244-246 value(): (C0 + sum lam - sum mu + sum_i (C W)_i . w_i)/L at fixed multipliers
    (triangles with lam = 0 dropped, est_dual_vcs.py:207)."""
    lam = np.zeros(0) if lam is None else np.asarray(lam)
    keep = lam > 0
    TIk = None if TI is None else np.asarray(TI)[keep]
    CW = apply_C(inst, W, plev, [Lv.sig for Lv in plev], TIk, lam[keep], vlev, [Lv.sig for Lv in vlev])
    g = np.einsum("ij,ij->i", CW, W)
    const = inst.C0 + float(lam.sum()) - mu_sum
    return (const + g.sum()) / inst.L, g, CW


def candidate_bound(dv, lmin_est, s, L):
    """est_dual_vcs.py:354-356: UB = dv + max(0, -lmin_est) sum(s) / L."""
    return dv + max(0.0, -lmin_est) * float(np.sum(s)) / L


# ------------------------------------------------------------------------------------------- row steps
def sweep_state(inst, V, plev, vlev, rho, wv):
    """Start-of-sweep state of sweeps() (alm_vcs.py:1368-1406): z, Y, Kq and the VCS stZ/Z/cnt (vcs_state)."""
    L_ = lib()
    V = _c(V, np.float64); n, k = V.shape; d = inst.d
    z = np.zeros(k); L_.orc_dTV(n, k, d, V, z)
    Ys, Kqs = [], []
    for Lv in plev:
        Y = cluster_sums(Lv.lab, d, V, Lv.P); Ys.append(Y)
        H = pair_H(Y, Lv.dsq); H = 0.5 * (H + H.T)
        kq = np.empty(Lv.P); L_.orc_kq(Lv.P, H, Lv.sig, Lv.rq, Lv.w, _c((Y * Y).sum(1), np.float64), rho, kq)
        Kqs.append(kq)
    vst = []
    for Lv in vlev:
        Yv = cluster_sums(Lv.lab, d, V, Lv.P)
        stZ = np.empty(Lv.nnz)
        L_.orc_vcs_sigt(n, k, V, d, Lv.lab, Yv, Lv.ptr, Lv.col, Lv.sig, Lv.rq, wv, rho, stZ)
        Z = np.empty((Lv.P, k)); cnt = np.empty(Lv.P)
        L_.orc_vcs_zinit(n, k, Lv.P, V, d, Lv.ptr, Lv.col, stZ, Z, cnt)
        vst.append(dict(Y=Yv, stZ=stZ, Z=Z, cnt=cnt))
    return dict(z=z, Y=Ys, Kq=Kqs, vcs=vst)


def pair_rows(Lv, Y, items, rho):
    """pair_all (alm_vcs.py:378-415) for the clusters `items` of one level at the current Y."""
    k = Y.shape[1]; M = np.zeros((Lv.P, k)); pdiag = np.zeros(Lv.P)
    lib().orc_pair_rows(len(items), _c(items, np.int64), Lv.P, k, _c(Y, np.float64), Lv.sig, Lv.rq, Lv.dsq, Lv.w,
                        rho, M, pdiag)
    return M, pdiag


def batch_step(inst, V, rows, plev, TI, lam, vlev, st, rho, tri_weight, wv, damp, kap2=1.0):
    """One batch of row steps in the Jacobi-within-batch form (alm_vcs.py:1408-1435 body for one batch, with
    batch_step6 256-351 per row).  `st` is the sweep state from sweep_state(); it is updated in place by the
    post-batch aggregate updates (_acc_rows, vcs_yupd, vcs_post).  Returns (Vnew, DD, parts)."""
    L_ = lib()
    V = _c(V, np.float64); n, k = V.shape; d = inst.d
    rows = _c(rows, np.int64); nr = len(rows)
    nl = len(plev)
    labs = _c(np.array([Lv.lab for Lv in plev], np.int64).reshape(nl, n), np.int64)
    Poff = np.r_[0, np.cumsum([Lv.P for Lv in plev])].astype(np.int64)
    GX = np.zeros((nr, k)); KX = np.zeros(nr)
    Vold = V[rows].copy()
    for Lv, s in zip(vlev, st["vcs"]):
        Y2 = _c(np.einsum("ij,ij->i", s["Y"], s["Y"]), np.float64)
        L_.orc_vcs_pre(nr, rows, k, V, d, Lv.lab, s["Y"], Y2, Lv.ptr, Lv.col, Lv.sig, s["stZ"], Lv.own, s["Z"],
                       s["cnt"], Lv.rq, wv, rho, kap2, GX, KX)
    Mall = np.zeros((int(Poff[-1]), k)); pdiag = np.zeros(int(Poff[-1])); Kq = np.zeros(int(Poff[-1]))
    for li, Lv in enumerate(plev):
        items = np.unique(Lv.lab[rows])
        M, pdg = pair_rows(Lv, st["Y"][li], items, rho)
        Mall[Poff[li]:Poff[li + 1]] = M; pdiag[Poff[li]:Poff[li + 1]] = pdg; Kq[Poff[li]:Poff[li + 1]] = st["Kq"][li]
    TI = np.zeros((0, 3), np.int64) if TI is None else _c(TI, np.int64).reshape(-1, 3)
    tptr, tcodes = incidence(n, TI)
    Vnew = V.copy(); DD = np.zeros((nr, k))
    L_.orc_batch_step(nr, rows, n, k, V, Vnew, inst.indptr, inst.indices, inst.data, d, _c(st["z"], np.float64),
                      inst.L, nl, labs if nl else np.zeros(1, np.int64), Poff, Mall if nl else np.zeros(1),
                      pdiag if nl else np.zeros(1), Kq if nl else np.zeros(1), tptr, tcodes, TI,
                      _c(lam if lam is not None else np.zeros(0), np.float64), rho * tri_weight, damp,
                      int(bool(vlev)), GX, KX, DD)
    parts = dict(GX=GX, KX=KX, Mall=Mall, pdiag=pdiag, Kq=Kq)
    # post-batch updates (alm_vcs.py:1425-1435)
    Ycat = np.concatenate(st["Y"]) if nl else np.zeros((0, k))
    L_.orc_acc_rows(nr, rows, k, DD, st["z"], nl, n, labs if nl else np.zeros(1, np.int64), Poff,
                    Ycat if nl else np.zeros(1))
    for li in range(nl):
        st["Y"][li][...] = Ycat[Poff[li]:Poff[li + 1]]
    for Lv, s in zip(vlev, st["vcs"]):
        for idx, i in enumerate(rows):             # vcs_yupd (vcsops.py:159-164), batch order
            s["Y"][Lv.lab[i]] += DD[idx]
        L_.orc_vcs_post(nr, rows, k, Vnew, _c(Vold, np.float64), d, Lv.lab, s["Y"], Lv.ptr, Lv.col, Lv.sig, s["stZ"],
                        Lv.rq, wv, rho, s["Z"], s["cnt"])
    return Vnew, DD, parts


# ------------------------------------------------------------------------------------------- separation
def _sep_family(family, inst, V, thresh, maxh, maxk, hub2, cap2, vtol, cap, nchunk=512, nb=2000):
    """separate_ref / separate1_ref (alm_vcs.py:965-984): histogram threshold, per-chunk counts, generation-order
    collection with caps, keep val > 0."""
    V = _c(V, np.float64); n, k = V.shape
    L_ = lib()
    buf = 1 << 16
    while True:
        tri = np.empty((buf, 3), np.int64); val = np.empty(buf)
        tot = L_.orc_sep_candidates(family, n, k, inst.indptr, inst.indices, V, thresh, maxh, maxk, hub2, cap2, vtol,
                                    buf, tri, val)
        if tot <= buf:
            tri = tri[:tot]; val = val[:tot]; break
        buf = int(tot)
    cs = (n + nchunk - 1) // nchunk
    ch = tri[:, 1] // cs
    bins = np.minimum(((val - vtol) / (2.0 - vtol) * nb).astype(np.int64), nb - 1)
    hist = np.zeros((nchunk, nb), np.int64)
    np.add.at(hist, (ch, bins), 1)
    cum = np.cumsum(hist.sum(0)[::-1])[::-1]
    ok = np.flatnonzero(cum <= cap)
    b0 = ok[0] if len(ok) else nb
    if b0 >= nb:
        return np.zeros((0, 3), np.int64), np.zeros(0)
    vmin = vtol + (2.0 - vtol) * b0 / nb
    counts = hist[:, b0:].sum(1)
    sel = val >= vmin
    # within each chunk keep the first counts[ch] candidates with vm >= vmin, in generation order
    rank = np.zeros(len(val), np.int64)
    if len(val):
        cs_ = ch[sel]
        r_ = np.arange(len(cs_)) - np.searchsorted(cs_, cs_, side="left")
        rank[np.flatnonzero(sel)] = r_
    keep = sel & (rank < counts[ch])
    return tri[keep], val[keep]


def separate(inst, V, thresh=0.3, maxh=100, vtol=1e-3, cap=0, nchunk=512, nb=2000):
    """Edge-arm wedge separation (alm_vcs.py:961-963, reference semantics of separate_ref 965-974)."""
    return _sep_family(0, inst, V, thresh, maxh, 0, 0, 0, vtol, cap, nchunk, nb)


def separate_both(inst, V, thresh, maxh, maxk, hub2, cap2, vtol, cap0, cap1, nchunk=512, nb=2000):
    """alm_vcs.py:938-954: (separate, separate1) in one call."""
    return (_sep_family(0, inst, V, thresh, maxh, maxk, hub2, cap2, vtol, cap0, nchunk, nb),
            _sep_family(1, inst, V, thresh, maxh, maxk, hub2, cap2, vtol, cap1, nchunk, nb))


def pool_merge(n, TI, lam, new, val, n1, v1, tri_add, tri1_add, room):
    """Main-loop pool merge (alm_vcs.py:1748-1756): tri1 candidates (values shifted by +10 on the edge family to keep
    both budgets), drop those already pooled, dedupe by key, keep the best min(tri_add + tri1_add, room)."""
    if tri1_add and len(n1):
        o1 = np.argsort(-v1, kind="stable")[:tri1_add]
        new = np.vstack([new, n1[o1]]); val = np.r_[val + 10.0, v1[o1]]
    if len(new):
        kn = (new[:, 0] * n + new[:, 1]) * n + new[:, 2]
        ex = np.sort((TI[:, 0] * n + TI[:, 1]) * n + TI[:, 2])
        pos = np.searchsorted(ex, kn); isnew = np.ones(len(kn), bool); ok = pos < len(ex)
        isnew[ok] = ex[pos[ok]] != kn[ok]
        new, val, kn = new[isnew], val[isnew], kn[isnew]
        _, fi = np.unique(kn, return_index=True); new, val = new[fi], val[fi]
        o = np.argsort(-val, kind="stable")[:min(tri_add + tri1_add, room)]; new = new[o]
        TI = np.vstack([TI, new]); lam = np.r_[lam, np.zeros(len(new))]
    return TI, lam


# ------------------------------------------------------------------------------------------- exact reduction
def reduce_exact(n, keys):
    """reduce_exact.py:1-50: leaf unions (degree-1 endpoint), true-twin unions (adjacent, N[u] = N[v], d^2 < 2m,
    d > 1), union-find with the smaller root kept (so every group is numbered by the rank of its minimum member),
    reduced keys/weights (edge counts between groups), volumes, C0 = #edges inside groups.  The reference's random
    hash only filters twin candidates before the exact neighbourhood comparison, so it does not enter the result."""
    keys = np.asarray(keys, np.int64)
    u = keys // n; v = keys % n; m = len(keys); L = 2 * m
    d = np.bincount(np.r_[u, v], minlength=n)
    import scipy.sparse as sp
    A = sp.csr_matrix((np.ones(2 * m, np.int8), (np.r_[u, v], np.r_[v, u])), shape=(n, n)); A.sort_indices()
    par = np.arange(n)

    def find(x):
        r = x
        while par[r] != r: r = par[r]
        while par[x] != r: par[x], x = r, par[x]
        return r

    def union(a, b):
        ra, rb = find(a), find(b)
        if ra != rb: par[max(ra, rb)] = min(ra, rb)

    leaf = (d[u] == 1) | (d[v] == 1)
    for a, b in zip(u[leaf], v[leaf]): union(a, b)
    cand = (d[u] == d[v]) & (d[u].astype(float) ** 2 < 2 * m) & (d[u] > 1)
    nT = 0
    for a, b in zip(u[cand], v[cand]):
        Na = set(A.indices[A.indptr[a]:A.indptr[a + 1]].tolist()) | {a}
        Nb = set(A.indices[A.indptr[b]:A.indptr[b + 1]].tolist()) | {b}
        if Na == Nb: union(a, b); nT += 1
    root = np.array([find(x) for x in range(n)]); _, grp = np.unique(root, return_inverse=True)
    N = int(grp.max()) + 1
    vol = np.bincount(grp, weights=d, minlength=N).astype(np.int64)
    gu, gv = grp[u], grp[v]; inside = gu == gv; C0e = int(inside.sum())
    a_ = np.minimum(gu[~inside], gv[~inside]); b_ = np.maximum(gu[~inside], gv[~inside])
    kk, w = np.unique(a_ * N + b_, return_counts=True)
    return dict(n=N, keys=kk.astype(np.int64), weights=w.astype(np.float64), vol=vol, group_of=grp.astype(np.int64),
                L_orig=L, leaf_edges=C0e, leaf_unions=int(leaf.sum()), twin_unions=nT)


def vcs_separate(V, d, lab, ptr, col, wv, nadd, tol, mode):
    """vcsops.py:333-414 (_sep_rows, separate): candidates (i, R) outside the working set with mean violation
    s'/vol(R minus i) < -tol, scored pen / mean / mass; the nadd best by score (ties: row, cluster ascending).
    Returns (rows, cols, scores) best first and the statistics (nviol, mass, nviol_ws, mass_ws)."""
    V = np.asarray(V, np.float64); d = np.asarray(d, np.float64); lab = np.unique(lab, return_inverse=True)[1]
    n = len(d); P = int(lab.max()) + 1
    vol = np.maximum(np.bincount(lab, weights=d, minlength=P), 1.0)
    rq = np.bincount(lab, minlength=P) / vol ** 2
    Y = np.zeros((P, V.shape[1])); np.add.at(Y, lab, d[:, None] * V)
    G = V @ Y.T
    own = lab[:, None] == np.arange(P)[None, :]
    s = G - np.where(own, d[:, None], 0.0)
    vR = vol[None, :] - np.where(own, d[:, None], 0.0)
    ok = vR > 0
    xb = np.where(ok, s / np.where(ok, vR, 1.0), 0.0)
    viol = ok & (xb < -tol)
    inws = np.zeros((n, P), bool)
    rows_ws = np.repeat(np.arange(n), np.diff(ptr)); inws[rows_ws, np.asarray(col, np.int64)] = True
    mass = -d[:, None] * s
    stats = np.array([viol.sum(), mass[viol].sum(), (viol & inws).sum(), mass[viol & inws].sum()], np.float64)
    cand = viol & ~inws
    ci, cR = np.nonzero(cand)
    sv = s[ci, cR]
    sc = {"pen": wv * rq[cR] * sv * sv, "mean": -xb[ci, cR], "mass": -d[ci] * sv}[mode]
    pos = sc > 0
    ci, cR, sc = ci[pos], cR[pos], sc[pos]
    o = np.lexsort((cR, ci, -sc))[:nadd]
    return ci[o].astype(np.int64), cR[o].astype(np.int32), sc[o], stats


def vcs_update_ws(n, ptr, col, sig, age, keep, ni, nR):
    """vcsops.py:388-430 (_merge, update_ws): drop entries with keep False, add (ni, nR) with sig 0 and age 0,
    every row sorted by cluster."""
    rows = np.repeat(np.arange(n), np.diff(ptr))
    r = np.r_[rows[keep], np.asarray(ni, np.int64)]; c = np.r_[np.asarray(col)[keep], np.asarray(nR, np.int64)]
    s = np.r_[np.asarray(sig)[keep], np.zeros(len(ni))]; a = np.r_[np.asarray(age)[keep], np.zeros(len(ni), np.uint8)]
    o = np.lexsort((c, r))
    nptr = np.r_[0, np.cumsum(np.bincount(r, minlength=n))].astype(np.int64)
    return nptr, c[o].astype(np.int32), s[o], a[o].astype(np.uint8)


def simple_graph(pairs, n_names=None):
    """graph.py:71-100 _from_pairs on integer pairs: names = sorted distinct ids (or range(n_names) when the pairs
    already index a name list), self-loops dropped, keys a * n_all + b deduplicated and sorted, isolated nodes set
    aside, the rest renumbered in name order.  Returns (n, u, v, kept names, isolated names, self-loops)."""
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    if n_names is None:
        names, inv = np.unique(pairs.ravel(), return_inverse=True)
        pairs = inv.reshape(-1, 2)
    else:
        names = np.arange(n_names, dtype=np.int64)
    a = np.minimum(pairs[:, 0], pairs[:, 1]); b = np.maximum(pairs[:, 0], pairs[:, 1])
    keep = a != b
    a, b = a[keep], b[keep]
    n_all = len(names)
    keys = np.unique(a * n_all + b); a, b = keys // n_all, keys % n_all
    used = np.zeros(n_all, bool); used[a] = True; used[b] = True
    new_id = np.cumsum(used) - 1
    return (int(used.sum()), new_id[a].astype(np.int64), new_id[b].astype(np.int64), names[used].astype(np.int64),
            names[~used].astype(np.int64), int((~keep).sum()))


def restrict_labels(r, n, keys, lab):
    """reduce_exact.py:51-62 for one label file: every group takes the label of its first member (the smallest
    original vertex in it); returns (lr, Q original, Q with the rules enforced, Q reduced) with exact Fractions."""
    keys = np.asarray(keys, np.int64); lab = np.asarray(lab, np.int64)
    u = keys // n; v = keys % n; L = r["L_orig"]; grp = r["group_of"]; N = r["n"]
    d = np.bincount(np.r_[u, v], minlength=n)
    order = np.argsort(grp, kind="stable"); gs = grp[order]
    firsts = order[np.r_[True, gs[1:] != gs[:-1]]]
    lr = lab[firsts]; lab2 = lr[grp]; P = int(lab.max()) + 1
    volc = np.bincount(lab2, weights=d, minlength=P).astype(np.int64)
    Qo = Fraction(2 * int((lab2[u] == lab2[v]).sum()), L) - Fraction(sum(int(x) ** 2 for x in volc), L * L)
    kk, w = r["keys"], r["weights"]
    volr = np.bincount(lr, weights=r["vol"], minlength=P).astype(np.int64)
    ein_r = int(w[lr[kk // N] == lr[kk % N]].sum())
    Qr = Fraction(2 * r["leaf_edges"] + 2 * ein_r, L) - Fraction(sum(int(x) ** 2 for x in volr), L * L)
    vo = np.bincount(lab, weights=d, minlength=P).astype(np.int64)
    Qorig = Fraction(2 * int((lab[u] == lab[v]).sum()), L) - Fraction(sum(int(x) ** 2 for x in vo), L * L)
    return lr.astype(np.int64), Qorig, Qo, Qr


# ------------------------------------------------------------------------------------------- exact modularity
def modularity_exact(m, u, v, d, labels):
    """modularity.py:21-33: Q = inside/m - sum_c vol_c^2 / (4 m^2) as a Fraction."""
    lab = np.unique(np.asarray(labels), return_inverse=True)[1]
    inside = int((lab[u] == lab[v]).sum())
    volc = np.bincount(lab, weights=d).astype(np.int64)
    return Fraction(inside, m) - Fraction(sum(int(x) ** 2 for x in volc), 4 * m * m)


# ------------------------------------------------------------------------------------------- timed CPU sample
def timed_sample(inst, V, TI, lam, rho, tri_weight, frac, tptr=None, tcodes=None):
    """Times the oracle's FP64 evaluation (value + G, no levels) of one instance on a bounded sample and extrapolates
    to one full evaluation.  Pieces, in the order of augmented() + CV() (alm_vcs.py:1496-1533, 1299-1312):
      full:   z = d^T V over all rows, tri_aug over all triangles (pt, gt, PHR term);
      sample: rows [0, S) holding a fraction `frac` of the edges: their quadA terms, their rows of A V,
              the degree correction -d_i z / L and their triangle rows T(pt) V.
    Returns dict(seconds_per_eval, sample_seconds, rows, frac_edges)."""
    import time
    L_ = lib()
    V = _c(V, np.float64); n, k = V.shape
    TI = _c(TI, np.int64).reshape(-1, 3); lam = _c(lam, np.float64); T = len(TI)
    if tptr is None:
        tptr, tcodes = incidence(n, TI)
    nnz = int(inst.indptr[-1])
    S = int(np.searchsorted(inst.indptr, frac * nnz)) if frac < 1 else n
    S = max(1, min(n, S))
    fe = float(inst.indptr[S]) / max(nnz, 1)
    out = np.empty((S, k)); rowbuf = np.empty(S); gt = np.empty(T); pt = np.empty(T); gmin = _D(0.0)
    z = np.zeros(k)
    t0 = time.perf_counter()
    L_.orc_dTV(n, k, inst.d, V, z)
    if T:
        L_.orc_tri_aug(T, k, TI, V, lam, rho * tri_weight, gt, pt, ctypes.byref(gmin))
    t1 = time.perf_counter()
    L_.orc_quadA(S, k, inst.indptr, inst.indices, inst.data, V, rowbuf)
    L_.orc_spmm(S, k, inst.indptr, inst.indices, inst.data, V, out)
    out -= np.outer(inst.d[:S], z) / inst.L
    if T:
        L_.orc_tri_apply(S, k, TI, pt, tptr, tcodes, V, out)
    t2 = time.perf_counter()
    return dict(seconds_per_eval=(t1 - t0) + (t2 - t1) / fe, sample_seconds=t2 - t0, rows=S, frac_edges=fe)


def sweeps(inst, V, perms, nbatch, plev=(), TI=None, lam=None, vlev=(), rho=0.02, tri_weight=1.0, wv=1.0, damp=0.0,
           kap2=1.0):
    """Batched Gauss-Seidel sweeps (alm_vcs.py:1360-1436) in the Jacobi-within-batch form: for every permutation,
    the start-of-sweep state, then np.array_split(perm, nbatch) batches of batch_step with the post-batch updates."""
    V = _c(V, np.float64).copy()
    for perm in np.atleast_2d(perms):
        st = sweep_state(inst, V, plev, vlev, rho, wv)
        for rows in np.array_split(np.asarray(perm, np.int64), nbatch):
            if len(rows) == 0:
                continue
            Vnew, _, _ = batch_step(inst, V, rows, plev, TI, lam, vlev, st, rho, tri_weight, wv, damp, kap2)
            V[rows] = Vnew[rows]
    return V
