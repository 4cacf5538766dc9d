#!/usr/bin/env python3
"""Generate the golden fixtures under tests/golden/ by running the REFERENCE implementation (Yahiahu/Lagbound).

Test infrastructure only: this script imports the reference from its source tree ($LAGBOUND_REF, or an importable
lagbound package from the reference project: oracle/refpath.py) and is run by hand in a container where that tree
exists, e.g. LAGBOUND_REF=<reference root> python tests/golden/make_golden.py. Its outputs (*.npz, *.json) are committed;
the tests read those and never the reference itself.

What it records (all citations are paths inside the reference project):

* eval_<name>.npz   -- one augmented-Lagrangian evaluation at a fixed (V, sigma, lam, VCS sigma, rho), composed only
                       from the reference's own Numba kernels in the order of ``augmented()``
                       (src/lagbound/_core/alm_vcs.py:1496-1533) and ``CV()`` (alm_vcs.py:1299-1312): value, primal,
                       per-term sums, effective multipliers pp / pt / ppv, violation counts and G = C(y_eff) V.
                       Also the fixed-multiplier (rho = 0) operator C(y) W and the candidate-bound pieces of
                       ``est_dual_vcs.value`` (src/lagbound/_core/est_dual_vcs.py:227-246).
                       Also one batch of row steps of ``batch_step6`` (alm_vcs.py:256-351) in the Jacobi-within-batch
                       form: every row of the batch is stepped by the reference kernel on its own copy of the
                       pre-batch V (rows=[i]), with the per-sweep Kq (``kq_level`` 417-428), the per-batch pair rows
                       (``pair_all`` 378-415) and the VCS pre-batch terms (``vcs_pre``, vcsops.py:127-156).
                       Then the post-batch aggregate updates (``_acc_rows`` 430-438, ``vcs_yupd``/``vcs_post``
                       vcsops.py:159-213) with one thread (deterministic order).
* sep_<name>.npz    -- triangle separation at a fixed V: ``separate`` (alm_vcs.py:961-963) and ``separate_both``
                       (alm_vcs.py:938-954), plus the pool merge of the main loop (alm_vcs.py:1735-1756) executed
                       from the reference file itself.
* reduce_<name>.npz -- ``reduce_exact.py`` run as a subprocess on small graphs with leaves and twins, with two
                       seeded label files (the restricted labels it writes and the modularities it prints).
* modularity.json   -- exact partition modularity (src/lagbound/modularity.py:21-33) as fractions.
* vsep_<name>.npz   -- VCS working-set separation (vcsops.py:364-414 separate) at a fixed V for the three scores,
                       with a small chunk size so that the sampled initial threshold and the buffer pruning run, and
                       the working-set merge that follows it in the main loop (update_ws, vcsops.py:417-430).
* init_<name>.npz   -- the solver's --init_partition start (alm_vcs.py:1198-1211, executed from the reference
                       file): greedy colouring of the cluster graph and V with its seeded noise.
* graph_<name>.npz  -- the simple graph of a pair list (src/lagbound/graph.py:71-100 _from_pairs through as_graph):
                       n, u, v, kept labels and isolated names, for pair lists with self-loops, reversed and repeated
                       pairs, nodes left isolated, negative and large ids.

Usage:  NUMBA_NUM_THREADS=1 python tests/golden/make_golden.py [--only eval|reduce|sep|vsep|init|graph|modularity]
"""
import json
import os
import re
import subprocess
import sys
import tempfile
import textwrap

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.refpath import reference_root  # noqa: E402

REF = reference_root()
CORE = os.path.join(REF, "src", "lagbound", "_core")
os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="lagbound_golden_numba_"))   # fresh: the kernels
# are compiled from an exec'd source, which Numba's on-disk cache cannot reload in a later process
os.environ.setdefault("NUMBA_NUM_THREADS", "1")
sys.path.insert(0, CORE)
sys.path.insert(0, os.path.join(REF, "src"))


def load_ref_kernels():
    """Execute the kernel section of alm_vcs.py (everything before its argparse block) under its real filename."""
    path = os.path.join(CORE, "alm_vcs.py")
    lines = open(path).read().split("\n")
    stop = next(i for i, l in enumerate(lines) if l.startswith("p = argparse.ArgumentParser"))
    ns = {"__name__": "lagbound_ref_kernels", "__file__": path}
    exec(compile("\n".join(lines[:stop]), path, "exec"), ns)
    return ns


K = load_ref_kernels()
import vcsops as VCS          # noqa: E402  (reference module)
from aggops import PairLevel  # noqa: E402  (reference module)


# ----------------------------------------------------------------------------------------------- instances
def sbm_keys(n, blocks, p_in, p_out, seed):
    rng = np.random.default_rng(seed)
    lab = np.repeat(np.arange(blocks), n // blocks)
    iu, ju = np.triu_indices(n, 1)
    p = np.where(lab[iu] == lab[ju], p_in, p_out)
    keep = rng.random(len(iu)) < p
    u, v = iu[keep], ju[keep]
    used = np.zeros(n, bool); used[u] = True; used[v] = True
    nid = np.cumsum(used) - 1
    n2 = int(used.sum())
    return n2, np.unique(nid[u] * n2 + nid[v]).astype(np.int64), lab[used]


def instance_from_keys(n, keys, weights=None, vol=None, L_orig=None, C0=0.0):
    """CSR exactly as alm_vcs.py:1105-1117 builds it."""
    u = keys // n; v = keys % n; m = len(keys); L = 2 * m
    d = np.bincount(np.r_[u, v], minlength=n).astype(float)
    W_ = weights if weights is not None else np.ones(m)
    A = sp.csr_matrix((np.r_[W_, W_], (np.r_[u, v], np.r_[v, u])), shape=(n, n))
    if vol is not None:
        d = vol.astype(float); L = int(L_orig)
    A.sort_indices()
    return dict(n=n, indptr=A.indptr.astype(np.int64), indices=A.indices.astype(np.int64),
                data=A.data.astype(np.float64), d=d, L=float(L), C0=float(C0))


def reduced_instance(edges_n, keys, tmp, labels=()):
    """Run the reference reduce_exact.py (with optional label files); returns the reduced instance, its raw outputs,
    the restricted label files it wrote and the three modularities it printed for each (original, rules enforced,
    reduced; six decimals)."""
    D = os.path.join(tmp, "data", "g"); os.makedirs(D, exist_ok=True)
    np.save(os.path.join(D, "keys.npy"), keys)
    json.dump({"n": int(edges_n), "m": int(len(keys))}, open(os.path.join(D, "graph.json"), "w"))
    files = []
    for i, lab in enumerate(labels):
        files.append(os.path.join(tmp, f"lab{i}.npy")); np.save(files[-1], np.asarray(lab, np.int64))
    res = subprocess.run([sys.executable, os.path.join(CORE, "reduce_exact.py"), "g"] + files, cwd=tmp, check=True,
                         stdout=subprocess.PIPE, text=True)
    Dz = os.path.join(tmp, "data", "g__rx")
    g = json.load(open(os.path.join(Dz, "graph.json"))); meta = json.load(open(os.path.join(Dz, "meta.json")))
    out = dict(n=g["n"], keys=np.load(os.path.join(Dz, "keys.npy")), weights=np.load(os.path.join(Dz, "weights.npy")),
               vol=np.load(os.path.join(Dz, "vol.npy")), group_of=np.load(os.path.join(Dz, "group_of.npy")), meta=meta)
    qlines = [ln for ln in res.stdout.splitlines() if "original Q" in ln]
    out["lr"] = [np.load(os.path.join(Dz, f"lab{i}.npy")) for i in range(len(labels))]
    out["q"] = [np.array([float(x) for x in re.findall(r"-?\d+\.\d+", ln)[:3]]) for ln in qlines]
    return out


def wedges(inst, T, seed):
    """Random wedge triples (a, b = centre, c), normalised (min, b, max), deduplicated."""
    rng = np.random.default_rng(seed)
    ip, ix = inst["indptr"], inst["indices"]; deg = np.diff(ip)
    cand = np.flatnonzero(deg >= 2)
    out = set()
    while len(out) < T:
        b = int(rng.choice(cand)); nb = ix[ip[b]:ip[b + 1]]
        a, c = rng.choice(nb, 2, replace=False)
        out.add((int(min(a, c)), b, int(max(a, c))))
    return np.array(sorted(out), np.int64)


# ----------------------------------------------------------------------------------------------- one evaluation
def ref_eval(inst, V, plev, TI, lam, vlev, rho, tri_weight, wv):
    """augmented() + CV() from reference kernels (alm_vcs.py:1496-1533, 1299-1312), nesplit off, no cuts."""
    ip, ix, ad, d, L, C0 = inst["indptr"], inst["indices"], inst["data"], inst["d"], inst["L"], inst["C0"]
    n, k = V.shape
    zz = d @ V
    qA = K["quadA"](ip, ix, ad, V)
    val0 = qA - float(zz @ zz) / L
    val = val0
    out = dict(quadA=qA, zz=zz, val0=val0)
    # pair levels (cluster_sums = Ysum, level_aug)
    labs = np.ascontiguousarray(np.array([Lv.lab for Lv in plev], np.int64).reshape(len(plev), n))
    Poff = np.r_[0, np.cumsum([Lv.P for Lv in plev])].astype(np.int64)
    Yall = np.zeros((int(Poff[-1]), k))
    if plev:
        K["cluster_sums"](labs, Poff, d, V, 1, Yall)
    pps, nviols, ltots = [], [], []
    for li, Lv in enumerate(plev):
        Y = Yall[Poff[li]:Poff[li + 1]]
        H = Y @ Y.T; H[np.diag_indices(Lv.P)] -= Lv.dsq; pp = np.empty_like(H)
        tot, nv = K["level_aug"](H, np.ascontiguousarray(Lv.sig), Lv.rq, float(Lv.w), float(rho), pp, 0, np.zeros((1, 1)))
        val -= tot; pps.append(pp); nviols.append(int(nv)); ltots.append(tot)
    rt = rho * tri_weight
    gt = np.empty(len(TI)); pt = np.empty(len(TI)); ttot = 0.0; gmin = np.inf
    if len(TI):
        ttot, gmin = K["tri_aug"](TI, V, lam, float(rt), gt, pt); val -= ttot
    vtots, ppvs, slks, stns, vnvs = [], [], [], [], []
    for Lv in vlev:
        Yv = np.ascontiguousarray(Lv.W @ V); ppv = np.empty(Lv.nnz); slk = np.empty(Lv.nnz, np.uint8); stn = np.empty(Lv.nnz)
        tot, nv = VCS.vcs_aug(Lv, V, d, Yv, wv, float(rho), ppv, slk, stn)
        val -= tot; vtots.append(tot); ppvs.append(ppv); slks.append(slk); stns.append(stn); vnvs.append(nv)
    out.update(value=val + C0, primal=val0 + C0, level_tot=np.array(ltots), nviol=np.array(nviols, np.int64),
               tri_tot=ttot, gmin=gmin, gt=gt, pt=pt, vcs_tot=np.array(vtots), vcs_nviol=np.array(vnvs, np.int64))
    for li, pp in enumerate(pps): out[f"pp{li}"] = pp
    for m, (ppv, slk, stn) in enumerate(zip(ppvs, slks, stns)):
        out[f"ppv{m}"] = ppv; out[f"slack{m}"] = slk; out[f"stn{m}"] = stn
    # G = C(y_eff) V  (CV with sigs = pp, w = pt, VCS sig = ppv)
    out["G"] = ref_CV(inst, V, plev, pps, TI, pt, vlev, ppvs)
    return out


def ref_CV(inst, X, plev, sigs, TI, w, vlev, vsigs):
    ip, ix, ad, d, L = inst["indptr"], inst["indices"], inst["data"], inst["d"], inst["L"]
    X = np.ascontiguousarray(X, dtype=np.float64)
    AXo = np.empty_like(X); K["spmm"](ip, ix, ad, X, AXo)
    out = AXo - np.outer(d, d @ X) / L
    for Lv, s in zip(plev, sigs):
        Y = Lv.W @ X
        out += d[:, None] * (s @ Y)[Lv.lab] - (np.diag(s)[Lv.lab] * d ** 2)[:, None] * X
    for Lv, s in zip(vlev, vsigs):
        out += VCS.vcs_apply(Lv, s, X, d)
    if len(w):
        ptr, codes = K["incidence"](X.shape[0], TI)
        K["tri_apply"](TI, w, ptr, codes, X, out)
    return out


# ----------------------------------------------------------------------------------------------- one batch of row steps
def ref_batch(inst, V, plev, TI, lam, vlev, rho, tri_weight, wv, rows, damp):
    ip, ix, ad, d, L = inst["indptr"], inst["indices"], inst["data"], inst["d"], inst["L"]
    n, k = V.shape
    nl = len(plev)
    labs = np.ascontiguousarray(np.array([Lv.lab for Lv in plev], np.int64).reshape(nl, n))
    Poff = np.r_[0, np.cumsum([Lv.P for Lv in plev])].astype(np.int64)
    sP = int(Poff[-1])
    Ycat = np.zeros((sP, k))
    if nl:
        K["cluster_sums"](labs, Poff, d, V, 1, Ycat)
    z = d @ V
    # per-sweep curvature Kq (sweeps(), alm_vcs.py:1388-1395, trace rule)
    Kq = np.zeros(sP)
    for li, Lv in enumerate(plev):
        Y = Ycat[Poff[li]:Poff[li + 1]]
        H = Y @ Y.T; H[np.diag_indices(Lv.P)] -= Lv.dsq; H = 0.5 * (H + H.T)
        K["kq_level"](H, np.ascontiguousarray(Lv.sig), Lv.r, (Y * Y).sum(1), float(rho), Kq[Poff[li]:Poff[li + 1]])
    # sigma CSR concatenated (alm_vcs.py:1374-1379)
    scsr = [K["sig_csr"](np.ascontiguousarray(Lv.sig)) for Lv in plev]
    if nl:
        sg_ptr = np.r_[0, np.cumsum(np.concatenate([np.diff(c[0]) for c in scsr]))].astype(np.int64)
        sg_idx = np.concatenate([c[1] + Poff[li] for li, c in enumerate(scsr)]).astype(np.int64)
        sg_val = np.concatenate([c[2] for c in scsr]); rq_all = np.concatenate([Lv.rq for Lv in plev])
        dsq_all = np.concatenate([Lv.dsq for Lv in plev])
    else:
        sg_ptr = np.zeros(1, np.int64); sg_idx = np.zeros(0, np.int64); sg_val = np.zeros(0)
        rq_all = np.zeros(0); dsq_all = np.zeros(0)
    Hoff = np.r_[0, np.cumsum([Lv.P ** 2 for Lv in plev])].astype(np.int64)
    CLO = np.zeros(sP, np.int64); CHI = np.zeros(sP, np.int64); PBASE = np.zeros(sP, np.int64)
    for li, Lv in enumerate(plev):
        o0, o1 = int(Poff[li]), int(Poff[li + 1]); Qg = np.arange(o0, o1, dtype=np.int64)
        CLO[o0:o1] = o0; CHI[o0:o1] = o1; PBASE[o0:o1] = Hoff[li] + (Qg - o0) * (o1 - o0) - o0
    ppbuf = np.zeros(max(1, int(Hoff[-1]))); eabuf = np.zeros(1)
    lw_all = np.array([float(Lv.w) for Lv in plev]) if nl else np.zeros(0)
    Pcnt = np.array([Lv.P for Lv in plev], np.int64)
    # VCS start-of-sweep state (vcs_state, vcsops.py:308-323)
    Yvs = [VCS.vcs_state(Lv, V, d, rho, wv, False) for Lv in vlev]
    state0 = {f"vcs_stZ{m}": Lv.stZ.copy() for m, Lv in enumerate(vlev)}
    state0.update({f"vcs_Z{m}": Lv.Z.copy() for m, Lv in enumerate(vlev)})
    state0.update({f"vcs_cnt{m}": Lv.cnt.copy() for m, Lv in enumerate(vlev)})
    nr = len(rows)
    GX = np.zeros((nr, k)); KX = np.zeros(nr)
    Vold = V[rows].copy()
    for Lv, Yv in zip(vlev, Yvs):
        VCS.vcs_pre(rows, V, d, Lv.lab, Yv, np.einsum("ij,ij->i", Yv, Yv), True, Lv.ptr, Lv.col, Lv.sig, Lv.stZ,
                    Lv.own, Lv.Z, Lv.cnt, Lv.rq, wv, float(rho), 1.0, GX, KX)
    Mall = np.zeros((sP, k)); pdiag = np.zeros(sP)
    if nl:
        mark = np.zeros(sP, np.int64)
        items, ilev = K["touched_all"](rows, labs, Poff, mark, 1)
        K["pair_all"](items, ilev, Ycat, CLO, CHI, PBASE, sg_ptr, sg_idx, sg_val, rq_all, dsq_all, lw_all, float(rho),
                      Mall, pdiag, 0, eabuf, ppbuf)
    tri_ptr, tri_codes = K["incidence"](n, TI)
    IABC = np.empty((len(tri_codes), 3), np.int32); K["inc_abc"](TI, tri_codes, IABC)
    LINC = np.empty(len(tri_codes)); K["inc_lam"](tri_codes, lam, LINC)
    rt = rho * tri_weight
    e3 = np.zeros((0, 3), np.int64); e2 = np.zeros((0, 2), np.int64); p1 = np.zeros(n + 1, np.int64); c0 = np.zeros(0, np.int64)
    Vnew = V.copy(); DD = np.zeros((nr, k))
    for idx, i in enumerate(rows):        # Jacobi within the batch: each row steps from the pre-batch V
        Vc = V.copy(); DDi = np.zeros((1, k))
        K["batch_step6"](np.array([i], np.int64), Vc, ip, ix, ad, d, z, float(L), labs, Poff, Mall, pdiag, Kq,
                         IABC, LINC, tri_ptr, tri_codes, float(rt), float(damp), np.zeros(n), 0.0, e3, np.zeros(0),
                         p1, c0, 0.0, e2, np.zeros(0), p1, c0, 0.0, 0, ppbuf, Hoff, Pcnt, False, 32, DDi,
                         bool(vlev), GX[idx:idx + 1], KX[idx:idx + 1])
        Vnew[i] = Vc[i]; DD[idx] = DDi[0]
    out = dict(rows=rows, damp=damp, Kq=Kq, Mall=Mall, pdiag=pdiag, GX=GX, KX=KX, Vnew=Vnew, DD=DD, z0=z, Y0=Ycat.copy())
    out.update(state0)
    # post-batch aggregate updates, one thread: _acc_rows, vcs_yupd, vcs_post
    z1 = z.copy(); Y1 = Ycat.copy()
    K["_acc_rows"](rows, DD, z1, labs, Poff, Y1)
    out.update(z1=z1, Y1=Y1)
    for m, (Lv, Yv) in enumerate(zip(vlev, Yvs)):
        VCS.vcs_yupd(rows, Lv.lab, DD, Yv)
        stZ = Lv.stZ.copy(); Z = Lv.Z.copy(); cnt = Lv.cnt.copy()
        VCS.vcs_post(rows, Vnew, Vold, d, Lv.lab, Yv, Lv.ptr, Lv.col, Lv.sig, stZ, Lv.rq, wv, float(rho), Z, cnt, 1,
                     np.zeros(Lv.P, np.int32))
        out[f"vcs_Y1_{m}"] = Yv.copy(); out[f"vcs_stZ1_{m}"] = stZ; out[f"vcs_Z1_{m}"] = Z; out[f"vcs_cnt1_{m}"] = cnt
    return out


# ----------------------------------------------------------------------------------------------- one fixture
def make_eval_fixture(name, inst, k, P, Pv, T, rho, tri_weight, w_pair, vc_weight, seed, nbatch=8, damp=0.0,
                      vcs_extra=0.2, stress=False):
    """stress=False: multipliers at the scale the PHR update produces (sig ~ rho r |h|), where the PHR terms are
    well conditioned.  stress=True: multipliers far above that scale, where (pp^2 - sig^2)/(2 rho r) cancels."""
    rng = np.random.default_rng(seed)
    n = inst["n"]; d = inst["d"]
    V = rng.standard_normal((n, k)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    # one pair level: random labels, symmetric sigma >= 0 with zeros
    plev = []
    if P:
        lab = rng.integers(0, P, n); lab[:P] = np.arange(P)
        Lv = PairLevel(lab, d)
        cnt = np.bincount(Lv.lab, minlength=Lv.P).astype(float)
        vol = np.maximum(np.bincount(Lv.lab, weights=d, minlength=Lv.P), 1.0)
        Lv.rq = cnt / vol ** 2; Lv.w = w_pair; Lv.r = np.outer(Lv.rq, Lv.rq) * w_pair
        if stress:
            S = rng.exponential(1.0, (Lv.P, Lv.P)) * (rng.random((Lv.P, Lv.P)) < 0.6) * 50.0
        else:
            Y = Lv.W @ V; H = Y @ Y.T; H[np.diag_indices(Lv.P)] -= Lv.dsq
            S = rho * Lv.r * np.abs(H) * rng.uniform(0, 3, (Lv.P, Lv.P)) * (rng.random((Lv.P, Lv.P)) < 0.6)
        Lv.sig = 0.5 * (S + S.T)
        plev.append(Lv)
    TI = wedges(inst, T, seed + 1) if T else np.zeros((0, 3), np.int64)
    lam = rng.exponential(0.05, len(TI)) * (rng.random(len(TI)) < 0.5)
    # one VCS level: neighbour pattern of its labels plus random extra entries, sigma >= 0 with zeros
    vlev = []
    wv = vc_weight * w_pair
    if Pv:
        labv = rng.integers(0, Pv, n); labv[:Pv] = np.arange(Pv)
        Lv = VCS.VCSLevel(labv, d)
        ip, ix = inst["indptr"], inst["indices"]
        rows_ = np.repeat(np.arange(n), np.diff(ip))
        pr = np.r_[np.arange(n), rows_, rng.integers(0, n, int(vcs_extra * n))]
        pc = np.r_[Lv.lab, Lv.lab[ix], rng.integers(0, Lv.P, int(vcs_extra * n))]
        pat = sp.csr_matrix((np.ones(len(pr)), (pr, pc)), shape=(n, Lv.P)); pat.sum_duplicates(); pat.sort_indices()
        if stress:
            sg = rng.exponential(2.0, pat.nnz) * (rng.random(pat.nnz) < 0.5)
        else:
            Yv = Lv.W @ V; rows_p = np.repeat(np.arange(n), np.diff(pat.indptr)); cols_p = pat.indices
            s_ = np.einsum("ij,ij->i", V[rows_p], Yv[cols_p]); dd = d[rows_p]
            g_ = dd * (s_ - np.where(cols_p == Lv.lab[rows_p], dd, 0.0))
            r_ = wv * Lv.rq[cols_p] / dd ** 2
            sg = rho * r_ * np.abs(g_) * rng.uniform(0, 3, pat.nnz) * (rng.random(pat.nnz) < 0.5)
        Lv.set_ws(pat.indptr.astype(np.int64), pat.indices.astype(np.int32), sg)
        vlev.append(Lv)
    ev = ref_eval(inst, V, plev, TI, lam, vlev, rho, tri_weight, wv)
    # fixed multipliers (rho = 0): the estimator's operator and value (est_dual_vcs.py:227-246); triangles with
    # lam = 0 are dropped there (est_dual_vcs.py:207), which does not change C(y).
    W = V.copy()
    C0 = inst["C0"]
    keep = lam > 0
    CW = ref_CV(inst, W, plev, [Lv.sig for Lv in plev], TI[keep], lam[keep], vlev, [Lv.sig for Lv in vlev])
    gvec = np.einsum("ij,ij->i", CW, W)
    const = C0 + lam.sum()
    est = dict(est_CW=CW, est_g=gvec, est_dv=(const + gvec.sum()) / inst["L"])
    # one batch of row steps
    order = np.random.default_rng(seed + 2).permutation(n).astype(np.int64)
    rows = np.array_split(order, nbatch)[0]
    bt = ref_batch(inst, V, plev, TI, lam, vlev, rho, tri_weight, wv, rows, damp)
    fx = dict(n=n, indptr=inst["indptr"], indices=inst["indices"], data=inst["data"], d=d, L=inst["L"], C0=C0,
              V=V, TI=TI, lam=lam, rho=rho, tri_weight=tri_weight, w_pair=w_pair, vc_weight=vc_weight,
              stress=int(stress))
    for li, Lv in enumerate(plev):
        fx[f"plab{li}"] = Lv.lab; fx[f"psig{li}"] = Lv.sig; fx[f"prq{li}"] = Lv.rq; fx[f"pdsq{li}"] = Lv.dsq
    fx["npl"] = len(plev)
    for m, Lv in enumerate(vlev):
        fx[f"vlab{m}"] = Lv.lab; fx[f"vptr{m}"] = Lv.ptr; fx[f"vcol{m}"] = Lv.col; fx[f"vsig{m}"] = Lv.sig
        fx[f"vrq{m}"] = Lv.rq; fx[f"vvol{m}"] = Lv.vol; fx[f"vown{m}"] = Lv.own
    fx["nvl"] = len(vlev)
    for key, val in ev.items(): fx["ev_" + key] = val
    for key, val in est.items(): fx[key] = val
    for key, val in bt.items(): fx["bt_" + key] = val
    path = os.path.join(HERE, f"eval_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, os.path.getsize(path), "bytes", "value", ev["value"])


# ----------------------------------------------------------------------------------------------- separation
def make_sep_fixture(name, inst, k, seed, tri_add, tri1_add, tri_max, pool_T):
    rng = np.random.default_rng(seed)
    n = inst["n"]
    V = rng.standard_normal((n, k)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    ip, ix = inst["indptr"], inst["indices"]
    thresh, maxh, maxk, hub2, cap2, vtol = 0.3, 100, 60, 8, 200, 1e-3
    # pool before separation (existing triangles, some with lam = 0 to be purged)
    TI = wedges(inst, pool_T, seed + 5) if pool_T else np.zeros((0, 3), np.int64)
    lam = rng.exponential(0.05, len(TI)) * (rng.random(len(TI)) < 0.5)
    keep = lam > 0; TIk = TI[keep]; lamk = lam[keep]
    room = max(0, tri_max - len(TIk))
    cap0 = int(min(tri_add, room) * 1.3) + 10; cap1 = int(tri1_add * 1.3) + 10
    new0, val0 = K["separate"](ip, ix, V, thresh, maxh, vtol, cap0)
    (nb0, vb0), (nb1, vb1) = K["separate_both"](ip, ix, V, thresh, maxh, maxk, hub2, cap2, vtol, cap0, cap1)
    # pool merge: the main loop's own lines, executed from the reference file (alm_vcs.py:1748-1756)
    lines = open(os.path.join(CORE, "alm_vcs.py")).read().split("\n")
    start = next(i for i, l in enumerate(lines) if "keep both budgets" in l) - 1
    assert lines[start].strip() == "if a.tri1_add:"
    block = textwrap.dedent("\n".join(lines[start:start + 9]))

    class A_: pass
    a_ = A_(); a_.tri_add = tri_add; a_.tri1_add = tri1_add
    ns = dict(np=np, a=a_, n=n, room=room, TI=TIk.copy(), lam=lamk.copy(), new=nb0.copy(), val=vb0.copy(),
              n1=nb1.copy(), v1=vb1.copy())
    exec(compile(block, os.path.join(CORE, "alm_vcs.py"), "exec"), ns)
    fx = dict(n=n, indptr=ip, indices=ix, V=V, thresh=thresh, maxh=maxh, maxk=maxk, hub2=hub2, cap2=cap2, vtol=vtol,
              tri_add=tri_add, tri1_add=tri1_add, tri_max=tri_max, TI0=TI, lam0=lam, cap0=cap0, cap1=cap1,
              sep_new=new0, sep_val=val0, both_new0=nb0, both_val0=vb0, both_new1=nb1, both_val1=vb1,
              pool_TI=ns["TI"], pool_lam=ns["lam"])
    path = os.path.join(HERE, f"sep_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, os.path.getsize(path), "bytes", "sep", len(new0), "both", len(nb0), len(nb1), "pool", len(ns["TI"]))


# ----------------------------------------------------------------------------------------------- reduction
def make_reduce_fixture(name, n, edges, tmp):
    edges = np.sort(np.asarray(edges, np.int64), axis=1)
    keys = np.unique(edges[:, 0] * n + edges[:, 1])
    rng = np.random.default_rng(n)
    labels = [rng.integers(0, 3, n), rng.integers(0, max(2, n // 4), n)]     # two partitions for the label loop
    r = reduced_instance(n, keys, tmp, labels)
    fx = dict(n=n, keys=keys, rn=r["n"], rkeys=r["keys"], rweights=r["weights"], rvol=r["vol"], group_of=r["group_of"],
              L_orig=r["meta"]["L_orig"], leaf_edges=r["meta"]["leaf_edges"], leaf_unions=r["meta"]["leaf_unions"],
              twin_unions=r["meta"]["twin_unions"])
    for i, lab in enumerate(labels):
        fx[f"lab{i}"] = np.asarray(lab, np.int64); fx[f"lr{i}"] = r["lr"][i]; fx[f"q{i}"] = r["q"][i]
    path = os.path.join(HERE, f"reduce_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, "n", n, "->", r["n"], "leaf", r["meta"]["leaf_unions"], "twin", r["meta"]["twin_unions"])
    return r


def make_vsep_fixture(name, inst, k, P, seed, cases, vcs_drop=5):
    """cases: (mode, nadd, tol, chunk_bytes) tuples; the first case's result is also merged into the working set."""
    rng = np.random.default_rng(seed)
    n = inst["n"]; d = inst["d"]
    V = rng.standard_normal((n, k)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    lab = rng.integers(0, P, n); lab[:P] = np.arange(P)
    Lv = VCS.VCSLevel(lab, d)
    ip, ix = inst["indptr"], inst["indices"]
    rows_ = np.repeat(np.arange(n), np.diff(ip))
    pr = np.r_[np.arange(n), rows_[::3], rng.integers(0, n, n)]
    pc = np.r_[Lv.lab, Lv.lab[ix[::3]], rng.integers(0, Lv.P, n)]
    pat = sp.csr_matrix((np.ones(len(pr)), (pr, pc)), shape=(n, Lv.P)); pat.sum_duplicates(); pat.sort_indices()
    sig = rng.exponential(0.5, pat.nnz) * (rng.random(pat.nnz) < 0.5)
    age = rng.integers(0, 8, pat.nnz).astype(np.uint8)
    Lv.set_ws(pat.indptr.astype(np.int64), pat.indices.astype(np.int32), sig, age)
    wv = 0.7
    fx = dict(n=n, d=d, V=V, lab=Lv.lab, ptr=Lv.ptr, col=Lv.col, sig=Lv.sig, age=Lv.age, wv=wv, ncase=len(cases),
              vcs_drop=vcs_drop)
    for c, (mode, nadd, tol, cb) in enumerate(cases):
        ai, aR, as_, st = VCS.separate(Lv, V, d, wv, nadd, tol, mode, chunk_bytes=cb)
        o = np.lexsort((aR, ai))
        fx.update({f"mode{c}": mode, f"nadd{c}": nadd, f"tol{c}": tol, f"rows{c}": ai[o].astype(np.int64),
                   f"cols{c}": aR[o].astype(np.int32), f"scores{c}": as_[o],
                   f"stats{c}": np.array([st["nviol"], st["mass"], st["nviol_ws"], st["mass_ws"]])})
        if c == 0:
            keep = Lv.age < vcs_drop
            VCS.update_ws(Lv, keep, ai, aR)
            fx.update(m_ptr=Lv.ptr, m_col=Lv.col, m_sig=Lv.sig, m_age=Lv.age)
            Lv.set_ws(fx["ptr"], fx["col"], fx["sig"], fx["age"])
    path = os.path.join(HERE, f"vsep_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, "n", n, "P", P, "ws", len(fx["col"]), [len(fx[f"rows{c}"]) for c in range(len(cases))])


def make_init_fixture(name, inst, lab, k, seed):
    lines = open(os.path.join(CORE, "alm_vcs.py")).read().split("\n")
    start = next(i for i, l in enumerate(lines) if l.startswith("elif a.init_partition:")) + 1
    end = next(i for i in range(start, len(lines)) if lines[i].strip().startswith("V += 1e-3")) + 1
    block = textwrap.dedent("\n".join(lines[start:end]))
    tmp = tempfile.mkdtemp(prefix="lagbound_init_")
    f = os.path.join(tmp, "lab.npy"); np.save(f, np.asarray(lab, np.int64))

    class A_: pass
    a_ = A_(); a_.k = k; a_.init_partition = f
    A = sp.csr_matrix((inst["data"], inst["indices"], inst["indptr"]), shape=(inst["n"], inst["n"]))
    ns = dict(np=np, sp=sp, a=a_, A=A, n=inst["n"], d=inst["d"], rng=np.random.default_rng(seed))
    exec(compile(block, os.path.join(CORE, "alm_vcs.py"), "exec"), ns)
    fx = dict(n=inst["n"], indptr=inst["indptr"], indices=inst["indices"], d=inst["d"], lab=np.asarray(lab, np.int64),
              k=k, seed=seed, V=ns["V"], colour=ns["col"])
    path = os.path.join(HERE, f"init_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, "P", int(np.max(lab)) + 1, "k", k)


def make_pw_fixture(name, inst, labs, k, seed, rho, w0, rules, phase2_w, phase2_at_it, outer):
    """The pair weight of --pw_rule (alm_vcs.py:1625-1653: mobility_ratio and the rule's min of the mobility and step
    weights, then set_pair_weight) and the phase-2 switch of the main loop (alm_vcs.py:1663-1667, by outer
    iteration), both executed from the reference file, at a fixed V and levels, for several rule strings."""
    rng = np.random.default_rng(seed)
    n = inst["n"]; d = inst["d"]
    V = rng.standard_normal((n, k)); V /= np.linalg.norm(V, axis=1, keepdims=True)
    lines = open(os.path.join(CORE, "alm_vcs.py")).read().split("\n")
    start = next(i for i, l in enumerate(lines) if l.startswith("def mobility_ratio(V, w=1.0):"))
    end = next(i for i in range(start, len(lines)) if lines[i].startswith("    set_pair_weight(W_AUTO)")) + 1
    block = "\n".join(lines[start:end])
    p2 = next(i for i, l in enumerate(lines) if l.startswith("    if not PH2[0] and ((a.phase2_at > 0"))
    block2 = textwrap.dedent("\n".join(lines[p2:p2 + 3]))
    A = sp.csr_matrix((inst["data"], inst["indices"], inst["indptr"]), shape=(n, n))
    fx = dict(n=n, indptr=inst["indptr"], indices=inst["indices"], data=inst["data"], d=d, L=inst["L"], V=V, rho=rho,
              w0=w0, nlev=len(labs), phase2_w=phase2_w, phase2_at_it=phase2_at_it, outer=outer, rules=list(rules))
    for li, lab in enumerate(labs):
        fx[f"lab{li}"] = np.asarray(lab, np.int64)
    for c, rule in enumerate(rules):
        levels = []
        for lab in labs:
            Lv = PairLevel(lab, d)
            cnt = np.bincount(Lv.lab, minlength=Lv.P).astype(float)
            vol = np.maximum(np.bincount(Lv.lab, weights=d, minlength=Lv.P), 1.0)
            Lv.rq = cnt / vol ** 2; Lv.r = np.outer(Lv.rq, Lv.rq) * w0
            levels.append(Lv)

        class A_: pass
        a_ = A_(); a_.pairlvl_weight = w0; a_.rho = rho; a_.pw_auto = 0.0; a_.pw_rule = rule
        a_.phase2_at = 0.0; a_.phase2_at_it = phase2_at_it; a_.phase2_w = phase2_w
        a_.phase2_inner = 300; a_.phase2_tri_every = 1; a_.phase2_est_every = 1; a_.inner = 1; a_.tri_every = 9
        a_.est_every = 0
        got = {}

        def set_pair_weight(w, _got=got, _a=a_):
            _a.pairlvl_weight = float(w); _got.setdefault("weights", []).append(float(w))
        ns = dict(np=np, a=a_, A=A, d=d, L=float(inst["L"]), n=n, levels=levels, nl=len(levels), V=V,
                  log=lambda *x, **y: None, set_pair_weight=set_pair_weight, time=__import__("time"))
        exec(compile(block, os.path.join(CORE, "alm_vcs.py"), "exec"), ns)
        R0 = ns["mobility_ratio"](V, w0)
        ns.update(PH2=[False], t0=__import__("time").time())
        switched = -1
        code2 = compile(block2 + "\n    _sw[0] = it", os.path.join(CORE, "alm_vcs.py"), "exec")
        for it in range(1, outer + 1):
            loc = dict(ns, it=it, _sw=[-1])          # PH2 is the same list in every copy: it switches once
            exec(code2, loc)
            if loc["_sw"][0] > 0 and switched < 0:
                switched = it
        fx.update({f"R0_{c}": R0, f"w_auto_{c}": ns["W_AUTO"], f"w_phase2_{c}": got["weights"][-1],
                   f"switch_it_{c}": switched, f"nweights_{c}": len(got["weights"])})
    path = os.path.join(HERE, f"pw_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, [(fx[f"w_auto_{c}"], fx[f"switch_it_{c}"]) for c in range(len(rules))])


def make_graph_fixture(name, pairs, names=None):
    import warnings
    from lagbound.graph import _from_pairs
    pairs = np.asarray(pairs, np.int64)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        g = _from_pairs(pairs, names=None if names is None else list(range(names)))
    fx = dict(pairs=pairs, n_names=-1 if names is None else names, n=g.n, u=g.u, v=g.v,
              labels=np.asarray(g.labels, np.int64), isolated=np.asarray(g.isolated, np.int64).reshape(-1))
    path = os.path.join(HERE, f"graph_{name}.npz")
    np.savez_compressed(path, **fx)
    print("wrote", path, "n", g.n, "m", g.m, "isolated", len(g.isolated))


def main(only=None):
    """only: None for every fixture, or one of "eval", "reduce", "sep", "vsep", "init", "pw", "graph",
    "modularity"."""
    want = lambda part: only is None or only == part
    import networkx as nx
    from lagbound import modularity, as_graph
    tmp = tempfile.mkdtemp(prefix="lagbound_golden_")
    # --- evaluation fixtures: an SBM instance and an exactly reduced (weighted, vol != degree, C0 > 0) instance
    n, keys, _ = sbm_keys(400, 4, 0.08, 0.01, seed=3)
    sbm = instance_from_keys(n, keys)
    if want("eval"):
        make_eval_fixture("sbm400_k16", sbm, k=16, P=6, Pv=9, T=1500, rho=0.02, tri_weight=1.0, w_pair=0.3,
                          vc_weight=1.0, seed=11, nbatch=5, damp=0.0)
    if want("eval"):
        make_eval_fixture("sbm400_k13", sbm, k=13, P=5, Pv=7, T=900, rho=0.5, tri_weight=2.0, w_pair=2.0,
                          vc_weight=0.5, seed=12, nbatch=4, damp=0.3)
    if want("eval"):
        make_eval_fixture("sbm400_k16_stress", sbm, k=16, P=6, Pv=9, T=1500, rho=0.02, tri_weight=1.0, w_pair=0.3,
                          vc_weight=1.0, seed=15, nbatch=5, damp=0.0, stress=True)
    # a graph with many leaves and twins, reduced by the reference
    rng = np.random.default_rng(5)
    n0, k0, _ = sbm_keys(360, 6, 0.12, 0.01, seed=7)
    e = np.c_[k0 // n0, k0 % n0].tolist()
    nxt = n0
    for hub in rng.choice(n0, 40, replace=False):           # leaves
        e.append((int(hub), nxt)); nxt += 1
    for a in rng.choice(n0, 30, replace=False):              # true twins of existing vertices
        nb = [b for (x, b) in e if x == a] + [x for (x, b) in e if b == a]
        for b in nb: e.append((nxt, int(b)))
        e.append((nxt, int(a))); nxt += 1
    r = make_reduce_fixture("sbm_leaves_twins", nxt, e, os.path.join(tmp, "r1"))
    red = instance_from_keys(r["n"], r["keys"], weights=r["weights"], vol=r["vol"], L_orig=r["meta"]["L_orig"],
                             C0=2.0 * r["meta"]["leaf_edges"])
    if want("eval"):
        make_eval_fixture("reduced_k8", red, k=8, P=4, Pv=6, T=700, rho=0.05, tri_weight=1.0, w_pair=0.7,
                          vc_weight=1.0, seed=13, nbatch=6, damp=0.1)
    if want("eval"):
        make_eval_fixture("reduced_k8_nolevels", red, k=8, P=0, Pv=0, T=0, rho=0.05, tri_weight=1.0, w_pair=0.7,
                          vc_weight=1.0, seed=14, nbatch=3, damp=0.0)
    # --- reduction fixtures from the reference's own test graphs and networkx graphs
    GRAPH = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (3, 4), (4, 5), (5, 6), (4, 6), (0, 7)]
    make_reduce_fixture("k4_leaf_triangle", 8, GRAPH, os.path.join(tmp, "r2"))
    G = nx.karate_club_graph(); g = as_graph(G)
    make_reduce_fixture("karate", g.n, np.c_[g.u, g.v], os.path.join(tmp, "r3"))
    G = nx.les_miserables_graph(); g = as_graph(G)
    make_reduce_fixture("lesmis", g.n, np.c_[g.u, g.v], os.path.join(tmp, "r4"))
    g = as_graph(nx.complete_graph(12))
    make_reduce_fixture("k12", g.n, np.c_[g.u, g.v], os.path.join(tmp, "r5"))
    g = as_graph(nx.disjoint_union(nx.complete_graph(5), nx.complete_graph(6)))
    make_reduce_fixture("k5_k6", g.n, np.c_[g.u, g.v], os.path.join(tmp, "r6"))
    # --- separation fixtures
    n, keys, _ = sbm_keys(600, 6, 0.05, 0.006, seed=21)
    inst = instance_from_keys(n, keys)
    if want("sep"):
        make_sep_fixture("sbm600_k4", inst, k=4, seed=22, tri_add=2000, tri1_add=1000, tri_max=20000, pool_T=800)
        make_sep_fixture("sbm600_k6_tight", inst, k=6, seed=23, tri_add=300, tri1_add=150, tri_max=1200, pool_T=1000)
    # --- VCS working-set separation
    if want("vsep"):
        n, keys, _ = sbm_keys(1800, 6, 0.03, 0.004, seed=41)
        inst = instance_from_keys(n, keys)
        make_vsep_fixture("sbm1800_p40", inst, k=8, P=40, seed=42,
                          cases=[("pen", 3000, 1e-4, 8 * 40 * 64), ("mean", 10 ** 9, 1e-4, 64 * 2 ** 20),
                                 ("mass", 700, 1e-3, 8 * 40 * 200)])
        make_vsep_fixture("sbm1800_p7", inst, k=5, P=7, seed=43,
                          cases=[("pen", 400, 1e-4, 8 * 7 * 64), ("mass", 10 ** 9, 1e-4, 64 * 2 ** 20)])
    # --- solver start from a partition
    if want("init"):
        n, keys, lab = sbm_keys(1200, 12, 0.05, 0.004, seed=51)
        inst = instance_from_keys(n, keys)
        make_init_fixture("sbm1200_b12_k8", inst, lab, k=8, seed=0)
        rng = np.random.default_rng(52)
        make_init_fixture("sbm1200_r60_k32", inst, rng.integers(0, 60, n), k=32, seed=3)
    # --- pair weight of --pw_rule and the phase-2 switch
    if want("pw"):
        n, keys, lab = sbm_keys(900, 6, 0.06, 0.004, seed=61)
        inst = instance_from_keys(n, keys)
        rng = np.random.default_rng(62)
        make_pw_fixture("sbm900", inst, [lab, rng.integers(0, 30, n)], k=12, seed=63, rho=0.02, w0=1.0,
                        rules=["default", "0.3", ",0.001", "0.05,0.2", "0.001,1"], phase2_w=0.2, phase2_at_it=4, outer=9)
    # --- simple graphs of pair lists
    if want("graph"):
        make_graph_fixture("cleaning", [[0, 1], [1, 0], [1, 1], [1, 2], [5, 6], [5, 6]])
        G = nx.karate_club_graph()
        make_graph_fixture("karate_edges", np.array(G.edges()))
        rng = np.random.default_rng(31)
        pr = rng.integers(-50, 400, (3000, 2)); pr[::7, 1] = pr[::7, 0]; pr[1::5] = pr[1::5, ::-1]
        pr = np.r_[pr, pr[:500], [[10 ** 12, -(10 ** 12)], [10 ** 12 + 3, 10 ** 12 + 3]]]
        make_graph_fixture("random_ids", pr)
        pn = rng.integers(0, 1000, (2500, 2)); pn[::3, 1] = pn[::3, 0]
        make_graph_fixture("named_isolated", pn, names=1200)
    if not want("modularity"):
        return
    # --- exact modularity
    mods = []
    for gname, G in [("karate", nx.karate_club_graph()), ("lesmis", nx.les_miserables_graph())]:
        g = as_graph(G); rng = np.random.default_rng(0)
        for c in (1, 2, 4, 9):
            lab = rng.integers(0, c, g.n)
            q = modularity(g, lab, exact=True)
            mods.append(dict(graph=gname, n=int(g.n), u=g.u.tolist(), v=g.v.tolist(), labels=lab.tolist(),
                             num=str(q.numerator), den=str(q.denominator)))
    json.dump(mods, open(os.path.join(HERE, "modularity.json"), "w"))
    print("wrote modularity.json", len(mods))


if __name__ == "__main__":
    main(sys.argv[2] if len(sys.argv) > 2 and sys.argv[1] == "--only" else None)
