#!/usr/bin/env python3
"""Drop-in for the augmented-Lagrangian solver stage (src/lagbound/_core/alm_vcs.py) on a B200.

Same command line, DATA_DIR input files, log lines, checkpoint NPZ (alm_vcs.py:1576-1589) and history JSON as the
reference script, for the configuration the pipeline launches (pipeline.py:116-128): cluster-pair levels, sparse
VCS levels, the triangle pool with both separation families, --init_partition / --resume starts, --pw_rule,
the proximal phase switch, checkpoints.  The state lives on the GPU; every outer iteration is
    sweeps (GPU)  ->  augmented value and effective multipliers (GPU)  ->  multiplier update (GPU)
    [-> VCS separation (GPU) + working-set merge (host)]  [-> triangle separation (GPU) + pool merge (host)]
Options of the reference that production does not use and this stage does not implement (nested or dense-VC
levels, neighbour / connectivity / pair cuts, momentum, line searches, ...) stop it with an error when set.

Extra options (not in the reference): --vdtype f64|f32|bf16 (storage of V on the GPU, default f32) and --device.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import signal
import sys
import threading
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

import numpy as np

from lagbound_b200 import Context, Problem
from lagbound_b200 import pool
from lagbound_b200.problem import locality_order
from lagbound_b200.stages.common import Logger, data_dir, load_instance


def parse(argv):
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--tag", required=True); p.add_argument("--pair_labels", nargs="*", default=[])
    p.add_argument("--resume", default=""); p.add_argument("--init_V", default="")
    p.add_argument("--init_partition", default="")
    p.add_argument("--k", type=int, default=32); p.add_argument("--seed", type=int, default=0)
    p.add_argument("--save", required=True); p.add_argument("--save_last", type=int, default=1)
    p.add_argument("--outer", type=int, default=10 ** 9); p.add_argument("--inner", type=int, default=3)
    p.add_argument("--nbatch", type=int, default=64); p.add_argument("--damp", type=float, default=0.0)
    p.add_argument("--time_limit", type=float, default=3600); p.add_argument("--rho", type=float, default=0.02)
    p.add_argument("--tri_weight", type=float, default=1.0)
    p.add_argument("--tri", type=int, default=1); p.add_argument("--tri_add", type=int, default=500000)
    p.add_argument("--tri_every", type=int, default=3); p.add_argument("--tri_max", type=int, default=5000000)
    p.add_argument("--tri_thresh", type=float, default=0.3); p.add_argument("--tri_maxh", type=int, default=100)
    p.add_argument("--est_every", type=int, default=100); p.add_argument("--est_mix", type=int, default=20)
    p.add_argument("--eig_tol", type=float, default=1e-4); p.add_argument("--init_mix", type=int, default=0)
    p.add_argument("--final_polish", type=float, default=0); p.add_argument("--final_batch", type=int, default=20)
    p.add_argument("--lb", type=float, default=float("nan"))
    p.add_argument("--max_clusters", type=int, default=0)
    p.add_argument("--pair_refresh", type=int, default=1)
    p.add_argument("--shift_p", type=int, default=8)
    p.add_argument("--extra_tri", default="")
    p.add_argument("--tri1_add", type=int, default=0)
    p.add_argument("--tri1_maxk", type=int, default=60); p.add_argument("--tri1_hub", type=int, default=8)
    p.add_argument("--tri1_cap", type=int, default=200)
    p.add_argument("--eig_maxiter", type=int, default=300)
    p.add_argument("--est_damp", type=float, default=0.5)
    p.add_argument("--nbr_cut", type=int, default=0); p.add_argument("--nbr_weight", type=float, default=1.0)
    p.add_argument("--extra_conn", default=""); p.add_argument("--conn_weight", type=float, default=1.0)
    p.add_argument("--diag_out", default=""); p.add_argument("--diag_labels", default="")
    p.add_argument("--extra_pairs", default=""); p.add_argument("--pair_weight", type=float, default=1.0)
    p.add_argument("--pair_add", type=int, default=0); p.add_argument("--pair_hubs", type=int, default=20000)
    p.add_argument("--pair_max", type=int, default=5000000)
    p.add_argument("--ne_split", type=int, default=0)
    p.add_argument("--pairlvl_weight", type=float, default=1.0)
    p.add_argument("--mom", type=float, default=0.0)
    p.add_argument("--est_escape", type=int, default=0); p.add_argument("--est_only", type=int, default=0)
    p.add_argument("--sep_polish", type=int, default=0); p.add_argument("--dual_step", type=float, default=0.0)
    p.add_argument("--dual_mode", default="full"); p.add_argument("--init_sig", default="")
    p.add_argument("--init_tri", type=int, default=0)
    p.add_argument("--ls_etas", default=""); p.add_argument("--ls_mode", default="shrink,full")
    p.add_argument("--ls_what", default="both"); p.add_argument("--ls_rounds", type=int, default=3)
    p.add_argument("--ls_add", default=""); p.add_argument("--ls_add_n", type=int, default=200000)
    p.add_argument("--ckpt_every", type=int, default=0)
    p.add_argument("--slow_bk", type=int, default=0)
    p.add_argument("--pw_auto", type=float, default=0.0); p.add_argument("--pw_rule", default="")
    p.add_argument("--phase2_at", type=float, default=0.0); p.add_argument("--phase2_at_it", type=int, default=0)
    p.add_argument("--phase2_inner", type=int, default=300); p.add_argument("--phase2_w", type=float, default=0.2)
    p.add_argument("--phase2_tri_every", type=int, default=1); p.add_argument("--phase2_est_every", type=int, default=1)
    p.add_argument("--kq_mode", default="trace")
    p.add_argument("--pair_nested", nargs=2, action="append", default=[])
    p.add_argument("--vc_labels", nargs="*", default=[]); p.add_argument("--vc_weight", type=float, default=1.0)
    p.add_argument("--vc_max_clusters", type=int, default=-1); p.add_argument("--vc_kap2", type=float, default=1.0)
    p.add_argument("--vcs_labels", nargs="*", default=[]); p.add_argument("--vcs_full", nargs="*", default=[])
    p.add_argument("--vcs_every", type=int, default=10); p.add_argument("--vcs_first", type=int, default=2)
    p.add_argument("--vcs_add", type=int, default=1000000); p.add_argument("--vcs_max", type=int, default=20000000)
    p.add_argument("--vcs_drop", type=int, default=5); p.add_argument("--vcs_tol", type=float, default=1e-4)
    p.add_argument("--vcs_score", default="pen")
    p.add_argument("--vdtype", default="f32", choices=["f64", "f32", "bf16"])
    p.add_argument("--device", type=int, default=0)
    a = p.parse_args(argv)
    unsupported = [f for f, on in [
        ("--pair_nested", bool(a.pair_nested)), ("--vc_labels", bool(a.vc_labels)), ("--vcs_full", bool(a.vcs_full)),
        ("--nbr_cut", bool(a.nbr_cut)), ("--extra_conn", bool(a.extra_conn)), ("--extra_pairs", bool(a.extra_pairs)),
        ("--pair_add", bool(a.pair_add)), ("--ne_split", bool(a.ne_split)), ("--mom", a.mom > 0),
        ("--pw_auto", a.pw_auto > 0), ("--kq_mode", a.kq_mode != "trace"), ("--pair_refresh", a.pair_refresh != 1),
        ("--slow_bk", bool(a.slow_bk)), ("--sep_polish", bool(a.sep_polish)), ("--dual_step", a.dual_step > 0),
        ("--ls_etas", bool(a.ls_etas)), ("--ls_add", bool(a.ls_add)), ("--diag_out", bool(a.diag_out)),
        ("--est_only", bool(a.est_only)), ("--est_escape", bool(a.est_escape)), ("--init_sig", bool(a.init_sig)),
        ("--final_polish", a.final_polish > 0), ("--vcs_score", a.vcs_score not in ("pen", "mean", "mass"))] if on]
    if unsupported:
        raise SystemExit(f"options not supported by the GPU solver stage: {' '.join(unsupported)}")
    if os.environ.get("ALM_CANON_SWEEPS", "0") == "1" or os.environ.get("VCS_EXACT", "0") == "1":
        raise SystemExit("ALM_CANON_SWEEPS / VCS_EXACT are not supported by the GPU solver stage")
    return a


def capped_labels(lab, d, cap, log, what):
    """Labels 0..P-1; with a cap, the cap - 1 largest-volume clusters are kept and the rest merged into one
    (alm_vcs.py:1133-1137, 1144-1149)."""
    lab = np.unique(lab, return_inverse=True)[1]
    if cap and lab.max() + 1 > cap:
        vol = np.bincount(lab, weights=d)
        keep = np.argsort(-vol)[:cap - 1]
        mp = np.full(len(vol), cap - 1)
        mp[keep] = np.arange(len(keep))
        lab = mp[lab]
        log(f"{what}: capped to {cap} clusters (merged volume share {1 - vol[keep].sum() / vol.sum():.4f})")
    return lab.astype(np.int64)


def colouring_start(lab, inst, k, rng, log):
    """V at a colouring-embedded partition matrix (alm_vcs.py:1198-1211): clusters in decreasing volume take the
    free colour of least accumulated volume among those unused by adjacent clusters (else the least loaded colour);
    V = indicator of the cluster's colour plus 1e-3 Gaussian noise."""
    import scipy.sparse as sp
    n, d = inst["n"], inst["d"]
    lab = np.unique(lab, return_inverse=True)[1]
    P = int(lab.max()) + 1
    rows = np.repeat(np.arange(n), np.diff(inst["indptr"]))
    Cg = sp.csr_matrix((np.ones(len(rows)), (lab[rows], lab[inst["indices"]])), shape=(P, P))
    vol = np.bincount(lab, weights=d, minlength=P)
    col = -np.ones(P, np.int64)
    cvol = np.zeros(k)
    for Q in np.argsort(-vol):
        nb = Cg.indices[Cg.indptr[Q]:Cg.indptr[Q + 1]]
        used = np.zeros(k, bool)
        used[col[nb][col[nb] >= 0]] = True
        free = np.flatnonzero(~used)
        col[Q] = free[np.argmin(cvol[free])] if len(free) else int(np.argmin(cvol))
        cvol[col[Q]] += vol[Q]
    V = np.zeros((n, k))
    V[np.arange(n), col[lab]] = 1.0
    V += 1e-3 * rng.standard_normal(V.shape)
    coo = Cg.tocoo()
    log(f"init partition: {P} clusters -> {k} colours, {int((col[coo.row] == col[coo.col]).sum())} clashing "
        f"cluster adjacencies")
    return V


class Level:
    """Host record of a cluster-pair level: labels, P, rq = |Q| / vol_Q^2 (alm_vcs.py:1181-1184)."""

    def __init__(self, lab, d):
        self.lab = np.asarray(lab, np.int64)
        self.P = int(self.lab.max()) + 1
        cnt = np.bincount(self.lab, minlength=self.P).astype(float)
        vol = np.maximum(np.bincount(self.lab, weights=d, minlength=self.P), 1.0)
        self.rq = cnt / vol ** 2


class VcsState:
    """Host view of a VCS level's working-set structure.  The multipliers and ages live on the GPU; after a device
    update (Problem.vcs_grow) the structure is fetched from the device when it is next read."""

    def __init__(self, lab, name=""):
        self.lab = np.unique(lab, return_inverse=True)[1].astype(np.int64)
        self.P = int(self.lab.max()) + 1
        self.name = name
        self._ptr = np.zeros(len(self.lab) + 1, np.int64)
        self._col = np.zeros(0, np.int32)
        self._device = None            # (problem, level) while the device copy is newer

    def set(self, ptr, col):
        self._ptr, self._col, self._device = np.asarray(ptr, np.int64), np.asarray(col, np.int32), None

    def mark_device(self, prob, level):
        self._device = (prob, level)

    def _sync(self):
        if self._device is not None:
            prob, level = self._device
            self._ptr, self._col = prob.get_vcs_structure(level)
            self._device = None

    @property
    def ptr(self):
        self._sync()
        return self._ptr

    @property
    def col(self):
        self._sync()
        return self._col

    @property
    def nnz(self):
        if self._device is not None:
            prob, level = self._device
            return int(prob.vcs_nnz[level])
        return int(self._ptr[-1])


def main(argv=None):
    a = parse(sys.argv[1:] if argv is None else argv)
    log = Logger(0)
    D = data_dir()
    inst = load_instance(a.tag, D)
    n, m, L, C0, d = inst["n"], inst["m"], inst["L"], inst["C0"], inst["d"]
    z0 = np.load(a.resume) if a.resume else None
    if z0 is not None:
        bad = [k_ for k_ in ("nvc",) if k_ in z0.files and int(z0[k_])]
        bad += [k_ for k_ in ("CI", "PI") if k_ in z0.files and len(z0[k_])]
        bad += [f"nested{li}" for li in range(int(z0["nlev"])) if f"nested{li}" in z0.files and int(z0[f"nested{li}"])]
        if "mu" in z0.files and np.any(z0["mu"]):
            bad.append("mu")
        if bad:
            raise SystemExit(f"checkpoint holds state the GPU solver stage does not support: {bad}")
    # ---- levels
    levels = []
    if z0 is not None and not a.pair_labels:
        for li in range(int(z0["nlev"])):
            assert int(z0[f"pair{li}"]), "only cluster-pair levels are supported"
            levels.append(Level(np.unique(z0[f"lab{li}"], return_inverse=True)[1], d))
    else:
        for f in a.pair_labels:
            levels.append(Level(capped_labels(np.load(f), d, a.max_clusters, log, f"level {f.split('/')[-1]}"), d))
    vcsl = [VcsState(np.load(f), f.split("/")[-1]) for f in a.vcs_labels]
    if z0 is not None and "nvcs" in z0.files:
        if not vcsl:
            vcsl = [VcsState(z0[f"vcslab{mm}"]) for mm in range(int(z0["nvcs"]))]
    rng = np.random.default_rng(a.seed)
    TI = np.zeros((0, 3), np.int64)
    lam = np.zeros(0)
    vcs_resume = {}
    if z0 is not None:
        V = z0["V"].astype(np.float64)
        TI, lam, merged = pool.normalise(z0["TI"], z0["lam"], n)
        if merged:
            log("merged duplicate triangles ->", len(TI))
        sig_resume = {li: z0[f"sig{li}"].astype(np.float64) for li, Lv in enumerate(levels)
                      if f"sig{li}" in z0.files and z0[f"sig{li}"].shape == (Lv.P, Lv.P)}
        for mm, Lv in enumerate(vcsl):
            if "nvcs" in z0.files and mm < int(z0["nvcs"]) and \
                    np.array_equal(Lv.lab, np.unique(z0[f"vcslab{mm}"], return_inverse=True)[1]):
                if int(z0[f"vcsfull{mm}"]):
                    raise SystemExit("full VCS levels are not supported by the GPU solver stage")
                vcs_resume[mm] = (z0[f"vcsptr{mm}"].astype(np.int64), z0[f"vcscol{mm}"].astype(np.int32),
                                  z0[f"vcssig{mm}"].astype(np.float64))
        z0.close()
    elif a.init_partition:
        sig_resume = {}
        V = colouring_start(np.load(a.init_partition), inst, a.k, rng, log)
    elif a.init_V:
        sig_resume = {}
        V = np.load(a.init_V).astype(np.float64)
    else:
        sig_resume = {}
        V = rng.standard_normal((n, a.k))
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    k = V.shape[1]
    if a.extra_tri:
        E = np.load(a.extra_tri)["TI"].astype(np.int64)
        E = np.stack([np.minimum(E[:, 0], E[:, 2]), E[:, 1], np.maximum(E[:, 0], E[:, 2])], 1)
        ke = pool.tri_keys(E, n)
        _, fi = np.unique(ke, return_index=True)
        E, ke = E[fi], ke[fi]
        E = E[~np.isin(ke, pool.tri_keys(TI, n))]
        TI = np.vstack([TI, E]) if len(TI) else E
        lam = np.concatenate([lam, np.zeros(len(E))])
        log(f"merged {len(E)} extra triangles -> {len(TI)}")
    for mm, Lv in enumerate(vcsl):
        if mm in vcs_resume:
            Lv.set(*vcs_resume[mm][:2])
            log(f"resumed vcs level {mm}: nnz {Lv.nnz} sig sum {vcs_resume[mm][2].sum():.4g}")
        log(f"VCS level {Lv.name}: P {Lv.P} active-set nnz {Lv.nnz} ({Lv.nnz * 33 / 2 ** 20:.0f} MB)")
    for Lv in levels:
        log("pair level clusters", Lv.P, "")
    # ---- device state
    ctx = Context(a.device)
    order = locality_order(levels[0].lab) if levels else (locality_order(vcsl[0].lab) if vcsl else None)
    prob = Problem(ctx, n, inst["indptr"], inst["indices"], inst["weights"], d, L, C0, k, dtype=a.vdtype,
                   order=order)
    prob.set_V(V)
    pw = float(a.pairlvl_weight)
    for li, Lv in enumerate(levels):
        prob.add_pair_level(Lv.lab, Lv.P, pw)
        if li in sig_resume:
            prob.set_pair_sigma(li, sig_resume[li])
    for mm, Lv in enumerate(vcsl):
        prob.add_vcs_level(Lv.lab, Lv.P, float(a.vc_weight) * pw)
        if mm in vcs_resume:
            prob.set_vcs_ws(mm, Lv.ptr, Lv.col, vcs_resume[mm][2])
    prob.set_pair_weight(pw, a.vc_weight)
    prob.set_triangles(TI, lam)

    def sweeps(nsw, rho, rt, damp):
        """nsw sweeps, each over a fresh rng.permutation(n) (alm_vcs.py:1384), split into nbatch batches."""
        if nsw:
            perms = np.stack([rng.permutation(n) for _ in range(nsw)])
            prob.sweeps(perms, rho, rt, damp, a.nbatch, a.vc_kap2)

    if a.init_mix:
        sweeps(a.init_mix, 0.0, 0.0, a.damp)
        V = prob.get_V()
    W_AUTO = None
    if a.pw_rule and levels:
        R0 = mobility_ratio(ctx, inst, V, levels, a.rho, pw)
        W_AUTO, msg = pair_weight_rule(a.pw_rule, R0, pw, a.rho, n, L)
        log(msg)
        pw = W_AUTO
        prob.set_pair_weight(pw, a.vc_weight)
    a.pairlvl_weight = pw

    writer = [None, None]      # the checkpoint being written in the background, and its error

    def flush():
        """Wait for the checkpoint being written; re-raise its error."""
        if writer[0] is not None:
            writer[0].join()
            writer[0] = None
            if writer[1] is not None:
                err, writer[1] = writer[1], None
                raise err

    def save(path, W=None):
        """Checkpoint in the reference's schema (alm_vcs.py:1576-1589); W defaults to the current V.  The arrays are
        read from the device here; the file is written by a background thread while the solver continues (one
        write at a time; the stage waits for it before it exits)."""
        TI_, lam_ = pool_TI(), prob.get_lam()
        W = prob.get_V() if W is None else W
        dd = {"TI": TI_, "lam": lam_, "V": W.astype(np.float32), "nlev": len(levels), "mu": np.zeros(n),
              "CI": np.zeros((0, 3), np.int64), "om": np.zeros(0), "PI": np.zeros((0, 2), np.int64), "psi": np.zeros(0)}
        for li, Lv in enumerate(levels):
            sg = prob.get_pair_sigma(li)
            dd[f"lab{li}"] = Lv.lab; dd[f"sig{li}"] = 0.5 * (sg + sg.T); dd[f"dense{li}"] = 1; dd[f"pair{li}"] = 1
        dd["nvc"] = 0
        dd["nvcs"] = len(vcsl)
        for mm, Lv in enumerate(vcsl):
            sg, _ = prob.get_vcs_ws(mm)
            dd[f"vcslab{mm}"] = Lv.lab; dd[f"vcsptr{mm}"] = Lv.ptr; dd[f"vcscol{mm}"] = Lv.col
            dd[f"vcssig{mm}"] = sg.astype(np.float32); dd[f"vcsfull{mm}"] = 0
        flush()

        def write():
            try:
                tmp = path.replace(".npz", ".tmp.npz")
                np.savez(tmp, **dd)
                os.replace(tmp, path)
            except BaseException as e:          # reported by the next flush()
                writer[1] = e
        writer[0] = threading.Thread(target=write, daemon=False)
        writer[0].start()

    stop = [False]

    def _stop(*_):
        stop[0] = True
    signal.signal(signal.SIGTERM, _stop)
    signal.signal(signal.SIGINT, _stop)

    TI_cur = [TI]          # host copy of the pool's triangles; None while the device pool is newer

    def pool_TI():
        if TI_cur[0] is None:
            TI_cur[0] = prob.get_triangles()
        return TI_cur[0]
    PH2 = False
    log(f"[C0/L {C0 / L:.6f}] n {n} m {m} k {k} levels {[Lv.P for Lv in levels]} ntri {len(lam)} rho {a.rho} "
        f"nbatch {a.nbatch}")
    hist = []
    best = np.inf
    rho = a.rho
    ev = prob.eval(rho, a.tri_weight, grad=False)
    log(f"start L {ev['value'] / L:.6f} primal {ev['primal'] / L:.6f}")
    tsweep = tsep = test = 0.0
    tvcs = 0.0
    for it in range(1, a.outer + 1):
        if not PH2 and phase2_due(a, it, time.time() - log.t0):
            PH2 = True
            pw = phase2_weight(a, W_AUTO); a.pairlvl_weight = pw
            prob.set_pair_weight(pw, a.vc_weight)
            a.inner = a.phase2_inner; a.tri_every = a.phase2_tri_every; a.est_every = a.phase2_est_every
            log(f"PHASE2 at outer {it}: inner {a.inner}, pairlvl_weight {a.pairlvl_weight:.4g}, tri_every "
                f"{a.tri_every}, est_every {a.est_every}")
        ts = time.time()
        sweeps(a.inner, rho, rho * a.tri_weight, a.damp)
        ctx.synchronize()
        tsweep += time.time() - ts
        ev = prob.eval(rho, a.tri_weight, grad=False)
        Lc, prim = ev["value"], ev["primal"]
        nviol = int(ev["nviol"])
        vcs_nv = int(ev["vcs_nviol"])
        tviol = float(max(0.0, -ev["gmin"])) if prob.T else 0.0
        prob.multiplier_update()
        vcs_msg = ""
        if vcsl and not stop[0] and it < a.outer and (it % a.vcs_every == 0 or it == a.vcs_first):
            for mm, Lv in enumerate(vcsl):
                ts = time.time()
                nz0 = Lv.nnz
                # keep age < vcs_drop, room = vcs_max - kept, separate and merge: all on the device
                ndrop, nnew, stv = prob.vcs_grow(mm, a.vcs_add, a.vcs_tol, a.vcs_score,
                                                 drop_age=a.vcs_drop if 0 < a.vcs_drop <= 255 else 0,
                                                 max_nnz=a.vcs_max)
                Lv.mark_device(prob, mm)
                tvcs += time.time() - ts
                vcs_msg += (f" vcs[{Lv.name}] nnz {nz0}->{Lv.nnz} (-{ndrop} +{nnew}) viol "
                            f"{stv['nviol']:.4g} (ws {stv['nviol_ws']:.4g}) mass/L2 {stv['mass'] / L ** 2:.4g} "
                            f"(ws {stv['mass_ws'] / L ** 2:.4g}) [{time.time() - ts:.1f}s]")
        sep_now = a.tri and it % a.tri_every == 0 and not stop[0]
        msg = ""
        if sep_now:
            ts = time.time()
            # purge lam = 0, separate when there is room, merge: the pool stays on the device
            _, nadd = prob.tri_pool_round(a.tri_thresh, a.tri_maxh, a.tri1_maxk, a.tri1_hub, a.tri1_cap, a.tri_add,
                                          a.tri1_add, a.tri_max)
            TI_cur[0] = None
            if nadd or prob.T < a.tri_max:
                msg = f" +{nadd}tri"
            tsep += time.time() - ts
        ntri = prob.T
        rec = dict(outer=it, t=round(time.time() - log.t0, 1), Laug=Lc / L, primal=prim / L, nviol=nviol,
                   tviol=tviol, ntri=int(ntri))
        if vcsl:
            sums = [prob.vcs_sig_stats(mm) for mm in range(len(vcsl))]
            vsig = float(sum(s_ for s_, _ in sums))
            rec.update(vcs_nnz=[Lv.nnz for Lv in vcsl], vcs_viol=vcs_nv, vcs_sig=vsig)
            msg += (f" vcsviol {vcs_nv} vcssig {vsig:.4g} nnz {[Lv.nnz for Lv in vcsl]} act {[c_ for _, c_ in sums]} "
                    f"[vcs sep {tvcs:.0f}s]" + vcs_msg)
        line = (f"it {it} L {Lc / L:.6f} prim {prim / L:.6f} viol {nviol} tviol {tviol:.3f} ntri {ntri}{msg} "
                f"[sweep {tsweep:.0f}s (rowsteps {tsweep:.0f}s) sep {tsep:.0f}s est {test:.0f}s]")
        last = stop[0] or it == a.outer or time.time() - log.t0 > a.time_limit
        if a.est_every > 0 and (it % a.est_every == 0 or last):
            ts = time.time()
            if a.save_last:
                save(a.save.replace(".npz", "_last.npz"))
            ub, lmin, W, dv = estimate_in_loop(a, prob, ctx, inst, levels, vcsl, pool_TI(), sweeps, log)
            test += time.time() - ts
            rec.update(est=ub, dv=dv, lmin=lmin)
            if ub < best:
                best = ub
                save(a.save, W)
                line += " *"
            if a.save_last:
                save(a.save.replace(".npz", "_last.npz"), W)
            line += f" EST {ub:.6f} (dv {dv:.6f}) best {best:.6f} lmin {lmin:.1e}"
        if (last and a.est_every <= 0) or (a.ckpt_every > 0 and it % a.ckpt_every == 0 and
                                           not (a.est_every > 0 and it % a.est_every == 0)):
            save(a.save.replace(".npz", "_last.npz"))
        log(line)
        hist.append(rec)
        if it % 20 == 0 or last:
            json.dump(hist, open(a.save.replace(".npz", ".history.json"), "w"))
        if last:
            break
    flush()
    log(f"BEST {best:.6f}  (estimate only)")
    prob.close()
    ctx.close()


def mobility_ratio(ctx, inst, V, levels, rho, w):
    """(alm_vcs.py:1625-1641) volume-weighted mean over rows of kappa_i / |(B V)_i| at pair weight w with every pair
    active (mobility_ratio_from).  B V comes from a level-free FP64 evaluation on the GPU."""
    n, d = inst["n"], inst["d"]
    k = V.shape[1]
    tmp = Problem(ctx, n, inst["indptr"], inst["indices"], inst["weights"], d, inst["L"], inst["C0"], k, dtype="f64")
    try:
        tmp.set_V(V)
        tmp.eval(grad=True, fixed=True)
        gB = np.linalg.norm(tmp.G(), axis=1)
    finally:
        tmp.close()
    return mobility_ratio_from(gB, d, V, levels, rho, w)


def mobility_ratio_from(gB, d, V, levels, rho, w):
    """(alm_vcs.py:1625-1641) sum_i d_i kappa_i / max(|(B V)_i|, 1e-9) / sum_i d_i with kappa_i = d_i^2 sum over
    levels of 2 rho (r y2 + diag(r) y2)[Q(i)], r = rq rq^T w, y2 = |Y_Q|^2, Y_Q = sum_{i in Q} d_i v_i; gB[i] =
    |(B V)_i|."""
    n, k = V.shape
    kap = np.zeros(n)
    for Lv in levels:
        Y = np.zeros((Lv.P, k))
        np.add.at(Y, Lv.lab, d[:, None] * V)
        y2 = (Y * Y).sum(1)
        r_ = np.outer(Lv.rq, Lv.rq) * w
        kap += d ** 2 * (2 * rho * (r_ @ y2 + np.diag(r_) * y2))[Lv.lab]
    return float(np.sum(d * kap / np.maximum(gB, 1e-9)) / d.sum())


def pair_weight_rule(rule, R0, w0, rho, n, L):
    """--pw_rule (alm_vcs.py:1647-1653): the pair weight min(c1 / R(1), c2 / (rho n^2 / L)) with R(1) = R0 / w0 the
    mobility ratio at weight 1 (R0 measured at the current weight w0); c1, c2 from the rule string "c1,c2" (empty
    parts and "default" / "on" / "1" keep 0.1 and 0.05).  Returns (weight, the reference's log line)."""
    R1 = R0 / w0
    pr = [] if rule in ("default", "on", "1") else rule.split(",")
    c1 = float(pr[0]) if len(pr) > 0 and pr[0] else 0.1
    c2 = float(pr[1]) if len(pr) > 1 and pr[1] else 0.05
    n2L = n * float(n) / L
    wm, wsp = c1 / R1, c2 / (rho * n2L)
    w = min(wm, wsp)
    msg = (f"pw_rule c1 {c1:g} c2 {c2:g}: R(1) {R1:.6g} (R at w {w0:g}: {R0:.4g}), n {n} L {L} n^2/L {n2L:.4g} rho "
           f"{rho:g} | w_mob = c1/R {wm:.6g}, w_step = c2/(rho n^2/L) {wsp:.6g} -> pairlvl_weight {w:.6g} "
           f"({'mob' if wm <= wsp else 'step'})")
    return w, msg


def phase2_due(a, it, elapsed):
    """The phase-2 switch condition of the main loop (alm_vcs.py:1663): after phase2_at seconds, or once the outer
    iteration passes phase2_at_it (the caller switches only once)."""
    return (a.phase2_at > 0 and elapsed > a.phase2_at) or (a.phase2_at_it > 0 and it > a.phase2_at_it)


def phase2_weight(a, w_auto):
    """The phase-2 pair weight (alm_vcs.py:1664): phase2_w times the rule's weight, or phase2_w itself without a
    rule."""
    return float(a.phase2_w * w_auto if w_auto is not None else a.phase2_w)


def estimate_in_loop(a, prob, ctx, inst, levels, vcsl, TI, sweeps, log):
    """The main loop's estimate (alm_vcs.py:1536-1566) at the current multipliers: est_mix plain-mixing sweeps of a
    copy of V, W rounded to FP32, g = rowdot(C W, W), then the uniform shift n max(0, -lambda_min(Diag(g) - C))
    (with --shift_p, a per-vertex shift from the shift_p lowest eigenpairs first).  Leaves V as it was."""
    import scipy.sparse.linalg as sla
    from lagbound_b200.estimator import FixedOperator
    n, L, C0, d = inst["n"], inst["L"], inst["C0"], inst["d"]
    V0 = prob.get_V()
    sweeps(a.est_mix, 0.0, 0.0, a.est_damp)
    W = prob.get_V().astype(np.float32).astype(np.float64)
    prob.set_V(V0)
    lam = prob.get_lam()
    pair = [(Lv.lab, Lv.P, prob.get_pair_sigma(li)) for li, Lv in enumerate(levels)]
    vcs = [(Lv.lab, Lv.P, Lv.ptr, Lv.col, prob.get_vcs_ws(mm)[0]) for mm, Lv in enumerate(vcsl)]
    op = FixedOperator(ctx, n, inst["indptr"], inst["indices"], inst["weights"], d, L, C0, pair, vcs, TI, lam)
    try:
        gd = np.einsum("ij,ij->i", op(W), W)
        t = np.zeros(n)

        def mv(x, tt):
            x = x.reshape(-1)
            return (gd + tt) * x - op(x.reshape(-1, 1))[:, 0]
        for _ in range(3 if a.shift_p > 0 else 0):
            A_ = sla.LinearOperator((n, n), matvec=lambda x, tt=t.copy(): mv(x, tt), dtype=float)
            ev, Q = sla.eigsh(A_, k=a.shift_p, which="SA", tol=a.eig_tol, maxiter=20000, ncv=max(48, 3 * a.shift_p))
            neg = ev < 0
            if not neg.any():
                break
            for j in np.flatnonzero(neg):
                q = Q[:, j]
                t += 1.02 * abs(ev[j]) * np.abs(q) * np.abs(q).sum()
        A_ = sla.LinearOperator((n, n), matvec=lambda x: mv(x, t), dtype=float)
        try:
            ev_, _ = sla.eigsh(A_, k=1, which="SA", tol=a.eig_tol, maxiter=a.eig_maxiter, ncv=32)
            lmin = float(ev_.min())
        except sla.ArpackNoConvergence as e_:
            lmin = float(np.min(e_.eigenvalues)) if len(e_.eigenvalues) else float("nan")
            log("eigsh not converged; lmin estimate", lmin)
        base = C0 + lam.sum() + gd.sum()
        ub = (base + t.sum() + n * max(0.0, -lmin)) / L
        return ub, lmin, W, base / L
    finally:
        op.close()


if __name__ == "__main__":
    main()
