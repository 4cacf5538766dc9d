#!/usr/bin/env python3
"""Drop-in for the bound-estimate stage (src/lagbound/_core/est_dual_vcs.py) on a B200.

Same command line, DATA_DIR input files, checkpoint input, log lines, JSON output (ub, dv, s_<scale> records with
lmin_est, escape_rounds, ...) and --saveW NPZ as the reference script for the checkpoints the solver writes
(cluster-pair levels, sparse VCS levels, triangles): the products C(y) X run on the GPU (FP64) and, by default,
the Riemannian polish and the LOBPCG blocks too.  --polish mix is refused with VCS levels, as in the reference.

Extra options (not in the reference): --device, --vectors gpu|host (default gpu: the polish and LOBPCG blocks stay
on the GPU, lagbound_b200/estimator_gpu.py; host: NumPy vectors and SciPy's LOBPCG as the reference, with only the
products on the GPU).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))

import numpy as np

from lagbound_b200 import Context
from lagbound_b200 import estimator as E
from lagbound_b200 import pool
from lagbound_b200.problem import locality_order
from lagbound_b200.stages.common import Logger, data_dir, load_instance


def parse(argv):
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--tag", required=True); p.add_argument("--ckpt", required=True)
    p.add_argument("--polish", default="mix")
    p.add_argument("--max_sweeps", type=int, default=200); p.add_argument("--polish_time", type=float, default=600)
    p.add_argument("--chk", type=int, default=5)
    p.add_argument("--ptol", type=float, default=2e-5)
    p.add_argument("--damp", type=float, default=0.5); p.add_argument("--nbatch", type=int, default=64)
    p.add_argument("--rgd_iters", type=int, default=400)
    p.add_argument("--scale", default="vol,ones")
    p.add_argument("--eig_extra", type=int, default=16)
    p.add_argument("--eig_maxiter", type=int, default=400); p.add_argument("--eig_tol", type=float, default=1e-9)
    p.add_argument("--eig_chunk", type=int, default=20)
    p.add_argument("--eig_atol", type=float, default=1e-5)
    p.add_argument("--eig_time", type=float, default=1200)
    p.add_argument("--dense", type=int, default=0)
    p.add_argument("--seed", type=int, default=0); p.add_argument("--out", default="")
    p.add_argument("--saveW", default=""); p.add_argument("--initV", default="")
    p.add_argument("--no_w_init", type=int, default=0); p.add_argument("--lb", type=float, default=float("nan"))
    p.add_argument("--escape", type=int, default=2)
    p.add_argument("--escape_min", type=float, default=0.002)
    p.add_argument("--escape_p", type=int, default=4)
    p.add_argument("--escape_ratio", type=float, default=0.3)
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--vectors", default="gpu", choices=["gpu", "host"])
    a = p.parse_args(argv)
    if a.dense:
        raise SystemExit("--dense is not supported by the GPU estimate stage")
    return a


def main(argv=None):
    a = parse(sys.argv[1:] if argv is None else argv)
    rng = np.random.default_rng(a.seed)
    log = Logger(1)
    D = data_dir()
    inst = load_instance(a.tag, D)
    n, m, L, C0, d = inst["n"], inst["m"], inst["L"], inst["C0"], inst["d"]
    z0 = np.load(a.ckpt)
    nl = int(z0["nlev"])
    pair = []
    for li in range(nl):
        if f"nested{li}" in z0.files and int(z0[f"nested{li}"]):
            raise SystemExit("nested levels are not supported by the GPU estimate stage")
        lab = np.unique(z0[f"lab{li}"], return_inverse=True)[1].astype(np.int64)
        P = int(lab.max()) + 1
        sig = z0[f"sig{li}"].astype(np.float64)
        assert sig.shape == (P, P) and (sig >= 0).all()
        pair.append((lab, P, sig))
    TI = z0["TI"].astype(np.int64)
    lam = z0["lam"].astype(np.float64)
    mu = z0["mu"].astype(np.float64) if "mu" in z0.files and z0["mu"].shape == (n,) else np.zeros(n)
    om = z0["om"].astype(np.float64) if "om" in z0.files else np.zeros(0)
    if mu.any() or (om > 0).any() or ("nvc" in z0.files and int(z0["nvc"])):
        raise SystemExit("neighbour / connectivity cuts and dense VC levels are not supported by the GPU estimate stage")
    vcs = []
    for mm in range(int(z0["nvcs"]) if "nvcs" in z0.files else 0):
        lab = np.unique(z0[f"vcslab{mm}"], return_inverse=True)[1].astype(np.int64)
        P = int(lab.max()) + 1
        ptr = z0[f"vcsptr{mm}"].astype(np.int64); col = z0[f"vcscol{mm}"].astype(np.int32)
        sig = z0[f"vcssig{mm}"].astype(np.float64)
        assert (sig >= 0).all() and ptr[-1] == len(col) and (col >= 0).all() and (col < P).all()
        vcs.append((lab, P, ptr, col, sig))
    V = z0["V"].astype(np.float64)
    z0.close()
    if a.initV:
        V = np.load(a.initV)["V"].astype(np.float64)
    assert (lam >= 0).all()
    if len(TI):
        TI, lam, merged = pool.normalise(TI, lam, n)
        if merged:
            log("merged duplicate triangles ->", len(TI))
        TI, lam = pool.purge(TI, lam)
    const = C0 + lam.sum()
    V /= np.maximum(np.linalg.norm(V, axis=1, keepdims=True), 1e-300)
    V = np.ascontiguousarray(V)
    k = V.shape[1]
    log(f"tag {a.tag} ckpt {a.ckpt} n {n} m {m} L {L} k {k} vc levels [] vcs levels {[(v[1], len(v[3])) for v in vcs]} "
        f"levels {[p_[1] for p_ in pair]} ntri {len(lam)} nconn 0 mu False C0/L {C0 / L:.6f} const/L {const / L:.6f}")
    if vcs and "mix" in a.polish.split("+"):
        raise SystemExit("--polish mix not supported with nested levels")
    ctx = Context(a.device)
    order = locality_order(pair[0][0]) if pair else None
    gpu = a.vectors == "gpu"
    if gpu:
        import torch
        from lagbound_b200 import estimator_gpu as EG
        op = EG.DeviceOperator(ctx, n, inst["indptr"], inst["indices"], inst["weights"], d, L, C0, pair, vcs, TI,
                               lam, order=order)
        V = torch.as_tensor(V, dtype=torch.float64, device=op.dev)
        M = EG
    else:
        op = E.FixedOperator(ctx, n, inst["indptr"], inst["indices"], inst["weights"], d, L, C0, pair, vcs, TI, lam,
                             order=order)
        M = E
    hist = []

    def do_polish(W):
        for meth in a.polish.split("+"):
            if meth == "rgd":
                W = M.polish_rgd(op, W, const, L, a.rgd_iters, a.polish_time, a.ptol, log, hist)
            elif meth == "mix":
                raise SystemExit("--polish mix is not supported by the GPU estimate stage; use rgd")
        return W

    tpol = time.time()
    dv0 = M.value(op, V, const, L)[0]
    V = do_polish(V)
    tpol = time.time() - tpol
    dv, g, CW = M.value(op, V, const, L)
    log(f"POLISHED dv {dv:.6f} (start {dv0:.6f}) in {tpol:.0f}s")
    res = dict(tag=a.tag, ckpt=a.ckpt, n=n, L=L, k=k, dv0=dv0, dv=dv, polish_time=tpol, polish_hist=hist, lb=a.lb)
    scales = a.scale.split(",")
    best = np.inf
    eigvecs = {}
    Vbest = V
    rounds = []
    for rnd in range(a.escape + 1):
        if gpu:
            recs, vecs = EG.eig_round(op, V, dv, g, d, L, a.seed + rnd, scales, a.eig_extra, a.eig_maxiter,
                                      a.eig_chunk, a.eig_atol, a.eig_time, bool(a.no_w_init), log)
        else:
            recs, vecs = E.eig_round(op, V, dv, g, d, L, rng, scales, a.eig_extra, a.eig_maxiter, a.eig_tol,
                                     a.eig_chunk, a.eig_atol, a.eig_time, bool(a.no_w_init), log)
        ub_r = min(r["ub"] for r in recs.values())
        rounds.append(dict(round=rnd, dv=dv, ub=ub_r, k=int(V.shape[1])))
        log(f"[round {rnd}] k {V.shape[1]} dv {dv:.6f} UB {ub_r:.6f}")
        if ub_r < best:
            best = ub_r
            Vbest = V
            res["dv"] = dv
            for s_, r_ in recs.items():
                res[f"s_{s_}"] = r_
            eigvecs = {s_: np.asarray(v_[1][:, :4].cpu() if gpu else v_[1][:, :4], np.float32)
                       for s_, v_ in vecs.items()}
        if rnd == a.escape:
            break
        th, Xe = vecs[scales[0]]
        if recs[scales[0]]["shift"] < a.escape_min:
            break
        V2, sel = M.escape_vectors(V, th, Xe, a.escape_ratio, a.escape_p)
        if not sel:
            break
        V = V2
        tp = time.time()
        V = do_polish(V)
        dv, g, CW = M.value(op, V, const, L)
        log(f"ESCAPE round {rnd + 1}: appended {len(sel)} eigenvectors (theta {th[sel]}), re-polished dv {dv:.6f} "
            f"k {V.shape[1]} ({time.time() - tp:.0f}s)")
    res["escape_rounds"] = rounds
    res["ub"] = best
    res["time"] = time.time() - log.t0
    res["operator_calls"] = op.calls
    if np.isfinite(a.lb):
        res["gap"] = (best - a.lb) / a.lb
    log(f"RESULT dv {res['dv']:.6f}  UB {best:.6f}" +
        (f"  gap {(best - a.lb) / a.lb * 100:.2f}%" if np.isfinite(a.lb) else "") + f"  total {time.time() - log.t0:.0f}s")
    if a.out:
        json.dump(res, open(a.out, "w"), indent=1)
    if a.saveW:
        Vb = Vbest.cpu().numpy() if gpu else Vbest
        np.savez(a.saveW, V=Vb.astype(np.float32), **{f"eig_{k_}": v_ for k_, v_ in eigvecs.items()})
    op.close()
    ctx.close()


if __name__ == "__main__":
    main()
