#!/usr/bin/env python3
"""Test infrastructure: the reference's own certificate chain (api.py:272-298: repair, estimate, repair, sparse
lifted certificate, independent verification) run on CPU on a workspace written by the GPU stages
(lagbound_b200/stages/workflow.py), so that the bound the GPU path reports is accepted or rejected by the
reference's verifier alone.  Runs where the reference source tree exists ($LAGBOUND_REF, or an importable
lagbound package from the reference project: oracle/refpath.py).  The certificate and verifier import pymetis for
their orderings: --ordering rcm gives them the stand-in under oracle/_stub (reverse Cuthill-McKee), --ordering nd
this library's nested dissection (lagbound_b200/dropin).

    python oracle/reference_chain.py <workdir> [--margin 2] [--method ldl] [--ordering rcm|nd]
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from refpath import reference_root  # noqa: E402

REF = reference_root()


def main():
    p = argparse.ArgumentParser()
    p.add_argument("workdir")
    p.add_argument("--ckpt", default="", help="checkpoint to certify (default: the best estimate of summary.json)")
    p.add_argument("--margin", type=float, default=2.0)
    p.add_argument("--method", default="ldl")
    p.add_argument("--polish_time", type=float, default=1500); p.add_argument("--eig_time", type=float, default=1200)
    p.add_argument("--reference_solve", type=float, default=0.0,
                   help="> 0: first run the reference's own solver phases (this many seconds in total, the GPU "
                        "workflow's proximal fraction) and estimates on the same reduced instance, and certify that")
    p.add_argument("--no_certify", action="store_true", help="stop after the estimates (large instances)")
    p.add_argument("--ordering", default="rcm", choices=["rcm", "nd"],
                   help="the pymetis the certificate and verifier import: rcm = the test stand-in under oracle/_stub "
                        "(reverse Cuthill-McKee), nd = lagbound_b200/dropin (this library's nested dissection)")
    a = p.parse_args()
    stub = os.path.join(HERE, "_stub") if a.ordering == "rcm" else \
        os.path.join(os.path.dirname(HERE), "lagbound_b200", "dropin")
    sys.path[:0] = [os.path.join(REF, "src"), stub]
    os.environ["PYTHONPATH"] = os.pathsep.join([os.path.join(REF, "src"), stub, os.environ.get("PYTHONPATH", "")])
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join("/tmp", "lagbound_numba_cache"))
    from lagbound.pipeline import Workspace
    ws = Workspace(None, a.workdir, threads=os.cpu_count())
    summary = json.load(open(os.path.join(ws.root, "summary.json")))
    ckpt = a.ckpt or (os.path.join(ws.root, "runs", os.path.basename(summary["best_ckpt"]))
                      if "best_ckpt" in summary else "")
    labels = os.path.join(ws.root, "data", "g", "partition.npy")
    t0 = time.time()
    ref_est = None
    if not os.path.exists(os.path.join(ws.root, "data", "g__rx", "graph.json")):
        ws.reduce([labels])              # a workspace holding only data/g: reduce with the reference
    if a.reference_solve > 0:
        init_r = ws.reduced_labels(labels)
        n_red = json.load(open(os.path.join(ws.root, "data", "g__rx", "graph.json")))["n"]
        nbatch = summary.get("nbatch") or (512 if n_red >= 512 * 64 else min(n_red, max(8, n_red // 64)))
        solver = dict(lb=float("nan"), outer=3000, nbatch=nbatch, max_clusters=6000)
        t_main = 0.7 * a.reference_solve
        main_ck, weight = ws.solve("ref_main", [init_r], init_r, time_limit=t_main, init=init_r, **solver)
        prox_ck, _ = ws.solve("ref_proximal", [init_r], init_r, time_limit=max(1.0, a.reference_solve - t_main),
                              resume=main_ck, pair_weight=weight, proximal=True, **solver)
        ests = {nm: ws.estimate(f"ref_est_{nm}", ck, float("nan")) for nm, ck in (("main", main_ck),
                                                                                   ("proximal", prox_ck))}
        best = min(ests, key=lambda k_: ests[k_]["ub"])
        ckpt = {"main": main_ck, "proximal": prox_ck}[best]
        ref_est = dict(pair_weight=weight, estimates={k_: v_["ub"] for k_, v_ in ests.items()},
                       solve_seconds=time.time() - t0)
    if a.no_certify:
        out = dict(reference_solve=ref_est, gpu_estimate=summary.get("estimate"),
                   planted_modularity=summary.get("planted_modularity"), seconds=time.time() - t0)
        json.dump(out, open(os.path.join(ws.root, "reference_chain_estimates.json"), "w"), indent=1)
        print(json.dumps(out))
        return
    fix_v = ws.repair(ckpt, ws.path("runs", "cert_fixV.npz"), 10)
    est = ws.estimate("cert_est", ckpt, float("nan"), init_v=fix_v, save_w=ws.path("runs", "cert_W.npz"),
                      polish_time=a.polish_time, eig_time=a.eig_time)
    w2 = ws.repair(ckpt, ws.path("runs", "cert_W2.npz"), 3, init_w=ws.path("runs", "cert_W.npz"))
    cert = ws.certify("certificate", ckpt, w2, est["json"], margin=a.margin)
    res = ws.verify(cert["file"], a.method, labels)
    def find(d, key):
        if isinstance(d, dict):
            if key in d:
                return d[key]
            for v in d.values():
                r = find(v, key)
                if r is not None:
                    return r
        return None
    out = dict(ordering=a.ordering, cert_fill=cert.get("fill"), cert_seconds=cert.get("seconds"),
               verify_nnzL=find(res, "nnzL"), verify_seconds=res.get("seconds"), ckpt=ckpt, reference_solve=ref_est, gpu_estimate=summary.get("estimate"), planted_modularity=summary.get("planted_modularity"),
               cpu_cert_estimate=est["ub"], certified_UB=float(cert["UB"]), verified=bool(res.get("passed")),
               verified_UB=float(res["UB"]) if res.get("passed") else None, verifier=res.get("fail"),
               seconds=time.time() - t0)
    name = "reference_chain_refsolve.json" if ref_est else "reference_chain.json"
    if a.ordering != "rcm":
        name = name.replace(".json", f"_{a.ordering}.json")
    json.dump(out, open(os.path.join(ws.root, name), "w"), indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
