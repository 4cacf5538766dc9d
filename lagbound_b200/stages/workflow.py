#!/usr/bin/env python3
"""The upper-bound workflow of the reference (api.py:224-270 _sdp_upper_bound, stages 2-6) run with the GPU stage
scripts only, for hosts without the reference package: exact reduction, solver main phase, proximal phase and the
bound estimates of both checkpoints, with the production flags of pipeline.py:105-170.  The certificate and its
verification (stages 7-8) are the reference's own scripts, run afterwards on the files this writes:

    python -m lagbound_b200.stages.workflow --workdir W --graph sbm [--time 120] [--n 2000] ...

The working directory has the reference's layout (data/g/..., data/g__rx/..., runs/...), so the reference's
repair / certify / verify stages can be pointed at it.  A summary is written to W/summary.json.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TAG = "g"


class Workspace:
    """The reference's workspace layout and stage launch convention (pipeline.py:29-76) for the GPU stages."""

    def __init__(self, root, keys=None, n=None, vdtype="f32"):
        self.root = os.path.abspath(root)
        self.data = os.path.join(self.root, "data")
        self.runs = os.path.join(self.root, "runs")
        self.vdtype = vdtype
        os.makedirs(os.path.join(self.data, TAG), exist_ok=True)
        os.makedirs(self.runs, exist_ok=True)
        if keys is not None:
            np.save(os.path.join(self.data, TAG, "keys.npy"), np.asarray(keys, np.int64))
            with open(os.path.join(self.data, TAG, "graph.json"), "w") as fh:
                json.dump({"n": int(n), "m": int(len(keys))}, fh)

    def path(self, *parts):
        return os.path.join(self.root, *parts)

    def run(self, script, args, log):
        env = dict(os.environ, DATA_DIR=self.data + os.sep, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
        log_path = os.path.join(self.runs, log)
        with open(log_path, "w") as fh:
            proc = subprocess.run([sys.executable, os.path.join(HERE, script)] + [str(x) for x in args], cwd=self.root,
                                  env=env, stdout=fh, stderr=subprocess.STDOUT)
        if proc.returncode != 0:
            tail = "".join(open(log_path).readlines()[-15:])
            raise RuntimeError(f"{script} failed (exit {proc.returncode}); log {log_path}:\n{tail}")
        return log_path

    def reduce(self, label_files):
        self.run("reduce_exact.py", [TAG] + list(label_files), "reduce.log")
        return TAG + "__rx"

    def reduced_labels(self, label_file):
        return os.path.join(self.data, TAG + "__rx", os.path.basename(label_file))

    def solve(self, name, pairs, vc, lb, time_limit, outer, nbatch, init=None, resume=None, pair_weight=None,
              proximal=False, max_clusters=6000, ckpt_every=None, vdtype=None):
        """pipeline.py:105-136 (same flags)."""
        args = ["--tag", TAG + "__rx", "--pair_labels"] + list(pairs) + [
            "--max_clusters", max_clusters, "--k", 32, "--nbatch", nbatch, "--inner", 1, "--est_every", 0,
            "--tri_max", 16000000, "--mom", 0, "--lb", lb, "--shift_p", 0, "--time_limit", time_limit, "--seed", 0,
            "--vcs_labels", vc, "--vcs_max", 150000000, "--vcs_add", 10000000, "--outer", outer,
            "--save", os.path.join("runs", name + ".npz"), "--vdtype", vdtype or self.vdtype]
        if proximal:
            args += ["--resume", resume, "--tri_add", 0, "--tri1_add", 0, "--tri_every", 1000000,
                     "--pairlvl_weight", pair_weight, "--phase2_at_it", 1, "--phase2_w", pair_weight,
                     "--phase2_inner", 4, "--phase2_tri_every", 1000000, "--phase2_est_every", 0,
                     "--ckpt_every", ckpt_every or 20]
        else:
            args += ["--tri_add", 600000, "--tri1_add", 300000, "--tri_every", 9, "--init_partition", init,
                     "--pw_rule", "default", "--ckpt_every", ckpt_every or 50]
        log = self.run("alm_vcs.py", args, name + ".log")
        weight = pair_weight
        for line in open(log):
            hit = re.search(r"-> pairlvl_weight ([0-9.eE+-]+)", line)
            if hit:
                weight = float(hit.group(1))
        return os.path.join(self.runs, name + "_last.npz"), weight

    def estimate(self, name, ckpt, lb, init_v=None, save_w=None, polish_time=900, eig_time=900):
        """pipeline.py:156-170 (same flags)."""
        out = os.path.join(self.runs, name + ".json")
        args = ["--tag", TAG + "__rx", "--ckpt", ckpt, "--lb", lb, "--polish", "rgd", "--polish_time", polish_time,
                "--scale", "vol", "--eig_time", eig_time, "--out", out]
        if init_v:
            args += ["--initV", init_v]
        if save_w:
            args += ["--saveW", save_w]
        self.run("est_dual_vcs.py", args, name + ".log")
        res = json.load(open(out))
        res["json"] = out
        return res


def chung_lu_instance(name, seed):
    """The Chung-Lu + planted-communities shape of a benchmark configuration ('c2': n = 300,000, mean degree 13;
    'c3': n = 2.4M, mean degree 52): (n, keys u * n + v with u < v, community labels)."""
    from lagbound_b200 import synth
    g = synth.config_graph(name, seed=seed)
    rows = np.repeat(np.arange(g.n), np.diff(g.indptr))
    up = rows < g.indices
    return g.n, np.unique(rows[up] * g.n + g.indices[up]), np.asarray(g.labels, np.int64)


def sbm_instance(n, blocks, p_in, p_out, seed):
    """Planted-partition SBM (seeded), isolated nodes dropped: (n, keys u * n + v with u < v, planted labels)."""
    from lagbound_b200 import synth
    g = synth.sbm(n, blocks, p_in, p_out, seed)
    rows = np.repeat(np.arange(g.n), np.diff(g.indptr))
    up = rows < g.indices
    return g.n, np.unique(rows[up] * g.n + g.indices[up]), np.asarray(g.labels, np.int64)


def networkx_instance(name, seed):
    """Zachary's karate club or Les Miserables (the reference tests' graphs, test_bounds.py) with a Louvain partition
    as the starting partition (the reference takes any incumbent through partition=, api.py:213-214): (n, keys,
    labels)."""
    import networkx as nx
    G = nx.karate_club_graph() if name == "karate" else nx.les_miserables_graph()
    nodes = list(G.nodes())
    idx = {v: i for i, v in enumerate(nodes)}
    n = len(nodes)
    keys = np.unique([min(idx[u], idx[v]) * n + max(idx[u], idx[v]) for u, v in G.edges() if u != v])
    lab = np.zeros(n, np.int64)
    for c, comm in enumerate(nx.community.louvain_communities(G, seed=seed)):
        for v in comm:
            lab[idx[v]] = c
    return n, keys.astype(np.int64), lab


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--workdir", required=True)
    p.add_argument("--graph", default="sbm", choices=["sbm", "c2", "c3", "karate", "lesmis"],
                   help="sbm: planted SBM (--n --blocks --p_in --p_out); c2 / c3: the Chung-Lu benchmark shapes; "
                        "karate / lesmis: the reference tests' graphs with a Louvain starting partition")
    p.add_argument("--n", type=int, default=2000); p.add_argument("--blocks", type=int, default=8)
    p.add_argument("--p_in", type=float, default=0.08); p.add_argument("--p_out", type=float, default=0.002)
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--time", type=float, default=120.0, help="solver time limit (main + proximal)")
    p.add_argument("--proximal_fraction", type=float, default=0.3)
    p.add_argument("--max_iterations", type=int, default=3000)
    p.add_argument("--polish_time", type=float, default=900); p.add_argument("--eig_time", type=float, default=900)
    p.add_argument("--vdtype", default="f32", choices=["f64", "f32", "bf16"])
    p.add_argument("--proximal_vdtype", default=None, choices=["f64", "f32", "bf16"],
                   help="storage of V in the proximal phase (default: --vdtype).  With --vdtype bf16 the BF16 rounding "
                        "of V (about 1e-3 on every inner product) makes the triangle separation add spurious "
                        "triangles whose multipliers loosen the bound; an FP32 proximal phase lets the multiplier "
                        "updates release them")
    a = p.parse_args(argv)
    t0 = time.time()
    if a.graph == "sbm":
        n, keys, lab = sbm_instance(a.n, a.blocks, a.p_in, a.p_out, a.seed)
    elif a.graph in ("karate", "lesmis"):
        n, keys, lab = networkx_instance(a.graph, a.seed)
    else:
        n, keys, lab = chung_lu_instance(a.graph, a.seed)
    ws = Workspace(a.workdir, keys, n, a.vdtype)
    init = ws.path("data", TAG, "partition.npy")
    np.save(init, np.unique(lab, return_inverse=True)[1].astype(np.int64))
    stages = []
    ws.reduce([init])
    stages.append(("reduce", time.time() - t0))
    init_r = ws.reduced_labels(init)
    red = json.load(open(ws.path("data", TAG + "__rx", "graph.json")))
    n_red = red["n"]
    nbatch = 512 if n_red >= 512 * 64 else min(n_red, max(8, n_red // 64))       # api.py:250
    solver = dict(lb=float("nan"), outer=a.max_iterations, nbatch=nbatch, max_clusters=6000)
    t_main = (1.0 - a.proximal_fraction) * a.time
    main_ckpt, weight = ws.solve("main", [init_r], init_r, time_limit=t_main, init=init_r, **solver)
    stages.append(("main phase", time.time() - t0))
    cands = [("main", main_ckpt)]
    t_prox = max(0.0, a.time - (time.time() - t0))
    if a.proximal_fraction > 0 and t_prox > 0:
        prox_ckpt, _ = ws.solve("proximal", [init_r], init_r, time_limit=t_prox, resume=main_ckpt, pair_weight=weight,
                                proximal=True, vdtype=a.proximal_vdtype, **solver)
        cands.append(("proximal", prox_ckpt))
        stages.append(("proximal phase", time.time() - t0))
    est = {name: ws.estimate(f"est_{name}", ck, float("nan"), polish_time=a.polish_time, eig_time=a.eig_time)
           for name, ck in cands}
    best = min(est, key=lambda k_: est[k_]["ub"])
    stages.append(("estimates", time.time() - t0))
    from fractions import Fraction
    u, v = keys // n, keys % n
    m = len(keys)
    li = np.unique(lab, return_inverse=True)[1]
    ins = int((li[u] == li[v]).sum())
    vol = np.bincount(li, weights=np.bincount(np.r_[u, v], minlength=n)).astype(np.int64)
    Q = Fraction(ins, m) - Fraction(sum(int(x) ** 2 for x in vol), 4 * m * m)
    summary = dict(graph=a.graph, n=n, m=int(m), n_reduced=n_red, nbatch=nbatch, pair_weight=weight, vdtype=a.vdtype,
                   proximal_vdtype=a.proximal_vdtype or a.vdtype,
                   planted_modularity=float(Q), estimates={k_: dict(ub=v_["ub"], dv=v_["dv"], json=v_["json"])
                                                           for k_, v_ in est.items()},
                   best=best, best_ckpt=dict(cands)[best], estimate=float(est[best]["ub"]), stages=stages,
                   seconds=time.time() - t0)
    json.dump(summary, open(ws.path("summary.json"), "w"), indent=1)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
