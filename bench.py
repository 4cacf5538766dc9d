#!/usr/bin/env python3
"""Benchmark of the augmented-Lagrangian inner loop on B200: AL gradient evaluations per second.

One step = one evaluation of the augmented Lagrangian at fixed multipliers: value + dual residuals + the full
half-gradient G = C(y_eff) V for all n rows (the Jacobi form of one inner iteration), through the library's C ABI.

Workload (default, the large single-graph shape the metric is quoted on): synthetic Chung-Lu graph with planted
communities, n = 2.4M, m = 62.4M (mean degree 52, exponent 2.3, max degree 1e5), 20,000 communities of log-normal
size (4, 1), mixing 0.25, unit weights; r = 32; 5M wedge triangle triples with multipliers 50 % zero / 50 % Exp(0.05);
V stored in BF16 with FP32 accumulation and FP64 reductions (also FP32 and FP64 forms, reported under "forms").
The inputs (1.3 GB in BF16) exceed the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c3|c2|c1]

N > 1 (torchrun, one process per GPU): independent replicas of the workload, no collective on the data path
(one graph's evaluation is not sharded across GPUs); value = all ranks' evaluations / max-over-ranks time.
--impl reference: the CPU oracle (a C restatement of the reference's Numba kernels, all host threads) on rank 0,
one full FP64 evaluation (value + G for every row) per step.

Besides the headline line's keys: "precision" (BF16 / FP32 results against the FP64 GPU form at the same stored V,
against the FP64 form at the original V, and against the FP64 oracle), "levels" (the same evaluation with one pair
level of the communities capped at 6000 clusters and one VCS level on the neighbour pattern), "batched" (512 graphs
in one batched problem per rank), and "cpu_baseline" (the oracle's full evaluation on the host cores).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "AL grad evals/s & HBM GB/s at n=2.4M r=32 vs FP64; p50/p99 time-to-bound"
WORKLOADS = {
    "c3": "Chung-Lu + planted communities n=2.4M m=62.4M (mean deg 52, gamma 2.3, max deg 1e5), 20k communities "
          "log-normal(4,1), mixing 0.25, unit weights; r=32; 5M wedge triples; BF16 V, FP32 accumulation, FP64 "
          "reductions",
    "c2": "Chung-Lu + planted communities n=300k m=1.95M (mean deg 13, gamma 2.1, max deg 2e4), 3000 communities, "
          "mixing 0.3; r=32; 1M wedge triples",
    "c1": "planted-partition SBM n=2000, 8 blocks, p_in 0.08, p_out 0.002; r=16; 20k wedge triples",
}
RHO, TRI_WEIGHT = 0.02, 1.0


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def algorithmic_bytes(n, nnz, r, T, s_v, s_g, weighted=False):
    """Algorithmic bytes of one evaluation (no levels): int32 CSR, V read once, d FP64, G written once, int32
    triples and FP64 multipliers.  Returns (whole evaluation, row kernel); the row kernel reads the triangles'
    vertex ids and effective multipliers pt (FP64) instead of lam."""
    csr = 4 * (n + 1) + 4 * nnz + (4 * nnz if weighted else 0)
    common = csr + s_v * n * r + 8 * n + s_g * n * r + 12 * T
    return common + 8 * T, common + 8 * T


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush(); self.f.seek(0)
        rows = [l.split(",") for l in self.f.read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_workload(name, device, triangles=None):
    from lagbound_b200 import synth
    t0 = time.time()
    g = synth.config_graph(name, seed=0, device=device)
    T = synth.CONFIG_TRIANGLES[name] if triangles is None else triangles
    TI = synth.wedge_triples_torch(g, T, seed=1, device=device) if device else synth.wedge_triples(g, T, seed=1)
    lam = synth.tri_multipliers(len(TI), seed=1)
    r = synth.CONFIG_RANK[name]
    V = synth.random_V(g.n, r, seed=0)
    return g, TI, lam, V, r, time.time() - t0


def host_cores():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


class CpuEval:
    """The oracle's FP64 evaluation (C, OpenMP on all host threads) of the whole instance: d^T V, tri_aug over every
    triangle, quadA and A V over every row, the degree correction and the triangle rows T(pt) V (the order of
    augmented() + CV(), alm_vcs.py:1496-1533, 1299-1312), with the same locality order of the rows as the GPU run.
    Nothing is sampled or extrapolated."""

    def __init__(self, g, TI, lam, V, order=None):
        from oracle import oracle as O
        from lagbound_b200 import synth
        if order is not None:
            g, inv = synth.permute_graph(g, order)
            TI = inv[TI]; V = V[order]
        self.O = O
        self.inst = O.Instance(g.n, g.indptr, g.indices, g.data, g.d, g.L, g.C0)
        self.TI = np.ascontiguousarray(TI, np.int64); self.lam = lam; self.V = np.ascontiguousarray(V)
        self.tptr, self.tcodes = O.incidence(g.n, self.TI)

    def seconds(self):
        r = self.O.timed_sample(self.inst, self.V, self.TI, self.lam, RHO, TRI_WEIGHT, 1.0, self.tptr, self.tcodes)
        assert r["frac_edges"] == 1.0
        return r["seconds_per_eval"]

    def sample_text(self):
        return (f"one full FP64 evaluation per step (n={self.inst.n}, nnz={int(self.inst.indptr[-1])}, "
                f"T={len(self.TI)}: value terms and G for every row), no sampling or extrapolation; same row order "
                f"as the GPU run")


def cpu_baseline(g, TI, lam, V, order=None, reps=3):
    ce = CpuEval(g, TI, lam, V, order)
    ce.seconds()                                   # warm-up (page-in of the instance)
    t = [ce.seconds() for _ in range(reps)]
    spe = sum(t) / len(t)
    return {"value": 1.0 / spe, "unit": "evals/s", "cores": host_cores(), "kind": "port",
            "sample": ce.sample_text() + f"; mean of {reps} after one warm-up"}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    # NCCL reduces device tensors; a CPU process group (gloo) host tensors
    t = torch.tensor([float(x)], device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args, world, rank):
    if rank != 0:
        return
    g, TI, lam, V, r, gen_s = build_workload(args.workload, "cuda" if _cuda() else None)
    from lagbound_b200.problem import locality_order
    order = locality_order(g.labels) if args.order == "partition" and g.labels is not None else None
    ce = CpuEval(g, TI, lam, V, order)
    for _ in range(args.warmup):
        ce.seconds()
    t = [ce.seconds() for _ in range(args.steps)]
    spe = sum(t) / len(t)
    cores = host_cores()
    value = 1.0 / spe
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": spe * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "n": g.n, "nnz": int(g.nnz), "T": int(len(TI)), "r": r},
            "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
                             "sample": ce.sample_text()},
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def time_form(ctx, g, TI, lam, V, r, dtype, steps, warmup, world, clocks_dev=None, order=None):
    """Device-timed evaluations of one storage form; returns (max-over-ranks ms total, phase ms, launches, problem)."""
    from lagbound_b200 import Problem
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, r, dtype, order=order)
    p.set_V(V)
    p.set_triangles(TI, lam)
    for _ in range(warmup):
        p.eval_async(RHO, TRI_WEIGHT, grad=True)
    ctx.synchronize()
    p.timing_collect()
    l0 = p.launch_count()
    barrier(world)
    ctx.synchronize()
    clk = None
    if clocks_dev is not None:
        clk = Clocks(clocks_dev)
        time.sleep(0.5)
    ctx.timer_start()
    for _ in range(steps):
        p.eval_async(RHO, TRI_WEIGHT, grad=True, timing=True)
    ms = ctx.timer_stop()
    clocks = clk.stop() if clk else None
    barrier(world)
    launches = p.launch_count() - l0
    phases, cnt = p.timing_collect()
    out = p.eval_fetch()
    ms_max = reduce_max(ms, world)
    return ms_max, {k: v / max(cnt, 1) for k, v in phases.items()}, launches, p, out, clocks


def time_batched(ctx, device, steps, warmup, world, count=512):
    """The batched shape: `count` graphs in FP32, grouped by rank into one batched problem per rank (each a
    block-diagonal CSR evaluated in the same launches); a step evaluates every group.  Device-timed with CUDA
    events on the library's stream."""
    from lagbound_b200 import BatchedProblem, synth
    from lagbound_b200.problem import locality_order
    t0 = time.time()
    graphs = synth.batch_graphs(count, seed=0, device=device)
    probs, B, rows, nnz, T = [], 0, 0, 0, 0
    for r in (8, 16, 32):
        grp = [g for g, rr in graphs if rr == r]
        if not grp:
            continue
        bp = BatchedProblem(ctx, grp, r, "f32", orders=[locality_order(g.labels) for g in grp])
        bp.set_V(synth.random_V(bp.n, r, seed=r))
        TI, lam = [], []
        for k, g in enumerate(grp):
            t = synth.wedge_triples_torch(g, 10 * g.n, seed=1000 + k, device=device)
            TI.append(t + bp.offsets[k]); lam.append(synth.tri_multipliers(len(t), seed=1000 + k))
            B += algorithmic_bytes(g.n, g.nnz, r, len(t), 4, 4)[0]
            rows += g.n; nnz += g.nnz; T += len(t)
        bp.set_triangles(np.concatenate(TI), np.concatenate(lam))
        probs.append((r, len(grp), bp))
    gen_s = time.time() - t0
    for _ in range(warmup):
        for _, _, bp in probs:
            bp.eval_async(RHO, TRI_WEIGHT, grad=True)
    ctx.synchronize()
    # the whole step captured in one CUDA graph (every problem was evaluated in the warm-up)
    with ctx.capture() as graph:
        for _, _, bp in probs:
            bp.eval_async(RHO, TRI_WEIGHT, grad=True)
    for _ in range(warmup):
        graph.launch()
    barrier(world)
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(steps):
        graph.launch()
    ms_graph = reduce_max(ctx.timer_stop(), world)
    kernels_graph = graph.kernels
    graph.close()
    for _, _, bp in probs:
        bp.timing_collect()
    barrier(world)
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(steps):
        for _, _, bp in probs:
            bp.eval_async(RHO, TRI_WEIGHT, grad=True, timing=True)
    ms = reduce_max(ctx.timer_stop(), world)
    per, phases = {}, {}
    for r, k, bp in probs:
        ph, cnt = bp.timing_collect()
        per[str(r)] = {"graphs": k, "rows": bp.n, "ms": round(sum(ph.values()) / max(cnt, 1), 4)}
        for key, v in ph.items():
            phases[key] = phases.get(key, 0.0) + v / max(cnt, 1)
    for _, _, bp in probs:
        bp.eval_fetch()
        bp.close()
    step_s = ms_graph / 1e3 / steps
    peak, peak_kind = load_peaks()
    return {"workload": "batched: %d graphs (planted-partition and Chung-Lu alternating), n log-uniform in [500, "
                        "50000], mean degree U[5, 40], r from {8, 16, 32}, 10 n triangle triples per graph, FP32 V; "
                        "one batched problem per rank, all of its graphs in the same launches" % count,
            "graphs": count, "rows": rows, "nnz": nnz, "triangles": T, "by_rank": per, "steps": steps,
            "ms_per_step": step_s * 1e3, "graph_evals_s": world * count / step_s, "batch_steps_s": world / step_s,
            "timing": "one CUDA graph per step (%d kernels), launched %d times after %d warm-up launches; the same "
                      "step launched directly with per-phase events: %.3f ms" % (kernels_graph, steps, warmup,
                                                                                 ms / steps),
            "hbm_gbs_eval": B / step_s / 1e9, "frac_of_peak": B / step_s / 1e9 / peak, "peak_kind": peak_kind,
            "algorithmic_bytes_per_step": B, "gpu_launches_per_step": kernels_graph,
            "phases_ms": {k: round(v, 4) for k, v in phases.items()},
            "gen_seconds": round(gen_s, 1)}


def rel_err(a, b):
    nb = float(np.linalg.norm(b))
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def precision_report(res, V, oracle_eval):
    """Errors of the reduced storage forms against FP64 (each result states its error against FP64): for each form
    f, (a) against the FP64 GPU form evaluated at f's stored V (the accumulation error alone), (b) against the FP64
    GPU form at the original V (storage rounding + accumulation), (c) against the FP64 oracle at f's stored V; value
    relative error, G relative Frobenius error and |G| relative error.  The FP64 form is itself checked against the
    oracle (c).  oracle_eval(V) -> (value, G) in the caller's row order."""
    p64 = res["f64"]["problem"]
    p64.set_V(V)
    o64 = p64.eval(RHO, TRI_WEIGHT, grad=True)
    G64 = p64.G()
    out = {}
    ov, oG = oracle_eval(V)
    out["f64"] = {"vs_oracle": {"value_rel": abs(o64["value"] - ov) / abs(ov), "G_rel": rel_err(G64, oG)}}
    for f in [f for f in res if f != "f64"]:
        p = res[f]["problem"]
        of = p.eval(RHO, TRI_WEIGHT, grad=True)
        Gf = p.G()
        Vs = p.get_V()                                # the V this form stores (rounded to its dtype)
        p64.set_V(Vs)
        os_ = p64.eval(RHO, TRI_WEIGHT, grad=True)
        Gs = p64.G()
        ov, oG = oracle_eval(Vs)
        n64 = float(np.linalg.norm(G64))
        out[f] = {
            "vs_f64_gpu_same_V": {"value_rel": abs(of["value"] - os_["value"]) / abs(os_["value"]),
                                  "G_rel": rel_err(Gf, Gs)},
            "vs_f64_gpu_original_V": {"value_rel": abs(of["value"] - o64["value"]) / abs(o64["value"]),
                                      "G_rel": rel_err(Gf, G64),
                                      "G_norm_rel": abs(float(np.linalg.norm(Gf)) - n64) / n64,
                                      "V_storage_rel": rel_err(Vs, V)},
            "vs_oracle": {"value_rel": abs(of["value"] - ov) / abs(ov), "G_rel": rel_err(Gf, oG)}}
        del Gf, Gs, oG
    p64.set_V(V)
    out["note"] = ("value = the augmented Lagrangian at fixed multipliers (rho 0.02, tri_weight 1); G = C(y_eff) V, "
                   "relative Frobenius error; the oracle is the FP64 C restatement of the reference's kernels")
    return out


def neighbour_pattern(g, lab, device):
    """VCS working set of aggops.neighbour_pattern (aggops.py:45-49): row i holds its own cluster and the clusters of
    its neighbours, columns sorted (drawn by torch on the GPU; input generation only)."""
    import torch
    dev = torch.device(device)
    P = int(lab.max()) + 1
    ip = torch.from_numpy(g.indptr).to(dev)
    ix = torch.from_numpy(np.ascontiguousarray(g.indices, np.int64)).to(dev)
    lt = torch.from_numpy(np.ascontiguousarray(lab, np.int64)).to(dev)
    rows = torch.repeat_interleave(torch.arange(g.n, device=dev), ip[1:] - ip[:-1])
    keys = torch.unique(torch.cat([torch.arange(g.n, device=dev) * P + lt, rows * P + lt[ix]]))
    del rows, ix
    r_ = keys // P
    ptr = torch.zeros(g.n + 1, dtype=torch.int64, device=dev)
    ptr[1:] = torch.cumsum(torch.bincount(r_, minlength=g.n), 0)
    col = (keys % P).to(torch.int32)
    out = ptr.cpu().numpy(), col.cpu().numpy()
    del keys, r_, ptr, col
    torch.cuda.empty_cache()
    return out


def time_levels(ctx, g, TI, lam, V, r, dtype, steps, warmup, world, order, device, with_oracle=True):
    """The evaluation with the production levels: one pair level = the planted communities capped at 6000 clusters
    (alm_vcs.py:1133-1137, --max_clusters 6000) and one VCS level on the communities with the neighbour-pattern
    working set; multipliers at the scale the PHR update produces (sig ~ rho r |h| for the pair level, half of the
    working-set entries active).  Device-timed like the headline; its algorithmic bytes add 8 P^2 (pair sigma) and
    12 nnz_vcs (int32 column + FP64 sigma per entry)."""
    from lagbound_b200 import Problem
    from lagbound_b200.stages.alm_vcs import capped_labels
    import scipy.sparse as sp
    t0 = time.time()
    rng = np.random.default_rng(7)
    w_pair, vc_weight = 0.03, 1.0
    lab_p = capped_labels(g.labels, g.d, 6000, lambda *a: None, "pair level")
    P = int(lab_p.max()) + 1
    cnt = np.bincount(lab_p, minlength=P).astype(float)
    vol = np.maximum(np.bincount(lab_p, weights=g.d, minlength=P), 1.0)
    rq = cnt / vol ** 2
    W = sp.csr_matrix((g.d, (lab_p, np.arange(g.n))), shape=(P, g.n))
    Y = W @ V
    H = Y @ Y.T
    H[np.diag_indices(P)] -= np.bincount(lab_p, weights=g.d * g.d, minlength=P)
    S = RHO * np.outer(rq, rq) * w_pair * np.abs(H) * rng.uniform(0, 3, (P, P)) * (rng.random((P, P)) < 0.6)
    sig = 0.5 * (S + S.T)
    del S, H, W
    lab_v = np.unique(g.labels, return_inverse=True)[1].astype(np.int64)
    Pv = int(lab_v.max()) + 1
    vptr, vcol = neighbour_pattern(g, lab_v, device)
    nnz_v = int(vptr[-1])
    vsig = rng.exponential(0.05, nnz_v) * (rng.random(nnz_v) < 0.5)
    wv = vc_weight * w_pair
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, r, dtype, order=order)
    p.set_V(V)
    p.set_triangles(TI, lam)
    lid = p.add_pair_level(lab_p, P, w_pair)
    p.set_pair_sigma(lid, sig)
    m = p.add_vcs_level(lab_v, Pv, wv)
    p.set_vcs_ws(m, vptr, vcol, vsig)
    setup_s = time.time() - t0
    for _ in range(warmup):
        p.eval_async(RHO, TRI_WEIGHT, grad=True)
    ctx.synchronize()
    p.timing_collect()
    barrier(world)
    ctx.synchronize()
    ctx.timer_start()
    for _ in range(steps):
        p.eval_async(RHO, TRI_WEIGHT, grad=True, timing=True)
    ms = reduce_max(ctx.timer_stop(), world)
    phases, cnt_ = p.timing_collect()
    step_s = ms / 1e3 / steps
    s_v = {"bf16": 2, "f32": 4, "f64": 8}[dtype]
    B = algorithmic_bytes(g.n, g.nnz, r, len(TI), s_v, 8 if dtype == "f64" else 4)[0] + 8 * P * P + 12 * nnz_v
    peak, peak_kind = load_peaks()
    out = {"workload": "the headline instance with one pair level (communities capped at %d clusters, --max_clusters "
                       "6000) and one VCS level (%d communities, neighbour-pattern working set of %d entries), %s V"
                       % (P, Pv, nnz_v, dtype.upper()),
           "P": P, "P_vcs": Pv, "nnz_vcs": nnz_v, "evals_s": world / step_s, "ms_per_step": step_s * 1e3,
           "algorithmic_bytes": B, "hbm_gbs_eval": B / step_s / 1e9, "frac_of_peak": B / step_s / 1e9 / peak,
           "peak_kind": peak_kind, "phases_ms": {k: round(v / max(cnt_, 1), 4) for k, v in phases.items()},
           "setup_seconds": round(setup_s, 1)}
    if with_oracle:
        from oracle import oracle as O
        o = p.eval(RHO, TRI_WEIGHT, grad=True)
        Gf = p.G()
        Vs = p.get_V()
        inst = O.Instance(g.n, g.indptr, g.indices, g.data, g.d, g.L, g.C0)
        pl = O.PairLevelData(lab_p, g.d, sig, w_pair)
        vl = O.VCSLevelData(lab_v, g.d, vptr, vcol, vsig)
        ref = O.evaluate(inst, Vs, [pl], TI, lam, [vl], RHO, TRI_WEIGHT, wv=wv, want_G=True)
        out["precision_vs_oracle"] = {"value_rel": abs(o["value"] - ref["value"]) / abs(ref["value"]),
                                      "G_rel": rel_err(Gf, ref["G"]), "nviol": [int(o["nviol"]),
                                                                                int(ref["nviol"].sum())],
                                      "vcs_nviol": [int(o["vcs_nviol"]), int(ref["vcs_nviol"].sum())]}
    p.close()
    return out


def time_sweeps(ctx, device, steps, warmup, nbatch=512):
    """The solver's inner iteration at the C2 shape: batched Gauss-Seidel sweeps (alm_vcs.py:1360-1436; per sweep a
    row permutation split into nbatch batches, per batch the pair rows, VCS pre/post terms, row steps and aggregate
    updates) on the Chung-Lu graph n = 300k, m = 1.95M, r = 32, FP32 V, with one pair level (the 3,000 communities),
    one VCS level on the neighbour pattern and 1M triangle triples; wall time of lb_sweeps (it synchronises) per sweep
    after `warmup` sweeps."""
    from lagbound_b200 import Problem, synth
    from lagbound_b200.problem import locality_order
    t0 = time.time()
    g = synth.config_graph("c2", seed=0, device=device)
    TI = synth.wedge_triples_torch(g, synth.CONFIG_TRIANGLES["c2"], seed=1, device=device)
    lam = synth.tri_multipliers(len(TI), seed=1)
    V = synth.random_V(g.n, 32, seed=0)
    lab = np.unique(g.labels, return_inverse=True)[1].astype(np.int64)
    P = int(lab.max()) + 1
    vptr, vcol = neighbour_pattern(g, lab, device)
    rng = np.random.default_rng(3)
    vsig = rng.exponential(0.05, len(vcol)) * (rng.random(len(vcol)) < 0.5)
    p = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, 32, "f32", order=locality_order(lab))
    p.set_V(V)
    p.set_triangles(TI, lam)
    lid = p.add_pair_level(lab, P, 0.03)
    p.set_pair_sigma(lid, np.zeros((P, P)))
    m = p.add_vcs_level(lab, P, 0.03)
    p.set_vcs_ws(m, vptr, vcol, vsig)
    setup_s = time.time() - t0
    perm_rng = np.random.default_rng(5)
    for _ in range(warmup):
        p.sweeps(perm_rng.permutation(g.n)[None], RHO, RHO * TRI_WEIGHT, 0.0, nbatch)
    ts = []
    for _ in range(steps):
        perm = perm_rng.permutation(g.n)[None]
        t = time.perf_counter()
        p.sweeps(perm, RHO, RHO * TRI_WEIGHT, 0.0, nbatch)
        ts.append(time.perf_counter() - t)
    p.close()
    return {"workload": "Gauss-Seidel sweeps at the C2 shape: n=%d, nnz=%d, r=32, FP32 V, pair level of %d communities, "
                        "VCS level on the neighbour pattern (%d entries), %d triangle triples, nbatch %d, community "
                        "row order" % (g.n, g.nnz, P, len(vcol), len(TI), nbatch),
            "ms_per_sweep": 1e3 * float(np.median(ts)), "ms_min": 1e3 * min(ts), "sweeps": steps,
            "rows_per_s": g.n / float(np.median(ts)), "setup_seconds": round(setup_s, 1),
            "timing": "wall clock around lb_sweeps (it synchronises), median over the sweeps"}


def gather_probe(ctx, ngather=125_000_000, reps=3):
    """The random row-gather ceiling of the device (lb_gather_probe): per footprint and row size, ms per 125M
    gathers, gathered GB/s and millions of rows per ms."""
    import ctypes
    from lagbound_b200 import _capi as C
    rows = []
    for rb in (64, 128):
        for mb in (4, 16, 32, 48, 64, 80, 96, 112, 128, 154):
            ms = ctypes.c_float()
            C.call("lb_gather_probe", ctx.h, int(mb * (1 << 20)), rb, ngather, reps, ctypes.byref(ms))
            rows.append({"row_bytes": rb, "footprint_mb": mb, "ms": round(ms.value, 4),
                         "gathered_gbs": round(ngather * rb / ms.value / 1e6, 1),
                         "mrows_per_ms": round(ngather / ms.value / 1e6, 2)})
    return rows


def time_serving(device, requests=40, rate=20.0, n_max=100_000, slots=32):
    """p50 / p99 time to a candidate bound on a Poisson stream of bound requests (the served configuration's shapes:
    Chung-Lu graphs with planted communities, n ~ Pareto(1.2) clipped to [1000, n_max], mean degree U[8, 50],
    r U{16..32}, BF16 V; 30 AL outer iterations and the GPU estimate per request), served with continuous batching
    against a 150 GB HBM budget (lagbound_b200.serving); two small warm-up requests first."""
    from lagbound_b200 import serving as S
    S.BoundServer(device, slots, 150e9).run(S.request_stream(2, rate, 99, n_max=2000, device=f"cuda:{device}"))
    t0 = time.time()
    reqs = S.request_stream(requests, rate, 0, n_max=n_max, device=f"cuda:{device}")
    gen_s = time.time() - t0
    res = S.BoundServer(device, slots, 150e9).run(reqs)
    st = S.latency_stats(res)
    st.update(workload=f"{requests} requests, Poisson {rate:g}/s, n Pareto(1.2) in [1000, {n_max}], mean degree "
                       f"U[8, 50], r U{{16..32}}, BF16 V, 30 outer iterations + estimate each; {slots} slots, 150 GB "
                       f"budget", time_to="candidate bound (solve + estimate, the GPU stages); the certificate and "
                                          "its verification are the reference's CPU stages",
              n_total=int(sum(q.n for q in reqs)), n_max_seen=int(max(q.n for q in reqs)),
              gen_seconds=round(gen_s, 1))
    return st


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=["c1", "c2", "c3"])
    ap.add_argument("--forms", default="bf16,f32,f64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-graphs line (key 'batched')")
    ap.add_argument("--no-serving", action="store_true", help="skip the served request stream (key 'serving')")
    ap.add_argument("--gather-probe", action="store_true",
                    help="time only the random row-gather probe (lb_gather_probe: 125M gathers of 64- and 128-byte "
                         "rows from footprints of 4 MB to 154 MB) and print that table (key 'gather_probe')")
    ap.add_argument("--sweep-only", action="store_true",
                    help="time only the solver's sweeps at the C2 shape (key 'sweep') and print that object")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the precision report and the levels variant (keys 'precision' and 'levels')")
    ap.add_argument("--triangles", type=int, default=None,
                    help="stored triples (default: the workload's; other values are for analysis and show in config.T)")
    ap.add_argument("--order", default="partition", choices=["partition", "natural"],
                    help="locality order of the rows: grouped by the starting partition (the planted communities "
                         "stand in for the solver's --init_partition labels) or the generator's vertex order")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    from lagbound_b200 import Context
    from lagbound_b200.problem import locality_order
    if args.gather_probe:
        ctx = Context(local)
        out = gather_probe(ctx)
        ctx.close()
        if rank == 0:
            print(json.dumps({"gather_probe": out}), flush=True)
        return
    if args.sweep_only:
        ctx = Context(local)
        out = time_sweeps(ctx, f"cuda:{local}", args.steps, args.warmup)
        ctx.close()
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    g, TI, lam, V, r, gen_s = build_workload(args.workload, f"cuda:{local}", args.triangles)
    order = locality_order(g.labels) if args.order == "partition" and g.labels is not None else None
    ctx = Context(local)
    forms = args.forms.split(",")
    head = forms[0]
    res = {}
    for f in forms:
        ms, phases, launches, p, out, clocks = time_form(ctx, g, TI, lam, V, r, f, args.steps, args.warmup, world,
                                                         clocks_dev=local if f == head else None, order=order)
        res[f] = dict(ms=ms, phases=phases, launches=launches, out=out, clocks=clocks, problem=p)
    hp = res[head]
    evals_s = world * args.steps / (hp["ms"] / 1e3)
    s_v = {"bf16": 2, "f32": 4, "f64": 8}[head]
    s_g = 8 if head == "f64" else 4
    B_eval, B_rows = algorithmic_bytes(g.n, g.nnz, r, len(TI), s_v, s_g)
    peak, peak_kind = load_peaks()
    t_rows = hp["phases"]["rows"] / 1e3
    achieved = B_rows / t_rows / 1e9
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            traffic = json.load(fh).get(f"k_rows {args.workload} {head}")
    except Exception:
        pass
    # end to end through the public C ABI with host buffers, every step: H2D of V (pinned, storage dtype), the
    # evaluation, D2H of the scalar results and of the whole gradient G (pinned, n x r in its dtype)
    p = hp["problem"]
    import torch
    tdt = {"bf16": torch.bfloat16, "f32": torch.float32, "f64": torch.float64}[head]
    Vh = torch.from_numpy(V).to(tdt).pin_memory()
    raw = Vh.view(torch.int16).numpy() if head == "bf16" else Vh.numpy()
    Gh = torch.empty((g.n, r), dtype=torch.float64 if head == "f64" else torch.float32).pin_memory().numpy()
    for _ in range(2):
        p.eval_host(raw, RHO, TRI_WEIGHT)
        p.G_raw(Gh)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        p.eval_host(raw, RHO, TRI_WEIGHT)
        p.G_raw(Gh)
    t_seq = reduce_max(time.perf_counter() - t0, world)
    # the same steps through lb_eval_host_pipelined: the V uploads and G downloads overlap the evaluations (two
    # pinned V and two pinned G buffers used alternately)
    Vh2 = Vh.clone().pin_memory()
    raw2 = Vh2.view(torch.int16).numpy() if head == "bf16" else Vh2.numpy()
    Gh2 = torch.empty_like(torch.from_numpy(Gh)).pin_memory().numpy()
    Vl = [raw if k % 2 == 0 else raw2 for k in range(args.steps)]
    Gl = [Gh if k % 2 == 0 else Gh2 for k in range(args.steps)]
    p.eval_host_pipelined(Vl[:2], Gl[:2], RHO, TRI_WEIGHT)
    barrier(world)
    t0 = time.perf_counter()
    p.eval_host_pipelined(Vl, Gl, RHO, TRI_WEIGHT)
    t_e2e = reduce_max(time.perf_counter() - t0, world)
    e2e = {"value": world * args.steps / t_e2e, "unit": "evals/s", "h2d_bytes_per_step": int(raw.nbytes),
           "d2h_bytes_per_step": int(Gh.nbytes) + 128,
           "sequential_value": world * args.steps / t_seq,
           "what": "per step: pinned host V -> device, evaluation, scalars and the whole G -> pinned host, all steps "
                   "in one lb_eval_host_pipelined call (uploads, evaluations and downloads on three streams, "
                   "overlapped); wall clock around the call.  sequential_value: the same steps as lb_eval_host + "
                   "lb_get_G_raw one after another"}
    del Gh, Gh2
    forms_out = {f: world * args.steps / (res[f]["ms"] / 1e3) for f in forms}
    line = {"metric": METRIC, "value": evals_s, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": hp["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": head, "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload], "n": g.n, "nnz": int(g.nnz), "T": int(len(TI)), "r": r,
                       "rho": RHO, "l2": "inputs > 126 MB L2 (V alone is %.0f MB); no flush" % (g.n * r * s_v / 1e6),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "row_order": "grouped by the starting partition (planted communities)" if order is not None
                       else "generator order (random ids)",
                       "gen_seconds": round(gen_s, 1),
                       "light_threshold": hp["problem"].light_threshold()[0]},
            "forms": {f"{f}_evals_s": v for f, v in forms_out.items()},
            "hbm_gbs_eval": evals_s / world * B_eval / 1e9,
            "roofline": {"bound": "hbm", "kernel": "k_rows (A V + fused epilogue + triangle rows)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes": B_rows, "traffic": traffic},
            "phases_ms": {k: round(v, 4) for k, v in hp["phases"].items()},
            "forms_phases_ms": {f: {k: round(v, 4) for k, v in res[f]["phases"].items()} for f in forms},
            "gpu_launches": int(hp["launches"]),
            "e2e": e2e,
            "clocks": hp["clocks"]}
    if "f64" in forms_out and head != "f64":
        line["forms"][f"{head}_over_f64"] = forms_out[head] / forms_out["f64"]
    extras = world == 1 and not args.no_extras
    if extras and "f64" in res:
        from oracle import oracle as O
        inst = O.Instance(g.n, g.indptr, g.indices, g.data, g.d, g.L, g.C0)

        def oracle_eval(X):
            o = O.evaluate(inst, X, (), TI, lam, (), RHO, TRI_WEIGHT, want_G=True)
            return o["value"], o["G"]
        t0 = time.time()
        line["precision"] = precision_report(res, V, oracle_eval)
        line["precision"]["seconds"] = round(time.time() - t0, 1)
    for f in forms:
        if f != head:
            res[f]["problem"].close()
    if extras:
        # attribution of the row kernel's time: the same instance and form without the triangle pool
        from lagbound_b200 import Problem
        p0 = Problem(ctx, g.n, g.indptr, g.indices, None, g.d, g.L, g.C0, r, head, order=order)
        p0.set_V(V)
        for _ in range(args.warmup):
            p0.eval_async(RHO, TRI_WEIGHT, grad=True)
        ctx.synchronize()
        p0.timing_collect()
        for _ in range(args.steps):
            p0.eval_async(RHO, TRI_WEIGHT, grad=True, timing=True)
        ph0, c0 = p0.timing_collect()
        p0.close()
        line["rows_attribution"] = {
            "rows_ms_with_triangles": round(hp["phases"]["rows"], 4),
            "rows_ms_without_triangles": round(ph0["rows"] / max(c0, 1), 4),
            "tri_kernel_ms": round(hp["phases"]["tri"], 4),
            "note": "row kernel (A V, epilogue, and with triangles the incidence rows T(pt) V: %d incidences) on the "
                    "same instance and form, with and without the %d stored triples" % (3 * len(TI), len(TI))}
        # the row kernel's gather rate against the device's random-gather ceiling (lb_gather_probe) for rows of the
        # same size, at a footprint L2 holds and at V's own footprint
        import ctypes
        from lagbound_b200 import _capi as C
        row_b = r * s_v
        if row_b in (64, 128):
            ceil = {}
            for key, mb in (("l2_resident_32mb", 32), ("at_v_footprint", max(1, int(round(g.n * row_b / 2 ** 20))))):
                ms = ctypes.c_float()
                C.call("lb_gather_probe", ctx.h, int(mb * (1 << 20)), int(row_b), 125_000_000, 3, ctypes.byref(ms))
                ceil[key] = {"footprint_mb": mb, "mrows_per_ms": round(125e6 / ms.value / 1e6, 2)}
            gathers = int(g.nnz) + 2 * 3 * len(TI)
            line["gather_ceiling"] = dict(ceil, row_bytes=int(row_b), row_kernel_gathers=gathers,
                                          row_kernel_mrows_per_ms=round(gathers / hp["phases"]["rows"] / 1e6, 2),
                                          note="random whole-row gathers from the footprint (bench.py --gather-probe); "
                                               "the row kernel's gathers: one per stored edge and two per triangle "
                                               "incidence, per ms of its phase time")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(g, TI, lam, V, order)
    hp["problem"].close()
    if extras:
        line["levels"] = time_levels(ctx, g, TI, lam, V, r, head, args.steps, args.warmup, world, order,
                                     f"cuda:{local}")
    if not args.no_batched:
        del g, TI, lam, V
        line["batched"] = time_batched(ctx, f"cuda:{local}", args.steps, args.warmup, world)
    ctx.close()
    if extras:
        ctx = Context(local)
        line["sweep"] = time_sweeps(ctx, f"cuda:{local}", min(args.steps, 5), 2)
        ctx.close()
    if extras and not args.no_serving:
        line["serving"] = time_serving(local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
