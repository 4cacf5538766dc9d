#!/usr/bin/env python3
"""Test infrastructure: the reference's own CPU evaluation timed against the oracle's C port, on the same instance,
V, triangles and host threads, so that the port that bench.py times on the GPU box (where the reference source is
not available) can be read as the reference's speed.

One evaluation = the pieces of augmented() + CV() at fixed multipliers (src/lagbound/_core/alm_vcs.py:1496-1533,
1299-1312; the triangle incidence built once, as the reference rebuilds it only when the pool changes):
    zz = d @ V; tri_aug over the triangles; quadA; AV = spmm; BV = AV - outer(d, zz) / L; tri_apply(pt) on BV.
The reference's kernels are its Numba functions, loaded from its file (NUMBA_NUM_THREADS = the thread count);
the port is oracle.timed_sample over every row (OpenMP, OMP_NUM_THREADS the same).

    LAGBOUND_REF=<reference root> python oracle/time_reference.py [--workload c2|c3] [--reps 3] > out.json
"""
import argparse
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
from refpath import reference_root  # noqa: E402

REF = reference_root()
CORE = os.path.join(REF, "src", "lagbound", "_core")


def load_ref_kernels():
    """Execute the kernel section of alm_vcs.py (everything before its argparse block) under its real filename."""
    path = os.path.join(CORE, "alm_vcs.py")
    lines = open(path).read().split("\n")
    stop = next(i for i, l in enumerate(lines) if l.startswith("p = argparse.ArgumentParser"))
    ns = {"__name__": "lagbound_ref_kernels", "__file__": path}
    exec(compile("\n".join(lines[:stop]), path, "exec"), ns)
    return ns


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2", choices=["c2", "c3"])
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    os.environ.setdefault("NUMBA_NUM_THREADS", str(threads))
    os.environ.setdefault("NUMBA_CACHE_DIR", tempfile.mkdtemp(prefix="lagbound_timing_numba_"))
    import numpy as np
    from lagbound_b200 import synth
    from lagbound_b200.problem import locality_order
    import oracle as O            # oracle/oracle.py (this directory is on sys.path)
    t0 = time.time()
    g = synth.config_graph(a.workload, seed=0)
    TI = synth.wedge_triples(g, synth.CONFIG_TRIANGLES[a.workload], seed=1)
    lam = synth.tri_multipliers(len(TI), seed=1)
    V = synth.random_V(g.n, synth.CONFIG_RANK[a.workload], seed=0)
    order = locality_order(g.labels)
    g, inv = synth.permute_graph(g, order)
    TI = np.ascontiguousarray(inv[TI], np.int64); V = np.ascontiguousarray(V[order])
    gen_s = time.time() - t0
    K = load_ref_kernels()
    ip, ix, data, d, L = g.indptr, np.asarray(g.indices, np.int64), g.data, g.d, g.L
    rho, rt = 0.02, 0.02
    tptr, tcodes = K["incidence"](g.n, TI)

    def ref_eval():
        zz = d @ V
        gt = np.empty(len(TI)); pt = np.empty(len(TI))
        ttot, gmin = K["tri_aug"](TI, V, lam, rt, gt, pt)
        qa = K["quadA"](ip, ix, data, V)
        AV = np.empty_like(V)
        K["spmm"](ip, ix, data, V, AV)
        BV = AV - np.outer(d, zz) / L
        K["tri_apply"](TI, pt, tptr, tcodes, V, BV)
        return qa - float(zz @ zz) / L - ttot, BV

    inst = O.Instance(g.n, ip, ix, data, d, L, 0.0)
    otptr, otcodes = O.incidence(g.n, TI)

    def port_eval():
        return O.timed_sample(inst, V, TI, lam, rho, 1.0, 1.0, otptr, otcodes)["seconds_per_eval"]

    tc = time.time()
    val, BV = ref_eval()                                   # JIT compilation and warm-up
    compile_s = time.time() - tc
    ref_t, port_t = [], []
    port_eval()
    for _ in range(a.reps):
        tt = time.perf_counter(); ref_eval(); ref_t.append(time.perf_counter() - tt)
        port_t.append(port_eval())
    ev = O.evaluate(inst, V, (), TI, lam, (), rho, 1.0, want_G=True)
    out = dict(workload=a.workload, n=g.n, nnz=int(g.nnz), T=int(len(TI)), r=int(V.shape[1]), threads=threads,
               reference_numba_s=min(ref_t), port_s=min(port_t), port_over_reference_speed=min(ref_t) / min(port_t),
               reference_all_s=ref_t, port_all_s=port_t, compile_s=round(compile_s, 1), gen_s=round(gen_s, 1),
               value_rel=abs(val - ev["value"]) / abs(ev["value"]),
               G_rel=float(np.linalg.norm(BV - ev["G"]) / np.linalg.norm(ev["G"])),
               note="same instance, row order, V, triangles and thread count; min over reps")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
