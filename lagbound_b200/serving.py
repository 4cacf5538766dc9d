"""Bound requests served with continuous batching on one GPU.

A request is a graph (with its planted or starting partition) and a solve budget; its answer is the candidate upper
bound of the pipeline's solve + estimate stages (alm_vcs.py main loop, est_dual_vcs.py value / eig_round) at that
budget.  The certificate and its verification stay the reference's CPU code.

The server admits a request when a worker slot and its device-memory estimate fit the HBM budget, and runs it on
its own host thread with its own library context (its own CUDA stream) and torch stream, so the kernels of requests
in flight overlap on the device; state (V, multipliers, triangle pool, pair level) stays resident for the whole
request.  Requests that arrive while others run are admitted as slots and memory free up.  Each request's work is
the same alone and in the mix (it owns its stream and state; only the floating-point order of the sweeps' atomics
differs from run to run).
"""
from __future__ import annotations

import math
import sys
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from lagbound_b200.problem import Context, Problem, locality_order

RHO, TRI_WEIGHT = 0.02, 1.0


@dataclass
class BoundRequest:
    rid: int
    n: int
    indptr: np.ndarray
    indices: np.ndarray
    d: np.ndarray
    L: float
    C0: float
    labels: np.ndarray
    r: int = 16
    dtype: str = "bf16"
    outers: int = 30             # AL outer iterations (one sweep each)
    tri_every: int = 10          # triangle-pool rounds (alm_vcs.py:1735-1756) every tri_every outers
    tri_add: int = 0             # triangles added per round (0: 2 n)
    eig_iters: int = 100         # LOBPCG iterations of the candidate bound
    graph: bool = True           # outer iterations replayed as CUDA graphs (lb_outer_loop)
    arrival: float = 0.0         # seconds after the stream's start
    phases: dict = field(default_factory=dict)   # wall seconds per phase of the request's work (filled by the solve)

    @classmethod
    def from_graph(cls, rid, g, **kw):
        return cls(rid, int(g.n), g.indptr, g.indices, np.asarray(g.d, np.float64), float(g.L), float(g.C0),
                   np.asarray(g.labels), **kw)

    @property
    def nnz(self):
        return int(len(self.indices))

    def device_bytes(self):
        """Estimate of the request's device memory: CSR, V and G, sweep buffers, triangle pool and incidences, pair
        level, the estimate's FP64 blocks (LOBPCG keeps about ten n x (r + 16) blocks)."""
        s_v = {"f64": 8, "f32": 4, "bf16": 2}[self.dtype]
        ld = max(self.r, 16 // s_v)
        ld = 1 << (ld - 1).bit_length()
        T = (self.tri_add or 2 * self.n) * max(1, self.outers // self.tri_every)
        P = int(np.max(self.labels)) + 1 if len(self.labels) else 1
        b = 12 * self.nnz + 40 * self.n + (s_v + 8) * self.n * ld + 80 * T + 16 * P * P + 8 * P * ld * 4
        b += 10 * 8 * self.n * (self.r + 16) + 3 * 8 * self.n * 64
        return int(b * 1.2) + (64 << 20)


@dataclass
class BoundResult:
    rid: int
    ub: float
    dv: float
    n: int
    arrival: float
    admitted: float
    done: float
    log: list = field(default_factory=list)

    @property
    def latency(self):
        return self.done - self.arrival


def solve_bound(ctx, req: BoundRequest):
    """One request on `ctx`: pair level on the request's partition (weight by the pw_rule), `outers` AL outer
    iterations (sweep, evaluation, multiplier update; triangle-pool rounds), then the candidate bound
    dv + max(0, -lambda_min) sum(s) / L with the GPU LOBPCG (scale "vol").  Returns (ub, dv)."""
    import torch
    from lagbound_b200 import estimator_gpu as E
    from lagbound_b200 import synth
    from lagbound_b200.stages.alm_vcs import Level, mobility_ratio
    clock = [time.perf_counter()]

    def phase(name):
        t = time.perf_counter()
        req.phases[name] = req.phases.get(name, 0.0) + t - clock[0]
        clock[0] = t

    n = req.n
    lab = np.unique(req.labels, return_inverse=True)[1].astype(np.int64)
    order = locality_order(lab)
    V = synth.random_V(n, req.r, seed=req.rid)
    inst = dict(n=n, indptr=req.indptr, indices=req.indices, weights=None, d=req.d, L=req.L, C0=req.C0)
    lv = Level(lab, req.d)
    # pw_rule (alm_vcs.py:1663-1688) with its default constants
    R1 = mobility_ratio(ctx, inst, V, [lv], RHO, 1.0)
    pw = min(0.1 / R1, 0.05 / (RHO * n * float(n) / req.L))
    p = Problem(ctx, n, req.indptr, req.indices, None, req.d, req.L, req.C0, req.r, req.dtype, order=order)
    try:
        p.set_V(V)
        p.add_pair_level(lab, lv.P, pw)
        p.set_triangles(np.zeros((0, 3), np.int64), np.zeros(0))
        rng = np.random.default_rng(req.rid)
        nbatch = 512 if n >= 512 * 64 else min(n, max(8, n // 64))       # api.py:250
        tri_add = req.tri_add or 2 * n
        phase("setup")
        it = 0
        while it < req.outers:
            # the outer iterations up to the next triangle round in one native call (a CUDA graph replayed), with
            # no host synchronisation or Python in between
            k = min(req.tri_every, req.outers - it)
            p.outer_loop(np.stack([rng.permutation(n) for _ in range(k)]), RHO, TRI_WEIGHT, 0.0, nbatch, 1.0,
                         graph=req.graph)
            it += k
            phase("outers")
            if it % req.tri_every == 0 and it < req.outers:
                p.tri_pool_round(0.3, 100, 60, 8, 200, tri_add, tri_add // 2, 16_000_000)
                phase("triangle_rounds")
        W = p.get_V()
        sig = p.get_pair_sigma(0)
        TI, lam = p.get_triangles(), p.get_lam()
    finally:
        p.close()
    phase("readback")
    op = E.DeviceOperator(ctx, n, req.indptr, req.indices, None, req.d, req.L, req.C0,
                          pair_levels=[(lab, lv.P, 0.5 * (sig + sig.T))], TI=TI, lam=lam, order=order)
    try:
        dev = torch.device(f"cuda:{ctx.device}")
        Wt = torch.as_tensor(W.astype(np.float32).astype(np.float64), device=dev)
        const = req.C0 + float(lam.sum())
        dv, g, _ = E.value(op, Wt, const, req.L)
        recs, _ = E.eig_round(op, Wt, dv, g, req.d, req.L, seed=req.rid, maxiter=req.eig_iters, log=lambda *a: None)
        phase("estimate")
        return float(recs["vol"]["ub"]), float(dv)
    finally:
        op.close()


class BoundServer:
    """Continuous batching of bound requests on one GPU: at most `slots` requests in flight and their estimated
    device memory within `hbm_budget` bytes; each runs on its own thread, context and streams."""

    def __init__(self, device=0, slots=8, hbm_budget=150e9, switch_interval=5e-4):
        self.device = int(device)
        self.slots = int(slots)
        # Python's thread switch interval while serving (None: unchanged; Python's default is 5 ms).  A request
        # thread gives up the GIL at every wait for the device and then waits up to this long for another thread to
        # hand it back; 0.5 ms measured best for 32 requests in flight
        self.switch_interval = switch_interval
        self.budget = float(hbm_budget)
        self.lock = threading.Condition()
        self.pending = []
        self.inflight = {}
        self.used = 0.0
        self.results = []
        self.errors = []
        self.t0 = None

    def _solve(self, req):
        """A request's work on the calling thread, with its own torch stream and library context: (ub, dv)."""
        import torch
        torch.cuda.set_device(self.device)
        with torch.cuda.stream(torch.cuda.Stream(device=self.device)):
            ctx = Context(self.device)
            try:
                return solve_bound(ctx, req)
            finally:
                ctx.close()

    def _run(self, req, need):
        t_adm = time.perf_counter() - self.t0
        try:
            ub, dv = self._solve(req)
            res = BoundResult(req.rid, ub, dv, req.n, req.arrival, t_adm, time.perf_counter() - self.t0,
                              log=[dict(req.phases)])
        except BaseException as e:                        # reported by run()
            res = None
            err = e
        with self.lock:
            self.used -= need
            del self.inflight[req.rid]
            if res is not None:
                self.results.append(res)
            else:
                self.errors.append((req.rid, err))
            self.lock.notify_all()

    def _admit(self):
        """Start pending requests (arrival order) while a slot and memory are free; a request larger than the whole
        budget is refused."""
        while self.pending and len(self.inflight) < self.slots:
            req = self.pending[0]
            need = req.device_bytes()
            if need > self.budget:
                self.pending.pop(0)
                self.errors.append((req.rid, MemoryError(f"request {req.rid} needs {need / 1e9:.1f} GB")))
                continue
            if self.used + need > self.budget and self.inflight:
                return
            self.pending.pop(0)
            self.used += need
            th = threading.Thread(target=self._run, args=(req, need), daemon=True)
            self.inflight[req.rid] = th
            th.start()

    def run(self, requests, timeout=3600.0):
        """Serve `requests` (arriving at req.arrival seconds after the start); returns the results in completion
        order.  Raises the first error of a request."""
        reqs = sorted(requests, key=lambda q: q.arrival)
        old_si = sys.getswitchinterval()
        if self.switch_interval:
            sys.setswitchinterval(self.switch_interval)
        try:
            return self._serve(reqs, timeout)
        finally:
            sys.setswitchinterval(old_si)

    def _serve(self, reqs, timeout):
        self.t0 = time.perf_counter()
        k = 0
        with self.lock:
            while k < len(reqs) or self.pending or self.inflight:
                now = time.perf_counter() - self.t0
                while k < len(reqs) and reqs[k].arrival <= now:
                    self.pending.append(reqs[k])
                    k += 1
                self._admit()
                if self.errors:
                    break
                wait = (reqs[k].arrival - now) if k < len(reqs) else 1.0
                if now > timeout:
                    raise TimeoutError("bound requests did not finish in time")
                self.lock.wait(timeout=max(1e-3, min(wait, 1.0)))
            while self.inflight:
                self.lock.wait(timeout=1.0)
        if self.errors:
            rid, e = self.errors[0]
            raise RuntimeError(f"request {rid} failed: {e!r}") from e
        return list(self.results)


def latency_stats(results):
    """p50 / p99 of the time from arrival to bound, throughput over the stream."""
    lat = np.array([r.latency for r in results])
    span = max(r.done for r in results) - min(r.arrival for r in results)
    wait = np.array([r.admitted - r.arrival for r in results])
    ph = {}
    for r in results:
        for k, v in (r.log[0] if r.log and isinstance(r.log[0], dict) else {}).items():
            ph[k] = ph.get(k, 0.0) + v / len(results)
    return {"requests": len(results), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "requests_per_s": len(results) / span if span > 0 else math.inf,
            "span_s": span, "mean_queue_s": float(wait.mean()),
            "mean_phase_s": {k: round(v, 4) for k, v in ph.items()}}


def request_stream(count, rate=20.0, seed=0, n_min=1000, n_max=1_000_000, alpha=1.2, device=None, **kw):
    """Poisson arrivals at `rate` per second; n ~ Pareto(alpha) clipped to [n_min, n_max], mean degree U[8, 50],
    r uniform in {16, ..., 32}; Chung-Lu graphs with planted communities (drawn by torch on `device` if given)."""
    from lagbound_b200 import synth
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for k in range(count):
        n = int(min(n_max, n_min * (1.0 - rng.random()) ** (-1.0 / alpha)))
        mean = float(rng.uniform(8, 50))
        r = int(rng.integers(16, 33))
        args = (n, mean, 2.3, max(50, n // 10), max(2, n // 150), 0.25)
        g = synth.chung_lu_communities_torch(*args, seed=seed * 1000 + k, device=device) if device else \
            synth.chung_lu_communities(*args, seed=seed * 1000 + k)
        out.append(BoundRequest.from_graph(k, g, r=r, arrival=float(t[k]), **kw))
    return out


def main(argv=None):
    """Serve a Poisson stream of bound requests and print one JSON line with p50 / p99 time-to-bound."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--requests", type=int, default=40)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--slots", type=int, default=32)
    ap.add_argument("--hbm_budget", type=float, default=150e9)
    ap.add_argument("--n_max", type=int, default=1_000_000)
    ap.add_argument("--outers", type=int, default=30)
    ap.add_argument("--dtype", default="bf16", choices=["bf16", "f32", "f64"])
    ap.add_argument("--no_graph", action="store_true", help="outer iterations launched directly, not as CUDA graphs")
    ap.add_argument("--switch_interval", type=float, default=5e-4,
                    help="Python thread switch interval while serving (seconds)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=2, help="small requests solved before the stream (module loading, "
                                                            "library initialisation)")
    a = ap.parse_args(argv)
    if a.warmup:
        BoundServer(a.device, a.slots, a.hbm_budget).run(
            request_stream(a.warmup, a.rate, a.seed + 99, n_max=2000, device=f"cuda:{a.device}", dtype=a.dtype,
                           outers=a.outers, graph=not a.no_graph))
    t0 = time.time()
    reqs = request_stream(a.requests, a.rate, a.seed, n_max=a.n_max, device=f"cuda:{a.device}", dtype=a.dtype,
                          outers=a.outers, graph=not a.no_graph)
    gen_s = time.time() - t0
    res = BoundServer(a.device, a.slots, a.hbm_budget, a.switch_interval).run(reqs)
    st = latency_stats(res)
    st.update(config=dict(requests=a.requests, rate_per_s=a.rate, slots=a.slots, hbm_budget_gb=a.hbm_budget / 1e9,
                          warmup_requests=a.warmup,
                          n="Pareto(1.2) clipped to [1000, %d]" % a.n_max, mean_degree="U[8, 50]", r="U{16..32}",
                          dtype=a.dtype, outers=a.outers, graphs=not a.no_graph,
                          time_to="candidate bound (solve + estimate)"),
              n_total=int(sum(q.n for q in reqs)), n_max_seen=int(max(q.n for q in reqs)),
              gen_seconds=round(gen_s, 1), ub=[round(r.ub, 6) for r in sorted(res, key=lambda r: r.rid)])
    print(json.dumps(st), flush=True)


if __name__ == "__main__":
    main()
