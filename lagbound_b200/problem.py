"""Host-side objects over the C ABI: a device context and one augmented-Lagrangian problem (graph, V, pair levels,
VCS levels, triangle pool) resident on the GPU.

The names mirror the reference's solver state (src/lagbound/_core/alm_vcs.py): V, levels with sig, VCS levels with a
working set (ptr, col, sig, age), the triangle pool (TI, lam), rho, tri_weight, pairlvl_weight.
"""
from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _capi as C

DTYPES = {"f64": C.LB_F64, "fp64": C.LB_F64, "float64": C.LB_F64, "f32": C.LB_F32, "fp32": C.LB_F32,
          "float32": C.LB_F32, "bf16": C.LB_BF16, "bfloat16": C.LB_BF16}


class Context:
    """One CUDA device and one stream; every problem created from it runs its work in order on that stream."""

    def __init__(self, device: int = 0, stream=None):
        """stream: None = the context's own stream; else a CUDA stream handle (an int, e.g. torch's
        current_stream().cuda_stream) that the context's work is queued on."""
        h = ctypes.c_void_p()
        if stream is None:
            C.call("lb_ctx_create", int(device), ctypes.byref(h))
        else:
            C.call("lb_ctx_create_on_stream", int(device), ctypes.c_void_p(int(stream)), ctypes.byref(h))
        self.h = h
        self.device = device
        self._problems = weakref.WeakSet()
        self._graphs = weakref.WeakSet()

    def synchronize(self):
        C.call("lb_ctx_synchronize", self.h)

    def set_cache(self, l2_fetch_bytes=0, v_persist_fraction=0.0):
        """L2 fetch granularity (32/64/128 bytes, 0 = leave) and the share of V kept persisting in L2."""
        C.call("lb_ctx_set_cache", self.h, int(l2_fetch_bytes), float(v_persist_fraction))

    def timer_start(self):
        C.call("lb_ctx_timer", self.h, 0, None)

    def timer_stop(self) -> float:
        ms = ctypes.c_float()
        C.call("lb_ctx_timer", self.h, 1, ctypes.byref(ms))
        return float(ms.value)

    def capture(self):
        """CUDA-graph capture of this context's stream: `with ctx.capture() as g: p.eval_async(...)` records the
        asynchronous calls made inside the block (each problem evaluated once before); g.launch() replays them."""
        return CudaGraph(self)

    def close(self):
        """Destroys the problems created from this context first, then the context."""
        if getattr(self, "h", None):
            for g in list(self._graphs):
                g.close()
            for p in list(self._problems):
                p.close()
            C.get_lib().lb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def locality_order(labels, degrees=None):
    """A locality order from a partition (the solver's starting partition or pair-level labels): rows grouped by
    label, labels in order of first appearance, rows in their original order inside a label."""
    lab = np.unique(np.asarray(labels), return_inverse=True)[1]
    return np.argsort(lab, kind="stable").astype(np.int64)


class CudaGraph:
    """A captured sequence of asynchronous calls on one context (see Context.capture)."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.h = None
        self.kernels = 0

    def __enter__(self):
        C.call("lb_ctx_capture_begin", self.ctx.h)
        return self

    def __exit__(self, et, ev, tb):
        h = ctypes.c_void_p()
        try:
            C.call("lb_ctx_capture_end", self.ctx.h, ctypes.byref(h))
        except Exception:
            if et is None:
                raise
            return False
        self.h = h
        k = ctypes.c_int64()
        C.call("lb_cuda_graph_kernels", self.h, ctypes.byref(k))
        self.kernels = int(k.value)
        self.ctx._graphs.add(self)
        return False

    def launch(self):
        C.call("lb_cuda_graph_launch", self.h)

    def close(self):
        if getattr(self, "h", None):
            C.get_lib().lb_cuda_graph_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Problem:
    """Device-resident instance (CSR, volumes, L, C0) plus V and the multiplier state."""

    def __init__(self, ctx: Context, n, indptr, indices, weights, d, L, C0, r, dtype="f64", order=None):
        """order: optional locality order (order[k] = caller row placed at internal row k), e.g.
        locality_order(labels); all inputs and outputs stay in the caller's row order."""
        self.ctx = ctx
        self.n = int(n)
        self.r = int(r)
        self.dtype = DTYPES[dtype] if isinstance(dtype, str) else int(dtype)
        ip = C.c(indptr, np.int64); ix = C.c(indices, np.int64)
        w = None if weights is None else C.c(weights, np.float64)
        dd = C.c(d, np.float64)
        h = ctypes.c_void_p()
        od = None if order is None else C.c(order, np.int64)
        C.call("lb_problem_create_ordered", ctx.h, self.n, C.ptr(ip), C.ptr(ix), C.ptr(w), C.ptr(dd), float(L),
               float(C0), self.r, self.dtype, C.ptr(od), ctypes.byref(h))
        self.h = h
        ctx._problems.add(self)
        self.L = float(L); self.C0 = float(C0)
        self.pair_P = []
        self.vcs_P = []
        self.vcs_nnz = []
        self.T = 0

    @classmethod
    def from_instance(cls, ctx, inst, r, dtype="f64", order=None):
        """From an object with n, indptr, indices, data, d, L, C0 (unit data -> unweighted)."""
        w = None if np.all(inst.data == 1.0) else inst.data
        return cls(ctx, inst.n, inst.indptr, inst.indices, w, inst.d, inst.L, inst.C0, r, dtype, order)

    def info(self):
        ld = ctypes.c_int32(); hv = ctypes.c_int64(); b = ctypes.c_int64()
        C.call("lb_problem_info", self.h, ctypes.byref(ld), ctypes.byref(hv), ctypes.byref(b))
        return dict(ld=ld.value, heavy_rows=hv.value, device_bytes=b.value)

    # ---------------------------------------------------------------------------------------- V
    def set_V(self, V):
        V = C.c(V, np.float64)
        assert V.shape == (self.n, self.r)
        C.call("lb_set_V", self.h, C.ptr(V))

    def set_V_raw(self, V):
        """V already in the storage dtype (bf16 given as uint16 / torch bf16 viewed as int16)."""
        assert V.flags["C_CONTIGUOUS"]
        C.call("lb_set_V_raw", self.h, C.ptr(V), self.dtype)

    def set_V_device(self, X, wait=True):
        """X: a CUDA FP64 tensor of shape (n, r), contiguous, in the caller's row order (torch).  wait=False only
        queues the conversion on the context's stream."""
        assert X.is_cuda and X.dtype.is_floating_point and X.element_size() == 8 and X.is_contiguous()
        assert tuple(X.shape) == (self.n, self.r)
        C.call("lb_set_V_device" if wait else "lb_set_V_device_async", self.h, ctypes.c_void_p(X.data_ptr()))

    def G_device(self, out, wait=True):
        """G of the last gradient evaluation into the CUDA FP64 tensor `out` of shape (n, r); wait=False only
        queues the copy on the context's stream."""
        assert out.is_cuda and out.element_size() == 8 and out.is_contiguous() and tuple(out.shape) == (self.n, self.r)
        C.call("lb_get_G_device" if wait else "lb_get_G_device_async", self.h, ctypes.c_void_p(out.data_ptr()))
        return out

    def get_V(self):
        out = np.empty((self.n, self.r))
        C.call("lb_get_V", self.h, C.ptr(out))
        return out

    # ---------------------------------------------------------------------------------------- levels
    def add_pair_level(self, lab, P=None, w=1.0):
        lab = C.c(lab, np.int64)
        P = int(lab.max()) + 1 if P is None else int(P)
        lv = ctypes.c_int32()
        C.call("lb_pair_level_add", self.h, P, C.ptr(lab), float(w), ctypes.byref(lv))
        self.pair_P.append(P)
        return lv.value

    def set_pair_sigma(self, level, sig):
        sig = C.c(sig, np.float64)
        C.call("lb_pair_level_set_sigma", self.h, int(level), C.ptr(sig))

    def get_pair_sigma(self, level):
        P = self.pair_P[level]; out = np.empty((P, P))
        C.call("lb_pair_level_get_sigma", self.h, int(level), C.ptr(out))
        return out

    def set_pair_weight(self, w, vc_weight=1.0):
        C.call("lb_set_pair_weight", self.h, float(w), float(vc_weight))

    def add_vcs_level(self, lab, P=None, wv=1.0):
        lab = C.c(lab, np.int64)
        P = int(lab.max()) + 1 if P is None else int(P)
        lv = ctypes.c_int32()
        C.call("lb_vcs_level_add", self.h, P, C.ptr(lab), float(wv), ctypes.byref(lv))
        self.vcs_P.append(P); self.vcs_nnz.append(0)
        return lv.value

    def set_vcs_ws(self, level, ptr, col, sig, age=None):
        ptr = C.c(ptr, np.int64); col = C.c(col, np.int32); sig = C.c(sig, np.float64)
        age = C.c(age, np.uint8)
        nnz = int(ptr[-1])
        C.call("lb_vcs_set_ws", self.h, int(level), nnz, C.ptr(ptr), C.ptr(col), C.ptr(sig), C.ptr(age))
        self.vcs_nnz[level] = nnz

    def get_vcs_ws(self, level):
        nnz = self.vcs_nnz[level]; sig = np.empty(nnz); age = np.empty(nnz, np.uint8)
        C.call("lb_vcs_get_ws", self.h, int(level), C.ptr(sig), C.ptr(age))
        return sig, age

    def set_triangles(self, TI, lam):
        TI = C.c(np.asarray(TI).reshape(-1, 3), np.int64); lam = C.c(lam, np.float64)
        C.call("lb_tri_set", self.h, len(TI), C.ptr(TI), C.ptr(lam))
        self.T = len(TI)

    def get_lam(self):
        out = np.empty(self.T)
        C.call("lb_tri_get_lam", self.h, C.ptr(out))
        return out

    # ---------------------------------------------------------------------------------------- evaluation
    @staticmethod
    def _flags(grad, fixed, timing=False):
        return (C.LB_EVAL_GRAD if grad else 0) | (C.LB_EVAL_FIXED if fixed else 0) | (C.LB_EVAL_TIMING if timing else 0)

    def eval(self, rho=0.02, tri_weight=1.0, grad=True, fixed=False) -> dict:
        out = C.EvalOut()
        C.call("lb_eval", self.h, float(rho), float(tri_weight), self._flags(grad, fixed), ctypes.byref(out))
        return out.as_dict()

    def eval_async(self, rho=0.02, tri_weight=1.0, grad=True, fixed=False, timing=False):
        C.call("lb_eval_async", self.h, float(rho), float(tri_weight), self._flags(grad, fixed, timing))

    def timing_collect(self):
        """Device ms per phase summed over the timed evaluations since the last collect, and their count."""
        ms = np.zeros(len(C.PHASES)); cnt = ctypes.c_int64()
        C.call("lb_timing_collect", self.h, C.ptr(ms), ctypes.byref(cnt))
        return dict(zip(C.PHASES, ms.tolist())), cnt.value

    LIGHT_THRESHOLDS = (0, 64, 128, 256, 512, 1024)

    def set_light_threshold(self, work):
        """Rows with at most `work` edges + 2 x triangle incidences run one per lane group (-1: autotune)."""
        C.call("lb_set_light_threshold", self.h, int(work))

    def light_threshold(self):
        v = ctypes.c_int32(); ms = np.zeros(len(self.LIGHT_THRESHOLDS), np.float32)
        C.call("lb_get_light_threshold", self.h, ctypes.byref(v), C.ptr(ms))
        return v.value, dict(zip(self.LIGHT_THRESHOLDS, ms.tolist()))

    def launch_count(self):
        v = ctypes.c_int64()
        C.call("lb_launch_count", self.h, ctypes.byref(v))
        return v.value

    def eval_fetch(self) -> dict:
        out = C.EvalOut()
        C.call("lb_eval_fetch", self.h, ctypes.byref(out))
        return out.as_dict()

    def eval_host(self, V_raw, rho=0.02, tri_weight=1.0, grad=True, fixed=False) -> dict:
        out = C.EvalOut()
        C.call("lb_eval_host", self.h, C.ptr(V_raw), float(rho), float(tri_weight), self._flags(grad, fixed),
               ctypes.byref(out))
        return out.as_dict()

    def eval_host_pipelined(self, V_list, G_list=None, rho=0.02, tri_weight=1.0, grad=True, fixed=False):
        """Evaluations of the host arrays V_list[k] (raw storage dtype, as eval_host takes them) with the copies
        overlapped; G_list[k] (optional, host n x r, as G_raw fills it) receives step k's gradient.  Pinned host
        arrays overlap their copies with the evaluations.  Returns one result dict per step."""
        ns = len(V_list)
        for V in V_list:
            assert V.flags["C_CONTIGUOUS"]
        vp = (ctypes.c_void_p * ns)(*[V.ctypes.data for V in V_list])
        gp = None
        if G_list is not None:
            assert len(G_list) == ns and grad
            for G in G_list:
                assert G.flags["C_CONTIGUOUS"]
            gp = (ctypes.c_void_p * ns)(*[G.ctypes.data for G in G_list])
        outs = (C.EvalOut * ns)()
        C.call("lb_eval_host_pipelined", self.h, ns, vp, gp, float(rho), float(tri_weight), self._flags(grad, fixed),
               outs)
        return [o.as_dict() for o in outs]

    def G_raw(self, out):
        """Copy the last gradient into `out` (host, n x r, FP64 for the FP64 form, FP32 otherwise; pinned memory
        for full-speed copies) in the caller's row order."""
        C.call("lb_get_G_raw", self.h, C.ptr(out))
        return out

    def G(self):
        out = np.empty((self.n, self.r))
        C.call("lb_get_G", self.h, C.ptr(out))
        return out

    def pair_pp(self, level):
        P = self.pair_P[level]; out = np.empty((P, P))
        C.call("lb_get_pair_pp", self.h, int(level), C.ptr(out))
        return out

    def tri_pt(self):
        pt = np.empty(self.T); gt = np.empty(self.T)
        C.call("lb_get_tri_pt", self.h, C.ptr(pt), C.ptr(gt))
        return pt, gt

    def vcs_ppv(self, level):
        nnz = self.vcs_nnz[level]
        ppv = np.empty(nnz); slk = np.empty(nnz, np.uint8); stn = np.empty(nnz)
        C.call("lb_get_vcs_ppv", self.h, int(level), C.ptr(ppv), C.ptr(slk), C.ptr(stn))
        return ppv, slk, stn

    def sweeps(self, perms, rho, rt, damp=0.0, nbatch=64, kap2=1.0):
        """Batched Gauss-Seidel sweeps (one row permutation per sweep, caller row ids)."""
        perms = C.c(np.atleast_2d(perms), np.int64)
        assert perms.shape[1] == self.n
        C.call("lb_sweeps", self.h, len(perms), float(rho), float(rt), float(damp), int(nbatch), C.ptr(perms),
               float(kap2))

    def outer_loop(self, perms, rho, tri_weight=1.0, damp=0.0, nbatch=64, kap2=1.0, iters=None, graph=True):
        """`iters` (default: one per row order) AL outer iterations in one native call: sweep k in the row order
        perms[k % len(perms)] with rt = rho tri_weight, evaluation without the gradient, multiplier update; with
        graph=True replayed as a CUDA graph of two iterations.  Returns the captured graph's kernel count (0: none)."""
        perms = C.c(np.atleast_2d(perms), np.int64)
        assert perms.shape[1] == self.n
        iters = len(perms) if iters is None else int(iters)
        k = ctypes.c_int64()
        C.call("lb_outer_loop", self.h, iters, C.ptr(perms), len(perms), float(rho), float(tri_weight), float(damp),
               int(nbatch), float(kap2), 1 if graph else 0, ctypes.byref(k))
        return int(k.value)

    def separate(self, thresh=0.3, maxh=100, maxk=60, hub2=8, cap2=200, vtol=1e-3, cap0=0, cap1=0, nchunk=512,
                 nbins=2000, families=(0, 1)):
        """Triangle separation at the current V (alm_vcs.py:938-984): returns {family: (triples, values)} with the
        reference's candidate arrays (caller vertex ids)."""
        n0 = ctypes.c_int64(); n1 = ctypes.c_int64()
        fam = (1 if 0 in families else 0) | (2 if 1 in families else 0)
        C.call("lb_separate", self.h, float(thresh), int(maxh), int(maxk), int(hub2), int(cap2), float(vtol),
               int(cap0), int(cap1), int(nchunk), int(nbins), fam, ctypes.byref(n0), ctypes.byref(n1))
        out = {}
        for f, cnt in ((0, n0.value), (1, n1.value)):
            if f not in families:
                continue
            tri = np.empty((cnt, 3), np.int64); val = np.empty(cnt)
            C.call("lb_separate_get", self.h, f, C.ptr(tri), C.ptr(val))
            out[f] = (tri, val)
        return out

    def tri_pool_round(self, thresh, maxh, maxk, hub2, cap2, tri_add, tri1_add, tri_max, vtol=1e-3, nchunk=512,
                       nbins=2000):
        """The solver's triangle-pool round on the device (alm_vcs.py:1735-1756): purge lam = 0, separate when
        there is room, merge the candidates.  Returns (purged, added)."""
        cnt = np.zeros(3, np.int64)
        C.call("lb_tri_pool_round", self.h, float(thresh), int(maxh), int(maxk), int(hub2), int(cap2), float(vtol),
               int(nchunk), int(nbins), int(tri_add), int(tri1_add), int(tri_max), C.ptr(cnt))
        self.T = int(cnt[2])
        return int(cnt[0]), int(cnt[1])

    def get_triangles(self):
        """The pool's triangles (T x 3 caller vertex ids, pool order)."""
        TI = np.empty((self.T, 3), np.int64)
        C.call("lb_tri_get", self.h, C.ptr(TI))
        return TI

    VCS_SCORES = {"pen": 0, "mean": 1, "mass": 2}

    def vcs_separate(self, level, nadd, tol=1e-4, mode="pen"):
        """VCS working-set separation (vcsops.py:364-414 separate) at the current V: (rows, cols, scores) of the
        nadd best violated entries outside the working set, best first, and the statistics dict of the reference."""
        cnt = ctypes.c_int64(); st = np.zeros(4)
        C.call("lb_vcs_separate", self.h, int(level), int(nadd), float(tol), self.VCS_SCORES[mode], ctypes.byref(cnt),
               C.ptr(st))
        rows = np.empty(cnt.value, np.int64); cols = np.empty(cnt.value, np.int32); sc = np.empty(cnt.value)
        C.call("lb_vcs_separate_get", self.h, C.ptr(rows), C.ptr(cols), C.ptr(sc))
        return rows, cols, sc, dict(nviol=st[0], mass=st[1], nviol_ws=st[2], mass_ws=st[3])

    def vcs_grow(self, level, nadd, tol=1e-4, mode="pen", drop_age=0, max_nnz=2 ** 62):
        """The solver's working-set round (alm_vcs.py:1713-1720) on the device: drop entries with age >= drop_age
        (0 keeps all), separate max(1, min(nadd, room)) entries with room = max(0, max_nnz - kept), add them (none
        at room 0).  Returns (dropped, added, statistics dict of the separation)."""
        st = np.zeros(4); cnt = np.zeros(3, np.int64)
        C.call("lb_vcs_grow", self.h, int(level), int(nadd), float(tol), self.VCS_SCORES[mode], int(drop_age),
               int(max_nnz), C.ptr(st), C.ptr(cnt))
        self.vcs_nnz[level] = int(cnt[2])
        return int(cnt[0]), int(cnt[1]), dict(nviol=st[0], mass=st[1], nviol_ws=st[2], mass_ws=st[3])

    def get_vcs_structure(self, level):
        """(ptr, col) of a VCS level's working set in the caller's row order."""
        ptr = np.empty(self.n + 1, np.int64); col = np.empty(self.vcs_nnz[level], np.int32)
        C.call("lb_vcs_get_structure", self.h, int(level), C.ptr(ptr), C.ptr(col))
        return ptr, col

    def vcs_sig_stats(self, level):
        """(sum of the working-set multipliers, number of positive ones) of a VCS level."""
        sm = ctypes.c_double(); act = ctypes.c_int64()
        C.call("lb_vcs_sig_stats", self.h, int(level), ctypes.byref(sm), ctypes.byref(act))
        return float(sm.value), int(act.value)

    def multiplier_update(self):
        C.call("lb_multiplier_update", self.h)

    def close(self):
        if getattr(self, "h", None):
            C.get_lib().lb_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchedProblem(Problem):
    """Several independent graphs evaluated together: one block-diagonal CSR with per-graph offsets, each graph with
    its own L and C0, one rank and dtype.  V, G and triangles are in the concatenated row numbering (graph g's rows
    start at offsets[g]); triangles must be grouped by graph in graph order.  Pair and VCS levels and sweeps are not
    available.  eval() returns the sums over the graphs, eval_graphs() the per-graph results."""

    def __init__(self, ctx: Context, graphs, r, dtype="f32", orders=None):
        """graphs: objects with n, indptr, indices, d, L, C0 (and data; non-unit data -> weighted); orders: optional
        per-graph locality orders (local row ids)."""
        self.ctx = ctx
        self.r = int(r)
        self.dtype = DTYPES[dtype] if isinstance(dtype, str) else int(dtype)
        ns = np.array([int(g.n) for g in graphs], np.int64)
        self.offsets = np.r_[0, np.cumsum(ns)].astype(np.int64)
        self.ngraphs = len(graphs)
        self.n = int(self.offsets[-1])
        nnz = np.array([len(g.indices) for g in graphs], np.int64)
        eoff = np.r_[0, np.cumsum(nnz)]
        indptr = np.concatenate([np.asarray(g.indptr[:-1], np.int64) + eoff[k] for k, g in enumerate(graphs)] +
                                [np.array([eoff[-1]], np.int64)])
        indices = np.concatenate([np.asarray(g.indices, np.int64) + self.offsets[k] for k, g in enumerate(graphs)])
        weighted = any(getattr(g, "data", None) is not None and not np.all(np.asarray(g.data) == 1.0) for g in graphs)
        w = np.concatenate([np.asarray(g.data, np.float64) for g in graphs]) if weighted else None
        d = np.concatenate([np.asarray(g.d, np.float64) for g in graphs])
        Ls = np.array([float(g.L) for g in graphs]); C0s = np.array([float(g.C0) for g in graphs])
        od = None
        if orders is not None:
            od = np.concatenate([np.asarray(o, np.int64) + self.offsets[k] for k, o in enumerate(orders)])
        h = ctypes.c_void_p()
        ip = C.c(indptr, np.int64); ix = C.c(indices, np.int64); dd = C.c(d, np.float64)
        rp = C.c(self.offsets, np.int64); Lc = C.c(Ls, np.float64); Cc = C.c(C0s, np.float64)
        wc = None if w is None else C.c(w, np.float64)
        oc = None if od is None else C.c(od, np.int64)
        C.call("lb_problem_create_batched", ctx.h, self.ngraphs, C.ptr(rp), self.n, C.ptr(ip), C.ptr(ix), C.ptr(wc),
               C.ptr(dd), C.ptr(Lc), C.ptr(Cc), self.r, self.dtype, C.ptr(oc), ctypes.byref(h))
        self.h = h
        ctx._problems.add(self)
        self.L = float(Ls.sum()); self.C0 = float(C0s.sum())
        self.pair_P = []
        self.vcs_P = []
        self.vcs_nnz = []
        self.T = 0

    def eval_graphs(self):
        """Per-graph results of the last evaluation: dict of arrays value, primal, quadA, zz, tri_tot."""
        out = np.empty((self.ngraphs, 5))
        C.call("lb_eval_graphs", self.h, C.ptr(out))
        return {k: out[:, j].copy() for j, k in enumerate(("value", "primal", "quadA", "zz", "tri_tot"))}

