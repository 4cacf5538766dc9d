"""The candidate-bound estimate (est_dual_vcs.py) with every n-sized vector on the GPU: the products C(y) X through
the library's fixed-multiplier evaluation on device pointers (lb_set_V_device / lb_get_G_device), the Riemannian
polish and a block LOBPCG on the pencil (Diag(g) - C, Diag(s)) in FP64 torch tensors (dense block algebra through
cuBLAS / cuSOLVER).  Same quantities, step rules and stopping rules as lagbound_b200/estimator.py, which follows
est_dual_vcs.py:248-389 with SciPy's LOBPCG on the host; here the eigensolver is a restatement of block LOBPCG
(Knyazev 2001: Rayleigh-Ritz on [X, W, P] with B-orthonormalised blocks, soft restart without P when the Gram
matrix loses definiteness)."""
from __future__ import annotations

import math
import time

import numpy as np

import ctypes

from . import _capi
from .problem import Context, Problem


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the GPU estimate needs a CUDA device")
    return torch


class DeviceOperator:
    """X -> C(y) X at fixed multipliers for CUDA FP64 tensors (one device problem per power-of-two block width).

    The problems live on a library context bound to torch's current stream at construction (the stream every call
    must then run on): the copy of X in, the evaluation and the copy of C(y) X out are queued behind the caller's
    torch work on that stream, with no host synchronisation."""

    MAX_WIDTH = 64

    def __init__(self, ctx, n, indptr, indices, weights, d, L, C0, pair_levels=(), vcs_levels=(), TI=None, lam=None,
                 order=None):
        self.torch = _torch()
        dev = self.torch.device(f"cuda:{ctx.device}")
        self.stream = self.torch.cuda.current_stream(dev)
        self.ctx = Context(ctx.device, stream=self.stream.cuda_stream)
        self.n = int(n)
        self.graph = (indptr, indices, weights, d, float(L), float(C0))
        self.pair_levels = list(pair_levels)
        self.vcs_levels = list(vcs_levels)
        self.TI = np.zeros((0, 3), np.int64) if TI is None else np.asarray(TI, np.int64).reshape(-1, 3)
        self.lam = np.zeros(0) if lam is None else np.asarray(lam, np.float64)
        self.order = order
        self.dev = self.torch.device(f"cuda:{ctx.device}")
        self._probs = {}
        self._buf = {}
        self.calls = 0

    def _problem(self, width):
        p = self._probs.get(width)
        if p is None:
            indptr, indices, weights, d, L, C0 = self.graph
            p = Problem(self.ctx, self.n, indptr, indices, weights, d, L, C0, width, dtype="f64", order=self.order)
            for lab, P, sig in self.pair_levels:
                lv = p.add_pair_level(lab, P)
                p.set_pair_sigma(lv, sig)
            for lab, P, ptr, col, sig in self.vcs_levels:
                lv = p.add_vcs_level(lab, P)
                p.set_vcs_ws(lv, ptr, col, sig)
            if len(self.TI):
                p.set_triangles(self.TI, self.lam)
            self._probs[width] = p
            t = self.torch
            self._buf[width] = (t.zeros(self.n, width, dtype=t.float64, device=self.dev),
                                t.empty(self.n, width, dtype=t.float64, device=self.dev))
        return p, self._buf[width]

    def __call__(self, X):
        t = self.torch
        assert t.cuda.current_stream(self.dev) == self.stream, "call on the stream the operator was built on"
        X = X.reshape(self.n, -1)
        out = t.empty_like(X)
        for c0 in range(0, X.shape[1], self.MAX_WIDTH):
            w = min(self.MAX_WIDTH, X.shape[1] - c0)
            width = 2
            while width < w:
                width *= 2
            p, (xin, gout) = self._problem(width)
            xin[:, :w] = X[:, c0:c0 + w]
            if w < width:
                xin[:, w:] = 0
            # one stream: the library's kernels run after the copy into xin and before the copy out of gout
            p.set_V_device(xin, wait=False)
            p.eval_async(grad=True, fixed=True)
            p.G_device(gout, wait=False)
            out[:, c0:c0 + w] = gout[:, :w]
        self.calls += 1
        return out

    def lobpcg(self, X, g, s, prec, maxiter):
        """Native block LOBPCG (lb_lobpcg) on the pencil (Diag(g) - C(y), Diag(s)) from the start block X (n x k
        CUDA FP64, k <= 64): the same iteration as lobpcg() below, run by the library on this operator's stream.
        Returns (theta, X) with theta a NumPy array."""
        t = self.torch
        k = X.shape[1]
        width = 2
        while width < k:
            width *= 2
        p, _ = self._problem(width)
        Xo = X.detach().clone().contiguous()
        th = np.zeros(k)
        done = ctypes.c_int32()
        _capi.call("lb_lobpcg", p.h, int(k), ctypes.c_void_p(Xo.data_ptr()), ctypes.c_void_p(g.data_ptr()),
                   ctypes.c_void_p(s.data_ptr()), ctypes.c_void_p(prec.data_ptr()), int(maxiter), _capi.ptr(th),
                   ctypes.byref(done))
        self.calls += 2 * int(done.value) + 1
        return th, Xo

    def close(self):
        for p in self._probs.values():
            p.close()
        self._probs = {}
        self._buf = {}
        if getattr(self, "ctx", None) is not None:
            self.ctx.close()
            self.ctx = None


def value(op, W, const, L):
    """(dv, g, C W) with g_i = (C W)_i . w_i (est_dual_vcs.py:245-246); dv a Python float."""
    CW = op(W)
    g = (CW * W).sum(1)
    return (const + float(g.sum())) / L, g, CW


def polish_rgd(op, V, const, L, iters=400, time_limit=600.0, ptol=2e-5, log=print, hist=None):
    """estimator.polish_rgd on the GPU (est_dual_vcs.py:276-308): preconditioned Riemannian ascent with BB steps in
    the D metric (alternating forms, clipped to [0.05, 50]) and the Zhang-Hager nonmonotone Armijo test."""
    hist = [] if hist is None else hist
    tp = time.time()
    f, g, CW = value(op, V, const, L)
    Cref, Q, alpha = f, 1.0, 2.0
    nr = CW.norm(dim=1).clamp_min(1e-12)
    Rr = CW - g[:, None] * V
    R = Rr / nr[:, None]
    hist.append(("rgd", 0, time.time() - tp, f))
    log(f"rgd start dv {f:.6f}")
    it, last_chk, bt = 0, f, 0
    while it < iters and time.time() - tp < time_limit:
        it += 1
        gr = float((Rr * R).sum()) / L
        for bt in range(12):
            Vn = V + alpha * R
            Vn = Vn / Vn.norm(dim=1, keepdim=True)
            fn, gn, CWn = value(op, Vn, const, L)
            if fn >= Cref + 1e-4 * alpha * gr:
                break
            alpha *= 0.5
        S = Vn - V
        nrn = CWn.norm(dim=1).clamp_min(1e-12)
        Rrn = CWn - gn[:, None] * Vn
        Rn = Rrn / nrn[:, None]
        Yd = Rn - R
        sy = float((S * (Yd * nrn[:, None])).sum())
        ss = float((S * (S * nrn[:, None])).sum())
        yy = float((Yd * (Yd * nrn[:, None])).sum())
        if sy < 0:
            alpha = (ss / (-sy)) if it % 2 else (-sy / yy)
        else:
            alpha = min(2 * alpha, 50.0)
        alpha = float(min(max(alpha, 0.05), 50.0))
        V, f, g, CW, R, Rr = Vn, fn, gn, CWn, Rn, Rrn
        Qn = 0.85 * Q + 1
        Cref = (0.85 * Q * Cref + f) / Qn
        Q = Qn
        if it % 10 == 0:
            hist.append(("rgd", it, time.time() - tp, f))
            log(f"rgd it {it} dv {f:.6f} alpha {alpha:.3g} bt {bt}")
            if f - last_chk < ptol * 2:
                break
            last_chk = f
    return V


def _b_orth(t, X, s, AX=None):
    """B-orthonormalise the columns of X (B = Diag(s)) by a Cholesky factor of X^T B X; AX follows.  None when the
    block is numerically dependent."""
    G = X.T @ (s[:, None] * X)
    G = 0.5 * (G + G.T)
    Lc, info = t.linalg.cholesky_ex(G)
    if int(info) != 0:
        return None, None
    Linv = t.linalg.solve_triangular(Lc, t.eye(G.shape[0], dtype=G.dtype, device=G.device), upper=False)
    X = X @ Linv.T
    return X, (None if AX is None else AX @ Linv.T)


def _b_orth_dev(t, X, s, AX=None):
    """_b_orth without a host synchronisation: returns (X, AX, ok) with ok a device boolean; when the block is
    numerically dependent (ok false) X and AX come back as NaN."""
    G = X.T @ (s[:, None] * X)
    G = 0.5 * (G + G.T)
    Lc, info = t.linalg.cholesky_ex(G)
    ok = info == 0
    Linv = t.linalg.solve_triangular(Lc, t.eye(G.shape[0], dtype=G.dtype, device=G.device), upper=False)
    Linv = t.where(ok, Linv, t.full_like(Linv, math.nan))
    return X @ Linv.T, (None if AX is None else AX @ Linv.T), ok


def lobpcg(Aop, s, prec, X, maxiter):
    """Block LOBPCG for the smallest eigenpairs of A x = theta B x, B = Diag(s) positive, preconditioner
    Diag(prec): Rayleigh-Ritz on span[X, W, P] each iteration (W = preconditioned residuals B-orthogonalised against
    X, P = the previous step's update).  Returns (theta ascending, X)."""
    t = _torch()
    b = X.shape[1]
    X, _ = _b_orth(t, X, s)
    if X is None:
        raise RuntimeError("LOBPCG start block is rank deficient")
    AX = Aop(X)
    Gm = X.T @ AX
    lam, C = t.linalg.eigh(0.5 * (Gm + Gm.T))
    X, AX = X @ C, AX @ C
    P = AP = None
    def gram(blocks, ablocks):
        S = t.cat(blocks, 1)
        AS = t.cat(ablocks, 1)
        gA = S.T @ AS
        gB = S.T @ (s[:, None] * S)
        gB = 0.5 * (gB + gB.T)
        Lc, info = t.linalg.cholesky_ex(gB)
        return S, AS, 0.5 * (gA + gA.T), gB, Lc, (info == 0) & t.isfinite(gB).all()

    for _ in range(maxiter):
        R = AX - (s[:, None] * X) * lam[None, :]
        W = prec[:, None] * R
        W = W - X @ (X.T @ (s[:, None] * W))
        # W and P are B-orthonormalised and the Gram matrices factored before the host looks at any outcome: one
        # synchronisation per iteration; the rare failures then take the same paths as checking each in turn
        W, _, okW = _b_orth_dev(t, W, s)
        AW = Aop(W)
        blocks, ablocks = [X, W], [AX, AW]
        okP = t.ones((), dtype=t.bool, device=X.device)
        if P is not None:
            Pn, APn, okP = _b_orth_dev(t, P, s, AP)
            blocks.append(Pn)
            ablocks.append(APn)
        S, AS, gA, gB, Lc, okB = gram(blocks, ablocks)
        fW, fP, fB = t.stack([okW, okP, okB]).tolist()
        if not fW:
            break                                              # residual block dependent
        if len(blocks) == 3 and not (fP and fB):
            # P dependent, or the Gram matrix not positive definite with it: soft restart without P
            S, AS, gA, gB, Lc, okB = gram(blocks[:2], ablocks[:2])
            fB = bool(okB)
        if not fB:
            break
        Linv = t.linalg.solve_triangular(Lc, t.eye(gB.shape[0], dtype=gB.dtype, device=gB.device), upper=False)
        th, Y = t.linalg.eigh(Linv @ gA @ Linv.T)
        Cc = Linv.T @ Y[:, :b]
        lam = th[:b]
        Xn = S @ Cc
        AXn = AS @ Cc
        P = S[:, b:] @ Cc[b:]
        AP = AS[:, b:] @ Cc[b:]
        X, AX = Xn, AXn
    return lam, X


def eig_round(op, V, dv, g, d, L, seed=0, scales=("vol",), extra=16, maxiter=400, chunk=20, atol=1e-5,
              time_limit=1200.0, no_w_init=False, log=print, native=True):
    """estimator.eig_round with the GPU LOBPCG: lambda_min of the pencil (Diag(g) - C, Diag(s)), block = [left
    singular vectors of W, random], Jacobi preconditioner 1 / (|g - diag C| + 0.01 s); the estimate is
    theta_1 - ||r_1|| after every `chunk` iterations, stopping when both the residual and the change of theta_1 are
    below atol in UB units, after maxiter iterations or time_limit seconds.  native: the LOBPCG chunks run in the
    library (lb_lobpcg) rather than as tensor operations (same iteration).  Returns ({scale: record},
    {scale: (theta, X)}) with NumPy theta and torch X."""
    t = _torch()
    n = g.shape[0]
    dev = g.device
    dT = t.as_tensor(d, dtype=t.float64, device=dev)
    diagM = g + dT ** 2 / L
    gen = t.Generator(device=dev)
    gen.manual_seed(int(seed))

    def Mop(X):
        return g[:, None] * X - op(X)

    recs, vecs = {}, {}
    for sname in scales:
        if sname == "ones":
            s = t.ones(n, dtype=t.float64, device=dev)
        elif sname == "vol":
            s = dT.clamp_min(1.0)
        elif sname == "sqrtvol":
            s = dT.clamp_min(1.0).sqrt() * math.sqrt(L / n)
        else:
            raise ValueError(f"unknown scale {sname}")
        te = time.time()
        b = V.shape[1] + extra
        sums = float(s.sum())
        if n < 5 * b:
            # a problem small against the block: the dense pencil, as SciPy's lobpcg does for n < 5 x block size
            Ds = 1.0 / s.sqrt()
            Mn = Mop(t.eye(n, dtype=t.float64, device=dev))
            th, Yd = t.linalg.eigh(0.5 * (Mn + Mn.T) * Ds[:, None] * Ds[None, :])
            X = Ds[:, None] * Yd
            th0 = float(th[0])
            lmin_est = th0
            shift = max(0.0, -lmin_est) * sums / L
            ub = dv + shift
            thn = th.cpu().numpy()
            recs[sname] = dict(theta=thn[:6].tolist(), resid=[0.0] * min(6, n), lmin_est=lmin_est, shift=shift, ub=ub,
                               sum_s=sums, eig_time=time.time() - te, eig_trace=[(0, time.time() - te, th0, 0.0)],
                               ub_ritz=ub, dv=dv, k=int(V.shape[1]), eigensolver="dense")
            log(f"[s={sname}] dense pencil (n {n} < 5 x block {b}): theta {thn[:4]} -> lmin {lmin_est:.3e}  shift "
                f"{shift:.6f}  UB {ub:.6f}")
            vecs[sname] = (thn, X)
            continue
        Uw, Sw, _ = t.linalg.svd(V, full_matrices=False)
        r_ = 0 if no_w_init else int((Sw > 1e-6 * Sw[0]).sum())
        X = t.cat([Uw[:, :r_], t.randn(n, b - r_, dtype=t.float64, device=dev, generator=gen)], 1)
        del Uw
        prec = 1.0 / (diagM.abs() + 1e-2 * s)
        it_tot, th_prev, trace = 0, math.inf, []
        g_ = g.contiguous()
        s_ = s.contiguous()
        prec_ = prec.contiguous()
        while True:
            if native and isinstance(op, DeviceOperator) and X.shape[1] <= op.MAX_WIDTH:
                _, X = op.lobpcg(X, g_, s_, prec_, chunk)
            else:
                _, X = lobpcg(Mop, s, prec, X, chunk)
            it_tot += chunk
            MX = Mop(X)
            xs = (X * (s[:, None] * X)).sum(0)
            th = (X * MX).sum(0) / xs
            o = t.argsort(th)
            th, X, MX, xs = th[o], X[:, o], MX[:, o], xs[o]
            Rres = MX - th[None, :] * (s[:, None] * X)
            rn = ((Rres * (Rres / s[:, None])).sum(0) / xs).sqrt()
            del MX, Rres
            th0, rn0 = float(th[0]), float(rn[0])
            trace.append((it_tot, time.time() - te, th0, rn0))
            log(f"  [s={sname}] lobpcg its {it_tot} theta1 {th0:.6e} r1 {rn0:.2e}  (shift-units: theta "
                f"{max(0, -th0) * sums / L:.6f} r {rn0 * sums / L:.2e})")
            if rn0 * sums / L < atol and abs(th0 - th_prev) * sums / L < atol:
                break
            if it_tot >= maxiter or time.time() - te > time_limit:
                break
            th_prev = th0
        lmin_est = th0 - rn0
        shift = max(0.0, -lmin_est) * sums / L
        ub = dv + shift
        thn, rnn = th.cpu().numpy(), rn.cpu().numpy()
        recs[sname] = dict(theta=thn[:6].tolist(), resid=rnn[:6].tolist(), lmin_est=lmin_est, shift=shift, ub=ub,
                           sum_s=sums, eig_time=time.time() - te, eig_trace=trace,
                           ub_ritz=dv + max(0.0, -th0) * sums / L, dv=dv, k=int(V.shape[1]), eigensolver="lobpcg-gpu")
        log(f"[s={sname}] theta {thn[:4]} resid {rnn[:4]} -> lmin_est {lmin_est:.3e}  shift {shift:.6f}  UB {ub:.6f}  "
            f"({time.time() - te:.0f}s)")
        vecs[sname] = (thn, X)
    return recs, vecs


def escape_vectors(V, th, Xe, ratio=0.3, maxp=4):
    """estimator.escape_vectors for torch blocks: append the bottom eigenvectors with theta_j < 0 and
    theta_j <= ratio theta_1 (at most maxp), scaled to max |entry| 0.5, and renormalise the rows."""
    t = _torch()
    sel = [j for j in range(len(th)) if th[j] < 0 and th[j] <= ratio * th[0]][:maxp]
    if not sel:
        return V, sel
    U = Xe[:, sel]
    U = 0.5 * U / U.abs().max(dim=0, keepdim=True).values
    W = t.cat([V, U], 1)
    return W / W.norm(dim=1, keepdim=True), sel
