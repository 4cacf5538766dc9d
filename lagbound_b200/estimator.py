"""Candidate-bound assembly at fixed multipliers (est_dual_vcs.py): C(y) X on the GPU for host FP64 blocks X, the
dual value dv of a factor W, the Riemannian polish of W and the pencil eigenvalue estimate of the bound.

    d(y) = C0 + sum(lam) + max_{X psd, diag X = 1} <C(y), X>,   C(y) = B + S_pair(sig) + S_vcs(sig) + T(lam)
    dv = (C0 + sum lam + sum_i g_i) / L,   g_i = (C(y) W)_i . w_i   (a lower bound on d(y)/L: W W^T is feasible)
    UB = dv + max(0, -mu_s) sum(s) / L,    mu_s = lambda_min of the pencil (Diag(g) - C(y), Diag(s))

(est_dual_vcs.py:1-21, 227-246, 310-364).  The products C(y) X are the library's fixed-multiplier evaluation
(LB_EVAL_FIXED); the rest is host FP64 vector work and SciPy's LOBPCG, as in the reference.
"""
from __future__ import annotations

import math
import time
import warnings

import numpy as np

from .problem import Problem


class FixedOperator:
    """X -> C(y) X at fixed multipliers for host FP64 blocks (one device problem per power-of-two block width)."""

    MAX_WIDTH = 64

    def __init__(self, ctx, n, indptr, indices, weights, d, L, C0, pair_levels=(), vcs_levels=(), TI=None, lam=None,
                 order=None):
        """pair_levels: [(lab, P, sig P x P)], vcs_levels: [(lab, P, ptr, col, sig)], TI/lam: triangle pool."""
        self.ctx = ctx
        self.n = int(n)
        self.graph = (indptr, indices, weights, d, float(L), float(C0))
        self.pair_levels = list(pair_levels)
        self.vcs_levels = list(vcs_levels)
        self.TI = np.zeros((0, 3), np.int64) if TI is None else np.asarray(TI, np.int64).reshape(-1, 3)
        self.lam = np.zeros(0) if lam is None else np.asarray(lam, np.float64)
        self.order = order
        self._probs = {}
        self.calls = 0
        self.columns = 0

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
        return p

    def __call__(self, X):
        X = np.asarray(X, np.float64)
        one = X.ndim == 1
        X = X.reshape(self.n, -1)
        out = np.empty_like(X)
        for c0 in range(0, X.shape[1], self.MAX_WIDTH):
            blk = X[:, c0:c0 + self.MAX_WIDTH]
            w = blk.shape[1]
            width = 2
            while width < w:
                width *= 2
            p = self._problem(width)
            if w < width:
                blk = np.concatenate([blk, np.zeros((self.n, width - w))], 1)
            p.set_V(np.ascontiguousarray(blk))
            p.eval(grad=True, fixed=True)
            out[:, c0:c0 + w] = p.G()[:, :w]
        self.calls += 1
        self.columns += X.shape[1]
        return out[:, 0] if one else out

    def close(self):
        for p in self._probs.values():
            p.close()
        self._probs = {}


def rowdot(X, Y):
    return np.einsum("ij,ij->i", X, Y)


def value(op, W, const, L):
    """(dv, g, C W): dv = (const + sum g) / L with g_i = (C W)_i . w_i (est_dual_vcs.py:245-246)."""
    CW = op(W)
    g = rowdot(CW, W)
    return (const + g.sum()) / L, g, CW


def polish_rgd(op, V, const, L, iters=400, time_limit=600.0, ptol=2e-5, log=print, hist=None):
    """Maximise <C, W W^T> over unit rows (est_dual_vcs.py:276-308): preconditioned Riemannian ascent
    W+ = rownormalize(W + alpha D^{-1} R), R = rows of CW minus their radial part, D = |CW rows|, with
    Barzilai-Borwein step sizes in the D metric (alternating long and short forms, clipped to [0.05, 50]) and a
    Zhang-Hager nonmonotone Armijo test (eta 0.85, up to 12 halvings).  Stops after `iters` steps, `time_limit`
    seconds, or when 10 steps gain less than 2 ptol."""
    hist = [] if hist is None else hist
    tp = time.time()
    f, g, CW = value(op, V, const, L)
    Cref, Q, alpha = f, 1.0, 2.0
    nr = np.maximum(np.linalg.norm(CW, axis=1), 1e-12)
    Rr = CW - g[:, None] * V
    R = Rr / nr[:, None]
    hist.append(("rgd", 0, time.time() - tp, f))
    log(f"rgd start dv {f:.6f}")
    it, last_chk = 0, f
    bt = 0
    while it < iters and time.time() - tp < time_limit:
        it += 1
        gr = float(np.einsum("ij,ij->", Rr, R)) / L
        for bt in range(12):
            Vn = V + alpha * R
            Vn /= np.linalg.norm(Vn, axis=1, keepdims=True)
            fn, gn, CWn = value(op, Vn, const, L)
            if fn >= Cref + 1e-4 * alpha * gr:
                break
            alpha *= 0.5
        S = Vn - V
        nrn = np.maximum(np.linalg.norm(CWn, axis=1), 1e-12)
        Rrn = CWn - gn[:, None] * Vn
        Rn = Rrn / nrn[:, None]
        Yd = Rn - R
        sy = float(np.einsum("ij,ij->", S, Yd * nrn[:, None]))
        ss = float(np.einsum("ij,ij->", S, S * nrn[:, None]))
        yy = float(np.einsum("ij,ij->", Yd, Yd * nrn[:, None]))
        if sy < 0:
            alpha = (ss / (-sy)) if it % 2 else (-sy / yy)
        else:
            alpha = min(2 * alpha, 50.0)
        alpha = float(np.clip(alpha, 0.05, 50.0))
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


def pencil_scale(name, d, L, n):
    """Pencil weights s (est_dual_vcs.py:315): vol = max(d, 1), ones, sqrtvol = sqrt(max(d, 1)) sqrt(L/n)."""
    if name == "ones":
        return np.ones(n)
    if name == "vol":
        return np.maximum(d, 1.0)
    if name == "sqrtvol":
        return np.sqrt(np.maximum(d, 1.0)) * math.sqrt(L / n)
    raise ValueError(f"unknown scale {name}")


def eig_round(op, V, dv, g, d, L, rng, scales=("vol",), extra=16, maxiter=400, tol=1e-9, chunk=20, atol=1e-5,
              time_limit=1200.0, no_w_init=False, log=print):
    """lambda_min of the pencil (Diag(g) - C, Diag(s)) by preconditioned block LOBPCG (est_dual_vcs.py:310-364):
    block = [left singular vectors of W, random], Jacobi preconditioner 1 / (|g - diag C| + 0.01 s); every `chunk`
    iterations the Ritz pairs are checked; the estimate is theta_1 - ||r_1|| (residual-hedged).  Returns
    ({scale: record}, {scale: (theta, X)})."""
    from scipy.sparse.linalg import LinearOperator, lobpcg
    n = len(g)
    diagC = -d ** 2 / L
    diagM = g - diagC

    def Mop(X):
        X = np.asarray(X, np.float64).reshape(n, -1)
        return g[:, None] * X - op(X)

    recs, vecs = {}, {}
    for sname in scales:
        s = pencil_scale(sname, d, L, n)
        te = time.time()
        b = V.shape[1] + extra
        Uw, Sw, _ = np.linalg.svd(V, full_matrices=False)
        r_ = 0 if no_w_init else int((Sw > 1e-6 * Sw[0]).sum())
        X0 = np.concatenate([Uw[:, :r_], rng.standard_normal((n, b - r_))], 1)
        del Uw
        prec = 1.0 / (np.abs(diagM) + 1e-2 * s)
        Aop = LinearOperator((n, n), matvec=lambda x: Mop(x)[:, 0], matmat=Mop, dtype=float)
        Bop = LinearOperator((n, n), matvec=lambda x: s * x.ravel(), matmat=lambda X: s[:, None] * X, dtype=float)
        Pop = LinearOperator((n, n), matvec=lambda x: prec * x.ravel(), matmat=lambda X: prec[:, None] * X,
                             dtype=float)
        sums = float(s.sum())
        Xe, it_tot, th_prev, trace = X0, 0, np.inf, []
        while True:
            with warnings.catch_warnings():
                warnings.simplefilter("ignore")
                ev, Xe = lobpcg(Aop, Xe, B=Bop, M=Pop, largest=False, maxiter=chunk, tol=tol)
            it_tot += chunk
            o = np.argsort(ev)
            Xe = Xe[:, o]
            MX = Mop(Xe)
            xs = np.einsum("ij,ij->j", Xe, s[:, None] * Xe)
            th = np.einsum("ij,ij->j", Xe, MX) / xs
            Rres = MX - th[None, :] * (s[:, None] * Xe)
            rn = np.sqrt(np.einsum("ij,ij->j", Rres, Rres / s[:, None]) / xs)
            del MX, Rres
            trace.append((it_tot, time.time() - te, float(th[0]), float(rn[0])))
            log(f"  [s={sname}] lobpcg its {it_tot} theta1 {th[0]:.6e} r1 {rn[0]:.2e}  (shift-units: theta "
                f"{max(0, -th[0]) * sums / L:.6f} r {rn[0] * sums / L:.2e})")
            if rn[0] * sums / L < atol and abs(th[0] - th_prev) * sums / L < atol:
                break
            if it_tot >= maxiter or time.time() - te > time_limit:
                break
            th_prev = th[0]
        lmin_est = float(th[0] - rn[0])
        shift = max(0.0, -lmin_est) * sums / L
        ub = dv + shift
        recs[sname] = dict(theta=th[:6].tolist(), resid=rn[:6].tolist(), lmin_est=lmin_est, shift=shift, ub=ub,
                           sum_s=sums, eig_time=time.time() - te, eig_trace=trace,
                           ub_ritz=dv + max(0.0, -float(th[0])) * sums / L, dv=dv, k=int(V.shape[1]))
        log(f"[s={sname}] theta {th[:4]} resid {rn[:4]} -> lmin_est {lmin_est:.3e}  shift {shift:.6f}  UB {ub:.6f}  "
            f"({time.time() - te:.0f}s)")
        vecs[sname] = (th, Xe)
    return recs, vecs


def escape_vectors(V, th, Xe, ratio=0.3, maxp=4):
    """Rank escape (est_dual_vcs.py:378-384): append the bottom pencil eigenvectors with theta_j < 0 and
    theta_j <= ratio theta_1 (at most maxp), scaled to max |entry| 0.5, and renormalise the rows.  Returns the new
    W and the chosen indices (empty: nothing to append)."""
    sel = [j for j in range(len(th)) if th[j] < 0 and th[j] <= ratio * th[0]][:maxp]
    if not sel:
        return V, sel
    U = Xe[:, sel]
    U = 0.5 * U / np.abs(U).max(axis=0, keepdims=True)
    W = np.concatenate([V, U], 1)
    W /= np.linalg.norm(W, axis=1, keepdims=True)
    return W, sel
