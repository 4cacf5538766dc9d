"""Seeded synthetic instances of the shapes the benchmarks are quoted on (the real graphs, e.g. ogbn-products, are
not available here).  Every generator returns a simple undirected graph as CSR (int64 indptr/indices, unit data,
sorted columns, no isolated nodes after relabelling), volumes d = degrees, L = 2m, C0 = 0.

* sbm(n, blocks, p_in, p_out)      planted-partition SBM (Bernoulli per pair), the small CPU-runnable case
* chung_lu_communities(...)        Chung-Lu power-law expected degrees w_i ~ i^(-1/(gamma-1)) scaled to a mean degree
                                   and clipped to [1, max_degree], planted communities with log-normal(mu, sigma)
                                   sizes rescaled to n; each edge's first endpoint is drawn proportional to w, the second
                                   inside the first's community with probability 1 - mixing (proportional to w there),
                                   else globally; duplicates and self-loops removed.  Vertex ids are a random permutation
                                   (no locality in the id order).
* wedge_triples(inst, T)           T random wedges (a, b = centre, c): uniform centre of degree >= 2, two distinct
                                   neighbours, normalised (min(a, c), b, max(a, c)), deduplicated.
* tri_multipliers(T)               lam: 50 % zero, 50 % exponential with mean 0.05.
"""
from __future__ import annotations

import numpy as np


class Graph:
    def __init__(self, n, indptr, indices, labels=None):
        self.n = int(n)
        self.indptr = indptr
        self.indices = indices
        self.data = np.ones(len(indices))
        self.d = np.diff(indptr).astype(np.float64)
        self.L = float(len(indices))
        self.C0 = 0.0
        self.labels = labels

    @property
    def nnz(self):
        return len(self.indices)


def _csr_from_pairs(n, u, v, labels=None):
    """Simple undirected graph from endpoint arrays: drop self-loops, dedupe, drop isolated nodes, CSR with sorted
    columns (one stable sort: reverse edges first, so every row lists its smaller neighbours, then its larger ones)."""
    a = np.minimum(u, v).astype(np.int64); b = np.maximum(u, v).astype(np.int64)
    keep = a != b
    keys = np.unique(a[keep] * n + b[keep])
    a = keys // n; b = keys % n
    used = np.zeros(n, bool); used[a] = True; used[b] = True
    nid = (np.cumsum(used) - 1).astype(np.int64)
    n2 = int(used.sum())
    a = nid[a]; b = nid[b]                           # still sorted by (a, b)
    rows = np.concatenate([b, a]); cols = np.concatenate([a, b])
    order = np.argsort(rows, kind="stable")
    cols = cols[order]
    indptr = np.r_[0, np.cumsum(np.bincount(rows, minlength=n2))].astype(np.int64)
    lab = None if labels is None else labels[used]
    return Graph(n2, indptr, cols, lab)


def permute_graph(g, order):
    """The same graph with row k = old row order[k] (columns renumbered, not re-sorted); returns (graph, inverse)."""
    order = np.asarray(order, np.int64)
    inv = np.empty_like(order); inv[order] = np.arange(len(order))
    deg = np.diff(g.indptr)[order]
    indptr = np.r_[0, np.cumsum(deg)].astype(np.int64)
    src = np.repeat(g.indptr[order] - indptr[:-1], deg) + np.arange(indptr[-1])
    out = Graph(g.n, indptr, inv[g.indices[src]], None if g.labels is None else g.labels[order])
    return out, inv


def sbm(n=2000, blocks=8, p_in=0.08, p_out=0.002, seed=0):
    rng = np.random.default_rng(seed)
    lab = np.repeat(np.arange(blocks), n // blocks)
    lab = np.r_[lab, np.full(n - len(lab), blocks - 1)]
    iu, ju = np.triu_indices(n, 1)
    p = np.where(lab[iu] == lab[ju], p_in, p_out)
    keep = rng.random(len(iu)) < p
    return _csr_from_pairs(n, iu[keep], ju[keep], lab)


def _chung_lu_setup(rng, n, mean_degree, gamma, max_degree, n_comm, size_mu, size_sigma, min_degree):
    # expected degrees: w_i = c i^(-1/(gamma-1)), c fitted so the clipped mean is mean_degree
    base = np.arange(1, n + 1, dtype=np.float64) ** (-1.0 / (gamma - 1.0))
    c = mean_degree / base.mean()
    for _ in range(30):
        w = np.clip(c * base, min_degree, max_degree)
        c *= mean_degree / w.mean()
    w = np.clip(c * base, min_degree, max_degree)
    w = w[rng.permutation(n)]                        # random id order
    # communities: log-normal sizes rescaled to n
    s = rng.lognormal(size_mu, size_sigma, n_comm)
    s = np.maximum(1, np.floor(s / s.sum() * n)).astype(np.int64)
    while s.sum() > n:
        s[np.argmax(s)] -= s.sum() - n
    s[np.argmax(s)] += n - s.sum()
    comm = np.repeat(np.arange(n_comm), s)[rng.permutation(n)]
    # vertices sorted by community; cumulative weights in that order
    order = np.argsort(comm, kind="stable")
    cw = np.cumsum(w[order])
    cstart = np.r_[0, np.cumsum(np.bincount(comm, minlength=n_comm))]
    cw0 = np.r_[0.0, cw]
    return w, comm, order, cw, cw0, cstart


def chung_lu_communities(n, mean_degree, gamma, max_degree, n_comm, mixing, size_mu=4.0, size_sigma=1.0, seed=0,
                         min_degree=1.0):
    rng = np.random.default_rng(seed)
    w, comm, order, cw, cw0, cstart = _chung_lu_setup(rng, n, mean_degree, gamma, max_degree, n_comm, size_mu,
                                                      size_sigma, min_degree)
    m_target = int(round(n * mean_degree / 2))
    cum_all = np.cumsum(w)
    total_w = cum_all[-1]

    def draw(k):
        u = np.minimum(np.searchsorted(cum_all, rng.random(k) * total_w, side="right"), n - 1)
        inside = rng.random(k) >= mixing
        v = np.minimum(np.searchsorted(cum_all, rng.random(k) * total_w, side="right"), n - 1)
        cu = comm[u[inside]]
        lo = cw0[cstart[cu]]; hi = cw0[cstart[cu + 1]]
        pos = np.searchsorted(cw, lo + rng.random(len(cu)) * (hi - lo), side="right")
        v[inside] = order[np.clip(pos, cstart[cu], cstart[cu + 1] - 1)]
        a = np.minimum(u, v); b = np.maximum(u, v); ok = a != b
        return a[ok] * n + b[ok]

    keys = np.unique(draw(int(m_target * 1.15) + 1000))
    while len(keys) < m_target:
        keys = np.unique(np.concatenate([keys, draw(int((m_target - len(keys)) * 1.5) + 1000)]))
    if len(keys) > m_target:
        keys = np.sort(keys[rng.permutation(len(keys))[:m_target]])
    return _csr_from_pairs(n, keys // n, keys % n, comm)


def chung_lu_communities_torch(n, mean_degree, gamma, max_degree, n_comm, mixing, size_mu=4.0, size_sigma=1.0,
                               seed=0, min_degree=1.0, device="cuda"):
    """chung_lu_communities with the edge draws, deduplication and CSR build done by torch on `device` (input
    generation only; seconds instead of minutes at 62M edges).  Same distribution, torch's seeded generator."""
    import torch
    rng = np.random.default_rng(seed)
    w, comm, order, cw, cw0, cstart = _chung_lu_setup(rng, n, mean_degree, gamma, max_degree, n_comm, size_mu,
                                                      size_sigma, min_degree)
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed) + 12345)
    T_ = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
    cum_all = T_(np.cumsum(w)); total_w = float(cum_all[-1])
    cw_t = T_(cw); cw0_t = T_(cw0); cstart_t = T_(cstart.astype(np.int64)); comm_t = T_(comm.astype(np.int64))
    order_t = T_(order.astype(np.int64))
    m_target = int(round(n * mean_degree / 2))

    def rand(k):
        return torch.rand(k, generator=gen, device=dev, dtype=torch.float64)

    def draw(k):
        u = torch.searchsorted(cum_all, rand(k) * total_w, right=True).clamp_(max=n - 1)
        inside = rand(k) >= mixing
        v = torch.searchsorted(cum_all, rand(k) * total_w, right=True).clamp_(max=n - 1)
        cu = comm_t[u[inside]]
        lo = cw0_t[cstart_t[cu]]; hi = cw0_t[cstart_t[cu + 1]]
        pos = torch.searchsorted(cw_t, lo + rand(len(cu)) * (hi - lo), right=True)
        pos = torch.minimum(torch.maximum(pos, cstart_t[cu]), cstart_t[cu + 1] - 1)
        v[inside] = order_t[pos]
        a = torch.minimum(u, v); b = torch.maximum(u, v); ok = a != b
        return a[ok] * n + b[ok]

    keys = torch.unique(draw(int(m_target * 1.15) + 1000))
    while len(keys) < m_target:
        keys = torch.unique(torch.cat([keys, draw(int((m_target - len(keys)) * 1.5) + 1000)]))
    if len(keys) > m_target:
        keys = torch.sort(keys[torch.randperm(len(keys), generator=gen, device=dev)[:m_target]]).values
    a = keys // n; b = keys % n
    used = torch.zeros(n, dtype=torch.bool, device=dev); used[a] = True; used[b] = True
    nid = torch.cumsum(used.to(torch.int64), 0) - 1
    n2 = int(used.sum())
    a = nid[a]; b = nid[b]
    rows = torch.cat([b, a]); cols = torch.cat([a, b])
    perm = torch.argsort(rows, stable=True)
    cols = cols[perm]
    indptr = torch.zeros(n2 + 1, dtype=torch.int64, device=dev)
    indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n2), 0)
    used_h = used.cpu().numpy()
    out = Graph(n2, indptr.cpu().numpy(), cols.cpu().numpy(), comm[used_h])
    del keys, a, b, rows, cols, perm, indptr
    torch.cuda.empty_cache() if dev.type == "cuda" else None
    return out


def wedge_triples_torch(g, T, seed=1, device="cuda"):
    """wedge_triples with torch on `device`."""
    import torch
    dev = torch.device(device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed) + 777)
    ip = torch.from_numpy(g.indptr).to(dev); ix = torch.from_numpy(g.indices).to(dev)
    deg = ip[1:] - ip[:-1]
    cand = torch.nonzero(deg >= 2).flatten()
    out = torch.zeros((0, 3), dtype=torch.int64, device=dev)
    while len(out) < T:
        k = int((T - len(out)) * 1.1) + 100
        b = cand[torch.randint(0, len(cand), (k,), generator=gen, device=dev)]
        db = deg[b].to(torch.float64)
        p1 = (torch.rand(k, generator=gen, device=dev, dtype=torch.float64) * db).to(torch.int64)
        p2 = (torch.rand(k, generator=gen, device=dev, dtype=torch.float64) * (db - 1)).to(torch.int64)
        p2 = p2 + (p2 >= p1).to(torch.int64)
        a = ix[ip[b] + p1]; c = ix[ip[b] + p2]
        tri = torch.stack([torch.minimum(a, c), b, torch.maximum(a, c)], 1)
        out = torch.unique(torch.cat([out, tri]), dim=0)
    out = out[torch.randperm(len(out), generator=gen, device=dev)[:T]]
    return out.cpu().numpy()


def wedge_triples(g, T, seed=1):
    rng = np.random.default_rng(seed)
    deg = np.diff(g.indptr)
    cand = np.flatnonzero(deg >= 2)
    out = np.zeros((0, 3), np.int64)
    while len(out) < T:
        k = int((T - len(out)) * 1.1) + 100
        b = cand[rng.integers(0, len(cand), k)]
        db = deg[b]
        p1 = (rng.random(k) * db).astype(np.int64)
        p2 = (rng.random(k) * (db - 1)).astype(np.int64)
        p2 = p2 + (p2 >= p1)
        a = g.indices[g.indptr[b] + p1]; c = g.indices[g.indptr[b] + p2]
        tri = np.stack([np.minimum(a, c), b, np.maximum(a, c)], 1)
        out = np.unique(np.concatenate([out, tri]), axis=0)
    return out[rng.permutation(len(out))[:T]]


def tri_multipliers(T, seed=1):
    rng = np.random.default_rng(seed)
    return rng.exponential(0.05, T) * (rng.random(T) < 0.5)


def random_V(n, r, seed=0):
    """i.i.d. N(0, 1) rows normalised to unit norm (alm_vcs.py:1215-1216 default init)."""
    V = np.random.default_rng(seed).standard_normal((n, r))
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    return V


# the named shapes of the benchmark configurations
def config_graph(name, seed=0, device=None):
    """c1 (SBM n=2000), c2 (n=300k), c3 (n=2.4M); with device='cuda' the Chung-Lu shapes are drawn by torch there."""
    if device is not None and name in ("c2", "c3"):
        args = CONFIG_ARGS[name]
        return chung_lu_communities_torch(*args, seed=seed, device=device)
    if name == "c1":
        return sbm(2000, 8, 0.08, 0.002, seed)
    if name == "c2":
        return chung_lu_communities(300_000, 13.0, 2.1, 20_000, 3000, 0.3, seed=seed)
    if name == "c3":
        return chung_lu_communities(2_400_000, 52.0, 2.3, 100_000, 20_000, 0.25, seed=seed)
    raise ValueError(name)


def batch_graphs(count=512, seed=0, device=None):
    """The batched shape: `count` independent graphs, n log-uniform in [500, 50,000], mean degree uniform in [5, 40],
    rank drawn from {8, 16, 32}; even-numbered graphs are planted-partition graphs (near-uniform expected degrees,
    blocks of ~200 rows, 20 % of the edges between blocks), odd-numbered ones Chung-Lu power-law graphs (exponent
    2.3, max degree n / 10) with planted communities.  Both come from the Chung-Lu generator (torch on `device`
    when given).  Returns a list of (graph, r)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(500), np.log(50_000))))
        mean = float(rng.uniform(5, 40))
        r = int(rng.choice([8, 16, 32]))
        if k % 2 == 0:
            args = (n, mean, 50.0, max(2.0 * mean, 10.0), max(2, n // 200), 0.2)
        else:
            args = (n, mean, 2.3, max(50, n // 10), max(2, n // 120), 0.25)
        kw = dict(seed=seed * 100003 + k)
        g = chung_lu_communities_torch(*args, device=device, **kw) if device else chung_lu_communities(*args, **kw)
        out.append((g, r))
    return out


CONFIG_ARGS = {"c2": (300_000, 13.0, 2.1, 20_000, 3000, 0.3), "c3": (2_400_000, 52.0, 2.3, 100_000, 20_000, 0.25)}
CONFIG_TRIANGLES = {"c1": 20_000, "c2": 1_000_000, "c3": 5_000_000}
CONFIG_RANK = {"c1": 16, "c2": 32, "c3": 32}
