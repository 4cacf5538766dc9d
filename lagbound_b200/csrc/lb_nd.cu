// Fill-reducing ordering for the certificate side: nested dissection by multilevel graph bisection, and the symbolic
// Cholesky fill of a given ordering.  Host code only (the ordering is sequential graph work).
//
// The reference's certificate and verifier order their sparse factorizations with METIS nested dissection through
// pymetis (src/lagbound/_core/certify_lifted_vc.py:247-251 nd_order, verify_cert.py:353-356); any symmetric
// ordering is valid for them, the ordering only sets the factor's fill and the time to a certified bound.  This is an
// independent nested dissection written from the published method (George 1973; the multilevel scheme of Karypis and
// Kumar 1998):
//   * connected components are ordered one after the other;
//   * a component larger than a leaf is split by a vertex separator S into A and B, ordered A, B, S (recursively);
//   * the separator comes from an edge bisection of a coarsened graph: heavy-edge matching until the graph is small,
//     greedy region growing from several seeds at the coarsest level, boundary Fiduccia-Mattheyses refinement on
//     the way back up, then a minimum vertex cover of the cut edges (Koenig, by bipartite matching) trimmed of
//     vertices with neighbours on one side only;
//   * leaves (at most LEAF vertices), and parts up to MDMAX vertices whose separator is large (dense parts such as
//     the triangle block of a lifted certificate), are ordered by minimum degree on their elimination graph.
// Every random choice uses a fixed seed, so the ordering is a function of the input graph.
#include <stdint.h>

#include <algorithm>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "lb_internal.cuh"

namespace lb {
namespace nd {

constexpr int LEAF = 160;          // components up to this size are ordered by minimum degree
constexpr int COARSE = 96;         // coarsening stops at this many vertices
constexpr int TRIALS = 6;          // region-growing seeds at the coarsest level
constexpr double BAL = 0.55;       // largest side of a bisection, as a share of the vertex weight
constexpr int MDMAX = 4096;        // largest part ordered by minimum degree when its separator is large
constexpr double SEPMAX = 0.12;    // separators above this share of the part count as large

struct Graph {
    int n = 0;
    std::vector<int> xadj, adj, ew, vw;   // CSR, edge weights, vertex weights
    int64_t total_vw() const { return std::accumulate(vw.begin(), vw.end(), (int64_t)0); }
};

// ------------------------------------------------------------------------------------------------ coarsening
// Heavy-edge matching in a seeded random order: v is matched with its unmatched neighbour of largest edge weight
// (the lighter one on ties) when their weight together stays below maxw; cmap gives the coarse vertex.
static int match(const Graph &g, std::mt19937_64 &rng, int64_t maxw, std::vector<int> &cmap) {
    const int n = g.n;
    std::vector<int> order(n), mate(n, -1);
    std::iota(order.begin(), order.end(), 0);
    std::shuffle(order.begin(), order.end(), rng);
    for (int v : order) {
        if (mate[v] >= 0) continue;
        int best = -1, bw = -1;
        for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) {
            const int u = g.adj[p];
            if (mate[u] >= 0 || u == v) continue;
            if ((int64_t)g.vw[u] + g.vw[v] > maxw) continue;
            if (g.ew[p] > bw || (g.ew[p] == bw && g.vw[u] < g.vw[best])) {
                best = u;
                bw = g.ew[p];
            }
        }
        if (best >= 0) {
            mate[v] = best;
            mate[best] = v;
        } else {
            mate[v] = v;
        }
    }
    cmap.assign(n, -1);
    int nc = 0;
    for (int v = 0; v < n; v++) {
        if (cmap[v] >= 0) continue;
        cmap[v] = nc;
        cmap[mate[v]] = nc;
        nc++;
    }
    return nc;
}

static Graph contract(const Graph &g, const std::vector<int> &cmap, int nc) {
    Graph c;
    c.n = nc;
    c.vw.assign(nc, 0);
    std::vector<std::vector<int>> members(nc);
    for (int v = 0; v < g.n; v++) {
        c.vw[cmap[v]] += g.vw[v];
        members[cmap[v]].push_back(v);
    }
    c.xadj.assign(nc + 1, 0);
    std::vector<int> slot(nc, -1);
    std::vector<int> nbr, wt;
    for (int a = 0; a < nc; a++) {
        nbr.clear();
        wt.clear();
        for (int v : members[a])
            for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) {
                const int b = cmap[g.adj[p]];
                if (b == a) continue;
                if (slot[b] < 0) {
                    slot[b] = (int)nbr.size();
                    nbr.push_back(b);
                    wt.push_back(0);
                }
                wt[slot[b]] += g.ew[p];
            }
        for (size_t k = 0; k < nbr.size(); k++) {
            c.adj.push_back(nbr[k]);
            c.ew.push_back(wt[k]);
            slot[nbr[k]] = -1;
        }
        c.xadj[a + 1] = (int)c.adj.size();
    }
    return c;
}

// ------------------------------------------------------------------------------------------------ bisection
static int64_t cut_of(const Graph &g, const std::vector<char> &side) {
    int64_t cut = 0;
    for (int v = 0; v < g.n; v++)
        for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++)
            if (side[v] != side[g.adj[p]]) cut += g.ew[p];
    return cut / 2;
}

// Region growing from `seed`: the vertex with the largest gain (edge weight into the region minus out of it) joins
// next (a lazy max-heap of gains), until the region holds half of the weight.
static void grow(const Graph &g, int seed, std::vector<char> &side) {
    const int64_t W = g.total_vw();
    side.assign(g.n, 1);
    std::vector<int64_t> gain(g.n);
    for (int v = 0; v < g.n; v++) {
        int64_t tot = 0;
        for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) tot += g.ew[p];
        gain[v] = -tot;
    }
    std::vector<std::pair<int64_t, int>> heap;
    heap.emplace_back(gain[seed], seed);
    int64_t inw = 0;
    int next_outside = 0;
    while (true) {
        int v = -1;
        while (!heap.empty()) {
            std::pop_heap(heap.begin(), heap.end());
            const auto top = heap.back();
            heap.pop_back();
            if (side[top.second] && top.first == gain[top.second]) {
                v = top.second;
                break;
            }
        }
        if (v < 0) {   // region closed off (a disconnected graph): continue from any vertex outside
            while (next_outside < g.n && !side[next_outside]) next_outside++;
            if (next_outside >= g.n) break;
            v = next_outside;
        }
        if (2 * (inw + g.vw[v]) > W + g.vw[v]) break;
        side[v] = 0;
        inw += g.vw[v];
        for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) {
            const int u = g.adj[p];
            if (!side[u]) continue;
            gain[u] += 2 * g.ew[p];
            heap.emplace_back(gain[u], u);
            std::push_heap(heap.begin(), heap.end());
        }
    }
}

// Boundary Fiduccia-Mattheyses: single-vertex moves in order of gain with a lock per pass, keeping the larger side
// within BAL of the weight; the best prefix of the moves is kept.  A few passes while the cut improves.
static void refine(const Graph &g, std::vector<char> &side, int passes) {
    const int64_t W = g.total_vw();
    const int64_t maxside = (int64_t)(BAL * (double)W) + 1;
    std::vector<int64_t> ext(g.n), inn(g.n);
    for (int pass = 0; pass < passes; pass++) {
        int64_t sw[2] = {0, 0};
        for (int v = 0; v < g.n; v++) sw[(int)side[v]] += g.vw[v];
        for (int v = 0; v < g.n; v++) {
            ext[v] = inn[v] = 0;
            for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++)
                (side[g.adj[p]] == side[v] ? inn[v] : ext[v]) += g.ew[p];
        }
        // candidates: boundary vertices in a lazy max-heap of (gain, vertex)
        std::vector<std::pair<int64_t, int>> heap;
        for (int v = 0; v < g.n; v++)
            if (ext[v] > 0) heap.emplace_back(ext[v] - inn[v], v);
        std::make_heap(heap.begin(), heap.end());
        std::vector<char> locked(g.n, 0);
        std::vector<int> moves;
        int64_t cur = 0, best = 0;
        size_t best_len = 0;
        const size_t limit = std::max<size_t>(64, (size_t)g.n / 4);
        while (!heap.empty() && moves.size() < limit) {
            std::pop_heap(heap.begin(), heap.end());
            const auto top = heap.back();
            heap.pop_back();
            const int v = top.second;
            if (locked[v] || top.first != ext[v] - inn[v]) continue;   // stale entry
            const int from = side[v], to = 1 - from;
            if (sw[to] + g.vw[v] > maxside) continue;
            locked[v] = 1;
            side[v] = (char)to;
            sw[from] -= g.vw[v];
            sw[to] += g.vw[v];
            cur += ext[v] - inn[v];
            std::swap(ext[v], inn[v]);
            moves.push_back(v);
            for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) {
                const int u = g.adj[p];
                if (side[u] == to) {
                    inn[u] += g.ew[p];
                    ext[u] -= g.ew[p];
                } else {
                    inn[u] -= g.ew[p];
                    ext[u] += g.ew[p];
                }
                if (!locked[u] && ext[u] > 0) {
                    heap.emplace_back(ext[u] - inn[u], u);
                    std::push_heap(heap.begin(), heap.end());
                }
            }
            if (cur > best) {
                best = cur;
                best_len = moves.size();
            }
        }
        for (size_t k = moves.size(); k > best_len; k--) side[moves[k - 1]] ^= 1;
        if (best <= 0) break;
    }
}

// Edge bisection of a connected graph by the multilevel scheme: coarsen, bisect the coarsest graph from several
// seeds, project back with refinement at every level.
static std::vector<char> bisect(const Graph &g0, std::mt19937_64 &rng) {
    std::vector<Graph> levels;
    std::vector<std::vector<int>> maps;
    const Graph *cur = &g0;
    const int64_t W = g0.total_vw();
    while (cur->n > COARSE) {
        std::vector<int> cmap;
        const int nc = match(*cur, rng, std::max<int64_t>(1, (int64_t)(1.5 * (double)W / COARSE)), cmap);
        if (nc > (int)(0.9 * cur->n)) break;      // matching stalled (e.g. a star): bisect at this level
        levels.push_back(contract(*cur, cmap, nc));
        maps.push_back(std::move(cmap));
        cur = &levels.back();
    }
    std::vector<char> side, best;
    int64_t bcut = INT64_MAX;
    std::uniform_int_distribution<int> pick(0, cur->n - 1);
    for (int t = 0; t < TRIALS; t++) {
        grow(*cur, pick(rng), side);
        refine(*cur, side, 4);
        const int64_t c = cut_of(*cur, side);
        if (c < bcut) {
            bcut = c;
            best = side;
        }
    }
    for (int l = (int)levels.size() - 1; l >= 0; l--) {
        const Graph &fine = l > 0 ? levels[l - 1] : g0;
        std::vector<char> s(fine.n);
        for (int v = 0; v < fine.n; v++) s[v] = best[maps[l][v]];
        refine(fine, s, 2);
        best.swap(s);
    }
    return best;
}

// Vertex separator from the edge cut: a minimum vertex cover of the bipartite graph of cut edges (Koenig's theorem:
// a maximum matching by augmenting paths, then the vertices of A not reached by alternating paths from unmatched A
// vertices plus the vertices of B reached), then trimmed: a separator vertex with no neighbour on one side joins that
// side (side[] updated).  sep[v] = 1 for separator vertices.
static void separator(const Graph &g, std::vector<char> &side, std::vector<char> &sep) {
    const int n = g.n;
    sep.assign(n, 0);
    std::vector<int> bnd;                       // boundary vertices (endpoints of cut edges)
    std::vector<int> bid(n, -1);
    for (int v = 0; v < n; v++)
        for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++)
            if (side[g.adj[p]] != side[v]) {
                bid[v] = (int)bnd.size();
                bnd.push_back(v);
                break;
            }
    if (bnd.empty()) return;
    // maximum matching between side-0 and side-1 boundary vertices (augmenting paths by iterative DFS)
    std::vector<int> mate(n, -1), seen(n, -1), parent(n, -1), stack;
    std::vector<int> it(n, 0);
    int stamp = 0;
    for (int root : bnd) {
        if (side[root] != 0 || mate[root] >= 0) continue;
        stamp++;
        stack.assign(1, root);
        seen[root] = stamp;
        it[root] = g.xadj[root];
        bool found = false;
        while (!stack.empty() && !found) {
            const int a = stack.back();
            if (it[a] >= g.xadj[a + 1]) {
                stack.pop_back();
                continue;
            }
            const int b = g.adj[it[a]++];
            if (side[b] == 0 || seen[b] == stamp) continue;
            seen[b] = stamp;
            parent[b] = a;
            if (mate[b] < 0) {                  // augment along a -> b and back up the stack
                int y = b;
                while (true) {
                    const int x = parent[y], nx = mate[x];
                    mate[x] = y;
                    mate[y] = x;
                    if (x == root) break;
                    y = nx;
                }
                found = true;
            } else {
                const int a2 = mate[b];
                if (seen[a2] != stamp) {
                    seen[a2] = stamp;
                    it[a2] = g.xadj[a2];
                    stack.push_back(a2);
                }
            }
        }
    }
    // alternating reachability from unmatched side-0 boundary vertices
    std::vector<char> reach(n, 0);
    std::vector<int> queue;
    for (int v : bnd)
        if (side[v] == 0 && mate[v] < 0) {
            reach[v] = 1;
            queue.push_back(v);
        }
    for (size_t h = 0; h < queue.size(); h++) {
        const int a = queue[h];
        for (int p = g.xadj[a]; p < g.xadj[a + 1]; p++) {
            const int b = g.adj[p];
            if (side[b] == 0 || reach[b]) continue;
            reach[b] = 1;
            const int a2 = mate[b];
            if (a2 >= 0 && !reach[a2]) {
                reach[a2] = 1;
                queue.push_back(a2);
            }
        }
    }
    for (int v : bnd) sep[v] = side[v] == 0 ? !reach[v] : reach[v];
    // trim: a separator vertex without neighbours on one side moves to that side (repeat until stable)
    bool changed = true;
    std::vector<char> cur(side);
    for (int v = 0; v < n; v++)
        if (sep[v]) cur[v] = 2;
    while (changed) {
        changed = false;
        for (int v : bnd) {
            if (cur[v] != 2) continue;
            bool n0 = false, n1 = false;
            for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) {
                const int c = cur[g.adj[p]];
                n0 |= c == 0;
                n1 |= c == 1;
            }
            if (!n1) {
                cur[v] = side[v] = 0;
                sep[v] = 0;
                changed = true;
            } else if (!n0) {
                cur[v] = side[v] = 1;
                sep[v] = 0;
                changed = true;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------ leaves
// Minimum-degree order of a small graph on its elimination graph (bit rows): the vertex of least current degree
// (lowest index on ties) is eliminated and its neighbours become a clique.
static void min_degree(const Graph &g, std::vector<int> &order) {
    const int n = g.n, w = (n + 63) / 64;
    std::vector<uint64_t> bits((size_t)n * w, 0);
    for (int v = 0; v < n; v++)
        for (int p = g.xadj[v]; p < g.xadj[v + 1]; p++) {
            const int u = g.adj[p];
            if (u != v) bits[(size_t)v * w + u / 64] |= 1ull << (u % 64);
        }
    std::vector<char> done(n, 0);
    order.clear();
    for (int step = 0; step < n; step++) {
        int bv = -1, bd = INT32_MAX;
        for (int v = 0; v < n; v++) {
            if (done[v]) continue;
            int dg = 0;
            for (int k = 0; k < w; k++) dg += __builtin_popcountll(bits[(size_t)v * w + k]);
            if (dg < bd) {
                bd = dg;
                bv = v;
            }
        }
        done[bv] = 1;
        order.push_back(bv);
        const uint64_t *rv = &bits[(size_t)bv * w];
        for (int u = 0; u < n; u++) {
            if (!((rv[u / 64] >> (u % 64)) & 1)) continue;
            uint64_t *ru = &bits[(size_t)u * w];
            for (int k = 0; k < w; k++) ru[k] |= rv[k];
            ru[u / 64] &= ~(1ull << (u % 64));
            ru[bv / 64] &= ~(1ull << (bv % 64));
        }
        std::fill(bits.begin() + (size_t)bv * w, bits.begin() + (size_t)(bv + 1) * w, 0ull);
    }
}

// ------------------------------------------------------------------------------------------------ driver
// The subgraph induced by `verts` (global ids) of the input graph (unit vertex and edge weights).
static Graph induced(const std::vector<int64_t> &xadj, const std::vector<int> &adj, const std::vector<int> &verts,
                     std::vector<int> &local) {
    Graph g;
    g.n = (int)verts.size();
    for (int k = 0; k < g.n; k++) local[verts[k]] = k;
    g.xadj.assign(g.n + 1, 0);
    for (int k = 0; k < g.n; k++) {
        const int v = verts[k];
        for (int64_t p = xadj[v]; p < xadj[v + 1]; p++) {
            const int u = local[adj[p]];
            if (u >= 0) {
                g.adj.push_back(u);
                g.ew.push_back(1);
            }
        }
        g.xadj[k + 1] = (int)g.adj.size();
    }
    g.vw.assign(g.n, 1);
    for (int v : verts) local[v] = -1;
    return g;
}

struct Task {
    std::vector<int> verts;
    int64_t lo, hi;   // positions [lo, hi) of the ordering
};

void order(int64_t n, const int64_t *indptr, const int64_t *indices, int64_t *perm) {
    // symmetric pattern without self loops or duplicates
    std::vector<std::vector<int>> nb((size_t)n);
    for (int64_t v = 0; v < n; v++)
        for (int64_t p = indptr[v]; p < indptr[v + 1]; p++) {
            const int64_t u = indices[p];
            LB_CHECK(u >= 0 && u < n, LB_ERR_INVALID, "nested dissection: column index outside [0, n)");
            if (u == v) continue;
            nb[v].push_back((int)u);
            nb[u].push_back((int)v);
        }
    std::vector<int64_t> xadj((size_t)n + 1, 0);
    std::vector<int> adj;
    for (int64_t v = 0; v < n; v++) {
        auto &a = nb[v];
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
        adj.insert(adj.end(), a.begin(), a.end());
        xadj[v + 1] = (int64_t)adj.size();
        std::vector<int>().swap(a);
    }
    std::vector<int> local((size_t)n, -1);
    std::mt19937_64 rng(0x5eed1e55ull);
    std::vector<Task> stack;
    {
        Task t;
        t.verts.resize((size_t)n);
        std::iota(t.verts.begin(), t.verts.end(), 0);
        t.lo = 0;
        t.hi = n;
        stack.push_back(std::move(t));
    }
    std::vector<int> comp, queue, ord;
    while (!stack.empty()) {
        Task t = std::move(stack.back());
        stack.pop_back();
        const int m = (int)t.verts.size();
        if (m == 0) continue;
        Graph g = induced(xadj, adj, t.verts, local);
        // connected components, in order of their smallest local vertex
        comp.assign(m, -1);
        int nc = 0;
        for (int s = 0; s < m; s++) {
            if (comp[s] >= 0) continue;
            queue.assign(1, s);
            comp[s] = nc;
            for (size_t h = 0; h < queue.size(); h++)
                for (int p = g.xadj[queue[h]]; p < g.xadj[queue[h] + 1]; p++)
                    if (comp[g.adj[p]] < 0) {
                        comp[g.adj[p]] = nc;
                        queue.push_back(g.adj[p]);
                    }
            nc++;
        }
        if (nc > 1) {
            std::vector<std::vector<int>> parts(nc);
            for (int k = 0; k < m; k++) parts[comp[k]].push_back(t.verts[k]);
            int64_t pos = t.lo;
            for (auto &pv : parts) {
                Task c;
                c.lo = pos;
                c.hi = pos + (int64_t)pv.size();
                pos = c.hi;
                c.verts = std::move(pv);
                stack.push_back(std::move(c));
            }
            continue;
        }
        if (m <= LEAF) {
            min_degree(g, ord);
            for (int k = 0; k < m; k++) perm[t.lo + k] = t.verts[ord[k]];
            continue;
        }
        std::vector<char> side, sep;
        side = bisect(g, rng);
        separator(g, side, sep);
        std::vector<int> A, B, S;
        for (int k = 0; k < m; k++) (sep[k] ? S : side[k] ? B : A).push_back(t.verts[k]);
        // no useful split (e.g. a clique), or a separator so large that dissection gains little over minimum degree
        // (dense parts such as the triangle block of a lifted certificate): minimum degree on the whole part
        if (A.empty() || B.empty() || (m <= MDMAX && (double)S.size() > SEPMAX * m)) {
            if (m <= MDMAX) {
                min_degree(g, ord);
                for (int k = 0; k < m; k++) perm[t.lo + k] = t.verts[ord[k]];
            } else {
                for (int k = 0; k < m; k++) perm[t.lo + k] = t.verts[k];
            }
            continue;
        }
        const int64_t sa = t.lo, sb = t.lo + (int64_t)A.size(), ss = t.hi - (int64_t)S.size();
        for (size_t k = 0; k < S.size(); k++) perm[ss + (int64_t)k] = S[k];
        Task ta, tb;
        ta.lo = sa;
        ta.hi = sb;
        ta.verts = std::move(A);
        tb.lo = sb;
        tb.hi = ss;
        tb.verts = std::move(B);
        stack.push_back(std::move(tb));
        stack.push_back(std::move(ta));
    }
}

// Nonzeros of the Cholesky factor L (diagonal included) of the pattern under the ordering perm (perm[k] = the
// vertex eliminated k-th): elimination tree by path compression, then every row's subtree marked once (Liu 1986);
// stops and returns -1 once the count passes cap.
int64_t fill(int64_t n, const int64_t *indptr, const int64_t *indices, const int64_t *perm, int64_t cap) {
    std::vector<int64_t> pos((size_t)n);
    for (int64_t k = 0; k < n; k++) pos[perm[k]] = k;
    // strictly-lower pattern in the new numbering: row k lists the columns i < k
    std::vector<std::vector<int64_t>> low((size_t)n);
    for (int64_t v = 0; v < n; v++)
        for (int64_t p = indptr[v]; p < indptr[v + 1]; p++) {
            const int64_t a = pos[v], b = pos[indices[p]];
            if (a > b) low[a].push_back(b);
            else if (b > a) low[b].push_back(a);
        }
    std::vector<int64_t> parent((size_t)n, -1), anc((size_t)n, -1);
    for (int64_t k = 0; k < n; k++)
        for (int64_t i : low[k]) {
            while (i != -1 && i < k) {
                const int64_t nx = anc[i];
                anc[i] = k;
                if (nx == -1) parent[i] = k;
                i = nx;
            }
        }
    std::vector<int64_t> mark((size_t)n, -1);
    int64_t nnz = n;
    for (int64_t k = 0; k < n; k++) {
        mark[k] = k;
        for (int64_t i : low[k]) {
            while (i != -1 && mark[i] != k) {
                mark[i] = k;
                nnz++;
                i = parent[i];
            }
        }
        if (cap > 0 && nnz > cap) return -1;
    }
    return nnz;
}

}  // namespace nd
}  // namespace lb

extern "C" int lb_nd_order(int64_t n, const int64_t *indptr, const int64_t *indices, int64_t *perm, int64_t *iperm) {
    try {
        LB_CHECK(n >= 0 && n < ((int64_t)1 << 31), LB_ERR_INVALID, "nested dissection: n must be in [0, 2^31)");
        LB_CHECK(n == 0 || (indptr && indices && perm), LB_ERR_INVALID, "nested dissection: null argument");
        if (n) lb::nd::order(n, indptr, indices, perm);
        if (iperm)
            for (int64_t k = 0; k < n; k++) iperm[perm[k]] = k;
        return LB_OK;
    } catch (const lb::Err &e) {
        return e.code;
    } catch (const std::bad_alloc &) {
        lb::set_error("nested dissection: out of host memory");
        return LB_ERR_NOMEM;
    } catch (...) {
        lb::set_error("nested dissection: unexpected exception");
        return LB_ERR_INVALID;
    }
}

extern "C" int lb_chol_fill(int64_t n, const int64_t *indptr, const int64_t *indices, const int64_t *perm,
                            int64_t cap, int64_t *nnz_L) {
    try {
        LB_CHECK(n >= 0 && nnz_L && (n == 0 || (indptr && indices && perm)), LB_ERR_INVALID,
                 "cholesky fill: null argument");
        std::vector<char> seen((size_t)n, 0);
        for (int64_t k = 0; k < n; k++) {
            LB_CHECK(perm[k] >= 0 && perm[k] < n && !seen[perm[k]], LB_ERR_INVALID,
                     "cholesky fill: perm is not a permutation of 0..n-1");
            seen[perm[k]] = 1;
        }
        for (int64_t p = 0; n && p < indptr[n]; p++)
            LB_CHECK(indices[p] >= 0 && indices[p] < n, LB_ERR_INVALID, "cholesky fill: column index outside [0, n)");
        *nnz_L = lb::nd::fill(n, indptr, indices, perm, cap);
        return LB_OK;
    } catch (const lb::Err &e) {
        return e.code;
    } catch (...) {
        lb::set_error("cholesky fill: unexpected exception");
        return LB_ERR_INVALID;
    }
}
