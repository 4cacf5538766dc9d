// Exact (optimum-preserving) graph reduction and exact partition modularity counts on the GPU.
//
// Reduction (src/lagbound/_core/reduce_exact.py:12-46): union every leaf edge (an endpoint of degree 1) and every true
// twin pair (adjacent u, v with N[u] = N[v], d^2 < 2m, d > 1); groups are the components of those unions, numbered by
// the rank of their smallest vertex (the reference's union-find keeps the smaller root, reduce_exact.py:24-25);
// reduced edges are the group pairs with their edge counts, volumes are degree sums, C0 counts the edges inside
// groups.  All integer work: the result is identical to the reference's.  The reference's random closed-neighbourhood
// hash (reduce_exact.py:31-33) only filters twin candidates before its exact set comparison; true twins always pass
// it, so comparing every candidate exactly gives the same unions and the same count.
//
// Components of the union graph are stars (a centre and its leaves), isolated edges and true-twin classes (cliques):
// a vertex with a leaf neighbour has no true twin, since the twin would be adjacent to the leaf too.  Their diameter
// is at most 2, so atomic-min label propagation with pointer jumping ends within a few rounds; the round count is
// bounded anyway and an overrun is an error, not a hang.
//
// Label restriction (reduce_exact.py:51-62): a group takes the label of its first (smallest) member; the counts of
// the exact identity Q(original, rules enforced) == Q(reduced) are returned for the caller to check.
//
// Modularity (src/lagbound/modularity.py:21-33): inside-edge count and sum of squared cluster volumes, from which
// Q = inside/m - sum_c vol_c^2 / (4 m^2) is formed exactly on the host.
//
// Simple graph (src/lagbound/graph.py:71-100 _from_pairs): node names (sorted distinct ids, or given), self-loops
// dropped, duplicate and reversed edges merged into sorted keys a * n_names + b (a < b), isolated nodes set aside and
// the rest renumbered in name order.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "lb_internal.cuh"

namespace lb {
namespace {

constexpr unsigned FULLR = 0xffffffffu;
constexpr int MAX_UNION_ROUNDS = 64;
typedef unsigned long long u64;

inline unsigned nblk(int64_t n, int per = 256) { return (unsigned)std::max<int64_t>(1, (n + per - 1) / per); }

// endpoints and degrees of keyed edges (u * n + v), and the (row * n + col) keys of both directions
__global__ void k_split(int64_t m, int64_t n, const int64_t *__restrict__ keys, int64_t *__restrict__ eu,
                        int64_t *__restrict__ ev, u64 *__restrict__ deg, int64_t *__restrict__ rc) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int64_t u = keys[e] / n, v = keys[e] % n;
    eu[e] = u;
    ev[e] = v;
    atomicAdd(deg + u, 1ull);
    atomicAdd(deg + v, 1ull);
    rc[e] = u * n + v;
    rc[m + e] = v * n + u;
}

// endpoint-count degrees of an edge list
__global__ void k_endpoint_deg(int64_t m, const int64_t *__restrict__ eu, const int64_t *__restrict__ ev,
                               u64 *__restrict__ deg) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    atomicAdd(deg + eu[e], 1ull);
    atomicAdd(deg + ev[e], 1ull);
}

// column of each sorted adjacency entry; a repeated (row, col) pair marks a duplicate edge
__global__ void k_cols(int64_t nnz, int64_t n, const int64_t *__restrict__ rc, int *__restrict__ cols,
                       int *__restrict__ dup) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    cols[e] = (int)(rc[e] % n);
    if (e > 0 && rc[e] == rc[e - 1]) *dup = 1;
}

__global__ void k_deg_to_i64(int64_t n, const u64 *__restrict__ deg, int64_t *__restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (int64_t)deg[i];
    else if (i == n) out[i] = 0;
}

// Leaf and twin decision, one warp per edge: flag 1 = leaf union, 2 = twin union, 0 = none.
__global__ void __launch_bounds__(256) k_unions(int64_t m, const int64_t *__restrict__ eu,
                                                const int64_t *__restrict__ ev, const u64 *__restrict__ deg,
                                                const int64_t *__restrict__ indptr, const int *__restrict__ cols,
                                                double two_m, unsigned char *__restrict__ flag,
                                                u64 *__restrict__ nunion) {
    const int lane = threadIdx.x & 31;
    const int64_t e = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (e >= m) return;
    const int64_t u = eu[e], v = ev[e];
    const int64_t du = (int64_t)deg[u], dv = (int64_t)deg[v];
    if (du == 1 || dv == 1) {
        if (lane == 0) {
            flag[e] = 1;
            atomicAdd(nunion, 1ull);
        }
        return;
    }
    if (!(du == dv && (double)du * (double)du < two_m && du > 1)) {
        if (lane == 0) flag[e] = 0;
        return;
    }
    // N[u] == N[v] for adjacent u, v  <=>  N(u) \ {v} == N(v) \ {u}; both sorted, du - 1 entries each
    const int *a = cols + indptr[u], *b = cols + indptr[v];
    int64_t lo = 0, hi = du;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    const int64_t pa = lo;   // position of v in N(u)
    lo = 0;
    hi = dv;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (b[mid] < u) lo = mid + 1; else hi = mid;
    }
    const int64_t pb = lo;   // position of u in N(v)
    bool same = true;
    for (int64_t t = lane; t < du - 1 && same; t += 32) same = a[t < pa ? t : t + 1] == b[t < pb ? t : t + 1];
    same = __all_sync(FULLR, same);
    if (lane == 0) {
        flag[e] = same ? 2 : 0;
        if (same) atomicAdd(nunion + 1, 1ull);
    }
}

__global__ void k_iota(int64_t n, int *__restrict__ label) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) label[i] = (int)i;
}

// Hooking: the endpoint with the larger label and that label's vertex take the smaller label.  Labels only decrease
// and always name a vertex of the same component, so label[x] <= x; at a fixed point of this and the jump below
// every label is a root (label[r] == r), constant on each component, hence the component's minimum.
__global__ void k_hook(int64_t m, const int64_t *__restrict__ eu, const int64_t *__restrict__ ev,
                       const unsigned char *__restrict__ flag, int *__restrict__ label, int *__restrict__ changed) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m || flag[e] == 0) return;
    const int u = (int)eu[e], v = (int)ev[e];
    const int lu = label[u], lv = label[v];
    if (lu == lv) return;
    const int mn = min(lu, lv);
    atomicMin(label + (lu < lv ? v : u), mn);
    atomicMin(label + max(lu, lv), mn);
    *changed = 1;
}

__global__ void k_jump(int64_t n, int *__restrict__ label, int *__restrict__ changed) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int l = label[x], ll = label[l];
    if (ll < l) {
        label[x] = ll;
        *changed = 1;
    }
}

__global__ void k_is_root(int64_t n, const int *__restrict__ label, int *__restrict__ isroot) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) isroot[x] = label[x] == (int)x ? 1 : 0;
}

__global__ void k_group(int64_t n, const int *__restrict__ label, const int *__restrict__ rank,
                        const u64 *__restrict__ deg, int64_t *__restrict__ grp, u64 *__restrict__ vol) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const int g = rank[label[x]];
    grp[x] = g;
    atomicAdd(vol + g, deg[x]);
}

// reduced edge keys min(gu, gv) * N + max(gu, gv); edges inside a group sort last under the INT64_MAX key
__global__ void k_red_keys(int64_t m, int64_t N, const int64_t *__restrict__ eu, const int64_t *__restrict__ ev,
                           const int64_t *__restrict__ grp, int64_t *__restrict__ rkeys, u64 *__restrict__ inside) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    const int64_t gu = grp[eu[e]], gv = grp[ev[e]];
    if (gu == gv) {
        atomicAdd(inside, 1ull);
        rkeys[e] = INT64_MAX;
    } else {
        rkeys[e] = min(gu, gv) * N + max(gu, gv);
    }
}

__global__ void k_red_decode(int64_t M, int64_t N, const int64_t *__restrict__ rk, const int *__restrict__ cnt,
                             int64_t *__restrict__ ru, int64_t *__restrict__ rv, u64 *__restrict__ rw) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= M) return;
    ru[e] = rk[e] / N;
    rv[e] = rk[e] % N;
    rw[e] = (u64)cnt[e];
}

// group label = label of the group's smallest member (its root)
__global__ void k_restrict(int64_t n, const int *__restrict__ label, const int *__restrict__ rank,
                           const int64_t *__restrict__ lab, int64_t *__restrict__ lr) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n && label[x] == (int)x) lr[rank[x]] = lab[x];
}

__global__ void k_expand(int64_t n, const int64_t *__restrict__ grp, const int64_t *__restrict__ lr,
                         int64_t *__restrict__ lab2) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) lab2[x] = lr[grp[x]];
}

// sum of w_e over edges whose endpoints share a label (w = 1 when null); warp-aggregated atomics
__global__ void k_inside(int64_t m, const int64_t *__restrict__ eu, const int64_t *__restrict__ ev,
                         const int64_t *__restrict__ lab, const u64 *__restrict__ w, u64 *__restrict__ out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    u64 c = 0;
    if (e < m && lab[eu[e]] == lab[ev[e]]) c = w ? w[e] : 1ull;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(FULLR, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

__global__ void k_label_vol(int64_t nv, const int64_t *__restrict__ lab, const u64 *__restrict__ wt,
                            u64 *__restrict__ volc) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < nv && wt[x]) atomicAdd(volc + lab[x], wt[x]);
}

__global__ void k_sumsq(int64_t P, const u64 *__restrict__ volc, u64 *__restrict__ out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    u64 s = c < P ? volc[c] * volc[c] : 0ull;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(FULLR, s, o);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

// ---------------------------------------------------------------------------------------------- simple graph
// position of each raw id among the sorted distinct ids (np.unique(..., return_inverse=True))
__global__ void k_lower_bound(int64_t cnt, const int64_t *__restrict__ vals, const int64_t *__restrict__ names,
                              int64_t nn, int64_t *__restrict__ inv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const int64_t x = vals[i];
    int64_t lo = 0, hi = nn;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (names[mid] < x) lo = mid + 1; else hi = mid;
    }
    inv[i] = lo;
}

// edge keys a * nn + b with a = min, b = max; self-loops get the INT64_MAX key (sorted last, dropped)
__global__ void k_pair_keys(int64_t m, const int64_t *__restrict__ ends, int64_t nn, int64_t *__restrict__ keys,
                            u64 *__restrict__ loops) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    u64 c = 0;
    if (e < m) {
        const int64_t x = ends[2 * e], y = ends[2 * e + 1];
        if (x == y) {
            keys[e] = INT64_MAX;
            c = 1;
        } else {
            keys[e] = min(x, y) * nn + max(x, y);
        }
    }
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(FULLR, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(loops, c);
}

__global__ void k_mark_used(int64_t m, const int64_t *__restrict__ keys, int64_t nn, int *__restrict__ used) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    used[keys[e] / nn] = 1;
    used[keys[e] % nn] = 1;
}

// kept names in order and isolated names in order, from the exclusive scan of the used flags
__global__ void k_split_nodes(int64_t nn, const int *__restrict__ used, const int *__restrict__ newid,
                              const int64_t *__restrict__ names, int64_t *__restrict__ kept,
                              int64_t *__restrict__ isolated) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const int64_t name = names ? names[i] : i;
    if (used[i]) kept[newid[i]] = name;
    else isolated[i - newid[i]] = name;
}

__global__ void k_renumber(int64_t m, const int64_t *__restrict__ keys, int64_t nn, const int *__restrict__ newid,
                           int64_t *__restrict__ u, int64_t *__restrict__ v) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m) return;
    u[e] = newid[keys[e] / nn];
    v[e] = newid[keys[e] % nn];
}

template <typename T> T fetch1(const DBuf &b, int64_t idx, cudaStream_t s) {
    T v{};
    LB_CUDA(cudaMemcpyAsync(&v, b.as<T>() + idx, sizeof(T), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    return v;
}

// inside count and sum of squared label volumes of one partition: edges (eu, ev, weights ew or unit), vertex
// weights vw, labels in [0, P)
void q_counts(int64_t nv, int64_t m, const int64_t *eu, const int64_t *ev, const int64_t *lab, const u64 *ew,
              const u64 *vw, int64_t P, DBuf &volc, DBuf &acc, cudaStream_t s, int64_t *ins, int64_t *s2) {
    volc.alloc(sizeof(u64) * std::max<int64_t>(P, 1));
    acc.alloc(2 * sizeof(u64));
    LB_CUDA(cudaMemsetAsync(volc.ptr, 0, sizeof(u64) * std::max<int64_t>(P, 1), s));
    LB_CUDA(cudaMemsetAsync(acc.ptr, 0, 2 * sizeof(u64), s));
    if (m) {
        k_inside<<<nblk(m), 256, 0, s>>>(m, eu, ev, lab, ew, acc.as<u64>());
        LB_LAUNCH_CHECK();
    }
    if (nv) {
        k_label_vol<<<nblk(nv), 256, 0, s>>>(nv, lab, vw, volc.as<u64>());
        LB_LAUNCH_CHECK();
    }
    k_sumsq<<<nblk(P), 256, 0, s>>>(P, volc.as<u64>(), acc.as<u64>() + 1);
    LB_LAUNCH_CHECK();
    u64 h[2];
    LB_CUDA(cudaMemcpyAsync(h, acc.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    *ins = (int64_t)h[0];
    *s2 = (int64_t)h[1];
}

}  // namespace

void reduce_run(Reduction &r, const int64_t *keys_h) {
    cudaStream_t s = r.ctx->stream;
    const int64_t n = r.n, m = r.m, nnz = 2 * m;
    DBuf keys, rc, rc_sorted, cols, dup, flag, nunion, changed, isroot, tmp, deg64, indptr, rkeys, rk_sorted, uniq,
        counts, nrun_d, inside;
    upload(keys, keys_h, (size_t)m, s);
    r.eu.alloc(sizeof(int64_t) * m);
    r.ev.alloc(sizeof(int64_t) * m);
    r.deg.alloc(sizeof(u64) * n);
    LB_CUDA(cudaMemsetAsync(r.deg.ptr, 0, sizeof(u64) * n, s));
    rc.alloc(sizeof(int64_t) * nnz);
    if (m) {
        k_split<<<nblk(m), 256, 0, s>>>(m, n, keys.as<int64_t>(), r.eu.as<int64_t>(), r.ev.as<int64_t>(),
                                        r.deg.as<u64>(), rc.as<int64_t>());
        LB_LAUNCH_CHECK();
    }
    // sorted adjacency (CSR with ascending columns) for the exact twin test
    int end_bit = 1;
    while (end_bit < 63 && ((int64_t)1 << end_bit) < n * n) end_bit++;
    rc_sorted.alloc(sizeof(int64_t) * nnz);
    cols.alloc(sizeof(int) * nnz);
    dup.alloc(sizeof(int));
    LB_CUDA(cudaMemsetAsync(dup.ptr, 0, sizeof(int), s));
    size_t tb = 0;
    if (m) {
        LB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, rc.as<int64_t>(), rc_sorted.as<int64_t>(), (int)nnz, 0,
                                               end_bit, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, rc.as<int64_t>(), rc_sorted.as<int64_t>(), (int)nnz, 0,
                                               end_bit, s));
        k_cols<<<nblk(nnz), 256, 0, s>>>(nnz, n, rc_sorted.as<int64_t>(), cols.as<int>(), dup.as<int>());
        LB_LAUNCH_CHECK();
    }
    LB_CHECK(fetch1<int>(dup, 0, s) == 0, LB_ERR_INVALID, "duplicate edge keys");
    deg64.alloc(sizeof(int64_t) * (n + 1));
    indptr.alloc(sizeof(int64_t) * (n + 1));
    k_deg_to_i64<<<nblk(n + 1), 256, 0, s>>>(n, r.deg.as<u64>(), deg64.as<int64_t>());
    LB_LAUNCH_CHECK();
    tb = 0;
    LB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, deg64.as<int64_t>(), indptr.as<int64_t>(), (int)(n + 1), s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, deg64.as<int64_t>(), indptr.as<int64_t>(), (int)(n + 1), s));
    // leaf and twin unions
    flag.alloc(m);
    nunion.alloc(2 * sizeof(u64));
    LB_CUDA(cudaMemsetAsync(nunion.ptr, 0, 2 * sizeof(u64), s));
    if (m) {
        k_unions<<<nblk(m, 8), 256, 0, s>>>(m, r.eu.as<int64_t>(), r.ev.as<int64_t>(), r.deg.as<u64>(),
                                            indptr.as<int64_t>(), cols.as<int>(), 2.0 * (double)m,
                                            flag.as<unsigned char>(), nunion.as<u64>());
        LB_LAUNCH_CHECK();
    }
    // components of the unions
    r.label.alloc(sizeof(int) * n);
    k_iota<<<nblk(n), 256, 0, s>>>(n, r.label.as<int>());
    LB_LAUNCH_CHECK();
    changed.alloc(sizeof(int));
    for (int round = 0; m; round++) {
        LB_CHECK(round < MAX_UNION_ROUNDS, LB_ERR_NUMERIC, "union components did not settle");
        LB_CUDA(cudaMemsetAsync(changed.ptr, 0, sizeof(int), s));
        k_hook<<<nblk(m), 256, 0, s>>>(m, r.eu.as<int64_t>(), r.ev.as<int64_t>(), flag.as<unsigned char>(),
                                       r.label.as<int>(), changed.as<int>());
        LB_LAUNCH_CHECK();
        for (int k = 0; k < 3; k++) {
            k_jump<<<nblk(n), 256, 0, s>>>(n, r.label.as<int>(), changed.as<int>());
            LB_LAUNCH_CHECK();
        }
        if (fetch1<int>(changed, 0, s) == 0) break;
    }
    // group number = rank of the group's root (its smallest member) among all roots
    isroot.alloc(sizeof(int) * n);
    r.rank.alloc(sizeof(int) * n);
    k_is_root<<<nblk(n), 256, 0, s>>>(n, r.label.as<int>(), isroot.as<int>());
    LB_LAUNCH_CHECK();
    tb = 0;
    LB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, isroot.as<int>(), r.rank.as<int>(), (int)n, s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, isroot.as<int>(), r.rank.as<int>(), (int)n, s));
    const int64_t N = n ? (int64_t)fetch1<int>(r.rank, n - 1, s) + fetch1<int>(isroot, n - 1, s) : 0;
    r.N = N;
    r.grp.alloc(sizeof(int64_t) * n);
    r.vol.alloc(sizeof(u64) * N);
    LB_CUDA(cudaMemsetAsync(r.vol.ptr, 0, sizeof(u64) * std::max<int64_t>(N, 1), s));
    k_group<<<nblk(n), 256, 0, s>>>(n, r.label.as<int>(), r.rank.as<int>(), r.deg.as<u64>(), r.grp.as<int64_t>(),
                                    r.vol.as<u64>());
    LB_LAUNCH_CHECK();
    // reduced edges: group-pair keys sorted and run-length encoded (run lengths = edge counts)
    inside.alloc(sizeof(u64));
    LB_CUDA(cudaMemsetAsync(inside.ptr, 0, sizeof(u64), s));
    rkeys.alloc(sizeof(int64_t) * m);
    rk_sorted.alloc(sizeof(int64_t) * m);
    uniq.alloc(sizeof(int64_t) * m);
    counts.alloc(sizeof(int) * m);
    nrun_d.alloc(sizeof(int));
    LB_CUDA(cudaMemsetAsync(nrun_d.ptr, 0, sizeof(int), s));
    if (m) {
        k_red_keys<<<nblk(m), 256, 0, s>>>(m, N, r.eu.as<int64_t>(), r.ev.as<int64_t>(), r.grp.as<int64_t>(),
                                           rkeys.as<int64_t>(), inside.as<u64>());
        LB_LAUNCH_CHECK();
        tb = 0;
        LB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, rkeys.as<int64_t>(), rk_sorted.as<int64_t>(), (int)m, 0,
                                               64, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, rkeys.as<int64_t>(), rk_sorted.as<int64_t>(), (int)m, 0,
                                               64, s));
        tb = 0;
        LB_CUDA(cub::DeviceRunLengthEncode::Encode(nullptr, tb, rk_sorted.as<int64_t>(), uniq.as<int64_t>(),
                                                   counts.as<int>(), nrun_d.as<int>(), (int)m, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRunLengthEncode::Encode(tmp.ptr, tb, rk_sorted.as<int64_t>(), uniq.as<int64_t>(),
                                                   counts.as<int>(), nrun_d.as<int>(), (int)m, s));
    }
    u64 unions[2];
    LB_CUDA(cudaMemcpyAsync(unions, nunion.ptr, sizeof(unions), cudaMemcpyDeviceToHost, s));
    r.inside = (int64_t)fetch1<u64>(inside, 0, s);
    const int64_t nrun = fetch1<int>(nrun_d, 0, s);
    r.leaf_unions = (int64_t)unions[0];
    r.twin_unions = (int64_t)unions[1];
    r.M = nrun - (r.inside > 0 ? 1 : 0);   // the last run holds the inside edges
    r.ru.alloc(sizeof(int64_t) * r.M);
    r.rv.alloc(sizeof(int64_t) * r.M);
    r.rw.alloc(sizeof(u64) * r.M);
    r.rkeys.alloc(sizeof(int64_t) * r.M);
    if (r.M) {
        k_red_decode<<<nblk(r.M), 256, 0, s>>>(r.M, N, uniq.as<int64_t>(), counts.as<int>(), r.ru.as<int64_t>(),
                                               r.rv.as<int64_t>(), r.rw.as<u64>());
        LB_LAUNCH_CHECK();
        LB_CUDA(cudaMemcpyAsync(r.rkeys.ptr, uniq.ptr, sizeof(int64_t) * r.M, cudaMemcpyDeviceToDevice, s));
    }
    LB_CUDA(cudaStreamSynchronize(s));
}

void reduce_get(const Reduction &r, int64_t *keys, double *weights, int64_t *vol, int64_t *group_of) {
    cudaStream_t s = r.ctx->stream;
    if (keys && r.M)
        LB_CUDA(cudaMemcpyAsync(keys, r.rkeys.ptr, sizeof(int64_t) * r.M, cudaMemcpyDeviceToHost, s));
    std::vector<u64> w(weights ? r.M : 0);
    if (weights && r.M) LB_CUDA(cudaMemcpyAsync(w.data(), r.rw.ptr, sizeof(u64) * r.M, cudaMemcpyDeviceToHost, s));
    if (vol && r.N) LB_CUDA(cudaMemcpyAsync(vol, r.vol.ptr, sizeof(int64_t) * r.N, cudaMemcpyDeviceToHost, s));
    if (group_of && r.n)
        LB_CUDA(cudaMemcpyAsync(group_of, r.grp.ptr, sizeof(int64_t) * r.n, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    for (size_t e = 0; e < w.size(); e++) weights[e] = (double)w[e];
}

void reduce_labels(Reduction &r, const int64_t *lab_h, int64_t P, int64_t *lr_out, int64_t *counts) {
    cudaStream_t s = r.ctx->stream;
    DBuf lab, lr, lab2, volc, acc;
    upload(lab, lab_h, (size_t)r.n, s);
    lr.alloc(sizeof(int64_t) * r.N);
    lab2.alloc(sizeof(int64_t) * r.n);
    if (r.n) {
        k_restrict<<<nblk(r.n), 256, 0, s>>>(r.n, r.label.as<int>(), r.rank.as<int>(), lab.as<int64_t>(),
                                             lr.as<int64_t>());
        LB_LAUNCH_CHECK();
        k_expand<<<nblk(r.n), 256, 0, s>>>(r.n, r.grp.as<int64_t>(), lr.as<int64_t>(), lab2.as<int64_t>());
        LB_LAUNCH_CHECK();
    }
    // the partition with the rules enforced, on the original graph
    q_counts(r.n, r.m, r.eu.as<int64_t>(), r.ev.as<int64_t>(), lab2.as<int64_t>(), nullptr, r.deg.as<u64>(), P, volc,
             acc, s, counts + 0, counts + 1);
    // the same partition on the reduced graph (edge counts as weights, group volumes as vertex weights)
    q_counts(r.N, r.M, r.ru.as<int64_t>(), r.rv.as<int64_t>(), lr.as<int64_t>(), r.rw.as<u64>(), r.vol.as<u64>(), P,
             volc, acc, s, counts + 2, counts + 3);
    // the partition as given, on the original graph
    q_counts(r.n, r.m, r.eu.as<int64_t>(), r.ev.as<int64_t>(), lab.as<int64_t>(), nullptr, r.deg.as<u64>(), P, volc,
             acc, s, counts + 4, counts + 5);
    if (lr_out && r.N) LB_CUDA(cudaMemcpyAsync(lr_out, lr.ptr, sizeof(int64_t) * r.N, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
}

void modularity_counts_run(Ctx &c, int64_t n, int64_t m, const int64_t *u_h, const int64_t *v_h,
                           const int64_t *lab_h, int64_t P, int64_t *inside, int64_t *sum_vol2) {
    cudaStream_t s = c.stream;
    DBuf u, v, lab, deg, volc, acc;
    upload(u, u_h, (size_t)m, s);
    upload(v, v_h, (size_t)m, s);
    upload(lab, lab_h, (size_t)n, s);
    deg.alloc(sizeof(u64) * n);
    LB_CUDA(cudaMemsetAsync(deg.ptr, 0, sizeof(u64) * std::max<int64_t>(n, 1), s));
    if (m) {
        k_endpoint_deg<<<nblk(m), 256, 0, s>>>(m, u.as<int64_t>(), v.as<int64_t>(), deg.as<u64>());
        LB_LAUNCH_CHECK();
    }
    q_counts(n, m, u.as<int64_t>(), v.as<int64_t>(), lab.as<int64_t>(), nullptr, deg.as<u64>(), P, volc, acc, s,
             inside, sum_vol2);
}

void simple_graph_run(SimpleGraph &g, const int64_t *pairs_h, int64_t m_in, int64_t n_names) {
    cudaStream_t s = g.ctx->stream;
    DBuf ends, vals, names, keys, keys_sorted, ukeys, nsel, loops, used, newid, tmp;
    const int64_t cnt = 2 * m_in;
    upload(vals, pairs_h, (size_t)cnt, s);
    size_t tb = 0;
    int64_t nn = n_names;
    if (n_names < 0) {
        // names = sorted distinct ids of all endpoints
        DBuf sorted;
        sorted.alloc(sizeof(int64_t) * cnt);
        names.alloc(sizeof(int64_t) * cnt);
        nsel.alloc(sizeof(int));
        LB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, vals.as<int64_t>(), sorted.as<int64_t>(), (int)cnt, 0, 64,
                                               s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, vals.as<int64_t>(), sorted.as<int64_t>(), (int)cnt, 0, 64,
                                               s));
        tb = 0;
        LB_CUDA(cub::DeviceSelect::Unique(nullptr, tb, sorted.as<int64_t>(), names.as<int64_t>(), nsel.as<int>(),
                                          (int)cnt, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceSelect::Unique(tmp.ptr, tb, sorted.as<int64_t>(), names.as<int64_t>(), nsel.as<int>(),
                                          (int)cnt, s));
        nn = fetch1<int>(nsel, 0, s);
        ends.alloc(sizeof(int64_t) * cnt);
        k_lower_bound<<<nblk(cnt), 256, 0, s>>>(cnt, vals.as<int64_t>(), names.as<int64_t>(), nn,
                                                ends.as<int64_t>());
        LB_LAUNCH_CHECK();
    }
    const int64_t *e_ptr = n_names < 0 ? ends.as<int64_t>() : vals.as<int64_t>();
    LB_CHECK(nn < ((int64_t)1 << 31), LB_ERR_INVALID, "too many distinct nodes");
    // keys, sorted and deduplicated
    keys.alloc(sizeof(int64_t) * m_in);
    keys_sorted.alloc(sizeof(int64_t) * m_in);
    ukeys.alloc(sizeof(int64_t) * m_in);
    loops.alloc(sizeof(u64));
    nsel.alloc(sizeof(int));
    LB_CUDA(cudaMemsetAsync(loops.ptr, 0, sizeof(u64), s));
    k_pair_keys<<<nblk(m_in), 256, 0, s>>>(m_in, e_ptr, nn, keys.as<int64_t>(), loops.as<u64>());
    LB_LAUNCH_CHECK();
    tb = 0;
    LB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.as<int64_t>(), keys_sorted.as<int64_t>(), (int)m_in, 0,
                                           64, s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, keys.as<int64_t>(), keys_sorted.as<int64_t>(), (int)m_in, 0,
                                           64, s));
    tb = 0;
    LB_CUDA(cub::DeviceSelect::Unique(nullptr, tb, keys_sorted.as<int64_t>(), ukeys.as<int64_t>(), nsel.as<int>(),
                                      (int)m_in, s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceSelect::Unique(tmp.ptr, tb, keys_sorted.as<int64_t>(), ukeys.as<int64_t>(), nsel.as<int>(),
                                      (int)m_in, s));
    g.self_loops = (int64_t)fetch1<u64>(loops, 0, s);
    const int64_t nu = fetch1<int>(nsel, 0, s);
    const int64_t m = nu - (g.self_loops > 0 ? 1 : 0);
    // used nodes, renumbered in name order
    used.alloc(sizeof(int) * nn);
    newid.alloc(sizeof(int) * nn);
    LB_CUDA(cudaMemsetAsync(used.ptr, 0, sizeof(int) * nn, s));
    if (m) {
        k_mark_used<<<nblk(m), 256, 0, s>>>(m, ukeys.as<int64_t>(), nn, used.as<int>());
        LB_LAUNCH_CHECK();
    }
    tb = 0;
    LB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, used.as<int>(), newid.as<int>(), (int)nn, s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, tb, used.as<int>(), newid.as<int>(), (int)nn, s));
    const int64_t n = nn ? (int64_t)fetch1<int>(newid, nn - 1, s) + fetch1<int>(used, nn - 1, s) : 0;
    g.n_names = nn;
    g.n = n;
    g.m = m;
    g.kept.alloc(sizeof(int64_t) * n);
    g.isolated.alloc(sizeof(int64_t) * (nn - n));
    g.u.alloc(sizeof(int64_t) * m);
    g.v.alloc(sizeof(int64_t) * m);
    k_split_nodes<<<nblk(nn), 256, 0, s>>>(nn, used.as<int>(), newid.as<int>(),
                                           n_names < 0 ? names.as<int64_t>() : nullptr, g.kept.as<int64_t>(),
                                           g.isolated.as<int64_t>());
    LB_LAUNCH_CHECK();
    if (m) {
        k_renumber<<<nblk(m), 256, 0, s>>>(m, ukeys.as<int64_t>(), nn, newid.as<int>(), g.u.as<int64_t>(),
                                           g.v.as<int64_t>());
        LB_LAUNCH_CHECK();
    }
    LB_CUDA(cudaStreamSynchronize(s));
}

void simple_graph_get(const SimpleGraph &g, int64_t *u, int64_t *v, int64_t *kept, int64_t *isolated) {
    cudaStream_t s = g.ctx->stream;
    if (u && g.m) LB_CUDA(cudaMemcpyAsync(u, g.u.ptr, sizeof(int64_t) * g.m, cudaMemcpyDeviceToHost, s));
    if (v && g.m) LB_CUDA(cudaMemcpyAsync(v, g.v.ptr, sizeof(int64_t) * g.m, cudaMemcpyDeviceToHost, s));
    if (kept && g.n) LB_CUDA(cudaMemcpyAsync(kept, g.kept.ptr, sizeof(int64_t) * g.n, cudaMemcpyDeviceToHost, s));
    if (isolated && g.n_names > g.n)
        LB_CUDA(cudaMemcpyAsync(isolated, g.isolated.ptr, sizeof(int64_t) * (g.n_names - g.n), cudaMemcpyDeviceToHost,
                                s));
    LB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace lb
