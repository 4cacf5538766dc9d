// Triangle separation (sm_100a) with the reference's exact outputs given the same V:
//   family 0, edge arms:      alm_vcs.py:554-565 _centre, 567-597 sep_hist / sep_collect, 965-974 separate_ref
//   family 1, one-edge arms:  alm_vcs.py:608-632 _centre1, 634-666 sep1_hist / sep1_collect, 976-984 separate1_ref
// (the reference's fused fast path separate_both, 938-954, returns the same arrays).
//
// Everything runs in the caller's vertex numbering (a locality order of the problem only changes where the V rows
// live).  Dot products are FP64, sequential in the column index, without FMA, as in the reference.
//   k_arm_count     arms per centre j: neighbours i with X_ij > thresh
//   k_arm_fill      arm lists of centres with at most maxh arms, in CSR order
//   k_arm_big       centres with more arms: the top maxh by value (ties by position), block-level exact selection
//   k_walk          family 1 second arms K (2-hop, not adjacent to j, deduplicated by id, X_jk > thresh; sorted by
//                   id, or the top maxk by value)
//   k_pairs         violations vm = xh_x + x_y - X_xy - 1 of every arm pair in generation order: histogram pass,
//                   per-centre count pass (bin >= b0, vm >= vmin), ordered write pass with the per-chunk caps
#include <math.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "lb_internal.cuh"

namespace lb {
namespace {

constexpr unsigned FULLS = 0xffffffffu;
constexpr int WALK_CAP = 2048;   // walk candidates per centre held in shared memory (hub2 * cap2 <= WALK_CAP)

template <typename T> __device__ __forceinline__ double tod(T x) { return (double)x; }
template <> __device__ __forceinline__ double tod<__nv_bfloat16>(__nv_bfloat16 x) { return (double)__bfloat162float(x); }

struct SepGraph {
    int64_t n;
    const int64_t *indptr;   // caller numbering, sorted columns
    const int *indices;
    const int *row;          // caller vertex -> row of V (nullptr: identity)
    int ld, r;
};

template <typename T>
__device__ __forceinline__ double vdot(const SepGraph &g, const T *V, int64_t a, int64_t b) {
    const T *va = V + (int64_t)(g.row ? g.row[a] : a) * g.ld;
    const T *vb = V + (int64_t)(g.row ? g.row[b] : b) * g.ld;
    double s = 0.0;
    for (int q = 0; q < g.r; q++) s = __dadd_rn(s, __dmul_rn(tod<T>(va[q]), tod<T>(vb[q])));
    return s;
}

// --------------------------------------------------------------------------------------------- arms
template <typename T>
__global__ void __launch_bounds__(256) k_arm_count(SepGraph g, const T *__restrict__ V, double thresh,
                                                   int *__restrict__ m) {
    const int lane = threadIdx.x & 31;
    const int64_t j = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (j >= g.n) return;
    const int64_t a = g.indptr[j], b = g.indptr[j + 1];
    int c = 0;
    for (int64_t e = a + lane; e < b; e += 32) c += vdot<T>(g, V, g.indices[e], j) > thresh ? 1 : 0;
    for (int off = 16; off; off >>= 1) c += __shfl_xor_sync(FULLS, c, off);
    if (lane == 0) m[j] = c;
}

// arms of centres with m <= maxh, in CSR order (ordered compaction)
template <typename T>
__global__ void __launch_bounds__(256) k_arm_fill(SepGraph g, const T *__restrict__ V, double thresh, int maxh,
                                                  const int *__restrict__ m, const int64_t *__restrict__ arm_ptr,
                                                  int *__restrict__ arm_idx, double *__restrict__ arm_val) {
    const int lane = threadIdx.x & 31;
    const int64_t j = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (j >= g.n || m[j] > maxh || m[j] == 0) return;
    const int64_t a = g.indptr[j], b = g.indptr[j + 1];
    int64_t o = arm_ptr[j];
    for (int64_t e0 = a; e0 < b; e0 += 32) {
        const int64_t e = e0 + lane;
        int i = 0;
        double s = 0.0;
        bool ok = false;
        if (e < b) {
            i = g.indices[e];
            s = vdot<T>(g, V, i, j);
            ok = s > thresh;
        }
        const unsigned bal = __ballot_sync(FULLS, ok);
        if (ok) {
            const int pos = __popc(bal & ((1u << lane) - 1u));
            arm_idx[o + pos] = i;
            arm_val[o + pos] = s;
        }
        o += __popc(bal);
    }
}

// centres with more than maxh arms (block per centre): all values into the pool, then maxh rounds of a block argmax
// over (value desc, position asc); the chosen arms are written in that order.
template <typename T>
__global__ void __launch_bounds__(256) k_arm_big(SepGraph g, const T *__restrict__ V, double thresh, int maxh,
                                                 const int *__restrict__ big, const int64_t *__restrict__ pool_ptr,
                                                 double *__restrict__ pool, const int64_t *__restrict__ arm_ptr,
                                                 int *__restrict__ arm_idx, double *__restrict__ arm_val) {
    __shared__ double sv[256];
    __shared__ int64_t se[256];
    const int64_t j = big[blockIdx.x];
    const int64_t a = g.indptr[j], b = g.indptr[j + 1];
    double *pv = pool + pool_ptr[blockIdx.x];
    for (int64_t e = a + threadIdx.x; e < b; e += blockDim.x) {
        const double s = vdot<T>(g, V, g.indices[e], j);
        pv[e - a] = s > thresh ? s : -INFINITY;
    }
    __syncthreads();
    const int64_t o = arm_ptr[j];
    for (int r = 0; r < maxh; r++) {
        double bv = -INFINITY;
        int64_t be = INT64_MAX;
        for (int64_t e = threadIdx.x; e < b - a; e += blockDim.x) {
            const double v = pv[e];
            if (v > bv || (v == bv && e < be)) {
                bv = v;
                be = e;
            }
        }
        sv[threadIdx.x] = bv;
        se[threadIdx.x] = be;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) {
                const double v2 = sv[threadIdx.x + w];
                const int64_t e2 = se[threadIdx.x + w];
                if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && e2 < se[threadIdx.x])) {
                    sv[threadIdx.x] = v2;
                    se[threadIdx.x] = e2;
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            arm_idx[o + r] = g.indices[a + se[0]];
            arm_val[o + r] = sv[0];
            pv[se[0]] = -INFINITY;
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------------------------------------- family 1 walk
__device__ __forceinline__ bool adjacent(const SepGraph &g, int64_t j, int x) {
    int64_t lo = g.indptr[j], hi = g.indptr[j + 1];
    const int64_t end = hi;
    while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (g.indices[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < end && g.indices[lo] == x;
}

// Block (128 threads) per centre.  MODE 0: count |K| (after the maxk cap) into kcnt; MODE 1: write K into
// k_idx/k_val at k_ptr.  K: the walk's candidates c (first cap2 neighbours of the first hub2 arms; not j, not
// adjacent to j), unique ids, X_cj > thresh, sorted by id; more than maxk: the top maxk by value (ties by id).
template <typename T, int MODE>
__global__ void __launch_bounds__(128) k_walk(SepGraph g, const T *__restrict__ V, double thresh, int hub2, int cap2,
                                              int maxk, const int *__restrict__ m, const int64_t *__restrict__ arm_ptr,
                                              const int *__restrict__ arm_idx, int *__restrict__ kcnt,
                                              const int64_t *__restrict__ k_ptr, int *__restrict__ k_idx,
                                              double *__restrict__ k_val) {
    __shared__ int cand[WALK_CAP];
    __shared__ double cval[WALK_CAP];
    __shared__ int s_n, s_m;
    __shared__ double rv[128];
    __shared__ int ri[128];
    for (int64_t j = blockIdx.x; j < g.n; j += gridDim.x) {
        const int64_t deg = g.indptr[j + 1] - g.indptr[j];
        const int mh = min(m[j], 0x7fffffff);
        const int mhc = mh;   // arms stored: min(m, maxh) (callers pass the capped list via arm_ptr)
        const int64_t ah = arm_ptr[j], nh_all = arm_ptr[j + 1] - ah;
        if (deg < 1 || nh_all == 0) {
            if (MODE == 0 && threadIdx.x == 0) kcnt[j] = 0;
            continue;
        }
        (void)mhc;
        const int nh = (int)min((int64_t)hub2, nh_all);
        // gather walk candidates (order irrelevant: they are sorted by id below)
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        for (int a = 0; a < nh; a++) {
            const int i2 = arm_idx[ah + a];
            const int64_t lo = g.indptr[i2], hi = min(g.indptr[i2 + 1], lo + (int64_t)cap2);
            for (int64_t e = lo + threadIdx.x; e < hi; e += blockDim.x) {
                const int c = g.indices[e];
                if (c == j || adjacent(g, j, c)) continue;
                const int pos = atomicAdd(&s_n, 1);
                if (pos < WALK_CAP) cand[pos] = c;
            }
        }
        __syncthreads();
        const int nc = min(s_n, WALK_CAP);
        // bitonic sort of cand[0..P) by id (padding with INT_MAX)
        int P = 1;
        while (P < nc) P <<= 1;
        for (int t = nc + threadIdx.x; t < P; t += blockDim.x) cand[t] = 0x7fffffff;
        __syncthreads();
        for (int kk = 2; kk <= P; kk <<= 1)
            for (int jj = kk >> 1; jj > 0; jj >>= 1) {
                for (int t = threadIdx.x; t < P; t += blockDim.x) {
                    const int x = t ^ jj;
                    if (x > t) {
                        const bool up = (t & kk) == 0;
                        const int u = cand[t], v = cand[x];
                        if ((u > v) == up) {
                            cand[t] = v;
                            cand[x] = u;
                        }
                    }
                }
                __syncthreads();
            }
        // unique ids with X_cj > thresh, compacted in id order (values into cval, -inf marks dropped)
        for (int t = threadIdx.x; t < nc; t += blockDim.x) {
            const int c = cand[t];
            double s = -INFINITY;
            if (t == 0 || cand[t - 1] != c) {
                const double v = vdot<T>(g, V, c, j);
                if (v > thresh) s = v;
            }
            cval[t] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int w = 0;
            for (int t = 0; t < nc; t++)
                if (cval[t] != -INFINITY) {
                    cand[w] = cand[t];
                    cval[w] = cval[t];
                    w++;
                }
            s_m = w;
        }
        __syncthreads();
        const int mk = s_m;
        const int keep = min(mk, maxk);
        if (MODE == 0) {
            if (threadIdx.x == 0) kcnt[j] = keep;
            __syncthreads();
            continue;
        }
        const int64_t ko = k_ptr[j];
        if (mk <= maxk) {
            for (int t = threadIdx.x; t < mk; t += blockDim.x) {
                k_idx[ko + t] = cand[t];
                k_val[ko + t] = cval[t];
            }
        } else {
            // top maxk by (value desc, id asc): maxk rounds of a block argmax
            for (int rnd = 0; rnd < maxk; rnd++) {
                double bv = -INFINITY;
                int bi = 0x7fffffff;
                for (int t = threadIdx.x; t < mk; t += blockDim.x) {
                    const double v = cval[t];
                    if (v > bv || (v == bv && t < bi)) {
                        bv = v;
                        bi = t;
                    }
                }
                rv[threadIdx.x] = bv;
                ri[threadIdx.x] = bi;
                __syncthreads();
                for (int w = blockDim.x / 2; w > 0; w >>= 1) {
                    if ((int)threadIdx.x < w) {
                        const double v2 = rv[threadIdx.x + w];
                        const int i2 = ri[threadIdx.x + w];
                        if (v2 > rv[threadIdx.x] || (v2 == rv[threadIdx.x] && i2 < ri[threadIdx.x])) {
                            rv[threadIdx.x] = v2;
                            ri[threadIdx.x] = i2;
                        }
                    }
                    __syncthreads();
                }
                if (threadIdx.x == 0) {
                    k_idx[ko + rnd] = cand[ri[0]];
                    k_val[ko + rnd] = rv[0];
                    cval[ri[0]] = -INFINITY;
                }
                __syncthreads();
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------------------------------------- pairs
struct PairArgs {
    int family;                    // 0: x < y over the arms; 1: x over the arms, y over K (skip equal ids)
    const int64_t *a_ptr;          // first list (arms)
    const int *a_idx;
    const double *a_val;
    const int64_t *b_ptr;          // second list (arms for family 0, K for family 1)
    const int *b_idx;
    const double *b_val;
    int64_t cs;                    // chunk size in centres
    int nb;
    double vtol, vmin;
    int b0;
    int *hist;                     // MODE 0
    int *cntbin, *cntv;            // MODE 1 (per centre)
    const int64_t *cbase;          // MODE 2: rank of the centre's first candidate inside its chunk
    const int64_t *climit;         // MODE 2: cap of the centre's chunk (counts[ch])
    const int64_t *coff;           // MODE 2: output offset of the centre's chunk
    int64_t *out_tri;
    double *out_val;
};

// Warp per centre; pairs in generation order (x, then y), 32 at a time.
template <typename T, int MODE>
__global__ void __launch_bounds__(256) k_pairs(SepGraph g, const T *__restrict__ V, PairArgs pa) {
    __shared__ int sh_hist[2048];
    const int lane = threadIdx.x & 31;
    if (MODE == 0) {
        for (int t = threadIdx.x; t < pa.nb; t += blockDim.x) sh_hist[t] = 0;
        __syncthreads();
    }
    const int64_t j = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (j < g.n) {
        const int64_t deg = g.indptr[j + 1] - g.indptr[j];
        const int64_t ha = pa.a_ptr[j], mh = pa.a_ptr[j + 1] - ha;
        const int64_t kb = pa.b_ptr[j], mk = pa.b_ptr[j + 1] - kb;
        const bool run = pa.family == 0 ? (deg >= 2 && mh >= 2) : (deg >= 1 && mh > 0 && mk > 0);
        int cb = 0, cv = 0;
        int64_t rank = MODE == 2 ? pa.cbase[j] : 0;
        const int64_t lim = MODE == 2 ? pa.climit[j] : 0;
        if (run) {
            for (int64_t x = 0; x < mh; x++) {
                const int hx = pa.a_idx[ha + x];
                const double xv = pa.a_val[ha + x];
                const int64_t y0 = pa.family == 0 ? x + 1 : 0;
                for (int64_t yb = y0; yb < mk; yb += 32) {
                    const int64_t y = yb + lane;
                    bool cand = false, inbin = false, ok = false;
                    int ky = 0;
                    double vm = 0.0;
                    if (y < mk) {
                        ky = pa.b_idx[kb + y];
                        if (!(pa.family == 1 && ky == hx)) {
                            const double s = vdot<T>(g, V, hx, ky);
                            vm = __dsub_rn(__dsub_rn(__dadd_rn(xv, pa.b_val[kb + y]), s), 1.0);
                            ok = true;
                            if (vm > pa.vtol) {
                                long long bin = (long long)(__dmul_rn(__dsub_rn(vm, pa.vtol) / __dsub_rn(2.0, pa.vtol),
                                                                      (double)pa.nb));
                                if (bin > pa.nb - 1) bin = pa.nb - 1;
                                if (MODE == 0) atomicAdd(&sh_hist[bin], 1);
                                inbin = bin >= pa.b0;
                            }
                            cand = vm >= pa.vmin;
                        }
                    }
                    (void)ok;
                    if (MODE == 1) {
                        cb += inbin ? 1 : 0;
                        cv += cand ? 1 : 0;
                    }
                    if (MODE == 2) {
                        const unsigned bal = __ballot_sync(FULLS, cand);
                        if (cand) {
                            const int64_t rk = rank + __popc(bal & ((1u << lane) - 1u));
                            if (rk < lim) {
                                const int64_t o = pa.coff[j] + rk;
                                pa.out_tri[3 * o] = min(hx, ky);
                                pa.out_tri[3 * o + 1] = j;
                                pa.out_tri[3 * o + 2] = max(hx, ky);
                                pa.out_val[o] = vm;
                            }
                        }
                        rank += __popc(bal);
                    }
                }
            }
        }
        if (MODE == 1) {
            for (int off = 16; off; off >>= 1) {
                cb += __shfl_xor_sync(FULLS, cb, off);
                cv += __shfl_xor_sync(FULLS, cv, off);
            }
            if (lane == 0) {
                pa.cntbin[j] = cb;
                pa.cntv[j] = cv;
            }
        }
    }
    if (MODE == 0) {
        __syncthreads();
        for (int t = threadIdx.x; t < pa.nb; t += blockDim.x)
            if (sh_hist[t]) atomicAdd(&pa.hist[t], sh_hist[t]);
    }
}

static inline unsigned nb8(int64_t n) { return (unsigned)((n + 7) / 8); }

}  // namespace

// --------------------------------------------------------------------------------------------- host
struct SepScratch {
    // the problem's scratch buffers of the separation (kept across rounds)
    DBuf &m, &arm_ptr, &arm_idx, &arm_val, &big, &pool_ptr, &pool, &kcnt, &k_ptr, &k_idx, &k_val, &hist, &cntbin,
         &cntv, &cbase, &climit, &coff;
    explicit SepScratch(Problem &p)
        : m(p.scratch("sep:m")),
          arm_ptr(p.scratch("sep:arm_ptr")),
          arm_idx(p.scratch("sep:arm_idx")),
          arm_val(p.scratch("sep:arm_val")),
          big(p.scratch("sep:big")),
          pool_ptr(p.scratch("sep:pool_ptr")),
          pool(p.scratch("sep:pool")),
          kcnt(p.scratch("sep:kcnt")),
          k_ptr(p.scratch("sep:k_ptr")),
          k_idx(p.scratch("sep:k_idx")),
          k_val(p.scratch("sep:k_val")),
          hist(p.scratch("sep:hist")),
          cntbin(p.scratch("sep:cntbin")),
          cntv(p.scratch("sep:cntv")),
          cbase(p.scratch("sep:cbase")),
          climit(p.scratch("sep:climit")),
          coff(p.scratch("sep:coff")) {}
};

// One family's histogram threshold, counts and ordered output (separate_ref semantics).
template <typename T>
static void run_pairs(Problem &p, const SepGraph &g, const T *V, PairArgs pa, int nchunk, int64_t cap,
                      SepScratch &sc, std::vector<int64_t> &tri_out, std::vector<double> &val_out, cudaStream_t s) {
    const int64_t n = g.n;
    const int nb = pa.nb;
    // histogram
    sc.hist.alloc(sizeof(int) * nb);
    LB_CUDA(cudaMemsetAsync(sc.hist.ptr, 0, sizeof(int) * nb, s));
    pa.hist = sc.hist.as<int>();
    pa.b0 = nb;
    pa.vmin = INFINITY;
    k_pairs<T, 0><<<nb8(n), 256, 0, s>>>(g, V, pa);
    LB_LAUNCH_CHECK();
    std::vector<int> hist(nb);
    LB_CUDA(cudaMemcpyAsync(hist.data(), sc.hist.ptr, sizeof(int) * nb, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    // b0 = first bin whose tail count (bins b0..nb-1) is <= cap (alm_vcs.py:967-970)
    int b0 = nb;
    {
        int64_t tail = 0;
        std::vector<int64_t> cum(nb + 1, 0);
        for (int b = nb - 1; b >= 0; b--) {
            tail += hist[b];
            cum[b] = tail;
        }
        for (int b = 0; b < nb; b++)
            if (cum[b] <= cap) {
                b0 = b;
                break;
            }
    }
    tri_out.clear();
    val_out.clear();
    if (b0 >= nb) return;
    const double vmin = pa.vtol + (2.0 - pa.vtol) * b0 / nb;
    pa.b0 = b0;
    pa.vmin = vmin;
    // per-centre counts
    sc.cntbin.alloc(sizeof(int) * n);
    sc.cntv.alloc(sizeof(int) * n);
    LB_CUDA(cudaMemsetAsync(sc.cntbin.ptr, 0, sizeof(int) * n, s));
    LB_CUDA(cudaMemsetAsync(sc.cntv.ptr, 0, sizeof(int) * n, s));
    pa.cntbin = sc.cntbin.as<int>();
    pa.cntv = sc.cntv.as<int>();
    k_pairs<T, 1><<<nb8(n), 256, 0, s>>>(g, V, pa);
    LB_LAUNCH_CHECK();
    std::vector<int> cb(n), cv(n);
    LB_CUDA(cudaMemcpyAsync(cb.data(), sc.cntbin.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaMemcpyAsync(cv.data(), sc.cntv.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    // counts[ch] = sum of bin >= b0 in the chunk; kept[ch] = min(counts, candidates); output offsets by chunk
    std::vector<int64_t> counts(nchunk, 0), ncand(nchunk, 0);
    for (int64_t j = 0; j < n; j++) {
        counts[j / pa.cs] += cb[j];
        ncand[j / pa.cs] += cv[j];
    }
    std::vector<int64_t> off(nchunk + 1, 0);
    for (int c = 0; c < nchunk; c++) off[c + 1] = off[c] + std::min(counts[c], ncand[c]);
    std::vector<int64_t> cbase(n), climit(n), coff(n);
    std::vector<int64_t> run(nchunk, 0);
    for (int64_t j = 0; j < n; j++) {
        const int64_t c = j / pa.cs;
        cbase[j] = run[c];
        run[c] += cv[j];
        climit[j] = counts[c];
        coff[j] = off[c];
    }
    const int64_t total = off[nchunk];
    if (total == 0) return;
    upload(sc.cbase, cbase, s);
    upload(sc.climit, climit, s);
    upload(sc.coff, coff, s);
    DBuf &otri = p.scratch("lb_sep:480:otri"), &oval = p.scratch("lb_sep:480:oval");
    otri.alloc(sizeof(int64_t) * 3 * total);
    oval.alloc(sizeof(double) * total);
    pa.cbase = sc.cbase.as<int64_t>();
    pa.climit = sc.climit.as<int64_t>();
    pa.coff = sc.coff.as<int64_t>();
    pa.out_tri = otri.as<int64_t>();
    pa.out_val = oval.as<double>();
    k_pairs<T, 2><<<nb8(n), 256, 0, s>>>(g, V, pa);
    LB_LAUNCH_CHECK();
    tri_out.resize(3 * total);
    val_out.resize(total);
    LB_CUDA(cudaMemcpyAsync(tri_out.data(), otri.ptr, sizeof(int64_t) * 3 * total, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaMemcpyAsync(val_out.data(), oval.ptr, sizeof(double) * total, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
}

template <typename T>
static void separate_typed(Problem &p, const SepParams &sp, cudaStream_t s) {
    const int64_t n = p.n;
    SepGraph g;
    g.n = n;
    g.indptr = p.permuted ? p.cindptr.as<int64_t>() : p.indptr.as<int64_t>();
    g.indices = p.permuted ? p.cindices.as<int>() : p.indices.as<int>();
    g.row = p.permuted ? p.inv_d.as<int>() : nullptr;
    g.ld = p.ld;
    g.r = p.r;
    const T *V = p.V.as<T>();
    SepScratch sc(p);
    // arms
    sc.m.alloc(sizeof(int) * n);
    k_arm_count<T><<<nb8(n), 256, 0, s>>>(g, V, sp.thresh, sc.m.as<int>());
    LB_LAUNCH_CHECK();
    std::vector<int> m(n);
    LB_CUDA(cudaMemcpyAsync(m.data(), sc.m.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    std::vector<int64_t> arm_ptr(n + 1, 0), pool_ptr{0};
    std::vector<int> big;
    const std::vector<int64_t> &ip = p.permuted ? p.cindptr_h : p.indptr_h;
    for (int64_t j = 0; j < n; j++) {
        arm_ptr[j + 1] = arm_ptr[j] + std::min(m[j], sp.maxh);
        if (m[j] > sp.maxh) {
            big.push_back((int)j);
            pool_ptr.push_back(pool_ptr.back() + (ip[j + 1] - ip[j]));
        }
    }
    upload(sc.arm_ptr, arm_ptr, s);
    sc.arm_idx.alloc(sizeof(int) * std::max<int64_t>(arm_ptr[n], 1));
    sc.arm_val.alloc(sizeof(double) * std::max<int64_t>(arm_ptr[n], 1));
    k_arm_fill<T><<<nb8(n), 256, 0, s>>>(g, V, sp.thresh, sp.maxh, sc.m.as<int>(), sc.arm_ptr.as<int64_t>(),
                                         sc.arm_idx.as<int>(), sc.arm_val.as<double>());
    LB_LAUNCH_CHECK();
    if (!big.empty()) {
        upload(sc.big, big, s);
        upload(sc.pool_ptr, pool_ptr, s);
        sc.pool.alloc(sizeof(double) * pool_ptr.back());
        k_arm_big<T><<<(unsigned)big.size(), 256, 0, s>>>(g, V, sp.thresh, sp.maxh, sc.big.as<int>(),
                                                          sc.pool_ptr.as<int64_t>(), sc.pool.as<double>(),
                                                          sc.arm_ptr.as<int64_t>(), sc.arm_idx.as<int>(),
                                                          sc.arm_val.as<double>());
        LB_LAUNCH_CHECK();
    }
    PairArgs pa{};
    pa.cs = (n + sp.nchunk - 1) / sp.nchunk;
    pa.nb = sp.nbins;
    pa.vtol = sp.vtol;
    pa.a_ptr = sc.arm_ptr.as<int64_t>();
    pa.a_idx = sc.arm_idx.as<int>();
    pa.a_val = sc.arm_val.as<double>();
    // family 0: pairs of arms
    if (sp.want0) {
        pa.family = 0;
        pa.b_ptr = pa.a_ptr;
        pa.b_idx = pa.a_idx;
        pa.b_val = pa.a_val;
        run_pairs<T>(p, g, V, pa, sp.nchunk, sp.cap0, sc, p.sep_tri[0], p.sep_val[0], s);
    } else {
        p.sep_tri[0].clear();
        p.sep_val[0].clear();
    }
    // family 1: arms x second arms from the walk
    if (sp.want1) {
        sc.kcnt.alloc(sizeof(int) * n);
        const unsigned wg = (unsigned)std::min<int64_t>(n, (int64_t)p.ctx->c.num_sms * 16);
        k_walk<T, 0><<<wg, 128, 0, s>>>(g, V, sp.thresh, sp.hub2, sp.cap2, sp.maxk, sc.m.as<int>(),
                                        sc.arm_ptr.as<int64_t>(), sc.arm_idx.as<int>(), sc.kcnt.as<int>(), nullptr,
                                        nullptr, nullptr);
        LB_LAUNCH_CHECK();
        std::vector<int> kc(n);
        LB_CUDA(cudaMemcpyAsync(kc.data(), sc.kcnt.ptr, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
        std::vector<int64_t> k_ptr(n + 1, 0);
        for (int64_t j = 0; j < n; j++) k_ptr[j + 1] = k_ptr[j] + kc[j];
        upload(sc.k_ptr, k_ptr, s);
        sc.k_idx.alloc(sizeof(int) * std::max<int64_t>(k_ptr[n], 1));
        sc.k_val.alloc(sizeof(double) * std::max<int64_t>(k_ptr[n], 1));
        k_walk<T, 1><<<wg, 128, 0, s>>>(g, V, sp.thresh, sp.hub2, sp.cap2, sp.maxk, sc.m.as<int>(),
                                        sc.arm_ptr.as<int64_t>(), sc.arm_idx.as<int>(), sc.kcnt.as<int>(),
                                        sc.k_ptr.as<int64_t>(), sc.k_idx.as<int>(), sc.k_val.as<double>());
        LB_LAUNCH_CHECK();
        pa.family = 1;
        pa.b_ptr = sc.k_ptr.as<int64_t>();
        pa.b_idx = sc.k_idx.as<int>();
        pa.b_val = sc.k_val.as<double>();
        run_pairs<T>(p, g, V, pa, sp.nchunk, sp.cap1, sc, p.sep_tri[1], p.sep_val[1], s);
    } else {
        p.sep_tri[1].clear();
        p.sep_val[1].clear();
    }
}

void separate_run(Problem &p, const SepParams &sp, cudaStream_t s) {
    LB_CHECK(sp.hub2 * sp.cap2 <= WALK_CAP, LB_ERR_INVALID, "hub2 * cap2 must be at most 2048");
    LB_CHECK(sp.nbins >= 1 && sp.nbins <= 2048, LB_ERR_INVALID, "nbins must be in [1, 2048]");
    if (p.permuted && p.cindptr_h.empty()) {
        // caller-numbered CSR and the caller -> internal row map, kept for separation
        const int64_t n = p.n;
        std::vector<int> inv(n);
        for (int64_t i = 0; i < n; i++) inv[i] = (int)p.inv_h[i];
        upload(p.inv_d, inv, s);
        p.cindptr_h.assign(n + 1, 0);
        for (int64_t i = 0; i < n; i++) {
            const int64_t k = p.inv_h[i];
            p.cindptr_h[i + 1] = p.cindptr_h[i] + (p.indptr_h[k + 1] - p.indptr_h[k]);
        }
        std::vector<int> idx_int(p.nnz), cidx(p.nnz);
        LB_CUDA(cudaMemcpy(idx_int.data(), p.indices.ptr, sizeof(int) * p.nnz, cudaMemcpyDeviceToHost));
        for (int64_t i = 0; i < n; i++) {
            const int64_t k = p.inv_h[i];
            int64_t o = p.cindptr_h[i];
            for (int64_t e = p.indptr_h[k]; e < p.indptr_h[k + 1]; e++) cidx[o++] = (int)p.order_h[idx_int[e]];
            std::sort(cidx.begin() + p.cindptr_h[i], cidx.begin() + p.cindptr_h[i + 1]);
        }
        upload(p.cindptr, p.cindptr_h, s);
        upload(p.cindices, cidx, s);
    }
    if (p.vdtype == LB_F64)
        separate_typed<double>(p, sp, s);
    else if (p.vdtype == LB_F32)
        separate_typed<float>(p, sp, s);
    else
        separate_typed<__nv_bfloat16>(p, sp, s);
}

}  // namespace lb
