// VCS working-set separation on the GPU (vcsops.py:333-414 _sep_rows / _sep_rows1 / separate).
//
// Every entry (i, R) outside level's working set with mean violation xbar = s' / vol(R minus i) < -tol is a
// candidate, where s' = v_i . Y_R - [R = R(i)] d_i and vol(R minus i) = vol_R - [R = R(i)] d_i must be > 0; its score
// is wv rq_R s'^2 (pen), -xbar (mean) or -d_i s' (mass), and the nadd best are kept.
//
// The products v_i . Y_R form an n x P x r contraction (the reference's chunked BLAS G = V Y^T): it runs here as
// 64 x 64 register-tiled FP64 tiles (the scores decide a selection, so they are kept in FP64; ties are broken by
// (row, cluster)).  The selection is a radix select on the bits of the positive FP64 scores: one pass counts the
// candidates and the reference's statistics and histograms the top 12 bits, two more passes refine the threshold
// bin by 12 bits each, and a last pass writes the candidates at or above the 36-bit threshold, which are then sorted
// exactly (score descending, then row and cluster ascending) and cut to nadd.  Each pass recomputes the tiles (no
// n x P intermediate is stored).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "lb_internal.cuh"

namespace lb {
namespace {

constexpr int TR = 64, TC = 64, KC = 16;   // rows x clusters of a tile, dimensions per shared-memory chunk
constexpr int HB = 12, NB = 1 << HB;      // histogram bits per pass
typedef unsigned long long u64;

template <typename T> __device__ __forceinline__ double to_d(T x) { return (double)x; }
template <> __device__ __forceinline__ double to_d(__nv_bfloat16 x) { return (double)__bfloat162float(x); }

template <typename T> struct VsepArgs {
    int64_t n;
    int P, r, ld, mode;
    const T *V;
    const double *Y, *d, *vol, *rq;
    const int *lab;
    const int64_t *ptr;
    const int *col;
    double tol, wv;
    // pass 0: statistics + histogram of key bits [52, 64); pass 1, 2: histogram of bits [shift, shift + 12) of the
    // candidates whose key >> (shift + 12) == prefix; pass 3: write candidates with key >> 28 >= prefix
    int pass, shift;
    u64 prefix;
    u64 *hist;
    double *stats;
    u64 *wcount;
    int64_t *out_idx;
    double *out_score;
    int64_t cap;
};

__device__ __forceinline__ bool in_ws(const int64_t *ptr, const int *col, int64_t i, int R) {
    int64_t lo = ptr[i], hi = ptr[i + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int c = col[mid];
        if (c == R) return true;
        if (c < R) lo = mid + 1; else hi = mid;
    }
    return false;
}

// Persistent blocks of 16 x 16 threads; thread (tx, ty) owns rows i0 + ty + 16 a and clusters c0 + tx + 16 b,
// a, b = 0..3 (interleaved so that a warp reads consecutive shared-memory words).
template <typename T> __global__ void __launch_bounds__(256) k_vsep(VsepArgs<T> a) {
    __shared__ double Vs[KC][TR];
    __shared__ double Ys[KC][TC];
    __shared__ unsigned int h[NB];
    __shared__ double red[4][8];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, tid = threadIdx.x;
    const bool counting = a.pass < 3;
    if (counting)
        for (int b = tid; b < NB; b += 256) h[b] = 0;
    double nv = 0, mv = 0, nw = 0, mw = 0;
    const int64_t nrt = (a.n + TR - 1) / TR;
    const int64_t nct = (a.P + TC - 1) / TC;
    const int nkc = (a.r + KC - 1) / KC;
    for (int64_t t = blockIdx.x; t < nrt * nct; t += gridDim.x) {
        const int64_t i0 = (t / nct) * TR;
        const int c0 = (int)(t % nct) * TC;
        double acc[4][4];
#pragma unroll
        for (int x = 0; x < 4; x++)
#pragma unroll
            for (int y = 0; y < 4; y++) acc[x][y] = 0.0;
        for (int kc = 0; kc < nkc; kc++) {
            __syncthreads();
            for (int e = tid; e < KC * TR; e += 256) {
                const int rr = e / KC, q = e % KC, qq = kc * KC + q;
                const int64_t i = i0 + rr;
                Vs[q][rr] = (i < a.n && qq < a.r) ? to_d(a.V[i * a.ld + qq]) : 0.0;
                const int c = c0 + rr;
                Ys[q][rr] = (c < a.P && qq < a.r) ? a.Y[(int64_t)c * a.ld + qq] : 0.0;
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < KC; q++) {
                double vr[4], yc[4];
#pragma unroll
                for (int x = 0; x < 4; x++) vr[x] = Vs[q][ty + 16 * x];
#pragma unroll
                for (int y = 0; y < 4; y++) yc[y] = Ys[q][tx + 16 * y];
#pragma unroll
                for (int x = 0; x < 4; x++)
#pragma unroll
                    for (int y = 0; y < 4; y++) acc[x][y] = fma(vr[x], yc[y], acc[x][y]);
            }
        }
        // epilogue: candidate test, statistics, histogram or write
#pragma unroll
        for (int x = 0; x < 4; x++) {
            const int64_t i = i0 + ty + 16 * x;
            if (i >= a.n) continue;
            const double di = a.d[i];
            const int Ri = a.lab[i];
#pragma unroll
            for (int y = 0; y < 4; y++) {
                const int R = c0 + tx + 16 * y;
                if (R >= a.P) continue;
                double s = acc[x][y], vR = a.vol[R];
                if (R == Ri) {
                    s = s - di;
                    vR = vR - di;
                }
                if (vR <= 0.0) continue;
                const double xb = s / vR;
                if (xb >= -a.tol) continue;
                const bool inws = in_ws(a.ptr, a.col, i, R);
                if (a.pass == 0) {
                    nv += 1.0;
                    mv += -di * s;
                    if (inws) {
                        nw += 1.0;
                        mw += -di * s;
                    }
                }
                if (inws) continue;
                const double sc = a.mode == 0 ? a.wv * a.rq[R] * s * s : (a.mode == 1 ? -xb : -di * s);
                if (!(sc > 0.0)) continue;
                const u64 key = (u64)__double_as_longlong(sc);
                if (a.pass == 0) {
                    atomicAdd(&h[key >> 52], 1u);
                } else if (a.pass < 3) {
                    if ((key >> (a.shift + HB)) == a.prefix) atomicAdd(&h[(key >> a.shift) & (NB - 1)], 1u);
                } else if ((key >> 28) >= a.prefix) {
                    const u64 pos = atomicAdd(a.wcount, 1ull);
                    if ((int64_t)pos < a.cap) {
                        a.out_idx[pos] = i * a.P + R;
                        a.out_score[pos] = sc;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (counting)
        for (int b = tid; b < NB; b += 256)
            if (h[b]) atomicAdd(a.hist + b, (u64)h[b]);
    if (a.pass == 0) {
        double v[4] = {nv, mv, nw, mw};
#pragma unroll
        for (int k = 0; k < 4; k++)
            for (int o = 16; o; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        const int w = tid >> 5, lane = tid & 31;
        if (lane == 0)
            for (int k = 0; k < 4; k++) red[k][w] = v[k];
        __syncthreads();
        if (tid < 4) {
            double sum = 0;
            for (int k = 0; k < 8; k++) sum += red[tid][k];
            if (sum != 0.0) atomicAdd(a.stats + tid, sum);
        }
    }
}

// highest bin b with cum_above + hist[b] >= need (cum_above = sum of the bins above b)
int pick_bin(const std::vector<u64> &hist, int64_t need, int64_t *above) {
    int64_t cum = 0;
    for (int b = NB - 1; b >= 0; b--) {
        if (cum + (int64_t)hist[b] >= need) {
            *above = cum;
            return b;
        }
        cum += (int64_t)hist[b];
    }
    *above = cum;
    return 0;
}

template <typename T>
void vsep_typed(Problem &p, VcsLevel &lv, int64_t nadd, double tol, int mode, int64_t *count, double *stats,
                cudaStream_t s, bool to_host) {
    vcs_cluster_sums(p, lv, s);
    DBuf &hist = p.scratch("lb_vsep:195:hist"), &st = p.scratch("lb_vsep:195:st"), &wc = p.scratch("lb_vsep:195:wc");
    hist.alloc(sizeof(u64) * NB);
    st.alloc(sizeof(double) * 4);
    wc.alloc(sizeof(u64));
    LB_CUDA(cudaMemsetAsync(st.ptr, 0, sizeof(double) * 4, s));
    VsepArgs<T> a{};
    a.n = p.n;
    a.P = lv.P;
    a.r = p.r;
    a.ld = p.ld;
    a.mode = mode;
    a.V = p.V.as<T>();
    a.Y = lv.Y.as<double>();
    a.d = p.d.as<double>();
    a.vol = lv.vol.as<double>();
    a.rq = lv.rq.as<double>();
    a.lab = lv.lab.as<int>();
    a.ptr = lv.ptr.as<int64_t>();
    a.col = lv.col.as<int>();
    a.tol = tol;
    a.wv = lv.wv;
    a.hist = hist.as<u64>();
    a.stats = st.as<double>();
    a.wcount = wc.as<u64>();
    int bps = 0;
    LB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_vsep<T>, 256, 0));
    const int64_t tiles = ((p.n + TR - 1) / TR) * ((lv.P + TC - 1) / TC);
    const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)p.ctx->c.num_sms * std::max(bps, 1)));
    std::vector<u64> hh(NB);
    auto run_pass = [&](int pass, int shift, u64 prefix) {
        LB_CUDA(cudaMemsetAsync(hist.ptr, 0, sizeof(u64) * NB, s));
        a.pass = pass;
        a.shift = shift;
        a.prefix = prefix;
        k_vsep<T><<<grid, 256, 0, s>>>(a);
        LB_LAUNCH_CHECK();
        p.launches++;
        if (pass < 3) {
            LB_CUDA(cudaMemcpyAsync(hh.data(), hist.ptr, sizeof(u64) * NB, cudaMemcpyDeviceToHost, s));
            LB_CUDA(cudaStreamSynchronize(s));
        }
    };
    // pass 0: all candidates
    run_pass(0, 52, 0);
    double sh[4];
    LB_CUDA(cudaMemcpy(sh, st.ptr, sizeof(sh), cudaMemcpyDeviceToHost));
    if (stats) std::memcpy(stats, sh, sizeof(sh));
    int64_t total = 0;
    for (u64 c : hh) total += (int64_t)c;
    u64 prefix36 = 0;
    int64_t expect = total;
    if (total > nadd && nadd > 0) {
        int64_t above = 0, above_all = 0, need = nadd;
        const int b1 = pick_bin(hh, need, &above);
        above_all += above;
        need -= above;
        run_pass(1, 40, (u64)b1);
        const int b2 = pick_bin(hh, need, &above);
        above_all += above;
        need -= above;
        run_pass(2, 28, ((u64)b1 << HB) | (u64)b2);
        const int b3 = pick_bin(hh, need, &above);
        above_all += above;
        prefix36 = ((u64)b1 << (2 * HB)) | ((u64)b2 << HB) | (u64)b3;
        expect = above_all + (int64_t)hh[b3];
    }
    p.vsep_idx.clear();
    p.vsep_score.clear();
    p.vsep_dev_count = 0;
    if (nadd <= 0 || total == 0) {
        *count = 0;
        return;
    }
    DBuf &idx = p.scratch("lb_vsep:268:idx"), &sc = p.scratch("lb_vsep:268:sc"), &idx2 = p.scratch("lb_vsep:268:idx2"),
         &sc2 = p.scratch("lb_vsep:268:sc2"), &tmp = p.scratch("lb_vsep:268:tmp");
    idx.alloc(sizeof(int64_t) * expect);
    sc.alloc(sizeof(double) * expect);
    idx2.alloc(sizeof(int64_t) * expect);
    sc2.alloc(sizeof(double) * expect);
    LB_CUDA(cudaMemsetAsync(wc.ptr, 0, sizeof(u64), s));
    a.out_idx = idx.as<int64_t>();
    a.out_score = sc.as<double>();
    a.cap = expect;
    run_pass(3, 28, prefix36);
    u64 written = 0;
    LB_CUDA(cudaMemcpyAsync(&written, wc.ptr, sizeof(u64), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    LB_CHECK((int64_t)written == expect, LB_ERR_NUMERIC, "VCS separation: candidate count changed between passes");
    // exact order: (row, cluster) ascending, then a stable sort by score descending
    const int ne = (int)expect;
    size_t tb = 0, tb2 = 0;
    LB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, idx.as<int64_t>(), idx2.as<int64_t>(), sc.as<double>(),
                                            sc2.as<double>(), ne, 0, 64, s));
    LB_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb2, sc2.as<double>(), sc.as<double>(),
                                                      idx2.as<int64_t>(), idx.as<int64_t>(), ne, 0, 64, s));
    tmp.alloc(std::max(tb, tb2));
    LB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, idx.as<int64_t>(), idx2.as<int64_t>(), sc.as<double>(),
                                            sc2.as<double>(), ne, 0, 64, s));
    LB_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.ptr, tb2, sc2.as<double>(), sc.as<double>(),
                                                      idx2.as<int64_t>(), idx.as<int64_t>(), ne, 0, 64, s));
    const int64_t keep = std::min<int64_t>(nadd, expect);
    p.vsep_P = lv.P;
    *count = keep;
    if (!to_host) {
        std::swap(p.vsep_dev.ptr, idx.ptr);
        std::swap(p.vsep_dev.owner, idx.owner);
        std::swap(p.vsep_dev.bytes, idx.bytes);
        p.vsep_dev_count = keep;
        return;
    }
    p.vsep_idx.resize(keep);
    p.vsep_score.resize(keep);
    LB_CUDA(cudaMemcpyAsync(p.vsep_idx.data(), idx.ptr, sizeof(int64_t) * keep, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaMemcpyAsync(p.vsep_score.data(), sc.ptr, sizeof(double) * keep, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
}

struct Positive {
    __host__ __device__ int64_t operator()(double x) const { return x > 0.0 ? 1 : 0; }
};

}  // namespace

void vcs_sig_stats_run(Problem &p, int level, double *sum, int64_t *active, cudaStream_t s) {
    VcsLevel &lv = *p.vlev[level];
    *sum = 0.0;
    *active = 0;
    if (lv.nnz == 0) return;
    DBuf &out = p.scratch("lb_vsep:321:out"), &tmp = p.scratch("lb_vsep:321:tmp");
    out.alloc(sizeof(double) + sizeof(int64_t));
    double *dsum = out.as<double>();
    int64_t *dcnt = reinterpret_cast<int64_t *>(out.as<char>() + sizeof(double));
    size_t tb = 0, tb2 = 0;
    cub::TransformInputIterator<int64_t, Positive, const double *> pos(lv.sig.as<double>(), Positive());
    LB_CUDA(cub::DeviceReduce::Sum(nullptr, tb, lv.sig.as<double>(), dsum, (int)lv.nnz, s));
    LB_CUDA(cub::DeviceReduce::Sum(nullptr, tb2, pos, dcnt, (int)lv.nnz, s));
    tmp.alloc(std::max(tb, tb2));
    LB_CUDA(cub::DeviceReduce::Sum(tmp.ptr, tb, lv.sig.as<double>(), dsum, (int)lv.nnz, s));
    LB_CUDA(cub::DeviceReduce::Sum(tmp.ptr, tb2, pos, dcnt, (int)lv.nnz, s));
    LB_CUDA(cudaMemcpyAsync(sum, dsum, sizeof(double), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaMemcpyAsync(active, dcnt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
}

void vcs_separate_run(Problem &p, int level, int64_t nadd, double tol, int mode, int64_t *count, double *stats,
                      cudaStream_t s, bool to_host) {
    VcsLevel &lv = *p.vlev[level];
    LB_CHECK((int64_t)lv.P * p.n < ((int64_t)1 << 62), LB_ERR_INVALID, "n * P too large");
    if (p.vdtype == LB_F64)
        vsep_typed<double>(p, lv, nadd, tol, mode, count, stats, s, to_host);
    else if (p.vdtype == LB_F32)
        vsep_typed<float>(p, lv, nadd, tol, mode, count, stats, s, to_host);
    else
        vsep_typed<__nv_bfloat16>(p, lv, nadd, tol, mode, count, stats, s, to_host);
}

}  // namespace lb
