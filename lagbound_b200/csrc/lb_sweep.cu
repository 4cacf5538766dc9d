// Batched Gauss-Seidel sweeps of the augmented Lagrangian (sm_100a): the inner loop of the reference's solver
// (src/lagbound/_core/alm_vcs.py:1360-1436 sweeps(), row step batch_step6 256-351, pair rows pair_all 378-415,
// Kq kq_level 417-428, aggregate updates _acc_rows 430-438; VCS terms vcsops.py:94-213).
//
// Per sweep: z = d^T V, cluster sums Y of every pair and VCS level, Kq per pair level (trace rule), the VCS
// start-of-sweep effective multipliers stZ with Z and cnt.  Per batch (a slice of the caller's row permutation):
//   k_vcs_pre      GX_i, KX_i of the VCS levels (vcs_pre)
//   k_mark/k_pair_rows   fresh M_Q = sum_R pp_QR Y_R and pp_QQ for the clusters of the batch (pair_all)
//   k_step         the row step of every batch row from the pre-batch V (Jacobi within a batch; the reference reads
//                  neighbour rows Hogwild-style while they change), V_new and DD = d_i (v_new - v_old)
//   k_commit       V[rows] = V_new, z += sum DD, Y[lab] += DD (FP64 atomics)
//   k_vcs_post     new effective multipliers of the moved rows, Z and cnt updates, stZ (vcs_post)
// The aggregate updates use FP64 atomics, so sweeps are not bit-reproducible run to run (the reference's are not
// either: its batches update V in place from many threads).
#include <math.h>

#include <algorithm>
#include <type_traits>

#include "lb_internal.cuh"
#include "lb_segsum.cuh"

namespace lb {
namespace {

constexpr unsigned FULLW = 0xffffffffu;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// entries in flight per lane group in the batch kernels' working-set loops (a lane holds VU x EPL doubles of Y)
template <typename T> constexpr int VU = 16 / VT<T>::EPL;
// neighbour rows (SU) and triangle records (TU, two rows each) in flight per lane group in k_step
constexpr int SU = 8, TU = 4;
// EPL doubles of an FP64 row (16-byte aligned: EPL is even)
template <int EPL> __device__ __forceinline__ void load_y(const double *p, double (&x)[EPL]) {
#pragma unroll
    for (int k = 0; k < EPL; k += 2) {
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p + k));
        x[k] = v.x;
        x[k + 1] = v.y;
    }
}

template <int NCH> __device__ __forceinline__ double grp_sum(double x) {
#pragma unroll
    for (int off = 1; off < NCH; off <<= 1) x += __shfl_xor_sync(FULLW, x, off);
    return x;
}

static inline unsigned nblk(int64_t work, int per) { return (unsigned)((work + per - 1) / per); }
// warps per block of the per-batch row kernels: a batch holds a few hundred rows, so small blocks spread them over
// all SMs
// warps per row of the per-batch row kernels (one row per block): enough to fill the SMs with the batch's rows,
// so a high-degree row is spread over up to 8 warps
static inline int batch_warps(int64_t nr, int nsm) {
    const int64_t w = (int64_t)nsm * 32 / std::max<int64_t>(nr, 1);
    return (int)std::max<int64_t>(1, std::min<int64_t>(8, w));
}

// ------------------------------------------------------------------------------------------------ per sweep
// Kq_Q = 2 rho (sum_R [pp_QR > 0] r_QR |Y_R|^2 + [pp_QQ > 0] r_QQ |Y_Q|^2), pp = sig - rho r h, h = Y_Q.Y_R - [Q=R]dsq
// (alm_vcs.py:417-428 kq_level, r = rq rq^T w).  Block per Q.
__global__ void __launch_bounds__(256) k_kq(int P, int ld, const double *__restrict__ Y, const double *__restrict__ sig,
                                            const double *__restrict__ rq, const double *__restrict__ dsq, double w,
                                            double rho, double *__restrict__ kq) {
    __shared__ double sh[256];
    __shared__ double yq[512];
    const int Q = blockIdx.x;
    for (int c = threadIdx.x; c < ld; c += blockDim.x) yq[c] = Y[(int64_t)Q * ld + c];
    __syncthreads();
    double s = 0.0, dg = 0.0;
    for (int R = threadIdx.x; R < P; R += blockDim.x) {
        const double *yr = Y + (int64_t)R * ld;
        double h = 0.0, y2 = 0.0;
        for (int c = 0; c < ld; c++) {
            h += yq[c] * yr[c];
            y2 += yr[c] * yr[c];
        }
        if (R == Q) h -= dsq[Q];
        const double r = (rq[Q] * rq[R]) * w;
        const double p = sig[(int64_t)Q * P + R] - rho * r * h;
        if (p > 0.0) {
            s += r * y2;
            if (R == Q) dg = r * y2;
        }
    }
    sh[threadIdx.x] = s + dg;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) sh[threadIdx.x] += sh[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) kq[Q] = 2 * rho * sh[0];
}

// VCS start-of-sweep effective multipliers (vcsops.py:94-108 vcs_sigt): warp per row.
template <typename T, int NCH>
__global__ void __launch_bounds__(256) k_vcs_sigt(int64_t n, int ld, const T *__restrict__ V, const double *__restrict__ d,
                                                  const int *__restrict__ lab, const double *__restrict__ Y,
                                                  const int64_t *__restrict__ ptr, const int *__restrict__ col,
                                                  const double *__restrict__ sig, const double *__restrict__ rq,
                                                  double wv, double rho, double *__restrict__ out) {
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int64_t i = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (i >= n) return;
    const int64_t a = ptr[i], b = ptr[i + 1];
    if (b == a) return;
    const double di = d[i];
    const int Ri = lab[i];
    double vi[EPL];
    load_d<T>(V + i * ld + ch * EPL, vi);
    for (int64_t e0 = a; e0 < b; e0 += NPW) {
        const int64_t e = e0 + sub;
        const bool act = e < b;
        const int R = act ? col[e] : 0;
        double s = 0.0;
        if (act) {
            const double *yr = Y + (int64_t)R * ld + ch * EPL;
#pragma unroll
            for (int k = 0; k < EPL; k++) s += vi[k] * yr[k];
        }
        s = grp_sum<NCH>(s);
        if (act && ch == 0) {
            if (rho <= 0.0 || di <= 0.0) {
                out[e] = sig[e];
            } else {
                const double g = (R == Ri) ? dmul(di, dsub(s, di)) : dmul(di, s);
                const double p = dsub(sig[e], dmul(dmul(rho, dmul(wv, rq[R]) / dmul(di, di)), g));
                out[e] = p > 0.0 ? p : 0.0;
            }
        }
    }
}

// cnt_R = #(stZ_e > 0) over the entries of column R (column view): warp per column, an exact integer count.
__global__ void k_vcs_cnt(int P, const int64_t *__restrict__ cptr, const int64_t *__restrict__ cent,
                          const double *__restrict__ stZ, double *__restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int R = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (R >= P) return;
    long long c = 0;
    for (int64_t q = cptr[R] + lane; q < cptr[R + 1]; q += 32) c += stZ[cent[q]] > 0.0 ? 1 : 0;
#pragma unroll
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[R] = (double)c;
}

// ------------------------------------------------------------------------------------------------ per batch
// VCS pre-batch terms (vcsops.py:127-156 vcs_pre, useY2): warp per batch row; lanes over entries (one lane group
// per entry) for the dot products, then the half-gradient GX (FP64) and curvature KX.
template <typename T, int NCH>
__global__ void __launch_bounds__(256) k_vcs_pre(int nr, const int *__restrict__ rows, int ld, const T *__restrict__ V,
                                                 const double *__restrict__ d, const int *__restrict__ lab,
                                                 const double *__restrict__ Y,
                                                 const int64_t *__restrict__ ptr, const int *__restrict__ col,
                                                 const double *__restrict__ sig, const double *__restrict__ stZ,
                                                 const int64_t *__restrict__ own, const double *__restrict__ Z,
                                                 const double *__restrict__ cnt, const double *__restrict__ rq,
                                                 double wv, double rho, double kap2, double *__restrict__ GX,
                                                 double *__restrict__ KX) {
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int idx = blockIdx.x, wid = threadIdx.x >> 5, W = blockDim.x >> 5;   // one row per block of W warps
    if (idx >= nr) return;
    const int64_t i = rows[idx];
    const double di = d[i];
    const int Ri = lab[i];
    double vi[EPL], acc[EPL];
    load_d<T>(V + i * ld + ch * EPL, vi);
#pragma unroll
    for (int k = 0; k < EPL; k++) acc[k] = 0.0;
    double kap = 0.0, pown = 0.0;
    const int64_t a = ptr[i], b = ptr[i + 1];
    // 32 entries at a time: their cluster, multiplier, rq and |Y_R|^2 loaded lane-parallel, then VU steps of one
    // entry per lane group with all VU rows Y_R in flight (group `sub` takes the entries = sub mod NPW, in order)
    for (int64_t e0 = a + 32 * wid; e0 < b; e0 += 32 * W) {   // the warps take interleaved chunks
        const int nin = (int)(b - e0 < 32 ? b - e0 : 32);
        const bool inl = lane < nin;
        const int Rl = inl ? col[e0 + lane] : 0;
        const double sgl = inl ? sig[e0 + lane] : 0.0, rql = inl ? rq[Rl] : 0.0;
        for (int u0 = 0; u0 < nin; u0 += NPW * VU<T>) {
            double yr[VU<T>][EPL];
            int R[VU<T>];
#pragma unroll
            for (int u = 0; u < VU<T>; u++) {
                const int j = u0 + u * NPW + sub;
                R[u] = __shfl_sync(FULLW, Rl, j & 31);
                if (j < nin) load_y<EPL>(Y + (int64_t)R[u] * ld + ch * EPL, yr[u]);
            }
#pragma unroll
            for (int u = 0; u < VU<T>; u++) {
                const int j = u0 + u * NPW + sub;
                const bool act = j < nin;
                const double sg = __shfl_sync(FULLW, sgl, j & 31), rqR = __shfl_sync(FULLW, rql, j & 31);
                double s = 0.0, y2R = 0.0;          // v_i . Y_R and |Y_R|^2 (useY2)
                if (act)
#pragma unroll
                    for (int k = 0; k < EPL; k++) {
                        s += vi[k] * yr[u][k];
                        y2R += yr[u][k] * yr[u][k];
                    }
                s = grp_sum<NCH>(s);
                y2R = grp_sum<NCH>(y2R);
                if (act) {
                    double p;
                    if (rho > 0.0 && di > 0.0) {
                        const double g = (R[u] == Ri) ? dmul(di, dsub(s, di)) : dmul(di, s);
                        const double rr = dmul(wv, rqR) / dmul(di, di);
                        p = dsub(sg, dmul(dmul(rho, rr), g));
                        if (p > 0.0) {
                            double y2 = y2R;
                            if (R[u] == Ri) y2 = y2 - 2 * di * s + di * di;
                            if (ch == 0) kap += rho * rr * di * di * y2;
                        } else {
                            p = 0.0;
                        }
                    } else {
                        p = sg;
                    }
                    if (R[u] == Ri) pown = p;     // same value in every lane of the group
                    if (p != 0.0)
#pragma unroll
                        for (int k = 0; k < EPL; k++) acc[k] += p * yr[u][k];
                }
            }
        }
    }
    // combine the lane groups: acc over groups with the same chunk, kap and pown over the warp
#pragma unroll
    for (int off = NCH; off < 32; off <<= 1) {
#pragma unroll
        for (int k = 0; k < EPL; k++) acc[k] += __shfl_xor_sync(FULLW, acc[k], off);
    }
    for (int off = 16; off; off >>= 1) kap += __shfl_xor_sync(FULLW, kap, off);
    // pown: the group that held the own entry has it; take the maximum magnitude over groups (others are 0)
    for (int off = NCH; off < 32; off <<= 1) {
        const double o = __shfl_xor_sync(FULLW, pown, off);
        if (o != 0.0) pown = o;
    }
    if (W > 1) {   // the warps' sums through shared memory, in warp order; warp 0 finishes the row
        extern __shared__ __align__(16) double rowsh[];   // W x (ld + 2)
        double *red = rowsh + wid * (ld + 2);
        if (sub == 0)
#pragma unroll
            for (int k = 0; k < EPL; k++) red[ch * EPL + k] = acc[k];
        if (lane == 0) {
            red[ld] = kap;
            red[ld + 1] = pown;
        }
        __syncthreads();
        if (wid != 0) return;
#pragma unroll
        for (int k = 0; k < EPL; k++) {
            double t = 0.0;
            for (int w = 0; w < W; w++) t += rowsh[w * (ld + 2) + ch * EPL + k];
            acc[k] = t;
        }
        kap = 0.0;
        pown = 0.0;
        for (int w = 0; w < W; w++) {
            kap += rowsh[w * (ld + 2) + ld];
            const double o = rowsh[w * (ld + 2) + ld + 1];
            if (o != 0.0) pown = o;
        }
    }
    const int64_t eo = own[i];
    const double sz = eo >= 0 ? stZ[eo] : 0.0;
    if (sub == 0) {
#pragma unroll
        for (int k = 0; k < EPL; k++) {
            const int c = ch * EPL + k;
            GX[(int64_t)idx * ld + c] += 0.5 * di * (acc[k] - pown * di * vi[k]) + 0.5 * di * (Z[(int64_t)Ri * ld + c] - sz * di * vi[k]);
        }
    }
    if (lane == 0) {
        if (rho > 0.0) kap += kap2 * rho * di * di * wv * rq[Ri] * (cnt[Ri] - (sz > 0.0 ? 1.0 : 0.0));
        KX[idx] += kap;
    }
}

// Touched clusters of the batch (one list per pair level, concatenated over levels): mark + compact.
__global__ void k_mark(int nr, const int *__restrict__ rows, const int *__restrict__ lab, int off,
                       unsigned *__restrict__ mark, unsigned stamp, int *__restrict__ list, int *__restrict__ count) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nr) return;
    const int Q = lab[rows[idx]];
    if (atomicExch(mark + off + Q, stamp) != stamp) {
        const int pos = atomicAdd(count, 1);
        list[pos] = off + Q;
    }
}

// Fresh pair rows (alm_vcs.py:378-415 pair_all) of the touched clusters: p_QR = max(0, sig_QR - rho r_QR h_QR),
// h_QR = Y_Q.Y_R - [Q=R] dsq_Q, r_QR = rq_Q rq_R w (p = sig at rho 0); M_Q = sum_R p_QR Y_R, pdiag_Q = p_QQ.
// Block per PR_Q touched clusters and one of gridDim.y contiguous ranges of R (partial rows into Mpart, summed in
// range order by k_pair_combine).  The range's Y rows stream through shared memory in tiles of rt rows (two buffers
// filled by asynchronous copies, the next tile in flight while one is used), each tile serving all PR_Q clusters of
// the block.  Each thread sums a 2 x 2 tile of M (two clusters, two columns) over one of S = 256 / ld interleaved
// slices of R, in R order; the slices are then added in order (FP64).
constexpr int PR_Q = 4;
constexpr int PR_MAXSPLIT = 16;         // R ranges per cluster group

__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Y-tile rows for a row width: two tiles within 96 KB, at most 128 rows
__host__ __device__ constexpr int pair_tile_rows(int ld) {
    return (48 * 1024) / ((ld + 2) * 8) > 128 ? 128 : ((48 * 1024) / ((ld + 2) * 8) < 16 ? 16 : (48 * 1024) / ((ld + 2) * 8));
}

template <int LD>
__global__ void __launch_bounds__(256) k_pair_rows(const int *__restrict__ list, const int *__restrict__ count,
                                                   int lo, int P, const double *__restrict__ Y,
                                                   const double *__restrict__ sig, const double *__restrict__ rq,
                                                   const double *__restrict__ dsq, double w, double rho,
                                                   double *__restrict__ Mpart, double *__restrict__ pdiag) {
    extern __shared__ __align__(16) double shp[];
    constexpr int ld = LD, rt = pair_tile_rows(LD);        // row width and tile rows known at compile time
    constexpr int ys = ld + 2;                             // tile row stride: 16-byte rows, staggered banks
    double *yq = shp, *ytb = yq + PR_Q * ld, *pt = ytb + 2 * rt * ys;
    __shared__ int qs[PR_Q];
    const int tid = threadIdx.x, nth = blockDim.x;
    const int t0 = blockIdx.x * PR_Q, cnt = *count;
    if (t0 >= cnt) return;
    const int nq = min(PR_Q, cnt - t0);
    // this block's range of R: whole tiles, split as evenly as the tiles allow
    const int ntiles = (P + rt - 1) / rt, sp = blockIdx.y, ns = gridDim.y;
    const int Rb = (int)((int64_t)ntiles * sp / ns) * rt, Re = min(P, (int)((int64_t)ntiles * (sp + 1) / ns) * rt);
    auto load_tile = [&](int buf, int R0) {
        constexpr int cpr = ld >> 1;                      // 16-byte chunks per row (ld is even)
        const int nr = min(rt, Re - R0);
        double *dst = ytb + buf * rt * ys;
        for (int j = tid; j < nr * cpr; j += nth) {
            const int r = j / cpr, c2 = 2 * (j % cpr);
            cp_async16(dst + r * ys + c2, Y + (int64_t)(R0 + r) * ld + c2);
        }
        cp_async_commit();
    };
    if (Rb < Re) load_tile(0, Rb);
    if (tid < PR_Q) qs[tid] = tid < nq ? list[t0 + tid] - lo : 0;
    __syncthreads();
    for (int j = tid; j < PR_Q * ld; j += nth) {
        const int q = j / ld, c = j % ld;
        yq[j] = q < nq ? Y[(int64_t)qs[q] * ld + c] : 0.0;
    }
    // M items: (cluster pair qp, column pair cp, slice sl of the tile rows); S = 256 / ld slices
    constexpr int hl = ld >> 1, S = 256 / ld > 1 ? 256 / ld : 1, items = ld * S;
    const int it_cp = tid % hl, it_qp = (tid / hl) & 1, it_sl = tid / ld;
    const bool it_on = tid < items && 2 * it_qp < nq;
    double m00 = 0.0, m01 = 0.0, m10 = 0.0, m11 = 0.0;
    for (int t = 0, R0 = Rb; R0 < Re; t++, R0 += rt) {
        const int nr = min(rt, Re - R0);
        if (R0 + rt < Re) load_tile((t + 1) & 1, R0 + rt);
        else cp_async_commit();                            // an empty group: the wait below counts uniformly
        cp_async_wait1();                                  // this thread's copies of tile t have landed
        __syncthreads();                                   // everyone's copies (and yq) visible
        const double *yt = ytb + (t & 1) * rt * ys;
        // p for (cluster pair, R): both dot products over the columns in order, two columns per shared load
        for (int j = tid; j < (PR_Q / 2) * rt; j += nth) {
            const int r = j % rt, qp = j / rt, q0 = 2 * qp, q1 = q0 + 1;
            if (r >= nr || q0 >= nq) continue;
            double h0 = 0.0, h1 = 0.0;
            if (rho > 0.0) {
                // even and odd columns in separate chains (four independent FMA chains), added at the end
                const double2 *b2 = reinterpret_cast<const double2 *>(yt + r * ys);
                const double2 *a0 = reinterpret_cast<const double2 *>(yq + q0 * ld);
                const double2 *a1 = reinterpret_cast<const double2 *>(yq + q1 * ld);
                double h0o = 0.0, h1o = 0.0;
#pragma unroll 8
                for (int c2 = 0; c2 < hl; c2++) {
                    const double2 y = b2[c2], x0 = a0[c2], x1 = a1[c2];
                    h0 += x0.x * y.x;
                    h0o += x0.y * y.y;
                    h1 += x1.x * y.x;
                    h1o += x1.y * y.y;
                }
                h0 += h0o;
                h1 += h1o;
            }
            const int R = R0 + r;
#pragma unroll
            for (int v = 0; v < 2; v++) {
                const int q = q0 + v;
                if (q >= nq) continue;
                const int Q = qs[q];
                double p;
                if (rho > 0.0) {
                    double h = v ? h1 : h0;
                    if (R == Q) h -= dsq[Q];
                    p = sig[(int64_t)Q * P + R] - (rho * ((rq[Q] * rq[R]) * w)) * h;
                    if (p < 0.0) p = 0.0;
                } else {
                    p = sig[(int64_t)Q * P + R];
                }
                pt[q * rt + r] = p;
                if (R == Q) pdiag[Q] = p;
            }
        }
        __syncthreads();
        // M: a 2 x 2 register tile (clusters 2qp, 2qp+1; columns 2cp, 2cp+1) over the slice's rows, in order
        if (it_on) {
            const bool two = 2 * it_qp + 1 < nq;
            const double *p0 = pt + (2 * it_qp) * rt, *p1 = two ? p0 + rt : p0;
            for (int r = it_sl; r < nr; r += S) {
                const double a = p0[r], c = two ? p1[r] : 0.0;
                if (a == 0.0 && c == 0.0) continue;
                const double2 y = reinterpret_cast<const double2 *>(yt + r * ys)[it_cp];
                m00 += a * y.x;
                m01 += a * y.y;
                m10 += c * y.x;
                m11 += c * y.y;
            }
        }
        __syncthreads();                                   // tile t and pt consumed before they are refilled
    }
    // slices summed in order through shared memory (the tile and p buffers are free now; the launch sizes them for
    // S x PR_Q x ld doubles): red[sl][q][c]
    double *red = ytb;
    if (it_on) {
        double *o = red + (size_t)it_sl * PR_Q * ld;
        o[(2 * it_qp) * ld + 2 * it_cp] = m00;
        o[(2 * it_qp) * ld + 2 * it_cp + 1] = m01;
        o[(2 * it_qp + 1) * ld + 2 * it_cp] = m10;
        o[(2 * it_qp + 1) * ld + 2 * it_cp + 1] = m11;
    }
    __syncthreads();
    // partial row of list entry t0 + q, range sp: Mpart[((t0 + q) * ns + sp) * ld + c]
    for (int j = tid; j < nq * ld; j += nth) {
        double m = 0.0;
        for (int sl = 0; sl < S; sl++) m += red[(size_t)sl * PR_Q * ld + j];
        Mpart[((int64_t)(t0 + j / ld) * ns + sp) * ld + j % ld] = m;
    }
}

// M_Q = sum of the partial rows over the R ranges, in range order
__global__ void k_pair_combine(const int *__restrict__ list, const int *__restrict__ count, int lo, int ld, int ns,
                               const double *__restrict__ Mpart, double *__restrict__ M) {
    const int cnt = *count;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < (int64_t)cnt * ld;
         j += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(j / ld), c = (int)(j % ld);
        double m = 0.0;
        for (int sp = 0; sp < ns; sp++) m += Mpart[((int64_t)t * ns + sp) * ld + c];
        M[(int64_t)(list[t] - lo) * ld + c] = m;
    }
}

// R ranges per touched-cluster group: about four blocks per SM, whole tiles per range
static inline int pair_splits(int64_t nt, int P, int ld, int nsm) {
    const int64_t groups = (nt + PR_Q - 1) / PR_Q, ntiles = (P + pair_tile_rows(ld) - 1) / pair_tile_rows(ld);
    const int64_t want = (4 * (int64_t)nsm + groups - 1) / std::max<int64_t>(groups, 1);
    return (int)std::max<int64_t>(1, std::min<int64_t>({want, ntiles, (int64_t)PR_MAXSPLIT}));
}
// shared memory: Y_Q rows, then the two tiles and the p tile, which the slice sums (S x PR_Q x ld, S = 256 / ld)
// reuse at the end
static inline size_t pair_rows_smem(int ld) {
    const size_t rt = (size_t)pair_tile_rows(ld), S = std::max(1, 256 / ld);
    return sizeof(double) * ((size_t)PR_Q * ld + std::max(2 * rt * (ld + 2) + PR_Q * rt, S * PR_Q * ld));
}

struct StepLevels {
    int npl;
    const int *plab[MAX_LEVELS];
    const double *M[MAX_LEVELS];
    const double *pdiag[MAX_LEVELS];
    const double *kq[MAX_LEVELS];
};

// Row step of batch_step6 (alm_vcs.py:256-351, production features) for the batch rows, warp per row, reading the
// pre-batch V; writes V_new rows (batch order) and DD = d_i (v_new - v_old) (FP64).
template <typename T, int NCH, bool WEIGHTED>
__global__ void __launch_bounds__(256) k_step(int nr, const int *__restrict__ rows, int64_t n, int ld,
                                              const int64_t *__restrict__ indptr, const int *__restrict__ indices,
                                              const float *__restrict__ wts, const T *__restrict__ V,
                                              const double *__restrict__ d, const double *__restrict__ z,
                                              double invL, StepLevels lv, const double *__restrict__ GX,
                                              const double *__restrict__ KX, int usevc, const int64_t *__restrict__ tptr,
                                              const int *__restrict__ tinc, const double *__restrict__ lam, double rt,
                                              double damp, T *__restrict__ Vnew, double *__restrict__ DD,
                                              T *__restrict__ Vold) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int idx = blockIdx.x, wid = threadIdx.x >> 5, W = blockDim.x >> 5;   // one row per block of W warps
    if (idx >= nr) return;
    const int64_t i = rows[idx];
    const double di = d[i];
    Acc vi[EPL];
    {
        const uint4 raw = ld_chunk(V + i * ld + ch * EPL);
        Unpack<T>::run(raw, vi);
        // the pre-batch row, for vcs_post (V changes at the commit)
        if (Vold && wid == 0 && sub == 0) *reinterpret_cast<uint4 *>(Vold + (int64_t)idx * ld + ch * EPL) = raw;
    }
    // neighbour sum
    Acc acc[EPL];
#pragma unroll
    for (int k = 0; k < EPL; k++) acc[k] = 0;
    // 32 edges at a time: neighbour ids (and weights) lane-parallel, then SU steps of one edge per lane group with
    // all SU neighbour rows in flight (group `sub` takes the edges = sub mod NPW, in order)
    const int64_t eb = indptr[i], ee = indptr[i + 1];
    for (int64_t e0 = eb + 32 * wid; e0 < ee; e0 += 32 * W) {   // the warps take interleaved chunks
        const int nin = (int)(ee - e0 < 32 ? ee - e0 : 32);
        const int jl = lane < nin ? indices[e0 + lane] : 0;
        const float wl = WEIGHTED && lane < nin ? wts[e0 + lane] : 1.0f;
        for (int u0 = 0; u0 < nin; u0 += NPW * SU) {
            uint4 raw[SU];
#pragma unroll
            for (int u = 0; u < SU; u++) {
                const int jj = u0 + u * NPW + sub;
                const int j = __shfl_sync(FULLW, jl, jj & 31);
                raw[u] = jj < nin ? ld_chunk(V + (int64_t)j * ld + ch * EPL) : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int u = 0; u < SU; u++) {
                const int jj = u0 + u * NPW + sub;
                const float wf = __shfl_sync(FULLW, wl, jj & 31);
                if (jj < nin) {
                    Acc x[EPL];
                    Unpack<T>::run(raw[u], x);
                    const Acc w = WEIGHTED ? (Acc)wf : (Acc)1;
#pragma unroll
                    for (int k = 0; k < EPL; k++) acc[k] += w * x[k];
                }
            }
        }
    }
    // triangles with pt = lam - rt (1 - tau) > 0: g -= pt q / 2, kap += rt |q|^2
    Acc accT[EPL];
#pragma unroll
    for (int k = 0; k < EPL; k++) accT[k] = 0;
    double kapT = 0.0;
    if (tptr) {
        const int64_t t0 = tptr[i], t1 = tptr[i + 1];
        // 32 incidence records at a time, lane-parallel (with their multipliers), then TU steps with both other
        // rows of each record in flight
        for (int64_t c0 = t0 + 32 * wid; c0 < t1; c0 += 32 * W) {
          const int nin = (int)(t1 - c0 < 32 ? t1 - c0 : 32);
          const bool inl = lane < nin;
          const int o1l = inl ? tinc[3 * (c0 + lane)] : 0, o2l = inl ? tinc[3 * (c0 + lane) + 1] : 0;
          const unsigned trl = inl ? (unsigned)tinc[3 * (c0 + lane) + 2] : 0u;
          const double laml = inl ? lam[trl & 0x3fffffffu] : 0.0;
          for (int u0 = 0; u0 < nin; u0 += NPW * TU) {
           uint4 r1[TU], r2[TU];
#pragma unroll
           for (int u = 0; u < TU; u++) {
               const int jj = u0 + u * NPW + sub;
               const int o1 = __shfl_sync(FULLW, o1l, jj & 31), o2 = __shfl_sync(FULLW, o2l, jj & 31);
               r1[u] = jj < nin ? ld_chunk(V + (int64_t)o1 * ld + ch * EPL) : make_uint4(0, 0, 0, 0);
               r2[u] = jj < nin ? ld_chunk(V + (int64_t)o2 * ld + ch * EPL) : make_uint4(0, 0, 0, 0);
           }
#pragma unroll
           for (int u = 0; u < TU; u++) {
            const int jj = u0 + u * NPW + sub;
            const bool act = jj < nin;
            const unsigned tr = __shfl_sync(FULLW, trl, jj & 31);
            const double lamt = __shfl_sync(FULLW, laml, jj & 31);
            Acc x1[EPL], x2[EPL];
            Unpack<T>::run(r1[u], x1);
            Unpack<T>::run(r2[u], x2);
            const unsigned role = tr >> 30;
            // (va, vb, vc) from the record: role 0 (i = a): c = o1, b = o2; role 1 (i = b): a = o1, c = o2;
            // role 2 (i = c): a = o1, b = o2
            double tau = 0.0, q2 = 0.0;
            Acc q[EPL];
#pragma unroll
            for (int k = 0; k < EPL; k++) {
                Acc va, vb, vc;
                if (role == 0) { va = vi[k]; vb = x2[k]; vc = x1[k]; }
                else if (role == 1) { va = x1[k]; vb = vi[k]; vc = x2[k]; }
                else { va = x1[k]; vb = x2[k]; vc = vi[k]; }
                tau += (double)(va * vb + vb * vc - va * vc);
                q[k] = role == 0 ? vb - vc : role == 1 ? va + vc : vb - va;
                q2 += (double)(q[k] * q[k]);
            }
            tau = grp_sum<NCH>(tau);
            q2 = grp_sum<NCH>(q2);
            if (act) {
                const double pt = lamt - rt * (1.0 - tau);
                if (pt > 0.0) {
                    const Acc h = (Acc)(0.5 * pt);
#pragma unroll
                    for (int k = 0; k < EPL; k++) accT[k] -= h * q[k];
                    if (ch == 0) kapT += rt * q2;
                }
            }
           }
          }
        }
    }
#pragma unroll
    for (int off = NCH; off < 32; off <<= 1) {
#pragma unroll
        for (int k = 0; k < EPL; k++) {
            acc[k] += __shfl_xor_sync(FULLW, acc[k], off);
            accT[k] += __shfl_xor_sync(FULLW, accT[k], off);
        }
    }
    for (int off = 16; off; off >>= 1) kapT += __shfl_xor_sync(FULLW, kapT, off);
    if (W > 1) {   // the warps' sums through shared memory (FP64), in warp order; warp 0 finishes the row
        extern __shared__ __align__(16) double rowsh[];   // W x (2 ld + 1)
        double *red = rowsh + wid * (2 * ld + 1);
        if (sub == 0)
#pragma unroll
            for (int k = 0; k < EPL; k++) {
                red[ch * EPL + k] = (double)acc[k];
                red[ld + ch * EPL + k] = (double)accT[k];
            }
        if (lane == 0) red[2 * ld] = kapT;
        __syncthreads();
        if (wid != 0) return;
#pragma unroll
        for (int k = 0; k < EPL; k++) {
            double t = 0.0, tT = 0.0;
            for (int w = 0; w < W; w++) {
                t += rowsh[w * (2 * ld + 1) + ch * EPL + k];
                tT += rowsh[w * (2 * ld + 1) + ld + ch * EPL + k];
            }
            acc[k] = (Acc)t;
            accT[k] = (Acc)tT;
        }
        kapT = 0.0;
        for (int w = 0; w < W; w++) kapT += rowsh[w * (2 * ld + 1) + 2 * ld];
    }
    // g in FP64: -(d_i/L)(z - d_i v_i) + A v + levels + GX + triangles
    double g[EPL];
    double kap = kapT;
#pragma unroll
    for (int k = 0; k < EPL; k++) {
        const int c = ch * EPL + k;
        g[k] = -(di * invL) * (z[c] - di * (double)vi[k]) + (double)acc[k] + (double)accT[k];
    }
    for (int l = 0; l < lv.npl; l++) {
        const int Q = lv.plab[l][i];
        const double pd = lv.pdiag[l][Q] * di;
        const double *mq = lv.M[l] + (int64_t)Q * ld + ch * EPL;
#pragma unroll
        for (int k = 0; k < EPL; k++) g[k] += di * (mq[k] - pd * (double)vi[k]);
        kap += di * di * lv.kq[l][Q];
    }
    if (usevc) {
#pragma unroll
        for (int k = 0; k < EPL; k++) g[k] += GX[(int64_t)idx * ld + ch * EPL + k];
        kap += KX[idx];
    }
    double gn = 0.0;
#pragma unroll
    for (int k = 0; k < EPL; k++) gn += g[k] * g[k];
    gn = grp_sum<NCH>(gn);
    const double w = 0.5 * kap + damp * sqrt(gn);
    double qn[EPL], nv = 0.0;
#pragma unroll
    for (int k = 0; k < EPL; k++) {
        qn[k] = g[k] + w * (double)vi[k];
        nv += qn[k] * qn[k];
    }
    nv = grp_sum<NCH>(nv);
    if (sub == 0) {
        if (nv <= 0.0) {
#pragma unroll
            for (int k = 0; k < EPL; k++) {
                Vnew[(int64_t)idx * ld + ch * EPL + k] = V[i * ld + ch * EPL + k];
                DD[(int64_t)idx * ld + ch * EPL + k] = 0.0;
            }
        } else {
            const double inv = 1.0 / sqrt(nv);
#pragma unroll
            for (int k = 0; k < EPL; k++) {
                const T vn = (T)(qn[k] * inv);
                Vnew[(int64_t)idx * ld + ch * EPL + k] = vn;
                // DD from the stored (rounded) new row, so the aggregates follow V exactly
                DD[(int64_t)idx * ld + ch * EPL + k] = di * ((double)(Acc)vn - (double)vi[k]);
            }
        }
    }
}

// V[rows] = V_new; z += DD; Y_l[lab_l[i]] += DD for every pair and VCS level (FP64 atomics).  Thread per element.
struct CommitLevels {
    int nl;
    const int *lab[2 * MAX_LEVELS];
    double *Y[2 * MAX_LEVELS];
};
template <typename T>
__global__ void k_commit(int nr, const int *__restrict__ rows, int ld, const T *__restrict__ Vnew, T *__restrict__ V,
                         const double *__restrict__ DD, double *__restrict__ z, CommitLevels cl) {
    const int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= (int64_t)nr * ld) return;
    const int idx = (int)(x / ld), c = (int)(x % ld);
    const int64_t i = rows[idx];
    V[i * ld + c] = Vnew[x];
    const double dd = DD[x];
    if (dd == 0.0) return;
    atomicAdd(z + c, dd);
    for (int l = 0; l < cl.nl; l++) atomicAdd(cl.Y[l] + (int64_t)cl.lab[l][i] * ld + c, dd);
}

// VCS post-batch update (vcsops.py:189-213 vcs_post): moved rows' new effective multipliers SN at the current Y,
// Z_R += d_i (SN v_new - stZ v_old), cnt_R += [SN > 0] - [stZ > 0], stZ = SN.  Warp per row, lane group per entry.
template <typename T, int NCH>
__global__ void __launch_bounds__(256) k_vcs_post(int nr, const int *__restrict__ rows, int ld, const T *__restrict__ V,
                                                  const T *__restrict__ Vold_batch, const double *__restrict__ d,
                                                  const int *__restrict__ lab, const double *__restrict__ Y,
                                                  const int64_t *__restrict__ ptr, const int *__restrict__ col,
                                                  const double *__restrict__ sig, double *__restrict__ stZ,
                                                  const double *__restrict__ rq, double wv, double rho,
                                                  double *__restrict__ Z, double *__restrict__ cnt) {
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int idx = blockIdx.x, wid = threadIdx.x >> 5, W = blockDim.x >> 5;   // one row per block of W warps
    if (idx >= nr) return;
    const int64_t i = rows[idx];
    const double di = d[i];
    const int Ri = lab[i];
    double vn[EPL], vo[EPL];
    load_d<T>(V + i * ld + ch * EPL, vn);
    load_d<T>(Vold_batch + (int64_t)idx * ld + ch * EPL, vo);
    const int64_t a = ptr[i], b = ptr[i + 1];
    // 32 entries at a time (cluster, multiplier, rq, old stZ lane-parallel; the old stZ of the whole chunk is read
    // before any of it is rewritten), then VU steps with their rows Y_R in flight
    for (int64_t e0 = a + 32 * wid; e0 < b; e0 += 32 * W) {   // the warps take interleaved chunks
        const int nin = (int)(b - e0 < 32 ? b - e0 : 32);
        const bool inl = lane < nin;
        const int Rl = inl ? col[e0 + lane] : 0;
        const double sgl = inl ? sig[e0 + lane] : 0.0, rql = inl ? rq[Rl] : 0.0, sol = inl ? stZ[e0 + lane] : 0.0;
        for (int u0 = 0; u0 < nin; u0 += NPW * VU<T>) {
            double yr[VU<T>][EPL];
            int R[VU<T>];
#pragma unroll
            for (int u = 0; u < VU<T>; u++) {
                const int j = u0 + u * NPW + sub;
                R[u] = __shfl_sync(FULLW, Rl, j & 31);
                if (j < nin) load_y<EPL>(Y + (int64_t)R[u] * ld + ch * EPL, yr[u]);
            }
#pragma unroll
            for (int u = 0; u < VU<T>; u++) {
                const int j = u0 + u * NPW + sub;
                const bool act = j < nin;
                const double sg = __shfl_sync(FULLW, sgl, j & 31), rqR = __shfl_sync(FULLW, rql, j & 31);
                const double so = __shfl_sync(FULLW, sol, j & 31);
                double s = 0.0;
                if (act)
#pragma unroll
                    for (int k = 0; k < EPL; k++) s += vn[k] * yr[u][k];
                s = grp_sum<NCH>(s);
                if (act) {
                    const int Rr = R[u];
                    double sn;
                    if (rho > 0.0 && di > 0.0) {
                        const double g = (Rr == Ri) ? dmul(di, dsub(s, di)) : dmul(di, s);
                        const double p = dsub(sg, dmul(dmul(rho, dmul(wv, rqR) / dmul(di, di)), g));
                        sn = p > 0.0 ? p : 0.0;
                    } else {
                        sn = sg;
                    }
                    if (sn != 0.0 || so != 0.0)
#pragma unroll
                        for (int k = 0; k < EPL; k++)
                            atomicAdd(Z + (int64_t)Rr * ld + ch * EPL + k, di * (sn * vn[k] - so * vo[k]));
                    if (ch == 0) {
                        if (sn > 0.0) {
                            if (!(so > 0.0)) atomicAdd(cnt + Rr, 1.0);
                        } else if (so > 0.0)
                            atomicAdd(cnt + Rr, -1.0);
                        stZ[e0 + j] = sn;
                    }
                }
            }
        }
    }
}

}  // namespace

// ------------------------------------------------------------------------------------------------ host driver
template <typename T, int NCH>
static void sweeps_typed(Problem &p, int nsw, double rho, double rt, double damp, int nbatch, const int *perms_dev,
                         double kap2, cudaStream_t s) {
    const int ld = p.ld;
    const int64_t n = p.n;
    T *V = p.V.as<T>();
    const int nl = (int)p.plev.size(), nv = (int)p.vlev.size();
    const bool usevc = nv > 0;
    // array_split(order, nbatch): the first n % nbatch batches hold one row more
    const int64_t bs = n / nbatch, extra = n % nbatch, maxb = bs + (extra ? 1 : 0);
    p.sw_Vnew.alloc(sizeof(T) * (size_t)maxb * ld);
    p.sw_Vold.alloc(sizeof(T) * (size_t)maxb * ld);
    p.sw_DD.alloc(sizeof(double) * (size_t)maxb * ld);
    p.sw_GX.alloc(sizeof(double) * (size_t)maxb * ld);
    p.sw_KX.alloc(sizeof(double) * (size_t)maxb);
    int64_t sumP = 0;
    for (auto *lv : p.plev) sumP += lv->P;
    p.sw_mark.alloc(sizeof(unsigned) * (size_t)std::max<int64_t>(sumP, 1));
    p.sw_list.alloc(sizeof(int) * (size_t)std::max<int64_t>(sumP, 1));
    p.sw_count.alloc(sizeof(int) * MAX_LEVELS);
    int64_t max_nt = 1;
    for (auto *lv : p.plev) max_nt = std::max<int64_t>(max_nt, std::min<int64_t>(lv->P, maxb));
    p.sw_mpart.alloc(sizeof(double) * (size_t)max_nt * PR_MAXSPLIT * ld);
    LB_CUDA(cudaMemsetAsync(p.sw_mark.ptr, 0, p.sw_mark.bytes, s));
    int64_t max_items = p.zplan.scratch_rows();
    for (auto *lv : p.plev) max_items = std::max(max_items, lv->plan.scratch_rows());
    for (auto *lv : p.vlev) max_items = std::max({max_items, lv->yplan.scratch_rows(), lv->zplan.scratch_rows()});
    p.partials.alloc(sizeof(double) * (size_t)std::max<int64_t>(max_items * ld, 1));
    double *segpart = p.partials.as<double>();
    unsigned stamp = 0;
    for (int sweep = 0; sweep < nsw; sweep++) {
        const int *perm = perms_dev + (int64_t)sweep * n;
        // --- start of sweep: z, Y, Kq, VCS state
        segsum_run<T, NCH>(p.zplan, V, ld, nullptr, nullptr, p.d.as<double>(), nullptr, segpart, p.z.as<double>(), s);
        for (auto *lv : p.plev) {
            segsum_run<T, NCH>(lv->plan, V, ld, lv->members.as<int>(), nullptr, p.d.as<double>(), nullptr, segpart,
                               lv->Y.as<double>(), s);
            if (rho > 0) {
                k_kq<<<lv->P, 256, 0, s>>>(lv->P, ld, lv->Y.as<double>(), lv->sig.as<double>(), lv->rq.as<double>(),
                                           lv->dsq.as<double>(), lv->w, rho, lv->kq.as<double>());
                LB_LAUNCH_CHECK();
            } else {
                LB_CUDA(cudaMemsetAsync(lv->kq.ptr, 0, sizeof(double) * lv->P, s));
            }
        }
        for (auto *lv : p.vlev) {
            segsum_run<T, NCH>(lv->yplan, V, ld, lv->members.as<int>(), nullptr, p.d.as<double>(), nullptr, segpart,
                               lv->Y.as<double>(), s);
            if (lv->nnz) {
                k_vcs_sigt<T, NCH><<<nblk(n, 8), 256, 0, s>>>(n, ld, V, p.d.as<double>(), lv->lab.as<int>(),
                                                              lv->Y.as<double>(), lv->ptr.as<int64_t>(),
                                                              lv->col.as<int>(), lv->sig.as<double>(),
                                                              lv->rq.as<double>(), lv->wv, rho, lv->stZ.as<double>());
                LB_LAUNCH_CHECK();
            }
            segsum_run<T, NCH>(lv->zplan, V, ld, lv->crow.as<int>(), lv->cent.as<int64_t>(), p.d.as<double>(),
                               lv->stZ.as<double>(), segpart, lv->Z.as<double>(), s);
            k_vcs_cnt<<<nblk(lv->P, 8), 256, 0, s>>>(lv->P, lv->cptr.as<int64_t>(), lv->cent.as<int64_t>(),
                                                       lv->stZ.as<double>(), lv->cnt.as<double>());
            LB_LAUNCH_CHECK();
        }
        // --- batches
        int64_t start = 0;
        for (int b = 0; b < nbatch; b++) {
            const int nr = (int)(bs + (b < extra ? 1 : 0));
            const int bw = batch_warps(nr, p.ctx->c.num_sms);
            const int *rows = perm + start;
            start += nr;
            if (nr == 0) continue;
            if (usevc) {
                LB_CUDA(cudaMemsetAsync(p.sw_GX.ptr, 0, sizeof(double) * (size_t)nr * ld, s));
                LB_CUDA(cudaMemsetAsync(p.sw_KX.ptr, 0, sizeof(double) * (size_t)nr, s));
                for (auto *lv : p.vlev) {
                    k_vcs_pre<T, NCH><<<nr, 32 * bw, bw > 1 ? sizeof(double) * bw * (ld + 2) : 0, s>>>(
                        nr, rows, ld, V, p.d.as<double>(), lv->lab.as<int>(), lv->Y.as<double>(),
                        lv->ptr.as<int64_t>(), lv->col.as<int>(), lv->sig.as<double>(), lv->stZ.as<double>(),
                        lv->own.as<int64_t>(), lv->Z.as<double>(), lv->cnt.as<double>(), lv->rq.as<double>(), lv->wv,
                        rho, kap2, p.sw_GX.as<double>(), p.sw_KX.as<double>());
                    LB_LAUNCH_CHECK();
                }
            }
            if (nl) {
                LB_CUDA(cudaMemsetAsync(p.sw_count.ptr, 0, sizeof(int) * MAX_LEVELS, s));
                stamp++;
                int64_t off = 0;
                for (int l = 0; l < nl; l++) {
                    auto *lv = p.plev[l];
                    k_mark<<<nblk(nr, 256), 256, 0, s>>>(nr, rows, lv->lab.as<int>(), (int)off, p.sw_mark.as<unsigned>(),
                                                         stamp, p.sw_list.as<int>() + off, p.sw_count.as<int>() + l);
                    LB_LAUNCH_CHECK();
                    const size_t sh = pair_rows_smem(ld);
                    const int64_t nt = std::min<int64_t>(lv->P, nr);
                    const int ns = pair_splits(nt, lv->P, ld, p.ctx->c.num_sms);
                    const dim3 grid(nblk(nt, PR_Q), ns);
#define LB_PR_CASE(LDV)                                                                                            \
    case LDV:                                                                                                      \
        if (sh > 48 * 1024)                                                                                        \
            LB_CUDA(cudaFuncSetAttribute(k_pair_rows<LDV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh)); \
        k_pair_rows<LDV><<<grid, 256, sh, s>>>(p.sw_list.as<int>() + off, p.sw_count.as<int>() + l, (int)off,     \
                                               lv->P, lv->Y.as<double>(), lv->sig.as<double>(), lv->rq.as<double>(), \
                                               lv->dsq.as<double>(), lv->w, rho, p.sw_mpart.as<double>(),            \
                                               lv->pdiag.as<double>());                                             \
        break;
                    switch (ld) {
                        LB_PR_CASE(2) LB_PR_CASE(4) LB_PR_CASE(8) LB_PR_CASE(16) LB_PR_CASE(32) LB_PR_CASE(64)
                        LB_PR_CASE(128) LB_PR_CASE(256)
                        default: LB_CHECK(false, LB_ERR_INVALID, "row width not supported");
                    }
#undef LB_PR_CASE
                    LB_LAUNCH_CHECK();
                    k_pair_combine<<<nblk(nt * ld, 256), 256, 0, s>>>(p.sw_list.as<int>() + off,
                                                                      p.sw_count.as<int>() + l, (int)off, ld, ns,
                                                                      p.sw_mpart.as<double>(), lv->M.as<double>());
                    LB_LAUNCH_CHECK();
                    off += lv->P;
                }
            }
            StepLevels sl{};
            sl.npl = nl;
            for (int l = 0; l < nl; l++) {
                sl.plab[l] = p.plev[l]->lab.as<int>();
                sl.M[l] = p.plev[l]->M.as<double>();
                sl.pdiag[l] = p.plev[l]->pdiag.as<double>();
                sl.kq[l] = p.plev[l]->kq.as<double>();
            }
            if (p.weighted)
                k_step<T, NCH, true><<<nr, 32 * bw, bw > 1 ? sizeof(double) * bw * (2 * ld + 1) : 0, s>>>(
                    nr, rows, n, ld, p.indptr.as<int64_t>(), p.indices.as<int>(), p.weights.as<float>(), V,
                    p.d.as<double>(), p.z.as<double>(), 1.0 / p.L, sl, p.sw_GX.as<double>(), p.sw_KX.as<double>(),
                    usevc ? 1 : 0, p.T ? p.tptr.as<int64_t>() : nullptr, p.T ? p.tinc.as<int>() : nullptr,
                    p.T ? p.lam.as<double>() : nullptr, rt, damp, p.sw_Vnew.as<T>(), p.sw_DD.as<double>(),
                    usevc ? p.sw_Vold.as<T>() : nullptr);
            else
                k_step<T, NCH, false><<<nr, 32 * bw, bw > 1 ? sizeof(double) * bw * (2 * ld + 1) : 0, s>>>(
                    nr, rows, n, ld, p.indptr.as<int64_t>(), p.indices.as<int>(), nullptr, V, p.d.as<double>(),
                    p.z.as<double>(), 1.0 / p.L, sl, p.sw_GX.as<double>(), p.sw_KX.as<double>(), usevc ? 1 : 0,
                    p.T ? p.tptr.as<int64_t>() : nullptr, p.T ? p.tinc.as<int>() : nullptr,
                    p.T ? p.lam.as<double>() : nullptr, rt, damp, p.sw_Vnew.as<T>(), p.sw_DD.as<double>(),
                    usevc ? p.sw_Vold.as<T>() : nullptr);
            LB_LAUNCH_CHECK();
            CommitLevels cl{};
            cl.nl = 0;
            for (auto *lv : p.plev) {
                cl.lab[cl.nl] = lv->lab.as<int>();
                cl.Y[cl.nl++] = lv->Y.as<double>();
            }
            for (auto *lv : p.vlev) {
                cl.lab[cl.nl] = lv->lab.as<int>();
                cl.Y[cl.nl++] = lv->Y.as<double>();
            }
            k_commit<T><<<nblk((int64_t)nr * ld, 256), 256, 0, s>>>(nr, rows, ld, p.sw_Vnew.as<T>(), V,
                                                                   p.sw_DD.as<double>(), p.z.as<double>(), cl);
            LB_LAUNCH_CHECK();
            for (auto *lv : p.vlev) {
                if (!lv->nnz) continue;
                k_vcs_post<T, NCH><<<nr, 32 * bw, 0, s>>>(
                    nr, rows, ld, V, p.sw_Vold.as<T>(), p.d.as<double>(), lv->lab.as<int>(), lv->Y.as<double>(),
                    lv->ptr.as<int64_t>(), lv->col.as<int>(), lv->sig.as<double>(), lv->stZ.as<double>(),
                    lv->rq.as<double>(), lv->wv, rho, lv->Z.as<double>(), lv->cnt.as<double>());
                LB_LAUNCH_CHECK();
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_perm_pick(int64_t n, int nperm, const int *__restrict__ pool,
                                                   const unsigned long long *__restrict__ ctr, int *__restrict__ dst) {
    const int64_t k = (int64_t)(*ctr % (unsigned long long)nperm);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = pool[k * n + i];
}
__global__ void k_ctr_inc(unsigned long long *ctr) { *ctr += 1ull; }

void perm_pick(Problem &p, cudaStream_t s) {
    const unsigned nb = (unsigned)std::min<int64_t>(nblk(p.n, 256), 4 * (int64_t)p.ctx->c.num_sms);
    k_perm_pick<<<nb, 256, 0, s>>>(p.n, p.sw_nperm, p.sw_perm_pool.as<int>(), p.sw_perm_ctr.as<unsigned long long>(),
                                   p.sw_perm_cur.as<int>());
    LB_LAUNCH_CHECK();
    k_ctr_inc<<<1, 1, 0, s>>>(p.sw_perm_ctr.as<unsigned long long>());
    LB_LAUNCH_CHECK();
}

void sweeps_run(Problem &p, int nsw, double rho, double rt, double damp, int nbatch, const int *perms_dev, double kap2,
                cudaStream_t s) {
    const int nch = (int)(p.ld * dtype_size(p.vdtype) / 16);
#define LB_SW_CASE(TT, NN)                                                                                          \
    if (nch == NN) {                                                                                               \
        sweeps_typed<TT, NN>(p, nsw, rho, rt, damp, nbatch, perms_dev, kap2, s);                                   \
        return;                                                                                                    \
    }
    if (p.vdtype == LB_F64) {
        LB_SW_CASE(double, 1) LB_SW_CASE(double, 2) LB_SW_CASE(double, 4) LB_SW_CASE(double, 8)
        LB_SW_CASE(double, 16) LB_SW_CASE(double, 32)
    } else if (p.vdtype == LB_F32) {
        LB_SW_CASE(float, 1) LB_SW_CASE(float, 2) LB_SW_CASE(float, 4) LB_SW_CASE(float, 8) LB_SW_CASE(float, 16)
        LB_SW_CASE(float, 32)
    } else {
        LB_SW_CASE(__nv_bfloat16, 1) LB_SW_CASE(__nv_bfloat16, 2) LB_SW_CASE(__nv_bfloat16, 4)
        LB_SW_CASE(__nv_bfloat16, 8) LB_SW_CASE(__nv_bfloat16, 16) LB_SW_CASE(__nv_bfloat16, 32)
    }
#undef LB_SW_CASE
    LB_CHECK(false, LB_ERR_INVALID, "row width not supported");
}

}  // namespace lb
