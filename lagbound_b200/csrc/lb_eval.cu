// Evaluation kernels of the augmented-Lagrangian inner loop (sm_100a).
//
// One evaluation (reference: src/lagbound/_core/alm_vcs.py:1496-1533 augmented() and 1299-1312 CV()) at fixed
// multipliers runs, on one stream:
//   1. k_segsum_items + k_seg_combine   z = d^T V, pair-level and VCS-level cluster sums Y = W V (FP64, fixed order)
//   2. k_pair_level                     per pair level: h = Y_Q.Y_R - [Q=R] dsq, pp = max(0, sig - rho r h),
//                                       M_Q = sum_R pp_QR Y_R, PHR term, #(h < -1e-9)
//   3. k_vcs_entries, Z segsum          per VCS working-set entry: ppv, PHR term, slack, next stZ; Z = S^T (d V)
//   4. k_tri                            per triangle: tau, gt, pt, PHR term, min gt
//   5. k_rows / k_heavy_*               per row: (A V)_i (warp per row, 16-byte vector loads of V rows, rows with
//                                       more than HEAVY_DEG edges split across warps), fused epilogue
//                                       G_i = (A V)_i - (d_i/L) z + sum_l d_i (M_Q - pp_QQ d_i v_i)
//                                             + VCS terms + T(pt) V rows (incidence-ordered, deterministic)
//                                       and the row dots v_i.(A V)_i of quadA
//   6. k_finalize                       FP64 reduction of all partials in a fixed order -> lb_eval_out
//
// A lane group of NCH lanes holds one V row (NCH 16-byte chunks); a warp keeps 32/NCH rows in flight.  V is
// BF16/FP32 (FP32 accumulation) or FP64 (FP64 accumulation); every reduction across rows is FP64.
#include <float.h>
#include <algorithm>
#include <mutex>
#include <type_traits>
#include <math.h>

#include "lb_internal.cuh"
#include "lb_segsum.cuh"

namespace lb {

#define LB_DISPATCH_T(DT, ...)                                                                              \
    switch (DT) {                                                                                           \
    case LB_F64: {                                                                                          \
        using T = double;                                                                                   \
        __VA_ARGS__;                                                                                        \
    } break;                                                                                                \
    case LB_F32: {                                                                                          \
        using T = float;                                                                                    \
        __VA_ARGS__;                                                                                        \
    } break;                                                                                                \
    case LB_BF16: {                                                                                         \
        using T = __nv_bfloat16;                                                                            \
        __VA_ARGS__;                                                                                        \
    } break;                                                                                                \
    default: LB_CHECK(false, LB_ERR_INVALID, "unknown dtype");                                             \
    }
#define LB_DISPATCH_NCH(NV, ...)                                                                            \
    switch (NV) {                                                                                           \
    case 1: { constexpr int NCH = 1; __VA_ARGS__; } break;                                                  \
    case 2: { constexpr int NCH = 2; __VA_ARGS__; } break;                                                  \
    case 4: { constexpr int NCH = 4; __VA_ARGS__; } break;                                                  \
    case 8: { constexpr int NCH = 8; __VA_ARGS__; } break;                                                  \
    case 16: { constexpr int NCH = 16; __VA_ARGS__; } break;                                                \
    case 32: { constexpr int NCH = 32; __VA_ARGS__; } break;                                                \
    default: LB_CHECK(false, LB_ERR_INVALID, "row width not supported (max 512 bytes per row)");           \
    }

constexpr unsigned FULL = 0xffffffffu;

// FP64 arithmetic without FMA contraction, for the formulas the reference evaluates as separate multiply and add
// (its Numba kernels are compiled without fastmath): the PHR effective multipliers p = sig - rho r g and the PHR
// terms (p^2 - sig^2)/(2 rho r), whose cancellation amplifies any difference in rounding.
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

template <int NCH, typename A, int E> __device__ __forceinline__ void reduce_groups(A (&acc)[E]) {
#pragma unroll
    for (int off = NCH; off < 32; off <<= 1)
#pragma unroll
        for (int k = 0; k < E; k++) acc[k] += __shfl_xor_sync(FULL, acc[k], off);
}
template <int NCH> __device__ __forceinline__ double reduce_in_group(double x) {
#pragma unroll
    for (int off = 1; off < NCH; off <<= 1) x += __shfl_xor_sync(FULL, x, off);
    return x;
}
template <int NCH> __device__ __forceinline__ float reduce_in_group_f(float x) {
#pragma unroll
    for (int off = 1; off < NCH; off <<= 1) x += __shfl_xor_sync(FULL, x, off);
    return x;
}
__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int off = 16; off; off >>= 1) x += __shfl_xor_sync(FULL, x, off);
    return x;
}
__device__ __forceinline__ double warp_min(double x) {
#pragma unroll
    for (int off = 16; off; off >>= 1) x = fmin(x, __shfl_xor_sync(FULL, x, off));
    return x;
}

// Block of NW warps: each warp contributes one value (lane 0); the block's sum (fixed order) goes to *out.
template <int NW> __device__ __forceinline__ void block_store_sum(double warp_val, double *out) {
    __shared__ double sh[NW];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) sh[w] = warp_val;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < NW; k++) s += sh[k];
        *out = s;
    }
}
template <int NW> __device__ __forceinline__ void block_store_min(double warp_val, double *out) {
    __shared__ double shm[NW];
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) shm[w] = warp_val;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = INFINITY;
#pragma unroll
        for (int k = 0; k < NW; k++) s = fmin(s, shm[k]);
        *out = s;
    }
}

// ============================================================================================ pair level
// A block per PT_Q consecutive clusters Q, the clusters R in tiles of PT_R: the tile's rows of Y staged in shared
// memory; h_QR = sum_c Y_Qc Y_Rc (sequential over the columns, FP64 multiply and add without contraction) minus dsq_Q
// on the diagonal; pp = max(0, sig - rho r h) with r = rq_Q rq_R w; the PHR term (pp^2 - sig^2)/(2 rho r) and the
// count of h < -1e-9 per Q; then M_Q += sum_R pp_QR Y_R over the tile (R ascending).  sig is read and pp written once
// (coalesced), Y comes from L2, and every sum runs in a fixed order.
constexpr int PT_Q = 16, PT_R = 32, PT_LDMAX = 64;
template <bool FIXED>
__global__ void __launch_bounds__(256) k_pair_level(int P, int ld, const double *__restrict__ Y,
                                                    const double *__restrict__ sig, const double *__restrict__ rq,
                                                    const double *__restrict__ dsq, double w, double rho,
                                                    double *__restrict__ pp, double *__restrict__ M,
                                                    double *__restrict__ pdiag, double *__restrict__ val_out,
                                                    double *__restrict__ cnt_out) {
    __shared__ double yq[PT_Q][PT_LDMAX + 1];
    __shared__ double yr[PT_R][PT_LDMAX + 1];
    __shared__ double ptile[PT_Q][PT_R + 1];
    const int t = threadIdx.x, q = t >> 4, rr = t & 15;
    const int Q = blockIdx.x * PT_Q + q;
    const bool qok = Q < P;
    for (int idx = t; idx < PT_Q * ld; idx += blockDim.x) {
        const int qq = idx / ld, c = idx % ld, QQ = blockIdx.x * PT_Q + qq;
        yq[qq][c] = QQ < P ? Y[(int64_t)QQ * ld + c] : 0.0;
    }
    const double rqQ = qok ? rq[Q] : 0.0;
    const double dsQ = qok ? dsq[Q] : 0.0;
    constexpr int MC = PT_LDMAX / 16;
    double m[MC];
#pragma unroll
    for (int j = 0; j < MC; j++) m[j] = 0.0;
    double val = 0.0, cnt = 0.0;
    for (int R0 = 0; R0 < P; R0 += PT_R) {
        __syncthreads();
        for (int idx = t; idx < PT_R * ld; idx += blockDim.x) {
            const int k = idx / ld, c = idx % ld;
            yr[k][c] = R0 + k < P ? Y[(int64_t)(R0 + k) * ld + c] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < PT_R / 16; j++) {
            const int k = rr + 16 * j, R = R0 + k;
            double p = 0.0;
            if (qok && R < P) {
                const double sg = sig[(int64_t)Q * P + R];
                if (FIXED) {
                    p = sg;
                } else {
                    double h = 0.0;
                    for (int c = 0; c < ld; c++) h = dadd(h, dmul(yq[q][c], yr[k][c]));
                    if (R == Q) h = dsub(h, dsQ);
                    const double r_ = dmul(rho, dmul(dmul(rqQ, rq[R]), w));
                    p = dsub(sg, dmul(r_, h));
                    if (p < 0.0) p = 0.0;
                    val = dadd(val, dsub(dmul(p, p), dmul(sg, sg)) / dmul(2.0, r_));
                    if (h < -1e-9) cnt += 1.0;
                }
                pp[(int64_t)Q * P + R] = p;
                if (R == Q) pdiag[Q] = p;
            }
            ptile[q][k] = p;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < MC; j++) {
            const int c = rr + 16 * j;
            if (c < ld) {
                double acc = m[j];
                for (int k = 0; k < PT_R; k++) acc += ptile[q][k] * yr[k][c];
                m[j] = acc;
            }
        }
    }
    if (qok) {
#pragma unroll
        for (int j = 0; j < MC; j++) {
            const int c = rr + 16 * j;
            if (c < ld) M[(int64_t)Q * ld + c] = m[j];
        }
    }
    if (!FIXED) {
        // the 16 threads of one Q are 16 consecutive lanes: a fixed-order tree over them
#pragma unroll
        for (int off = 8; off; off >>= 1) {
            val += __shfl_xor_sync(FULL, val, off);
            cnt += __shfl_xor_sync(FULL, cnt, off);
        }
        if (qok && rr == 0) {
            val_out[Q] = val;
            cnt_out[Q] = cnt;
        }
    }
}

// ============================================================================================ VCS entries
// A warp per item (grid-stride over the items: warp w takes items w, w + W, ...): a row i and at most VSEG of its
// working-set entries (rows with more entries are split into several items).  The item's columns and multipliers are loaded by the whole warp at once; then a lane group per entry:
// s = v_i.Y_R, g = d_i (s - [R = R(i)] d_i), ppv = max(0, sig - rho r g) with r = wv rq_R / d_i^2 (vcsops.py:246-288
// _vcs_aug_rows), PHR term, slack, stn; and, for the row kernel's VCS term, the item's sum of ppv_e Y_R (FP64, entries
// of a lane group in order, then the lane groups in a fixed tree), written to SY_i when the row has one item, else to
// the item's partial slot (summed in slot order by k_vcs_sy_combine).  Lane ch of a lane group holds the 16-byte column
// pairs j = ch + NCH k of the FP64 rows (k < EPL/2), so that every load instruction of a lane group reads NCH
// consecutive pairs of the gathered Y row.
template <typename T> __device__ __forceinline__ void load_pair_d(const T *p, double &a, double &b);
template <> __device__ __forceinline__ void load_pair_d<double>(const double *p, double &a, double &b) {
    const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
    a = v.x;
    b = v.y;
}
template <> __device__ __forceinline__ void load_pair_d<float>(const float *p, double &a, double &b) {
    const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
    a = v.x;
    b = v.y;
}
template <> __device__ __forceinline__ void load_pair_d<__nv_bfloat16>(const __nv_bfloat16 *p, double &a, double &b) {
    const unsigned u = __ldg(reinterpret_cast<const unsigned *>(p));
    a = (double)__uint_as_float(u << 16);
    b = (double)__uint_as_float(u & 0xffff0000u);
}
template <typename T, int NCH, bool FIXED>
__global__ void __launch_bounds__(256, 3) k_vcs_items(int64_t nitems, int ld, const int4 *__restrict__ items,
                                                   const T *__restrict__ V, const double *__restrict__ d,
                                                   const int *__restrict__ lab, const double *__restrict__ Y,
                                                   const int *__restrict__ col, const double *__restrict__ sig,
                                                   const double *__restrict__ rq,
                                                   const double *__restrict__ inv2a, double wv, double rho,
                                                   double *__restrict__ ppv, uint8_t *__restrict__ slack,
                                                   double *__restrict__ stn, double *__restrict__ SY,
                                                   double *__restrict__ SYpart, double *__restrict__ val_out,
                                                   double *__restrict__ cnt_out) {
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH, PL = VSEG / 32;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int64_t wid = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5), W = (int64_t)gridDim.x * 8;
    double val = 0.0, cnt = 0.0;
    for (int64_t it = wid; it < nitems; it += W) {
        const int4 item = items[it];               // row, first entry, end entry, partial slot (-1: write SY)
        const int64_t i = item.x;
        const int e0 = item.y, e1 = item.z;
        const double di = d[i];
        const int Ri = lab[i];
        const double dd = dmul(di, di), idd = 1.0 / dd;        // d_i^2 and its reciprocal, once per item
        double vi[EPL], sy[EPL];
#pragma unroll
        for (int k = 0; k < EPL / 2; k++) load_pair_d<T>(V + i * ld + 2 * (ch + NCH * k), vi[2 * k], vi[2 * k + 1]);
#pragma unroll
        for (int k = 0; k < EPL; k++) sy[k] = 0.0;
        int cl[PL];
        double sl[PL];
#pragma unroll
        for (int u = 0; u < PL; u++) {
            const int e = e0 + 32 * u + lane;
            cl[u] = e < e1 ? __ldcs(col + e) : 0;
            sl[u] = e < e1 ? __ldcs(sig + e) : 0.0;
        }
#pragma unroll 2
        for (int st = 0; st < VSEG / NPW; st++) {
            const int pos = st * NPW + sub, e = e0 + pos;
            if (e0 + st * NPW >= e1) break;                      // uniform over the warp
            const bool act = e < e1;
            const int src = pos & 31, slot = pos >> 5;
            int R = 0;
            double sg = 0.0;
#pragma unroll
            for (int u = 0; u < PL; u++) {
                const int cu = __shfl_sync(FULL, cl[u], src);
                const double su = __shfl_sync(FULL, sl[u], src);
                if (u == slot) {
                    R = cu;
                    sg = su;
                }
            }
            double y[EPL];
            if (act) {
                const double2 *yp = reinterpret_cast<const double2 *>(Y + (int64_t)R * ld) + ch;
#pragma unroll
                for (int k = 0; k < EPL / 2; k++) {
                    const double2 v2 = __ldg(yp + NCH * k);
                    y[2 * k] = v2.x;
                    y[2 * k + 1] = v2.y;
                }
            } else {
#pragma unroll
                for (int k = 0; k < EPL; k++) y[k] = 0.0;
            }
            double s = 0.0;
            if (!FIXED) {
#pragma unroll
                for (int k = 0; k < EPL; k++) s += vi[k] * y[k];
            }
            s = reduce_in_group<NCH>(s);
            if (act) {
                double p = sg, q_ = sg;
                double g = dmul(di, s);
                if (R == Ri) g = dmul(di, dsub(s, di));
                if (!FIXED && di > 0.0) {
                    // r = rho wv rq_R / d_i^2 and 1 / (2 r) = d_i^2 / (2 rho wv rq_R) from per-item and per-cluster
                    // reciprocals (no division per entry; within a few units in the last place of the quotients)
                    const double r_ = dmul(dmul(rho, dmul(wv, rq[R])), idd);
                    p = dsub(sg, dmul(r_, g));
                    if (p < 0.0) p = 0.0;
                    const double qq = dsub(p, dmul(r_, g));
                    q_ = qq > 0.0 ? qq : 0.0;
                    if (ch == 0) val = dadd(val, dmul(dsub(dmul(p, p), dmul(sg, sg)), dmul(dd, inv2a[R])));
                }
                if (ch == 0) {
                    ppv[e] = p;
                    stn[e] = FIXED ? p : q_;
                    if (!FIXED) {
                        slack[e] = (p == 0.0 && g > 0.0) ? 1 : 0;
                        if (g < -1e-9) cnt += 1.0;
                    }
                }
#pragma unroll
                for (int k = 0; k < EPL; k++) sy[k] += p * y[k];
            }
        }
        reduce_groups<NCH>(sy);
        if (sub == 0) {
            double2 *dst = reinterpret_cast<double2 *>(item.w < 0 ? SY + i * ld : SYpart + (int64_t)item.w * ld) + ch;
#pragma unroll
            for (int k = 0; k < EPL / 2; k++) dst[NCH * k] = make_double2(sy[2 * k], sy[2 * k + 1]);
        }
    }
    // one partial per warp (no block barrier: warps finish their items at different times)
    if (!FIXED) {
        val = warp_sum(val);
        cnt = warp_sum(cnt);
        if (lane == 0) {
            val_out[wid] = val;
            cnt_out[wid] = cnt;
        }
    }
}

// 1 / (2 rho wv rq_R) per cluster of a VCS level (the PHR term's divisor without d_i^2), once per evaluation.
__global__ void k_vcs_inv2a(int P, double rho, double wv, const double *__restrict__ rq, double *__restrict__ out) {
    const int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R < P) out[R] = 1.0 / dmul(2.0, dmul(rho, dmul(wv, rq[R])));
}

// SY_i of the rows split into several items: the items' partial rows summed in slot order (thread per column).
__global__ void __launch_bounds__(256) k_vcs_sy_combine(int64_t nmulti, int ld, const int *__restrict__ rows,
                                                        const int *__restrict__ slot_ptr,
                                                        const double *__restrict__ SYpart, double *__restrict__ SY) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nmulti * ld) return;
    const int64_t h = idx / ld;
    const int c = (int)(idx % ld);
    double s = 0.0;
    for (int k = slot_ptr[h]; k < slot_ptr[h + 1]; k++) s += SYpart[(int64_t)k * ld + c];
    SY[(int64_t)rows[h] * ld + c] = s;
}

// ============================================================================================ triangles
// Lane group per triangle: tau = sum_q (v_a v_b + v_b v_c - v_a v_c), gt = 1 - tau, pt = max(0, lam - rt gt)
// (alm_vcs.py:498-509 tri_aug); block partials of the PHR term, min gt and sum lam.
template <typename T, int NCH, bool FIXED>
__global__ void __launch_bounds__(256) k_tri(int64_t T_, int ld, const T *__restrict__ V, const int *__restrict__ tri,
                                             const double *__restrict__ lam, double rt, double *__restrict__ pt,
                                             double *__restrict__ gt, double *__restrict__ val_out,
                                             double *__restrict__ gmin_out, double *__restrict__ lam_out) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int64_t W = (int64_t)gridDim.x * 8 * NPW;
    double val = 0.0, gmin = INFINITY, ls = 0.0;
    for (int64_t base = ((int64_t)blockIdx.x * 8 + (threadIdx.x >> 5)) * NPW; base < T_; base += W) {
        const int64_t t = base + sub;
        const bool act = t < T_;
        Acc tau = 0;
        if (act && !FIXED) {
            const int a = __ldg(tri + 3 * t), b = __ldg(tri + 3 * t + 1), c = __ldg(tri + 3 * t + 2);
            Acc va[EPL], vb[EPL], vc[EPL];
            VT<T>::load(V + (int64_t)a * ld + ch * EPL, va);
            VT<T>::load(V + (int64_t)b * ld + ch * EPL, vb);
            VT<T>::load(V + (int64_t)c * ld + ch * EPL, vc);
#pragma unroll
            for (int k = 0; k < EPL; k++) tau += va[k] * vb[k] + vb[k] * vc[k] - va[k] * vc[k];
        }
        double taud = (double)tau;
        taud = reduce_in_group<NCH>(taud);
        if (act && ch == 0) {
            const double l = lam[t];
            ls += l;
            if (FIXED) {
                pt[t] = l;
            } else {
                const double g = dsub(1.0, taud);
                double p = dsub(l, dmul(rt, g));
                if (p < 0.0) p = 0.0;
                pt[t] = p;
                gt[t] = g;
                val += dsub(dmul(p, p), dmul(l, l)) / dmul(2.0, rt);
                gmin = fmin(gmin, g);
            }
        }
    }
    val = warp_sum(val);
    ls = warp_sum(ls);
    gmin = warp_min(gmin);
    block_store_sum<8>(val, val_out + blockIdx.x);
    __syncthreads();
    block_store_sum<8>(ls, lam_out + blockIdx.x);
    __syncthreads();
    block_store_min<8>(gmin, gmin_out + blockIdx.x);
}

// ============================================================================================ rows
struct LevelArgs {
    int npl = 0, nvl = 0;
    const int *plab[MAX_LEVELS];
    const double *M[MAX_LEVELS];
    const double *pdiag[MAX_LEVELS];
    const int *vlab[MAX_LEVELS];
    const double *ppv[MAX_LEVELS];
    const double *SY[MAX_LEVELS];
    const double *Zv[MAX_LEVELS];
    const int64_t *own[MAX_LEVELS];
};

template <typename T> struct RowArgs {
    int64_t n;
    int ld;
    const int64_t *indptr;
    const int *indices;
    const float *w;
    const T *V;
    const double *d;
    double invL;
    const double *z;
    const int64_t *tptr;
    const int *tinc;
    const double *pt;
    LevelArgs lv;
    void *G;
    int write_G;
    double *part_quad;
    double *row_quad;                  // v_i . (A V)_i per row (summed in a fixed order by k_rowsum)
    const int *gid;                    // batched problems: graph of each row (null otherwise)
    const double *ginvL;               // batched problems: 1 / L per graph
    // heavy rows: items (row, kind, e0, e1), kind 0 = edge segment, 1 = triangle-incidence segment
    const int64_t *heavy_items;
    const int *heavy_rows;
    const int64_t *heavy_item_ptr;
    void *heavy_part;
    int64_t n_heavy_items, n_heavy;
};

// A row is heavy (split across warps) when it has more than HEAVY_DEG edges or HEAVY_TRI triangle incidences;
// the host builds the heavy items with the same rule.
__device__ __forceinline__ bool is_heavy(int64_t deg, int64_t ntri) { return deg > HEAVY_DEG || ntri > HEAVY_TRI; }

// Lanes of the lane group that holds `lane` (NCH consecutive lanes).
template <int NCH> __device__ __forceinline__ unsigned group_mask(int lane) {
    return NCH >= 32 ? FULL : (((1u << NCH) - 1u) << (lane & ~(NCH - 1)));
}

// Sum of w_e V[j_e] over edges [e0, e1) by a whole warp (32/NCH lane groups) in tiles of 32 KT edges: every lane
// loads KT column indices (coalesced), the next tile's while the current tile's rows are in flight; lane group `sub`
// takes the tile positions congruent to sub modulo 32/NCH, KT NCH of them, so that every lane keeps NCH KT (eight for
// NCH <= 8) row loads in flight.
template <typename T, int NCH, bool WEIGHTED>
__device__ __forceinline__ void spmm_tiles(const RowArgs<T> &a, int64_t e0, int64_t e1, int sl, int sub, int ch,
                                           typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, NPR = 32 / NCH, KT = NCH < 8 ? 8 / NCH : 1, UN = NCH < 8 ? NCH : 8;
    constexpr int TILE = 32 * KT;
    const int64_t ntiles = (e1 - e0 + TILE - 1) / TILE;
    int jn[KT];
    float wn[KT];
    auto fetch = [&](int64_t t) {
#pragma unroll
        for (int k = 0; k < KT; k++) {
            const int64_t e = e0 + t * TILE + 32 * k + sl;
            // column indices and weights are read once: streaming loads (evict first) keep V rows in L1/L2
            jn[k] = e < e1 ? __ldcs(a.indices + e) : 0;
            if (WEIGHTED) wn[k] = e < e1 ? __ldcs(a.w + e) : 0.f;
        }
    };
    if (ntiles > 0) fetch(0);
    for (int64_t t = 0; t < ntiles; t++) {
        int jl[KT];
        float wl[KT];
#pragma unroll
        for (int k = 0; k < KT; k++) {
            jl[k] = jn[k];
            wl[k] = wn[k];
        }
        const int64_t base = e0 + t * TILE;
#pragma unroll
        for (int u0 = 0; u0 < KT * NCH; u0 += UN) {
            uint4 raw[UN];
            Acc wt[UN];
#pragma unroll
            for (int u = 0; u < UN; u++) {
                const int k = (u0 + u) / NCH, pos = sub + NPR * ((u0 + u) % NCH);
                const int j = __shfl_sync(FULL, jl[k], pos);
                wt[u] = (Acc)(WEIGHTED ? __shfl_sync(FULL, wl[k], pos) : 1.f);
                raw[u] = base + 32 * k + pos < e1 ? ld_chunk(a.V + (int64_t)j * a.ld + ch * EPL)
                                                  : make_uint4(0, 0, 0, 0);
            }
            if (u0 + UN >= KT * NCH && t + 1 < ntiles) fetch(t + 1);
#pragma unroll
            for (int u = 0; u < UN; u++) {
                if (WEIGHTED) {
                    Acc x[EPL];
                    Unpack<T>::run(raw[u], x);
#pragma unroll
                    for (int k = 0; k < EPL; k++) acc[k] += wt[u] * x[k];
                } else {
                    Accum<T>::add(acc, raw[u]);
                }
            }
        }
    }
}

// Triangle rows T(pt) V (alm_vcs.py:106-120 tri_apply) from the incidence records [t0, t1) of one row, by a sub-warp
// of SW lanes (one record per lane group per round, `nrounds` uniform over the warp), added into acc.
template <typename T, int NCH, int SW>
__device__ __forceinline__ void tri_rows(const RowArgs<T> &a, int64_t t0, int64_t t1, int64_t nrounds, int sub,
                                         int ch, typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, NPR = SW / NCH;
    for (int64_t q = 0; q < nrounds; q++) {
        const int64_t e = t0 + q * NPR + sub;
        if (e >= t1) continue;
        const int o1 = __ldcs(a.tinc + 3 * e), o2 = __ldcs(a.tinc + 3 * e + 1);
        const unsigned tr = (unsigned)__ldcs(a.tinc + 3 * e + 2);
        const double p = __ldg(a.pt + (tr & 0x3fffffffu));
        if (p == 0.0) continue;
        const Acc h = (Acc)(0.5 * p);
        Acc x1[EPL], x2[EPL];
        Unpack<T>::run(ld_chunk(a.V + (int64_t)o1 * a.ld + ch * EPL), x1);
        Unpack<T>::run(ld_chunk(a.V + (int64_t)o2 * a.ld + ch * EPL), x2);
        if ((tr >> 30) == 1u) {
#pragma unroll
            for (int k = 0; k < EPL; k++) acc[k] -= h * (x1[k] + x2[k]);
        } else {
#pragma unroll
            for (int k = 0; k < EPL; k++) acc[k] += h * (x1[k] - x2[k]);
        }
    }
}

// Sum over the lane groups of one sub-warp of SW lanes.
template <int NCH, int SW, typename A, int E> __device__ __forceinline__ void reduce_sub(A (&acc)[E]) {
#pragma unroll
    for (int off = NCH; off < SW; off <<= 1)
#pragma unroll
        for (int k = 0; k < E; k++) acc[k] += __shfl_xor_sync(FULL, acc[k], off);
}
// Maximum over the sub-warps of a warp (every lane holds its sub-warp's value).
template <int SW> __device__ __forceinline__ int64_t max_over_subwarps(int64_t x) {
#pragma unroll
    for (int off = SW; off < 32; off <<= 1) x = max(x, (int64_t)__shfl_xor_sync(FULL, (long long)x, off));
    return x;
}

// v_i . (A V)_i of the row held by the lane group (every lane of the warp calls it: it shuffles).
template <typename T, int NCH>
__device__ __forceinline__ double row_dot(const typename VT<T>::Acc (&vi)[VT<T>::EPL],
                                          const typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    double q = 0.0;
#pragma unroll
    for (int k = 0; k < VT<T>::EPL; k++) q += (double)vi[k] * (double)acc[k];
    return reduce_in_group<NCH>(q);
}

// Fused epilogue of row i: acc = (A V)_i + (T(pt) V)_i, complete in the lanes of the row's lane group; vi = the row's
// own chunk, di its volume.  Only lanes of an active row (act) with sub == 0 store G.
template <typename T, int NCH, bool HAS_LV, typename TG>
__device__ __forceinline__ void row_epilogue(const RowArgs<T> &a, int64_t i, bool act, int sub, int ch,
                                             const typename VT<T>::Acc (&vi)[VT<T>::EPL], double di,
                                             const typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL;
    if (act && sub == 0 && a.write_G) {
        // degree correction with the row's graph's d^T V and L (batched problems run the HAS_LV instances, so the
        // plain instance keeps its registers)
        double dl = di * a.invL;
        const double *zg = a.z;
        if (HAS_LV && a.gid) {
            const int gi = a.gid[i];
            dl = di * a.ginvL[gi];
            zg = a.z + (int64_t)gi * a.ld;
        }
        const int c0 = ch * EPL;
        Acc g[EPL];
#pragma unroll
        for (int k = 0; k < EPL; k++) g[k] = acc[k] - (Acc)(dl * zg[c0 + k]);
        if (HAS_LV) {
            for (int l = 0; l < a.lv.npl; l++) {
                const int Q = a.lv.plab[l][i];
                const double *mq = a.lv.M[l] + (int64_t)Q * a.ld + c0;
                const double pd = a.lv.pdiag[l][Q] * di;
#pragma unroll
                for (int k = 0; k < EPL; k++) g[k] += (Acc)(di * (mq[k] - pd * (double)vi[k]));
            }
            for (int m = 0; m < a.lv.nvl; m++) {
                const int Ri = a.lv.vlab[m][i];
                // sum over the row's working-set entries of ppv_e Y_R, formed by k_vcs_items
                const double *syr = a.lv.SY[m] + i * a.ld + c0;
                double sy[EPL];
#pragma unroll
                for (int k = 0; k < EPL; k++) sy[k] = syr[k];
                const int64_t eo = a.lv.own[m][i];
                const double ow = eo >= 0 ? a.lv.ppv[m][eo] : 0.0;
                const double *zr = a.lv.Zv[m] + (int64_t)Ri * a.ld + c0;
#pragma unroll
                for (int k = 0; k < EPL; k++)
                    g[k] += (Acc)(0.5 * di * (sy[k] + zr[k]) - (ow * di * di) * (double)vi[k]);
            }
        }
        TG gs[EPL];
#pragma unroll
        for (int k = 0; k < EPL; k++) gs[k] = (TG)g[k];
        Store<TG>::st_cs(reinterpret_cast<TG *>(a.G) + i * a.ld + c0, gs, EPL);
    }
}

// Degree-binned rows.  Within each chunk of ROW_CHUNK consecutive rows (a locality order keeps a community together)
// the host schedule lists the rows by increasing work (edges + 2 x triangle incidences).  The first nlight rows of a
// chunk (work at most the light threshold) run one row per lane group (NCH lanes, 32/NCH rows per warp); the other
// non-heavy rows run one row per warp with coalesced index tiles.  A block takes a chunk from a global counter; its
// warps pull rows of the chunk from shared counters, the one-per-warp rows first and every kind heaviest first, so
// that the warps reach the chunk's barrier together.
//
// A light row's lane group walks its edges GSTEP at a time: the group's lanes load the GSTEP column indices together
// (one coalesced load each, shared by shuffles within the group), issue the GSTEP row loads, load the next step's
// indices while those are in flight, then accumulate in edge order.
#ifndef LB_GSTEP
#define LB_GSTEP 8
#endif
#ifndef LB_ROWS_MINB
#define LB_ROWS_MINB 3
#endif
constexpr int GSTEP = LB_GSTEP;
template <typename T, int NCH, bool WEIGHTED>
__device__ __forceinline__ void group_edges(const RowArgs<T> &a, int64_t e0, int64_t e1, int ch, unsigned gm,
                                            typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, IPL = (GSTEP + NCH - 1) / NCH;
    int jn[IPL];
    float wn[IPL];
    auto fetch = [&](int64_t base, int lim) {
#pragma unroll
        for (int k = 0; k < IPL; k++) {
            const int p = ch + NCH * k;
            const bool in = p < lim && p < GSTEP;
            jn[k] = in ? __ldcs(a.indices + base + p) : 0;
            if (WEIGHTED) wn[k] = in ? __ldcs(a.w + base + p) : 0.f;
        }
    };
    const int64_t nstep = (e1 - e0) / GSTEP;
    int64_t e = e0;
    if (nstep > 0) fetch(e0, GSTEP);
    for (int64_t st = 0; st < nstep; st++, e += GSTEP) {
        uint4 raw[GSTEP];
        Acc w[GSTEP];
#pragma unroll
        for (int u = 0; u < GSTEP; u++) {
            const int j = __shfl_sync(gm, jn[u / NCH < IPL ? u / NCH : 0], u % NCH, NCH);
            w[u] = (Acc)(WEIGHTED ? __shfl_sync(gm, wn[u / NCH < IPL ? u / NCH : 0], u % NCH, NCH) : 1.f);
            raw[u] = ld_chunk(a.V + (int64_t)j * a.ld + ch * EPL);
        }
        if (st + 1 < nstep) fetch(e + GSTEP, GSTEP);
#pragma unroll
        for (int u = 0; u < GSTEP; u++) {
            if (WEIGHTED) {
                Acc x[EPL];
                Unpack<T>::run(raw[u], x);
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] += w[u] * x[k];
            } else {
                Accum<T>::add(acc, raw[u]);
            }
        }
    }
    const int rem = (int)(e1 - e);
    if (rem > 0) {
        fetch(e, rem);
        uint4 raw[GSTEP];
        Acc w[GSTEP];
#pragma unroll
        for (int u = 0; u < GSTEP; u++) {
            const int j = __shfl_sync(gm, jn[u / NCH < IPL ? u / NCH : 0], u % NCH, NCH);
            w[u] = (Acc)(WEIGHTED ? __shfl_sync(gm, wn[u / NCH < IPL ? u / NCH : 0], u % NCH, NCH) : 1.f);
            raw[u] = u < rem ? ld_chunk(a.V + (int64_t)j * a.ld + ch * EPL) : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < GSTEP; u++) {
            if (WEIGHTED) {
                Acc x[EPL];
                Unpack<T>::run(raw[u], x);
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] += w[u] * x[k];
            } else {
                Accum<T>::add(acc, raw[u]);
            }
        }
    }
}

// The triangle incidences of a light row, four at a time: records, then multipliers, then the rows.
template <typename T, int NCH>
__device__ __forceinline__ void group_tris(const RowArgs<T> &a, int64_t t0, int64_t t1, int ch,
                                           typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL;
    for (int64_t t = t0; t < t1; t += 4) {
        int o1[4], o2[4];
        unsigned tr[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const bool in = t + u < t1;
            o1[u] = in ? __ldcs(a.tinc + 3 * (t + u)) : 0;
            o2[u] = in ? __ldcs(a.tinc + 3 * (t + u) + 1) : 0;
            tr[u] = in ? (unsigned)__ldcs(a.tinc + 3 * (t + u) + 2) : 0u;
        }
        double p[4];
#pragma unroll
        for (int u = 0; u < 4; u++) p[u] = t + u < t1 ? __ldg(a.pt + (tr[u] & 0x3fffffffu)) : 0.0;
        uint4 r1[4], r2[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const bool on = p[u] != 0.0;
            r1[u] = on ? ld_chunk(a.V + (int64_t)o1[u] * a.ld + ch * EPL) : make_uint4(0, 0, 0, 0);
            r2[u] = on ? ld_chunk(a.V + (int64_t)o2[u] * a.ld + ch * EPL) : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (p[u] == 0.0) continue;
            const Acc h = (Acc)(0.5 * p[u]);
            Acc x1[EPL], x2[EPL];
            Unpack<T>::run(r1[u], x1);
            Unpack<T>::run(r2[u], x2);
            if ((tr[u] >> 30) == 1u) {
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] -= h * (x1[k] + x2[k]);
            } else {
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] += h * (x1[k] - x2[k]);
            }
        }
    }
}

// ---------------------------------------------------------------------------------------------- staged gathers
// With LB_STAGED the unweighted row gathers land in shared memory through asynchronous copies (cp.async, 16 bytes per
// lane, no register held while in flight) in two stages of GSTEP slots per lane: a lane issues the next step's copies
// before it waits for and consumes the current step's, and every lane reads back only the slots it filled itself.
#ifndef LB_STAGED
#define LB_STAGED 1
#endif
__device__ __forceinline__ void cp16(uint4 *dst, const void *src, bool on) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    const int n = on ? 16 : 0;   // 0: the slot is zero-filled and nothing is read
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// a lane's slot u of stage g in its warp's staging area (2 stages x GSTEP slots x 32 lanes of 16 bytes)
__device__ __forceinline__ uint4 *stage_slot(uint4 *stg, int g, int u, int lane) {
    return stg + ((g * GSTEP + u) << 5) + lane;
}

template <typename T, int NCH>
__device__ __forceinline__ void group_edges_staged(const RowArgs<T> &a, int64_t e0, int64_t e1, int ch, unsigned gm,
                                                   int lane, uint4 *stg, typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    constexpr int EPL = VT<T>::EPL, IPL = (GSTEP + NCH - 1) / NCH;
    const int64_t nst = (e1 - e0 + GSTEP - 1) / GSTEP;
    if (nst == 0) return;
    int jn[IPL];
    auto fetch = [&](int64_t st) {
        const int64_t base = e0 + st * GSTEP;
#pragma unroll
        for (int k = 0; k < IPL; k++) {
            const int p = ch + NCH * k;
            jn[k] = (p < GSTEP && base + p < e1) ? __ldcs(a.indices + base + p) : 0;
        }
    };
    auto issue = [&](int64_t st) {
        const int64_t base = e0 + st * GSTEP;
#pragma unroll
        for (int u = 0; u < GSTEP; u++) {
            const int j = __shfl_sync(gm, jn[u / NCH < IPL ? u / NCH : 0], u % NCH, NCH);
            cp16(stage_slot(stg, (int)(st & 1), u, lane), a.V + (int64_t)j * a.ld + ch * EPL, base + u < e1);
        }
        cp_commit();
    };
    fetch(0);
    issue(0);
    if (nst > 1) fetch(1);
    for (int64_t st = 0; st < nst; st++) {
        if (st + 1 < nst) {
            issue(st + 1);
            if (st + 2 < nst) fetch(st + 2);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        const int cnt = (int)min((int64_t)GSTEP, e1 - e0 - st * GSTEP);
#pragma unroll
        for (int u = 0; u < GSTEP; u++)
            if (u < cnt) Accum<T>::add(acc, *stage_slot(stg, (int)(st & 1), u, lane));
    }
}

// The warp path: tiles of 32 KT edges, KT NCH (= GSTEP) positions per lane group, two stages.
template <typename T, int NCH>
__device__ __forceinline__ void spmm_tiles_staged(const RowArgs<T> &a, int64_t e0, int64_t e1, int lane, int sub,
                                                  int ch, uint4 *stg, typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    constexpr int EPL = VT<T>::EPL, NPR = 32 / NCH, KT = NCH < 8 ? 8 / NCH : 1, NPOS = KT * NCH;
    constexpr int TILE = 32 * KT;
    const int64_t ntiles = (e1 - e0 + TILE - 1) / TILE;
    if (ntiles == 0) return;
    int jn[KT];
    auto fetch = [&](int64_t t) {
#pragma unroll
        for (int k = 0; k < KT; k++) {
            const int64_t e = e0 + t * TILE + 32 * k + lane;
            jn[k] = e < e1 ? __ldcs(a.indices + e) : 0;
        }
    };
    // positions beyond one stage (FP64 rows of 16 or 32 chunks, or fewer slots than positions) are issued and
    // consumed in single-stage rounds
    constexpr int ROUND = NPOS < GSTEP ? NPOS : GSTEP;
    // the copies of tile t, positions u0 .. u0 + ROUND - 1, into stage g
    auto issue = [&](int64_t t, int u0, int g) {
        const int64_t base = e0 + t * TILE;
#pragma unroll
        for (int u = 0; u < ROUND; u++) {
            const int q = u0 + u, k = q < NPOS ? q / NCH : 0, pos = sub + NPR * (q % NCH);
            const int j = __shfl_sync(FULL, jn[k], pos);
            cp16(stage_slot(stg, g, u, lane), a.V + (int64_t)j * a.ld + ch * EPL, q < NPOS && base + 32 * k + pos < e1);
        }
        cp_commit();
    };
    if (NPOS <= GSTEP) {
        fetch(0);
        issue(0, 0, 0);
        if (ntiles > 1) fetch(1);
        for (int64_t t = 0; t < ntiles; t++) {
            if (t + 1 < ntiles) {
                issue(t + 1, 0, (int)((t + 1) & 1));
                if (t + 2 < ntiles) fetch(t + 2);
                cp_wait<1>();
            } else {
                cp_wait<0>();
            }
#pragma unroll
            for (int u = 0; u < ROUND; u++) Accum<T>::add(acc, *stage_slot(stg, (int)(t & 1), u, lane));
        }
    } else {
        for (int64_t t = 0; t < ntiles; t++) {
            fetch(t);
#pragma unroll
            for (int u0 = 0; u0 < NPOS; u0 += ROUND) {
                issue(t, u0, 0);
                cp_wait<0>();
#pragma unroll
                for (int u = 0; u < ROUND; u++)
                    if (u0 + u < NPOS) Accum<T>::add(acc, *stage_slot(stg, 0, u, lane));
            }
        }
    }
}

// Triangle incidences of a light row, four per step: records and multipliers (cooperative, one record per lane),
// then the eight rows staged; the next step's records are loaded while the rows are in flight.
template <typename T, int NCH>
__device__ __forceinline__ void group_tris_staged(const RowArgs<T> &a, int64_t t0, int64_t t1, int ch, unsigned gm,
                                                  int lane, uint4 *stg, typename VT<T>::Acc (&acc)[VT<T>::EPL]) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, TS = 4, SL = TS > NCH ? TS / NCH : 1;
    int o1[SL], o2[SL];
    unsigned tr[SL];
    auto fetch = [&](int64_t t) {
#pragma unroll
        for (int k = 0; k < SL; k++) {
            const int pos = ch + NCH * k;
            const bool in = pos < TS && t + pos < t1;
            o1[k] = in ? __ldcs(a.tinc + 3 * (t + pos)) : 0;
            o2[k] = in ? __ldcs(a.tinc + 3 * (t + pos) + 1) : 0;
            tr[k] = in ? (unsigned)__ldcs(a.tinc + 3 * (t + pos) + 2) : 0u;
        }
    };
    if (t1 <= t0) return;
    fetch(t0);
    for (int64_t t = t0; t < t1; t += TS) {
        double p[SL];
#pragma unroll
        for (int k = 0; k < SL; k++) {
            const int pos = ch + NCH * k;
            p[k] = (pos < TS && t + pos < t1) ? __ldg(a.pt + (tr[k] & 0x3fffffffu)) : 0.0;
        }
        double pu[TS];
        bool neg[TS];
#pragma unroll
        for (int u = 0; u < TS; u++) {
            const int src = u % NCH, slot = u / NCH < SL ? u / NCH : 0;
            const int a1 = __shfl_sync(gm, o1[slot], src, NCH), a2 = __shfl_sync(gm, o2[slot], src, NCH);
            const unsigned r = __shfl_sync(gm, tr[slot], src, NCH);
            pu[u] = __shfl_sync(gm, p[slot], src, NCH);
            neg[u] = (r >> 30) == 1u;
            const bool on = t + u < t1 && pu[u] != 0.0;
            cp16(stage_slot(stg, 0, 2 * u, lane), a.V + (int64_t)a1 * a.ld + ch * EPL, on);
            cp16(stage_slot(stg, 0, 2 * u + 1, lane), a.V + (int64_t)a2 * a.ld + ch * EPL, on);
        }
        cp_commit();
        if (t + TS < t1) fetch(t + TS);
        cp_wait<0>();
#pragma unroll
        for (int u = 0; u < TS; u++) {
            if (!(t + u < t1) || pu[u] == 0.0) continue;
            const Acc h = (Acc)(0.5 * pu[u]);
            Acc x1[EPL], x2[EPL];
            Unpack<T>::run(*stage_slot(stg, 0, 2 * u, lane), x1);
            Unpack<T>::run(*stage_slot(stg, 0, 2 * u + 1, lane), x2);
            if (neg[u]) {
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] -= h * (x1[k] + x2[k]);
            } else {
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] += h * (x1[k] - x2[k]);
            }
        }
    }
}

constexpr int ROW_CHUNK = 256;
template <typename T, int NCH, bool WEIGHTED, bool HAS_LV, typename TG>
__global__ void __launch_bounds__(256, LB_ROWS_MINB) k_rows(RowArgs<T> a, const int *__restrict__ sched,
                                                 const int *__restrict__ nlight,
                                                 unsigned long long *__restrict__ counter) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    __shared__ long long s_base;
    __shared__ int s_light, s_rest;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const unsigned gm = group_mask<NCH>(lane);
    extern __shared__ uint4 lb_stage[];
    uint4 *stg = lb_stage + (threadIdx.x >> 5) * (2 * GSTEP * 32);
    // staged gathers measured faster for FP32 and FP64 rows, slower for BF16 (its 64-byte rows gain less from the
    // freed registers than they pay in shared-memory traffic)
    constexpr bool STAGED = LB_STAGED && !WEIGHTED && !std::is_same<T, __nv_bfloat16>::value;
    while (true) {
        if (threadIdx.x == 0) {
            s_base = (long long)atomicAdd(counter, (unsigned long long)ROW_CHUNK);
            s_light = 0;
            s_rest = 0;
        }
        __syncthreads();
        const int64_t base = s_base;
        if (base >= a.n) break;
        const int cnt = (int)min((int64_t)ROW_CHUNK, a.n - base);
        const int nl = nlight[base / ROW_CHUNK];
        // the other rows first, heaviest first, one row per warp (the light rows then even out the warps' finish)
        while (true) {
            int r = 0;
            if (lane == 0) r = atomicAdd(&s_rest, 1);
            r = __shfl_sync(FULL, r, 0);
            if (cnt - 1 - r < nl) break;
            const int64_t i = sched[base + cnt - 1 - r];
            const int64_t e0 = a.indptr[i], e1 = a.indptr[i + 1];
            const int64_t t0 = a.tptr ? a.tptr[i] : 0, t1 = a.tptr ? a.tptr[i + 1] : 0;
            if (is_heavy(e1 - e0, t1 - t0)) continue;
            Acc vi[EPL], acc[EPL];
            Unpack<T>::run(ld_chunk(a.V + i * a.ld + ch * EPL), vi);
            const double di = a.d[i];
#pragma unroll
            for (int k = 0; k < EPL; k++) acc[k] = 0;
            if (STAGED)
                spmm_tiles_staged<T, NCH>(a, e0, e1, lane, sub, ch, stg, acc);
            else
                spmm_tiles<T, NCH, WEIGHTED>(a, e0, e1, lane, sub, ch, acc);
            reduce_sub<NCH, 32>(acc);
            const double q = row_dot<T, NCH>(vi, acc);
            const int64_t nrounds = (t1 - t0 + NPW - 1) / NPW;
            if (nrounds > 0) {
                // every lane group now holds (A V)_i: keep it in group 0 only and add the triangle partials
                if (sub != 0)
#pragma unroll
                    for (int k = 0; k < EPL; k++) acc[k] = 0;
                tri_rows<T, NCH, 32>(a, t0, t1, nrounds, sub, ch, acc);
                reduce_sub<NCH, 32>(acc);
            }
            row_epilogue<T, NCH, HAS_LV, TG>(a, i, true, sub, ch, vi, di, acc);
            if (lane == 0) a.row_quad[i] = q;
        }
        // light rows: one row per lane group
        while (true) {
            int r = 0;
            if (lane == 0) r = atomicAdd(&s_light, NPW);
            r = __shfl_sync(FULL, r, 0);
            if (r >= nl) break;
            const int my = nl - 1 - (r + sub);       // heaviest light rows first
            const bool act = my >= 0;
            int64_t i = 0, t0 = 0, t1 = 0;
            Acc vi[EPL], acc[EPL];
            double di = 0.0;
#pragma unroll
            for (int k = 0; k < EPL; k++) {
                acc[k] = 0;
                vi[k] = 0;
            }
            if (act) {
                i = sched[base + my];
                const int64_t e0 = a.indptr[i], e1 = a.indptr[i + 1];
                if (a.tptr) {
                    t0 = a.tptr[i];
                    t1 = a.tptr[i + 1];
                }
                Unpack<T>::run(ld_chunk(a.V + i * a.ld + ch * EPL), vi);
                di = a.d[i];
                if (STAGED)
                    group_edges_staged<T, NCH>(a, e0, e1, ch, gm, lane, stg, acc);
                else
                    group_edges<T, NCH, WEIGHTED>(a, e0, e1, ch, gm, acc);
            }
            const double q = row_dot<T, NCH>(vi, acc);
            if (act) {
                if (STAGED)
                    group_tris_staged<T, NCH>(a, t0, t1, ch, gm, lane, stg, acc);
                else
                    group_tris<T, NCH>(a, t0, t1, ch, acc);
            }
            row_epilogue<T, NCH, HAS_LV, TG>(a, i, act, 0, ch, vi, di, acc);
            if (act && ch == 0) a.row_quad[i] = q;
        }
        __syncthreads();
    }
}

// Fixed-order partial sums of the per-row quad terms: block b sums rows [b n / nb, (b + 1) n / nb).
__global__ void __launch_bounds__(256) k_rowsum(int64_t n, const double *__restrict__ row_quad,
                                                double *__restrict__ part) {
    const int64_t nb = gridDim.x, b = blockIdx.x;
    const int64_t r0 = n * b / nb, r1 = n * (b + 1) / nb;
    double s = 0.0;
    for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) s += row_quad[i];
    s = warp_sum(s);
    block_store_sum<8>(s, part + b);
}

// One warp per heavy item: a 1024-edge segment of A V or a 256-record segment of T(pt) V.
template <typename T, int NCH, bool WEIGHTED>
__global__ void __launch_bounds__(256) k_heavy_part(RowArgs<T> a) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int64_t it = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (it >= a.n_heavy_items) return;
    const int64_t kind = a.heavy_items[4 * it + 1], e0 = a.heavy_items[4 * it + 2], e1 = a.heavy_items[4 * it + 3];
    Acc acc[EPL];
#pragma unroll
    for (int k = 0; k < EPL; k++) acc[k] = 0;
    if (kind == 0)
        spmm_tiles<T, NCH, WEIGHTED>(a, e0, e1, lane, sub, ch, acc);
    else
        tri_rows<T, NCH, 32>(a, e0, e1, (e1 - e0 + 32 / NCH - 1) / (32 / NCH), sub, ch, acc);
    reduce_groups<NCH>(acc);
    if (sub == 0) {
        Acc *dst = reinterpret_cast<Acc *>(a.heavy_part) + it * a.ld + ch * EPL;
#pragma unroll
        for (int k = 0; k < EPL; k++) dst[k] = acc[k];
    }
}

// One warp per heavy row: its item partials summed in item order, then the epilogue.
template <typename T, int NCH, bool HAS_LV, typename TG>
__global__ void __launch_bounds__(256) k_heavy_fin(RowArgs<T> a) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int64_t h = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (h < a.n_heavy) {
        const int64_t i = a.heavy_rows[h];
        Acc acc[EPL], accT[EPL];
#pragma unroll
        for (int k = 0; k < EPL; k++) {
            acc[k] = 0;
            accT[k] = 0;
        }
        Acc vi[EPL];
        Unpack<T>::run(ld_chunk(a.V + i * a.ld + ch * EPL), vi);
        const double di = a.d[i];
        const Acc *src = reinterpret_cast<const Acc *>(a.heavy_part);
        for (int64_t it = a.heavy_item_ptr[h]; it < a.heavy_item_ptr[h + 1]; it++) {
            const bool tri = a.heavy_items[4 * it + 1] != 0;
#pragma unroll
            for (int k = 0; k < EPL; k++) {
                const Acc v = src[it * a.ld + ch * EPL + k];
                if (tri)
                    accT[k] += v;
                else
                    acc[k] += v;
            }
        }
        const double quad = row_dot<T, NCH>(vi, acc);
#pragma unroll
        for (int k = 0; k < EPL; k++) acc[k] += accT[k];
        row_epilogue<T, NCH, HAS_LV, TG>(a, i, true, sub, ch, vi, di, acc);
        if (lane == 0) a.row_quad[i] = quad;
    }
}

// ============================================================================================ finalize
struct FinArgs {
    const double *part;
    int64_t off_quad, n_quad;        // row quad partials (light + heavy)
    int64_t off_lv, n_lv;            // pair-level value partials
    int64_t off_lc, n_lc;            // pair-level counts
    int64_t off_vv, n_vv;            // VCS value partials
    int64_t off_vc, n_vc;            // VCS counts
    int64_t off_tv, n_tv;            // triangle value partials
    int64_t off_tg, n_tg;            // triangle min gt partials
    int64_t off_tl, n_tl;            // lambda sums
    const double *z;
    int ld;
    double L, C0;
    int fixed;
    lb_eval_out *out;
    const double *gsum;               // batched problems: (sum of zz_g, sum of zz_g / L_g); null otherwise
};

// Batched problems: quadA_g over the graph's rows and the triangle PHR term over the graph's triangles (the
// per-triangle formula of k_tri), each graph's ranges cut into GRAPH_SLICES slices (block (g, slice)); partial sums
// in a fixed order.
constexpr int GRAPH_SLICES = 16;
__global__ void __launch_bounds__(256) k_graph_part(const int64_t *__restrict__ gptr, const int64_t *__restrict__ gtptr,
                                                    const double *__restrict__ row_quad, const double *__restrict__ pt,
                                                    const double *__restrict__ lam, double rt, int fixed,
                                                    double *__restrict__ part) {
    __shared__ double sh[2][256];
    const int g = blockIdx.x, sl = blockIdx.y, ns = gridDim.y;
    const int64_t r0 = gptr[g], nr = gptr[g + 1] - r0, t0 = gtptr[g], nt = gtptr[g + 1] - t0;
    double q = 0.0, tv = 0.0;
    for (int64_t i = r0 + nr * sl / ns + threadIdx.x; i < r0 + nr * (sl + 1) / ns; i += blockDim.x) q += row_quad[i];
    if (!fixed && pt)
        for (int64_t t = t0 + nt * sl / ns + threadIdx.x; t < t0 + nt * (sl + 1) / ns; t += blockDim.x) {
            const double p = pt[t], l = lam[t];
            tv += dsub(dmul(p, p), dmul(l, l)) / dmul(2.0, rt);
        }
    sh[0][threadIdx.x] = q;
    sh[1][threadIdx.x] = tv;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * ((int64_t)g * ns + sl)] = sh[0][0];
        part[2 * ((int64_t)g * ns + sl) + 1] = sh[1][0];
    }
}

// per graph (thread per graph): the slices in order, zz_g = |d_g^T V_g|^2, value_g and primal_g
__global__ void k_graph_fin(int G, int ld, const double *__restrict__ part, const double *__restrict__ z,
                            const double *__restrict__ gL, const double *__restrict__ gC0, double *__restrict__ gout) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    double q = 0.0, tv = 0.0, zz = 0.0;
    for (int sl = 0; sl < GRAPH_SLICES; sl++) {
        q += part[2 * ((int64_t)g * GRAPH_SLICES + sl)];
        tv += part[2 * ((int64_t)g * GRAPH_SLICES + sl) + 1];
    }
    for (int c = 0; c < ld; c++) zz += z[(int64_t)g * ld + c] * z[(int64_t)g * ld + c];
    const double val0 = q - zz / gL[g];
    gout[5 * g + 0] = val0 - tv + gC0[g];
    gout[5 * g + 1] = val0 + gC0[g];
    gout[5 * g + 2] = q;
    gout[5 * g + 3] = zz;
    gout[5 * g + 4] = tv;
}

// the totals over the graphs that k_finalize uses in place of |z|^2 and |z|^2 / L, from k_graph_fin's zz_g (one
// block, graphs strided over the threads, then a tree: a fixed order)
__global__ void __launch_bounds__(256) k_graph_zz(int G, const double *__restrict__ gout,
                                                  const double *__restrict__ gL, double *__restrict__ gsum) {
    __shared__ double sh[2][256];
    double s = 0.0, sl = 0.0;
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        const double zz = gout[5 * g + 3];
        s += zz;
        sl += zz / gL[g];
    }
    sh[0][threadIdx.x] = s;
    sh[1][threadIdx.x] = sl;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        gsum[0] = sh[0][0];
        gsum[1] = sh[1][0];
    }
}

__device__ double block_sum_fixed(const double *x, int64_t nel) {
    __shared__ double sh[512];
    double s = 0.0;
    for (int64_t k = threadIdx.x; k < nel; k += blockDim.x) s += x[k];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}
__device__ double block_min_fixed(const double *x, int64_t nel) {
    __shared__ double sh[512];
    double s = INFINITY;
    for (int64_t k = threadIdx.x; k < nel; k += blockDim.x) s = fmin(s, x[k]);
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) sh[threadIdx.x] = fmin(sh[threadIdx.x], sh[threadIdx.x + w]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(512) k_finalize(FinArgs f) {
    const double quad = block_sum_fixed(f.part + f.off_quad, f.n_quad);
    const double lv = block_sum_fixed(f.part + f.off_lv, f.n_lv);
    const double lc = block_sum_fixed(f.part + f.off_lc, f.n_lc);
    const double vv = block_sum_fixed(f.part + f.off_vv, f.n_vv);
    const double vc = block_sum_fixed(f.part + f.off_vc, f.n_vc);
    const double tv = block_sum_fixed(f.part + f.off_tv, f.n_tv);
    const double tl = block_sum_fixed(f.part + f.off_tl, f.n_tl);
    const double tg = block_min_fixed(f.part + f.off_tg, f.n_tg);
    if (threadIdx.x == 0) {
        double zz = 0.0, zzL;
        if (f.gsum) {
            zz = f.gsum[0];
            zzL = f.gsum[1];
        } else {
            for (int c = 0; c < f.ld; c++) zz += f.z[c] * f.z[c];
            zzL = zz / f.L;
        }
        lb_eval_out o;
        o.quadA = quad;
        o.zz = zz;
        const double val0 = quad - zzL;
        o.primal = val0 + f.C0;
        o.level_tot = f.fixed ? 0.0 : lv;
        o.tri_tot = f.fixed ? 0.0 : tv;
        o.vcs_tot = f.fixed ? 0.0 : vv;
        o.value = val0 - o.level_tot - o.tri_tot - o.vcs_tot + f.C0;
        o.gmin = tg;
        o.nviol = (int64_t)lc;
        o.vcs_nviol = (int64_t)vc;
        o.lam_sum = tl;
        for (int k = 0; k < 5; k++) o.reserved[k] = 0.0;
        *f.out = o;
    }
}

// ============================================================================================ conversions
template <typename T> __device__ __forceinline__ T from_double(double x);
template <> __device__ __forceinline__ double from_double<double>(double x) { return x; }
template <> __device__ __forceinline__ float from_double<float>(double x) { return (float)x; }
template <> __device__ __forceinline__ __nv_bfloat16 from_double<__nv_bfloat16>(double x) {
    return __double2bfloat16(x);
}
template <typename T> __device__ __forceinline__ double to_double(T x) { return (double)x; }
template <> __device__ __forceinline__ double to_double<__nv_bfloat16>(__nv_bfloat16 x) {
    return (double)__bfloat162float(x);
}

// V / G between the caller's n x r row-major layout and the internal n x ld layout; ord (internal row -> caller row)
// applies the locality order (nullptr: identity).
template <typename T>
__global__ void k_from_f64(int64_t n, int r, int ld, const double *__restrict__ src, T *__restrict__ V,
                           const int *__restrict__ ord) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * ld) return;
    const int64_t k = idx / ld;
    const int c = (int)(idx % ld);
    const int64_t i = ord ? (int64_t)ord[k] : k;
    V[idx] = from_double<T>(c < r ? src[i * r + c] : 0.0);
}
template <typename T>
__global__ void k_raw_in(int64_t n, int r, int ld, const T *__restrict__ src, T *__restrict__ V,
                         const int *__restrict__ ord) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * ld) return;
    const int64_t k = idx / ld;
    const int c = (int)(idx % ld);
    const int64_t i = ord ? (int64_t)ord[k] : k;
    V[idx] = c < r ? src[i * r + c] : from_double<T>(0.0);
}
template <typename T>
__global__ void k_to_f64(int64_t n, int r, int ld, const T *__restrict__ V, double *__restrict__ out,
                         const int *__restrict__ ord) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * r) return;
    const int64_t k = idx / r;
    const int c = (int)(idx % r);
    const int64_t i = ord ? (int64_t)ord[k] : k;
    out[i * r + c] = to_double<T>(V[k * ld + c]);
}

template <typename T>
__global__ void k_raw_out(int64_t n, int r, int ld, const T *__restrict__ V, T *__restrict__ out,
                          const int *__restrict__ ord) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n * r) return;
    const int64_t k = idx / r;
    const int c = (int)(idx % r);
    const int64_t i = ord ? (int64_t)ord[k] : k;
    out[i * r + c] = V[k * ld + c];
}

__global__ void k_age_update(int64_t nnz, const uint8_t *__restrict__ slack, uint8_t *__restrict__ age) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    // vcsops.py:300-305 age_update
    if (slack[e]) {
        if (age[e] < 255) age[e] = age[e] + 1;
    } else
        age[e] = 0;
}

// ============================================================================================ host side
static inline unsigned nblk(int64_t work, int per) { return (unsigned)((work + per - 1) / per); }

// Persistent grid: as many 256-thread blocks as fit on the device at once (capped by the work).
// Blocks per SM of a kernel at 256 threads and `smem` dynamic shared bytes (cached per kernel), times the SM count,
// capped by the work.
template <typename K> static unsigned occ_grid(K kernel, int64_t work_blocks, int num_sms, size_t smem = 0) {
    static std::mutex mu;
    static std::vector<std::pair<std::pair<int, const void *>, int>> cache;   // (device, kernel) -> blocks per SM
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    const std::pair<int, const void *> key(dev, (const void *)kernel);
    int per = 0;
    for (auto &c : cache)
        if (c.first == key) per = c.second;
    if (per == 0) {
        if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 256, smem) != cudaSuccess) {
            cudaGetLastError();
            per = 1;
        }
        per = std::max(per, 1);
        cache.emplace_back(key, per);
    }
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(work_blocks, (int64_t)per * num_sms));
}

void SegPlan::build(const std::vector<int64_t> &seg_ptr, cudaStream_t s) {
    nseg = (int64_t)seg_ptr.size() - 1;
    std::vector<int64_t> e0, e1, sip(nseg + 1, 0);
    std::vector<int> sg;
    for (int64_t q = 0; q < nseg; q++) {
        sip[q] = (int64_t)e0.size();
        for (int64_t a = seg_ptr[q]; a < seg_ptr[q + 1]; a += SEGSUM_CHUNK) {
            e0.push_back(a);
            e1.push_back(std::min<int64_t>(seg_ptr[q + 1], a + SEGSUM_CHUNK));
            sg.push_back((int)q);
        }
    }
    sip[nseg] = (int64_t)e0.size();
    nitems = (int64_t)e0.size();
    upload(item_e0, e0, s);
    upload(item_e1, e1, s);
    upload(item_seg, sg, s);
    upload(seg_item_ptr, sip, s);
    int64_t most = 0;
    for (int64_t q = 0; q < nseg; q++) most = std::max(most, sip[q + 1] - sip[q]);
    ngroups = 0;
    if (most > SEGSUM_GROUP) {
        std::vector<int64_t> gip, sgp(nseg + 1, 0);
        for (int64_t q = 0; q < nseg; q++) {
            sgp[q] = (int64_t)gip.size();
            for (int64_t a = sip[q]; a < sip[q + 1]; a += SEGSUM_GROUP) gip.push_back(a);
        }
        sgp[nseg] = (int64_t)gip.size();
        ngroups = (int64_t)gip.size();
        gip.push_back(nitems);
        upload(group_item_ptr, gip, s);
        upload(seg_group_ptr, sgp, s);
    }
}

// dynamic shared memory of k_rows: the staging areas of its 8 warps (staged unweighted builds only)
template <typename T> static size_t rows_smem(bool weighted) {
    return (LB_STAGED && !weighted && !std::is_same<T, __nv_bfloat16>::value) ? (size_t)8 * 2 * GSTEP * 32 * sizeof(uint4)
                                                                                : 0;
}

template <typename T, int NCH, typename TG>
static unsigned rows_grid(bool weighted, bool has_lv, int64_t n, int nsm) {
    const int64_t work = nblk(n, ROW_CHUNK);
    const size_t sm = rows_smem<T>(weighted);
    if (weighted)
        return has_lv ? occ_grid(k_rows<T, NCH, true, true, TG>, work, nsm, sm)
                      : occ_grid(k_rows<T, NCH, true, false, TG>, work, nsm, sm);
    return has_lv ? occ_grid(k_rows<T, NCH, false, true, TG>, work, nsm, sm)
                  : occ_grid(k_rows<T, NCH, false, false, TG>, work, nsm, sm);
}

template <typename T, int NCH, typename TG>
static void launch_rows(const RowArgs<T> &a, const int *sched, const int *nlight, unsigned long long *ctr,
                        bool weighted, bool has_lv, unsigned grid, cudaStream_t s) {
    if (weighted) {
        if (has_lv)
            k_rows<T, NCH, true, true, TG><<<grid, 256, rows_smem<T>(true), s>>>(a, sched, nlight, ctr);
        else
            k_rows<T, NCH, true, false, TG><<<grid, 256, rows_smem<T>(true), s>>>(a, sched, nlight, ctr);
    } else {
        if (has_lv)
            k_rows<T, NCH, false, true, TG><<<grid, 256, rows_smem<T>(false), s>>>(a, sched, nlight, ctr);
        else
            k_rows<T, NCH, false, false, TG><<<grid, 256, rows_smem<T>(false), s>>>(a, sched, nlight, ctr);
    }
    LB_LAUNCH_CHECK();
}

// grid of k_vcs_items for one VCS level (enough resident blocks to fill the GPU; warps stride over the items); its
// 8 warps per block each write one partial
template <typename T, int NCH>
static int64_t vcs_grid(const VcsLevel &lv, bool fixed, int nsm) {
    if (lv.nitems == 0) return 0;
    const int64_t want = nblk(lv.nitems, 8);
    return fixed ? occ_grid(k_vcs_items<T, NCH, true>, want, nsm) : occ_grid(k_vcs_items<T, NCH, false>, want, nsm);
}

// Evaluation items of a VCS level's working set (after every change of the working set): each row's entries in
// items of at most VSEG; a row of several items gets consecutive partial slots.  SY starts at zero, so rows without
// entries contribute nothing.
void vcs_build_items(Problem &p, VcsLevel &lv, cudaStream_t s) {
    const int64_t n = p.n;
    std::vector<int64_t> ptr_h((size_t)n + 1);
    LB_CUDA(cudaMemcpyAsync(ptr_h.data(), lv.ptr.ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    std::vector<int4> items;
    std::vector<int> mrows, mslot{0};
    items.reserve((size_t)n);
    int slot = 0;
    for (int64_t i = 0; i < n; i++) {
        const int64_t a = ptr_h[i], b = ptr_h[i + 1];
        if (b <= a) continue;
        if (b - a <= VSEG) {
            items.push_back(make_int4((int)i, (int)a, (int)b, -1));
            continue;
        }
        for (int64_t e = a; e < b; e += VSEG)
            items.push_back(make_int4((int)i, (int)e, (int)std::min<int64_t>(b, e + VSEG), slot++));
        mrows.push_back((int)i);
        mslot.push_back(slot);
    }
    lv.nitems = (int64_t)items.size();
    lv.nmulti = (int64_t)mrows.size();
    lv.nslots = slot;
    upload(lv.items, items, s);
    upload(lv.multi_rows, mrows, s);
    upload(lv.multi_slot_ptr, mslot, s);
    lv.SY.alloc(sizeof(double) * (size_t)std::max<int64_t>(n, 1) * p.ld);
    LB_CUDA(cudaMemsetAsync(lv.SY.ptr, 0, sizeof(double) * (size_t)n * p.ld, s));
    lv.SYpart.alloc(sizeof(double) * (size_t)std::max(slot, 1) * p.ld);
    LB_CUDA(cudaStreamSynchronize(s));
}

struct Layout {
    int64_t off_quad, n_quad, off_lv, n_lv, off_lc, n_lc, off_vv, n_vv, off_vc, n_vc, off_tv, n_tv, off_tg, n_tg,
        off_tl, n_tl, total;
};

template <typename T, int NCH>
static void eval_typed(Problem &p, double rho, double tri_weight, int flags, cudaStream_t s) {
    const bool fixed = (flags & LB_EVAL_FIXED) != 0;
    const bool timing = (flags & LB_EVAL_TIMING) != 0;
    auto mark = [&]() {
        if (timing) LB_CUDA(cudaEventRecord(p.next_event(), s));
    };
    mark();
    const int ld = p.ld;
    const T *V = p.V.as<T>();
    const int64_t n = p.n;
    // --- partial-sum layout
    Layout lay{};
    // batched problems take the level instances of the row kernels (their per-graph degree correction lives there)
    const bool has_lv = !p.plev.empty() || !p.vlev.empty() || p.ngraphs > 0;
    using TG = typename std::conditional<std::is_same<T, double>::value, double, float>::type;
    const int nsm = p.ctx->c.num_sms;
    const unsigned nb_rows = rows_grid<T, NCH, TG>(p.weighted, has_lv, n, nsm);
    const int64_t nb_heavy = nblk(p.n_heavy, 8);
    int64_t sumP = 0;
    for (auto *lv : p.plev) sumP += lv->P;
    int64_t nb_vcs = 0;
    for (auto *lv : p.vlev) nb_vcs += 8 * vcs_grid<T, NCH>(*lv, fixed, nsm);
    constexpr int NPW = 32 / NCH;
    const int64_t nb_tri = fixed ? occ_grid(k_tri<T, NCH, true>, nblk(nblk(p.T, NPW), 8), nsm)
                                 : occ_grid(k_tri<T, NCH, false>, nblk(nblk(p.T, NPW), 8), nsm);
    int64_t o = 0;
    lay.off_quad = o; lay.n_quad = nb_rows + nb_heavy; o += lay.n_quad;
    lay.off_lv = o; lay.n_lv = sumP; o += sumP;
    lay.off_lc = o; lay.n_lc = sumP; o += sumP;
    lay.off_vv = o; lay.n_vv = nb_vcs; o += nb_vcs;
    lay.off_vc = o; lay.n_vc = nb_vcs; o += nb_vcs;
    lay.off_tv = o; lay.n_tv = nb_tri; o += nb_tri;
    lay.off_tg = o; lay.n_tg = nb_tri; o += nb_tri;
    lay.off_tl = o; lay.n_tl = nb_tri; o += nb_tri;
    // scratch for segmented-sum partials: max items over all plans
    int64_t max_items = p.zplan.scratch_rows();
    for (auto *lv : p.plev) max_items = std::max(max_items, lv->plan.scratch_rows());
    for (auto *lv : p.vlev) max_items = std::max({max_items, lv->yplan.scratch_rows(), lv->zplan.scratch_rows()});
    const int64_t seg_off = o;
    lay.total = o + max_items * ld;
    p.partials.alloc(sizeof(double) * (size_t)std::max<int64_t>(lay.total, 1));
    double *part = p.partials.as<double>();
    if (lay.total > seg_off || lay.total > 0) LB_CUDA(cudaMemsetAsync(part, 0, sizeof(double) * seg_off, s));
    double *segpart = part + seg_off;
    // --- 1. aggregates
    segsum_run<T, NCH>(p.zplan, V, ld, nullptr, nullptr, p.d.as<double>(), nullptr, segpart, p.z.as<double>(), s);
    for (auto *lv : p.plev)
        segsum_run<T, NCH>(lv->plan, V, ld, lv->members.as<int>(), nullptr, p.d.as<double>(), nullptr, segpart,
                       lv->Y.as<double>(), s);
    for (auto *lv : p.vlev)
        segsum_run<T, NCH>(lv->yplan, V, ld, lv->members.as<int>(), nullptr, p.d.as<double>(), nullptr, segpart,
                       lv->Y.as<double>(), s);
    mark();
    // --- 2. pair levels
    int64_t lo = 0;
    for (auto *lv : p.plev) {
        LB_CHECK(ld <= PT_LDMAX, LB_ERR_INVALID, "pair levels need rows of at most 64 elements");
        const unsigned nbq = (unsigned)nblk(lv->P, PT_Q);
        if (fixed)
            k_pair_level<true><<<nbq, 256, 0, s>>>(lv->P, ld, lv->Y.as<double>(), lv->sig.as<double>(),
                                                  lv->rq.as<double>(), lv->dsq.as<double>(), lv->w, rho,
                                                  lv->pp.as<double>(), lv->M.as<double>(), lv->pdiag.as<double>(),
                                                  part + lay.off_lv + lo, part + lay.off_lc + lo);
        else
            k_pair_level<false><<<nbq, 256, 0, s>>>(lv->P, ld, lv->Y.as<double>(), lv->sig.as<double>(),
                                                   lv->rq.as<double>(), lv->dsq.as<double>(), lv->w, rho,
                                                   lv->pp.as<double>(), lv->M.as<double>(), lv->pdiag.as<double>(),
                                                   part + lay.off_lv + lo, part + lay.off_lc + lo);
        LB_LAUNCH_CHECK();
        lo += lv->P;
    }
    mark();
    // --- 3. VCS levels
    int64_t vo = 0;
    for (auto *lv : p.vlev) {
        const int64_t vgrid = vcs_grid<T, NCH>(*lv, fixed, nsm);
        if (lv->nitems) {
            const unsigned nbi = (unsigned)vgrid;
            lv->inv2a.alloc(sizeof(double) * (size_t)std::max(lv->P, 1));
            if (!fixed) {
                k_vcs_inv2a<<<nblk(lv->P, 256), 256, 0, s>>>(lv->P, rho, lv->wv, lv->rq.as<double>(),
                                                             lv->inv2a.as<double>());
                LB_LAUNCH_CHECK();
            }
            if (fixed)
                k_vcs_items<T, NCH, true><<<nbi, 256, 0, s>>>(
                    lv->nitems, ld, lv->items.as<int4>(), V, p.d.as<double>(), lv->lab.as<int>(), lv->Y.as<double>(),
                    lv->col.as<int>(), lv->sig.as<double>(), lv->rq.as<double>(), lv->inv2a.as<double>(), lv->wv, rho,
                    lv->ppv.as<double>(), lv->slack.as<uint8_t>(), lv->stn.as<double>(), lv->SY.as<double>(),
                    lv->SYpart.as<double>(),
                    part + lay.off_vv + vo, part + lay.off_vc + vo);
            else
                k_vcs_items<T, NCH, false><<<nbi, 256, 0, s>>>(
                    lv->nitems, ld, lv->items.as<int4>(), V, p.d.as<double>(), lv->lab.as<int>(), lv->Y.as<double>(),
                    lv->col.as<int>(), lv->sig.as<double>(), lv->rq.as<double>(), lv->inv2a.as<double>(), lv->wv, rho,
                    lv->ppv.as<double>(), lv->slack.as<uint8_t>(), lv->stn.as<double>(), lv->SY.as<double>(),
                    lv->SYpart.as<double>(),
                    part + lay.off_vv + vo, part + lay.off_vc + vo);
            LB_LAUNCH_CHECK();
            if (lv->nmulti) {
                k_vcs_sy_combine<<<nblk(lv->nmulti * ld, 256), 256, 0, s>>>(
                    lv->nmulti, ld, lv->multi_rows.as<int>(), lv->multi_slot_ptr.as<int>(), lv->SYpart.as<double>(),
                    lv->SY.as<double>());
                LB_LAUNCH_CHECK();
            }
        }
        vo += 8 * vgrid;
        // Z_R = sum over the entries of column R of ppv_e d_i v_i (rows ascending)
        segsum_run<T, NCH>(lv->zplan, V, ld, lv->crow.as<int>(), lv->cent.as<int64_t>(), p.d.as<double>(),
                       lv->ppv.as<double>(), segpart, lv->Z.as<double>(), s);
        if (lv->zplan.nitems == 0 && lv->P)
            LB_CUDA(cudaMemsetAsync(lv->Z.ptr, 0, sizeof(double) * (size_t)lv->P * ld, s));
    }
    mark();
    // --- 4. triangles
    if (p.T) {
        const double rt = rho * tri_weight;
        if (fixed)
            k_tri<T, NCH, true><<<nb_tri, 256, 0, s>>>(p.T, ld, V, p.tri.as<int>(), p.lam.as<double>(), rt,
                                                       p.pt.as<double>(), p.gt.as<double>(), part + lay.off_tv,
                                                       part + lay.off_tg, part + lay.off_tl);
        else
            k_tri<T, NCH, false><<<nb_tri, 256, 0, s>>>(p.T, ld, V, p.tri.as<int>(), p.lam.as<double>(), rt,
                                                        p.pt.as<double>(), p.gt.as<double>(), part + lay.off_tv,
                                                        part + lay.off_tg, part + lay.off_tl);
        LB_LAUNCH_CHECK();
    }
    mark();
    // --- 5. rows
    RowArgs<T> a{};
    a.n = n;
    a.ld = ld;
    a.indptr = p.indptr.as<int64_t>();
    a.indices = p.indices.as<int>();
    a.w = p.weighted ? p.weights.as<float>() : nullptr;
    a.V = V;
    a.d = p.d.as<double>();
    a.invL = 1.0 / p.L;
    a.z = p.z.as<double>();
    a.tptr = p.T ? p.tptr.as<int64_t>() : nullptr;
    a.tinc = p.T ? p.tinc.as<int>() : nullptr;
    a.pt = p.T ? p.pt.as<double>() : nullptr;
    a.lv.npl = (int)p.plev.size();
    for (int l = 0; l < a.lv.npl; l++) {
        a.lv.plab[l] = p.plev[l]->lab.as<int>();
        a.lv.M[l] = p.plev[l]->M.as<double>();
        a.lv.pdiag[l] = p.plev[l]->pdiag.as<double>();
    }
    a.lv.nvl = (int)p.vlev.size();
    for (int m = 0; m < a.lv.nvl; m++) {
        auto *lv = p.vlev[m];
        a.lv.vlab[m] = lv->lab.as<int>();
        a.lv.ppv[m] = lv->ppv.as<double>();
        a.lv.SY[m] = lv->SY.as<double>();
        a.lv.Zv[m] = lv->Z.as<double>();
        a.lv.own[m] = lv->own.as<int64_t>();
    }
    a.G = p.G.ptr;
    a.write_G = (flags & LB_EVAL_GRAD) ? 1 : 0;
    a.part_quad = part + lay.off_quad;
    p.row_quad.alloc(sizeof(double) * std::max<int64_t>(n, 1));
    a.row_quad = p.row_quad.as<double>();
    a.gid = p.ngraphs ? p.gid.as<int>() : nullptr;
    a.ginvL = p.ngraphs ? p.ginvL.as<double>() : nullptr;
    a.heavy_items = p.heavy_items.as<int64_t>();
    a.heavy_rows = p.heavy_rows.as<int>();
    a.heavy_item_ptr = p.heavy_item_ptr.as<int64_t>();
    a.heavy_part = p.heavy_part.ptr;
    a.n_heavy_items = p.n_heavy_items;
    a.n_heavy = p.n_heavy;
    p.row_counter.alloc(sizeof(unsigned long long));
    unsigned long long *ctr = p.row_counter.as<unsigned long long>();
    const int nch_chunks = (int)nblk(n, ROW_CHUNK);
    auto run_rows = [&](int li) {
        LB_CUDA(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long), s));
        launch_rows<T, NCH, TG>(a, p.sched.as<int>(), p.nlight.as<int>() + (int64_t)li * nch_chunks, ctr, p.weighted,
                                has_lv, nb_rows, s);
    };
    if (p.light_idx < 0) {
        // autotune once per problem: time each light-row threshold on this evaluation's inputs, keep the fastest
        cudaEvent_t e0, e1;
        LB_CUDA(cudaEventCreate(&e0));
        LB_CUDA(cudaEventCreate(&e1));
        float best = 1e30f;
        int best_i = 0;
        for (int li = 0; li < N_LIGHT; li++) {
            run_rows(li);                   // untimed first launch (module loading, cold caches)
            LB_CUDA(cudaEventRecord(e0, s));
            run_rows(li);
            LB_CUDA(cudaEventRecord(e1, s));
            LB_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            LB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            p.tune_ms[li] = ms;
            if (ms < best) {
                best = ms;
                best_i = li;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        p.light_idx = best_i;
    }
    run_rows(p.light_idx);
    if (p.n_heavy) {
        if (p.weighted)
            k_heavy_part<T, NCH, true><<<nblk(p.n_heavy_items, 8), 256, 0, s>>>(a);
        else
            k_heavy_part<T, NCH, false><<<nblk(p.n_heavy_items, 8), 256, 0, s>>>(a);
        LB_LAUNCH_CHECK();
        if (has_lv)
            k_heavy_fin<T, NCH, true, TG><<<nb_heavy, 256, 0, s>>>(a);
        else
            k_heavy_fin<T, NCH, false, TG><<<nb_heavy, 256, 0, s>>>(a);
        LB_LAUNCH_CHECK();
    }
    k_rowsum<<<(unsigned)lay.n_quad, 256, 0, s>>>(n, a.row_quad, part + lay.off_quad);
    LB_LAUNCH_CHECK();
    mark();
    // --- 6. finalize
    FinArgs f{};
    f.part = part;
    f.off_quad = lay.off_quad; f.n_quad = lay.n_quad;
    f.off_lv = lay.off_lv; f.n_lv = lay.n_lv;
    f.off_lc = lay.off_lc; f.n_lc = lay.n_lc;
    f.off_vv = lay.off_vv; f.n_vv = lay.n_vv;
    f.off_vc = lay.off_vc; f.n_vc = lay.n_vc;
    f.off_tv = lay.off_tv; f.n_tv = lay.n_tv;
    f.off_tg = lay.off_tg; f.n_tg = lay.n_tg;
    f.off_tl = lay.off_tl; f.n_tl = lay.n_tl;
    f.z = p.z.as<double>();
    f.ld = ld;
    f.L = p.L;
    f.C0 = p.C0;
    f.fixed = fixed ? 1 : 0;
    f.out = p.scal.as<lb_eval_out>();
    f.gsum = nullptr;
    if (p.ngraphs) {
        p.gpart.alloc(sizeof(double) * 2 * GRAPH_SLICES * (size_t)p.ngraphs);
        k_graph_part<<<dim3(p.ngraphs, GRAPH_SLICES), 256, 0, s>>>(
            p.gptr.as<int64_t>(), p.gtptr.as<int64_t>(), p.row_quad.as<double>(), p.T ? p.pt.as<double>() : nullptr,
            p.T ? p.lam.as<double>() : nullptr, rho * tri_weight, fixed ? 1 : 0, p.gpart.as<double>());
        LB_LAUNCH_CHECK();
        k_graph_fin<<<nblk(p.ngraphs, 128), 128, 0, s>>>(p.ngraphs, ld, p.gpart.as<double>(), p.z.as<double>(),
                                                         p.gL.as<double>(), p.gC0.as<double>(), p.gout.as<double>());
        LB_LAUNCH_CHECK();
        k_graph_zz<<<1, 256, 0, s>>>(p.ngraphs, p.gout.as<double>(), p.gL.as<double>(), p.gsum.as<double>());
        LB_LAUNCH_CHECK();
        f.gsum = p.gsum.as<double>();
    }
    k_finalize<<<1, 512, 0, s>>>(f);
    LB_LAUNCH_CHECK();
    mark();
    // kernels launched by this evaluation
    int64_t nl = 1 + 1 + 1 + (p.T ? 1 : 0) + (p.n_heavy ? 2 : 0) + (p.ngraphs ? 3 : 0);   // + per-graph sums
    auto seg = [](const SegPlan &pl) { return pl.nseg ? (pl.nitems ? 2 : 1) : 0; };
    nl += seg(p.zplan);
    for (auto *lv : p.plev) nl += seg(lv->plan) + 1;
    for (auto *lv : p.vlev)
        nl += seg(lv->yplan) + seg(lv->zplan) + (lv->nitems ? (fixed ? 1 : 2) : 0) + (lv->nmulti ? 1 : 0);
    p.launches += nl;
}

// Access-policy window over V on the evaluation stream: a share of V's lines persisting in L2 (the random gathers of
// the inter-community edges), the rest streaming.
void apply_l2_window(Problem &p, cudaStream_t s) {
    const Ctx &c = p.ctx->c;
    if (c.v_persist <= 0 || c.persist_max == 0 || c.window_max == 0) return;
    const size_t bytes = std::min(p.V.bytes, c.window_max);
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.base_ptr = p.V.ptr;
    v.accessPolicyWindow.num_bytes = bytes;
    v.accessPolicyWindow.hitRatio = (float)std::min(1.0, c.v_persist * (double)c.persist_max / (double)bytes);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    LB_CUDA(cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &v));
}

void eval_run(Problem &p, double rho, double tri_weight, int flags, cudaStream_t s) {
    apply_l2_window(p, s);
    const int nch = (int)(p.ld * dtype_size(p.vdtype) / 16);
    LB_DISPATCH_T(p.vdtype, LB_DISPATCH_NCH(nch, eval_typed<T, NCH>(p, rho, tri_weight, flags, s)));
    p.have_eval = true;
    p.last_flags = flags;
}

// Y_R = sum_{i in R} d_i v_i of one VCS level at the current V (the evaluation's deterministic segmented sums).
void vcs_cluster_sums(Problem &p, VcsLevel &lv, cudaStream_t s) {
    const int nch = (int)(p.ld * dtype_size(p.vdtype) / 16);
    DBuf part;
    part.alloc(sizeof(double) * (size_t)std::max<int64_t>(lv.yplan.scratch_rows(), 1) * p.ld);
    LB_DISPATCH_T(p.vdtype, LB_DISPATCH_NCH(nch, segsum_run<T, NCH>(lv.yplan, p.V.as<T>(), p.ld, lv.members.as<int>(),
                                                                    nullptr, p.d.as<double>(), nullptr,
                                                                    part.as<double>(), lv.Y.as<double>(), s)));
    LB_CUDA(cudaStreamSynchronize(s));
}

static const int *ord_of(const Problem &p) { return p.permuted ? p.order_d.as<int>() : nullptr; }

void convert_V_from_f64(Problem &p, const double *src, cudaStream_t s) {
    const int64_t tot = p.n * p.ld;
    LB_DISPATCH_T(p.vdtype,
                  k_from_f64<T><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, src, p.V.as<T>(), ord_of(p)));
    LB_LAUNCH_CHECK();
}
void convert_V_raw(Problem &p, const void *src, cudaStream_t s) {
    const int64_t tot = p.n * p.ld;
    LB_DISPATCH_T(p.vdtype, k_raw_in<T><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, (const T *)src,
                                                                        p.V.as<T>(), ord_of(p)));
    LB_LAUNCH_CHECK();
}
void convert_V_to_f64(const Problem &p, double *out, cudaStream_t s) {
    const int64_t tot = p.n * p.r;
    LB_DISPATCH_T(p.vdtype,
                  k_to_f64<T><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, p.V.as<T>(), out, ord_of(p)));
    LB_LAUNCH_CHECK();
}
void G_raw(const Problem &p, void *out, cudaStream_t s) {
    const int64_t tot = p.n * p.r;
    if (p.vdtype == LB_F64)
        k_raw_out<double><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, p.G.as<double>(), (double *)out, ord_of(p));
    else
        k_raw_out<float><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, p.G.as<float>(), (float *)out, ord_of(p));
    LB_LAUNCH_CHECK();
}
void G_to_f64(const Problem &p, double *out, cudaStream_t s) {
    const int64_t tot = p.n * p.r;
    if (p.vdtype == LB_F64)
        k_to_f64<double><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, p.G.as<double>(), out, ord_of(p));
    else
        k_to_f64<float><<<nblk(tot, 256), 256, 0, s>>>(p.n, p.r, p.ld, p.G.as<float>(), out, ord_of(p));
    LB_LAUNCH_CHECK();
}

// Row schedule of k_rows: per chunk of ROW_CHUNK rows, the rows by increasing work (edges + 2 x incidences, stable;
// heavy rows last), and for every light threshold LIGHT_WORK[li] the number of light rows at the front of each chunk.
static void build_schedule(Problem &p, cudaStream_t s) {
    const bool tri = !p.tptr_h.empty();
    const int64_t nch = (p.n + ROW_CHUNK - 1) / ROW_CHUNK;
    std::vector<int> sched((size_t)p.n), nlight((size_t)(N_LIGHT * nch));
    std::vector<std::pair<int64_t, int>> buf;
    for (int64_t c = 0; c < nch; c++) {
        const int64_t a = c * ROW_CHUNK, b = std::min<int64_t>(p.n, a + ROW_CHUNK);
        buf.clear();
        for (int64_t i = a; i < b; i++) {
            const int64_t deg = p.indptr_h[i + 1] - p.indptr_h[i];
            const int64_t nt = tri ? p.tptr_h[i + 1] - p.tptr_h[i] : 0;
            const bool heavy = deg > HEAVY_DEG || nt > HEAVY_TRI;
            buf.emplace_back(heavy ? INT64_MAX : deg + 2 * nt, (int)i);
        }
        std::stable_sort(buf.begin(), buf.end(), [](const std::pair<int64_t, int> &x, const std::pair<int64_t, int> &y) {
            return x.first < y.first;
        });
        for (int64_t k = 0; k < b - a; k++) sched[a + k] = buf[k].second;
        for (int li = 0; li < N_LIGHT; li++) {
            int nl = 0;
            while (nl < b - a && buf[nl].first <= LIGHT_WORK[li]) nl++;
            nlight[(size_t)li * nch + c] = nl;
        }
    }
    upload(p.sched, sched, s);
    upload(p.nlight, nlight, s);
}

// Heavy rows (is_heavy): items (row, kind, e0, e1) of at most SEG_EDGES edges / SEG_TRI incidences.
void build_heavy(Problem &p, cudaStream_t s) {
    build_schedule(p, s);
    std::vector<int64_t> items, iptr{0};
    std::vector<int> rows;
    const bool tri = !p.tptr_h.empty();
    for (int64_t i = 0; i < p.n; i++) {
        const int64_t e0 = p.indptr_h[i], e1 = p.indptr_h[i + 1];
        const int64_t t0 = tri ? p.tptr_h[i] : 0, t1 = tri ? p.tptr_h[i + 1] : 0;
        if (!(e1 - e0 > HEAVY_DEG || t1 - t0 > HEAVY_TRI)) continue;
        rows.push_back((int)i);
        for (int64_t e = e0; e < e1; e += SEG_EDGES) {
            items.insert(items.end(), {i, 0, e, std::min<int64_t>(e1, e + SEG_EDGES)});
        }
        for (int64_t t = t0; t < t1; t += SEG_TRI) {
            items.insert(items.end(), {i, 1, t, std::min<int64_t>(t1, t + SEG_TRI)});
        }
        iptr.push_back((int64_t)items.size() / 4);
    }
    p.n_heavy = (int64_t)rows.size();
    p.n_heavy_items = (int64_t)items.size() / 4;
    if (p.n_heavy) {
        upload(p.heavy_items, items, s);
        upload(p.heavy_rows, rows, s);
        upload(p.heavy_item_ptr, iptr, s);
        p.heavy_part.alloc(sizeof(double) * (size_t)p.n_heavy_items * p.ld);
    }
}

void multiplier_update(Problem &p, cudaStream_t s) {
    // alm_vcs.py:1704 Lv.sig = pp; 1709-1710 VCS sig = ppv + age_update; 1723 lam = pt
    for (auto *lv : p.plev) {
        std::swap(lv->sig.ptr, lv->pp.ptr);
        std::swap(lv->sig.owner, lv->pp.owner);
        std::swap(lv->sig.bytes, lv->pp.bytes);
    }
    for (auto *lv : p.vlev) {
        if (lv->nnz) {
            k_age_update<<<nblk(lv->nnz, 256), 256, 0, s>>>(lv->nnz, lv->slack.as<uint8_t>(), lv->age.as<uint8_t>());
            LB_LAUNCH_CHECK();
        }
        std::swap(lv->sig.ptr, lv->ppv.ptr);
        std::swap(lv->sig.owner, lv->ppv.owner);
        std::swap(lv->sig.bytes, lv->ppv.bytes);
    }
    if (p.T) {
        std::swap(p.lam.ptr, p.pt.ptr);
        std::swap(p.lam.owner, p.pt.owner);
        std::swap(p.lam.bytes, p.pt.bytes);
    }
}

}  // namespace lb
