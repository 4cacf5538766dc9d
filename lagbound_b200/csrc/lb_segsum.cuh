// Deterministic segmented row sums (FP64) shared by the evaluation and the sweeps: out[s] = sum over the entries of
// segment s of coef_e * V[row_e], computed in fixed-size work items (one warp each) whose partials are combined in
// item order.
#pragma once

#include "lb_internal.cuh"

namespace lb {
namespace seg {
constexpr unsigned FULL = 0xffffffffu;
static inline unsigned nblk(int64_t work, int per) { return (unsigned)((work + per - 1) / per); }
template <int NCH, typename A, int E> __device__ __forceinline__ void reduce_groups(A (&acc)[E]) {
#pragma unroll
    for (int off = NCH; off < 32; off <<= 1)
#pragma unroll
        for (int k = 0; k < E; k++) acc[k] += __shfl_xor_sync(FULL, acc[k], off);
}
// ============================================================================================ segmented sums
// part[item] = sum_{e in [e0,e1)} coef_e * V[row_e]   (FP64), coef_e = d[row_e] (MODE 0) or s_e * d[row_e] (MODE 1,
// s_e = sval[ent_e]).  Rows: row_e = rows[e] (or e when rows == nullptr).  The warp loads the rows, volumes and
// multipliers of 32 entries at once (one per lane, independent gathers), then its lane groups take the entries
// sub, sub + NPW, ... of the chunk with their row loads in flight together; every lane group adds its entries in
// entry order.
template <typename T, int NCH, int MODE>
__global__ void __launch_bounds__(256) k_segsum_items(const T *__restrict__ V, int ld, int64_t nitems,
                                                      const int64_t *__restrict__ e0s, const int64_t *__restrict__ e1s,
                                                      const int *__restrict__ rows, const int64_t *__restrict__ ent,
                                                      const double *__restrict__ d, const double *__restrict__ sval,
                                                      double *__restrict__ part) {
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    const int lane = threadIdx.x & 31, sub = lane / NCH, ch = lane % NCH;
    const int64_t it = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (it >= nitems) return;
    const int64_t e0 = e0s[it], e1 = e1s[it];
    double acc[EPL];
#pragma unroll
    for (int k = 0; k < EPL; k++) acc[k] = 0.0;
    for (int64_t cb = e0; cb < e1; cb += 32) {
        const int64_t e = cb + lane;
        const bool in = e < e1;
        const int64_t ie = in ? (rows ? (int64_t)__ldcs(rows + e) : e) : 0;
        const double ce = in ? d[ie] : 0.0;
        const double se = (MODE == 1 && in) ? sval[__ldcs(ent + e)] : 1.0;
        const int cnt = (int)min((int64_t)32, e1 - cb);
#pragma unroll 4
        for (int u = 0; u < 32 / NPW; u++) {
            const int src = u * NPW + sub;
            const int64_t i = __shfl_sync(FULL, ie, src);
            const double c = __shfl_sync(FULL, ce, src);
            const double sv = __shfl_sync(FULL, se, src);
            if (src >= cnt || (MODE == 1 && sv == 0.0)) continue;
            double x[EPL];
            load_d<T>(V + i * ld + ch * EPL, x);
            if (MODE == 1) {
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] += sv * (c * x[k]);
            } else {
#pragma unroll
                for (int k = 0; k < EPL; k++) acc[k] += c * x[k];
            }
        }
    }
    reduce_groups<NCH>(acc);
    if (sub == 0) {
#pragma unroll
        for (int k = 0; k < EPL; k++) part[it * ld + ch * EPL + k] = acc[k];
    }
}

// out[s] = sum of the partials of segment s; block per segment, thread (column c, slice k) sums the items
// k, k + S, ... in order, slices combined in order (S = 256 / ld).
static __global__ void __launch_bounds__(256) k_seg_combine(int64_t nseg, int ld, const int64_t *__restrict__ seg_item_ptr,
                                                     const double *__restrict__ part, double *__restrict__ out) {
    __shared__ double sh[256];
    const int64_t s = blockIdx.x;
    const int S = 256 / ld;
    const int c = threadIdx.x % ld, k = threadIdx.x / ld;
    const int64_t a = seg_item_ptr[s], b = seg_item_ptr[s + 1];
    double acc = 0.0;
    if (k < S)
        for (int64_t it = a + k; it < b; it += S) acc += part[it * ld + c];
    sh[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < ld) {
        double t = 0.0;
        for (int q = 0; q < S; q++) t += sh[q * ld + threadIdx.x];
        out[s * ld + threadIdx.x] = t;
    }
}

// First level of a two-level combine: grp[g] = sum of the partials of the items of group g, block per group, thread
// (column c, slice k) sums the items k, k + S, ... in order, slices combined in order (S = 256 / ld).
static __global__ void __launch_bounds__(256) k_seg_groups(int64_t ngroups, int ld,
                                                    const int64_t *__restrict__ group_item_ptr,
                                                    const double *__restrict__ part, double *__restrict__ grp) {
    __shared__ double sh[256];
    const int64_t g = blockIdx.x;
    const int S = 256 / ld;
    const int c = threadIdx.x % ld, k = threadIdx.x / ld;
    const int64_t a = group_item_ptr[g], b = group_item_ptr[g + 1];
    double acc = 0.0;
    if (k < S)
        for (int64_t it = a + k; it < b; it += S) acc += part[it * ld + c];
    sh[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < ld) {
        double t = 0.0;
        for (int q = 0; q < S; q++) t += sh[q * ld + threadIdx.x];
        grp[g * ld + threadIdx.x] = t;
    }
}

}  // namespace seg

template <typename T, int NCH>
static void segsum_run(const SegPlan &pl, const T *V, int ld, const int *rows, const int64_t *ent, const double *d,
                   const double *sval, double *part, double *out, cudaStream_t s) {
    if (pl.nseg == 0) return;
    if (pl.nitems) {
        if (sval)
            seg::k_segsum_items<T, NCH, 1><<<seg::nblk(pl.nitems, 8), 256, 0, s>>>(V, ld, pl.nitems, pl.item_e0.as<int64_t>(),
                                                                       pl.item_e1.as<int64_t>(), rows, ent, d, sval,
                                                                       part);
        else
            seg::k_segsum_items<T, NCH, 0><<<seg::nblk(pl.nitems, 8), 256, 0, s>>>(V, ld, pl.nitems, pl.item_e0.as<int64_t>(),
                                                                       pl.item_e1.as<int64_t>(), rows, ent, d, sval,
                                                                       part);
        LB_LAUNCH_CHECK();
    }
    if (pl.ngroups) {
        double *grp = part + pl.nitems * ld;
        seg::k_seg_groups<<<(unsigned)pl.ngroups, 256, 0, s>>>(pl.ngroups, ld, pl.group_item_ptr.as<int64_t>(), part,
                                                              grp);
        LB_LAUNCH_CHECK();
        seg::k_seg_combine<<<(unsigned)pl.nseg, 256, 0, s>>>(pl.nseg, ld, pl.seg_group_ptr.as<int64_t>(), grp, out);
    } else {
        seg::k_seg_combine<<<(unsigned)pl.nseg, 256, 0, s>>>(pl.nseg, ld, pl.seg_item_ptr.as<int64_t>(), part, out);
    }
    LB_LAUNCH_CHECK();
}

}  // namespace lb
