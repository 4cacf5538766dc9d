// VCS working sets on the device: the column view and caller map of a working set, and the solver's working-set
// update (alm_vcs.py:1713-1720: drop aged entries, separate, vcsops.py:457-464 update_ws) without a host round trip.
//
// A working set is a row CSR in internal row order (ptr int64, col int32 ascending in each row, sig f64, age u8).
// The update keeps the entries with age < drop_age, merges in the separation's selection (sorted by (row, cluster))
// with sig 0 and age 0, and rebuilds what the evaluation reads: the entry of (i, lab_i), the column view (entries
// sorted by cluster, rows ascending: a stable radix sort of the row-major entries by cluster) and, for a locality
// order, the map to the caller's entry order (rows in the caller's order, entries in each row as stored).
// Everything is integer work over the entries, HBM-bound: warp per row for the per-row passes, one CUB radix sort.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "lb_internal.cuh"

namespace lb {
namespace {

constexpr int WPB = 8;   // warps per 256-thread block

unsigned grid_for(int64_t units, int per_block) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((units + per_block - 1) / per_block, (int64_t)1 << 20));
}

int bits_for(uint64_t x) {   // bits needed for values in [0, x)
    int b = 1;
    while (b < 64 && (((uint64_t)1 << b) < x)) b++;
    return b;
}

// row of every entry
__global__ void k_rowof(int64_t n, const int64_t *__restrict__ ptr, int *__restrict__ rowof) {
    const int lane = threadIdx.x & 31;
    for (int64_t k = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5); k < n; k += (int64_t)gridDim.x * WPB)
        for (int64_t e = ptr[k] + lane; e < ptr[k + 1]; e += 32) rowof[e] = (int)k;
}

// own[k] = the entry (k, lab_k), or -1 (columns ascending in a row: binary search)
__global__ void k_own(int64_t n, const int64_t *__restrict__ ptr, const int *__restrict__ col,
                      const int *__restrict__ lab, int64_t *__restrict__ own) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = ptr[k], hi = ptr[k + 1];
        const int c = lab[k];
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (col[mid] < c) lo = mid + 1;
            else hi = mid;
        }
        own[k] = (lo < ptr[k + 1] && col[lo] == c) ? lo : -1;
    }
}

__global__ void k_iota64(int64_t m, int64_t *__restrict__ x) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = i;
}

// column view from the entries sorted by column: crow = row of each entry, cptr[c] = first position of column c
__global__ void k_colview(int64_t nnz, int P, const int *__restrict__ sorted_col, const int64_t *__restrict__ cent,
                          const int *__restrict__ rowof, int *__restrict__ crow, int64_t *__restrict__ cptr) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
        crow[q] = rowof[cent[q]];
        const int c = sorted_col[q], cp = q ? sorted_col[q - 1] : -1;
        for (int b = cp + 1; b <= c; b++) cptr[b] = q;     // columns (cp, c] start here
        if (q == nnz - 1)
            for (int b = c + 1; b <= P; b++) cptr[b] = nnz;
    }
}

// caller map: ccnt[order[k]] = entries of internal row k
__global__ void k_caller_counts(int64_t n, const int64_t *__restrict__ ptr, const int *__restrict__ order,
                                int64_t *__restrict__ ccnt) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        ccnt[order[k]] = ptr[k + 1] - ptr[k];
}

__global__ void k_ent_map(int64_t n, const int64_t *__restrict__ ptr, const int *__restrict__ order,
                          const int64_t *__restrict__ cptr_caller, int64_t *__restrict__ emap) {
    const int lane = threadIdx.x & 31;
    for (int64_t k = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5); k < n; k += (int64_t)gridDim.x * WPB) {
        const int64_t e0 = ptr[k], base = cptr_caller[order[k]];
        for (int64_t e = e0 + lane; e < ptr[k + 1]; e += 32) emap[e] = base + (e - e0);
    }
}

template <typename E>
__global__ void k_to_caller(int64_t nnz, const int64_t *__restrict__ emap, const E *__restrict__ src,
                            E *__restrict__ dst) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        dst[emap[e]] = src[e];
}

// kept entries per row: age < drop (drop <= 0 keeps every entry)
__global__ void k_keep_count(int64_t n, const int64_t *__restrict__ ptr, const uint8_t *__restrict__ age, int drop,
                             int64_t *__restrict__ kcnt) {
    const int lane = threadIdx.x & 31;
    for (int64_t k = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5); k < n; k += (int64_t)gridDim.x * WPB) {
        int64_t c = 0;
        for (int64_t e = ptr[k] + lane; e < ptr[k + 1]; e += 32) c += (drop <= 0 || age[e] < drop) ? 1 : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) kcnt[k] = c;
    }
}

// first selected key of each row (keys row * P + cluster, ascending): aptr[k] for k in [0, n]
__global__ void k_add_ptr(int64_t n, int64_t P, int64_t A, const int64_t *__restrict__ akeys,
                          int64_t *__restrict__ aptr) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t key = k * P;
        int64_t lo = 0, hi = A;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (akeys[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        aptr[k] = lo;
    }
}

// the kept entries of each row, compacted in order to kptr[k]
__global__ void k_compact(int64_t n, const int64_t *__restrict__ ptr, const int *__restrict__ col,
                          const double *__restrict__ sig, const uint8_t *__restrict__ age, int drop,
                          const int64_t *__restrict__ kptr, int *__restrict__ tcol, double *__restrict__ tsig,
                          uint8_t *__restrict__ tage) {
    const int lane = threadIdx.x & 31;
    for (int64_t k = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5); k < n; k += (int64_t)gridDim.x * WPB) {
        int64_t o = kptr[k];
        for (int64_t e0 = ptr[k]; e0 < ptr[k + 1]; e0 += 32) {
            const int64_t e = e0 + lane;
            const bool in = e < ptr[k + 1];
            const uint8_t a = in ? age[e] : 0;
            const bool kp = in && (drop <= 0 || a < drop);
            const unsigned m = __ballot_sync(0xffffffffu, kp);
            if (kp) {
                const int64_t q = o + __popc(m & ((1u << lane) - 1u));
                tcol[q] = col[e];
                tsig[q] = sig[e];
                tage[q] = a;
            }
            o += __popc(m);
        }
    }
}

// merge of the kept entries [kptr[k], kptr[k+1]) and the selected ones [aptr[k], aptr[k+1]) of each row by cluster;
// a selected entry equal to a kept one sets *clash (the separation only selects entries outside the working set)
__global__ void k_merge(int64_t n, int64_t P, const int64_t *__restrict__ kptr, const int *__restrict__ tcol,
                        const double *__restrict__ tsig, const uint8_t *__restrict__ tage,
                        const int64_t *__restrict__ aptr, const int64_t *__restrict__ akeys,
                        int64_t *__restrict__ nptr, int *__restrict__ ncol, double *__restrict__ nsig,
                        uint8_t *__restrict__ nage, int *__restrict__ clash) {
    const int lane = threadIdx.x & 31;
    for (int64_t k = (int64_t)blockIdx.x * WPB + (threadIdx.x >> 5); k < n; k += (int64_t)gridDim.x * WPB) {
        const int64_t k0 = kptr[k], k1 = kptr[k + 1], a0 = aptr[k], a1 = aptr[k + 1], base = k0 + a0;
        if (lane == 0) {
            nptr[k] = base;
            if (k == n - 1) nptr[n] = k1 + a1;
        }
        for (int64_t j = k0 + lane; j < k1; j += 32) {   // kept: rank among kept + selected with a smaller cluster
            const int64_t key = k * P + tcol[j];
            int64_t lo = a0, hi = a1;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (akeys[mid] < key) lo = mid + 1;
                else hi = mid;
            }
            const int64_t q = base + (j - k0) + (lo - a0);
            ncol[q] = tcol[j];
            nsig[q] = tsig[j];
            nage[q] = tage[j];
        }
        for (int64_t a = a0 + lane; a < a1; a += 32) {   // selected: rank among selected + kept with a smaller cluster
            const int c = (int)(akeys[a] - k * P);
            int64_t lo = k0, hi = k1;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                if (tcol[mid] < c) lo = mid + 1;
                else hi = mid;
            }
            if (lo < k1 && tcol[lo] == c) atomicExch(clash, 1);
            const int64_t q = base + (a - a0) + (lo - k0);
            ncol[q] = c;
            nsig[q] = 0.0;
            nage[q] = 0;
        }
    }
}

void swap_buf(DBuf &a, DBuf &b) {
    std::swap(a.ptr, b.ptr);
    std::swap(a.owner, b.owner);
    std::swap(a.bytes, b.bytes);
}

// exclusive prefix sum of cnt[0, n) into out[0, n] (out[n] = total)
void excl_scan(const int64_t *cnt, int64_t *out, int64_t n, DBuf &tmp, cudaStream_t s) {
    LB_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    if (n == 0) return;
    size_t tb = 0;
    LB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, cnt, out + 1, (int)n, s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceScan::InclusiveSum(tmp.ptr, tb, cnt, out + 1, (int)n, s));
}

}  // namespace

void vcs_rebuild_views(Problem &p, VcsLevel &lv, cudaStream_t s) {
    const int64_t n = p.n, nnz = lv.nnz;
    LB_CHECK(nnz < ((int64_t)1 << 31), LB_ERR_INVALID, "working set too large (2^31 entries)");
    const int64_t *ptr = lv.ptr.as<int64_t>();
    const unsigned gw = grid_for(n, WPB), gt = grid_for(n, 256);
    lv.own.alloc(sizeof(int64_t) * std::max<int64_t>(n, 1));
    k_own<<<gt, 256, 0, s>>>(n, ptr, lv.col.as<int>(), lv.lab.as<int>(), lv.own.as<int64_t>());
    LB_LAUNCH_CHECK();
    const size_t e1 = (size_t)std::max<int64_t>(nnz, 1);
    lv.crow.alloc(sizeof(int) * e1);
    lv.cent.alloc(sizeof(int64_t) * e1);
    lv.cptr.alloc(sizeof(int64_t) * ((size_t)lv.P + 1));
    lv.ppv.alloc(sizeof(double) * e1);
    lv.stn.alloc(sizeof(double) * e1);
    lv.stZ.alloc(sizeof(double) * e1);
    lv.slack.alloc(e1);
    std::vector<int64_t> cptr_h((size_t)lv.P + 1, 0);
    if (nnz) {
        DBuf &rowof = p.scratch("lb_vgrow:226:rowof"), &keys = p.scratch("lb_vgrow:226:keys"),
             &vals = p.scratch("lb_vgrow:226:vals"), &tmp = p.scratch("lb_vgrow:226:tmp");
        rowof.alloc(sizeof(int) * nnz);
        keys.alloc(sizeof(int) * nnz);
        vals.alloc(sizeof(int64_t) * nnz);
        k_rowof<<<gw, 256, 0, s>>>(n, ptr, rowof.as<int>());
        LB_LAUNCH_CHECK();
        k_iota64<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, vals.as<int64_t>());
        LB_LAUNCH_CHECK();
        // stable by cluster over the row-major entries: rows ascending within a cluster
        size_t tb = 0;
        const int eb = bits_for((uint64_t)lv.P);
        LB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, lv.col.as<int>(), keys.as<int>(), vals.as<int64_t>(),
                                                lv.cent.as<int64_t>(), (int)nnz, 0, eb, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, lv.col.as<int>(), keys.as<int>(), vals.as<int64_t>(),
                                                lv.cent.as<int64_t>(), (int)nnz, 0, eb, s));
        k_colview<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, lv.P, keys.as<int>(), lv.cent.as<int64_t>(),
                                                     rowof.as<int>(), lv.crow.as<int>(), lv.cptr.as<int64_t>());
        LB_LAUNCH_CHECK();
        LB_CUDA(cudaMemcpyAsync(cptr_h.data(), lv.cptr.ptr, sizeof(int64_t) * cptr_h.size(), cudaMemcpyDeviceToHost,
                                s));
    } else {
        LB_CUDA(cudaMemsetAsync(lv.cptr.ptr, 0, sizeof(int64_t) * cptr_h.size(), s));
    }
    if (p.permuted && nnz) {
        DBuf &ccnt = p.scratch("lb_vgrow:251:ccnt"), &cptr_caller = p.scratch("lb_vgrow:251:cptr_caller"),
             &tmp = p.scratch("lb_vgrow:251:tmp");
        ccnt.alloc(sizeof(int64_t) * n);
        cptr_caller.alloc(sizeof(int64_t) * (n + 1));
        k_caller_counts<<<gt, 256, 0, s>>>(n, ptr, p.order_d.as<int>(), ccnt.as<int64_t>());
        LB_LAUNCH_CHECK();
        excl_scan(ccnt.as<int64_t>(), cptr_caller.as<int64_t>(), n, tmp, s);
        lv.ent_map.alloc(sizeof(int64_t) * nnz);
        k_ent_map<<<gw, 256, 0, s>>>(n, ptr, p.order_d.as<int>(), cptr_caller.as<int64_t>(),
                                     lv.ent_map.as<int64_t>());
        LB_LAUNCH_CHECK();
    }
    LB_CUDA(cudaStreamSynchronize(s));
    lv.zplan.build(cptr_h, s);
    vcs_build_items(p, lv, s);
    p.launches += 5;
}

void vcs_grow_run(Problem &p, int level, int64_t nadd, double tol, int mode, int drop_age, int64_t max_nnz,
                  double *stats, int64_t *counts, cudaStream_t s) {
    VcsLevel &lv = *p.vlev[level];
    const int64_t n = p.n, nnz0 = lv.nnz, P = lv.P;
    const unsigned gw = grid_for(n, WPB), gt = grid_for(n + 1, 256);
    DBuf &kcnt = p.scratch("lb_vgrow:273:kcnt"), &kptr = p.scratch("lb_vgrow:273:kptr"),
         &tmp = p.scratch("lb_vgrow:273:tmp");
    kcnt.alloc(sizeof(int64_t) * std::max<int64_t>(n, 1));
    kptr.alloc(sizeof(int64_t) * (n + 1));
    k_keep_count<<<gw, 256, 0, s>>>(n, lv.ptr.as<int64_t>(), lv.age.as<uint8_t>(), drop_age, kcnt.as<int64_t>());
    LB_LAUNCH_CHECK();
    excl_scan(kcnt.as<int64_t>(), kptr.as<int64_t>(), n, tmp, s);
    int64_t K = 0;
    LB_CUDA(cudaMemcpyAsync(&K, kptr.as<int64_t>() + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    // alm_vcs.py:1717-1719: room = max(0, vcs_max - kept); separate max(1, min(vcs_add, room)); none join at room 0
    const int64_t room = std::max<int64_t>(0, max_nnz - K);
    int64_t got = 0;
    vcs_separate_run(p, level, std::max<int64_t>(1, std::min<int64_t>(nadd, room)), tol, mode, &got, stats, s, false);
    const int64_t A = room > 0 ? got : 0;
    const int64_t nnz = K + A;
    LB_CHECK(nnz < ((int64_t)1 << 31), LB_ERR_INVALID, "working set too large (2^31 entries)");
    // the selection in (row, cluster) order
    DBuf &akeys = p.scratch("lb_vgrow:290:akeys"), &aptr = p.scratch("lb_vgrow:290:aptr");
    akeys.alloc(sizeof(int64_t) * std::max<int64_t>(A, 1));
    if (A) {
        size_t tb = 0;
        const int eb = bits_for((uint64_t)n * (uint64_t)P);
        LB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, p.vsep_dev.as<int64_t>(), akeys.as<int64_t>(), (int)A, 0,
                                               eb, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, p.vsep_dev.as<int64_t>(), akeys.as<int64_t>(), (int)A, 0,
                                               eb, s));
    }
    aptr.alloc(sizeof(int64_t) * (n + 1));
    k_add_ptr<<<gt, 256, 0, s>>>(n, P, A, akeys.as<int64_t>(), aptr.as<int64_t>());
    LB_LAUNCH_CHECK();
    // kept entries compacted, then merged with the selection
    const size_t k1 = (size_t)std::max<int64_t>(K, 1), e1 = (size_t)std::max<int64_t>(nnz, 1);
    DBuf &tcol = p.scratch("lb_vgrow:306:tcol"), &tsig = p.scratch("lb_vgrow:306:tsig"),
         &tage = p.scratch("lb_vgrow:306:tage"), &nptr = p.scratch("lb_vgrow:306:nptr"),
         &ncol = p.scratch("lb_vgrow:306:ncol"), &nsig = p.scratch("lb_vgrow:306:nsig"),
         &nage = p.scratch("lb_vgrow:306:nage"), &clash = p.scratch("lb_vgrow:306:clash");
    tcol.alloc(sizeof(int) * k1);
    tsig.alloc(sizeof(double) * k1);
    tage.alloc(k1);
    k_compact<<<gw, 256, 0, s>>>(n, lv.ptr.as<int64_t>(), lv.col.as<int>(), lv.sig.as<double>(), lv.age.as<uint8_t>(),
                                 drop_age, kptr.as<int64_t>(), tcol.as<int>(), tsig.as<double>(), tage.as<uint8_t>());
    LB_LAUNCH_CHECK();
    nptr.alloc(sizeof(int64_t) * (n + 1));
    ncol.alloc(sizeof(int) * e1);
    nsig.alloc(sizeof(double) * e1);
    nage.alloc(e1);
    clash.alloc(sizeof(int));
    LB_CUDA(cudaMemsetAsync(clash.ptr, 0, sizeof(int), s));
    k_merge<<<gw, 256, 0, s>>>(n, P, kptr.as<int64_t>(), tcol.as<int>(), tsig.as<double>(), tage.as<uint8_t>(),
                               aptr.as<int64_t>(), akeys.as<int64_t>(), nptr.as<int64_t>(), ncol.as<int>(),
                               nsig.as<double>(), nage.as<uint8_t>(), clash.as<int>());
    LB_LAUNCH_CHECK();
    int clash_h = 0;
    LB_CUDA(cudaMemcpyAsync(&clash_h, clash.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    LB_CHECK(!clash_h, LB_ERR_NUMERIC, "VCS working-set update: a selected entry is already in the working set");
    swap_buf(lv.ptr, nptr);
    swap_buf(lv.col, ncol);
    swap_buf(lv.sig, nsig);
    swap_buf(lv.age, nage);
    lv.nnz = nnz;
    p.launches += 4;
    vcs_rebuild_views(p, lv, s);
    p.vsep_dev_count = 0;
    p.have_eval = false;
    if (counts) {
        counts[0] = nnz0 - K;
        counts[1] = A;
        counts[2] = nnz;
    }
}

void vcs_entries_to_caller(const Problem &p, const VcsLevel &lv, const void *src, void *dst_host, int esize,
                           cudaStream_t s) {
    const int64_t nnz = lv.nnz;
    if (!dst_host || nnz == 0) return;
    if (!p.permuted) {
        LB_CUDA(cudaMemcpyAsync(dst_host, src, (size_t)esize * nnz, cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
        return;
    }
    DBuf tmp;
    tmp.alloc((size_t)esize * nnz);
    const unsigned g = grid_for(nnz, 256);
    const int64_t *em = lv.ent_map.as<int64_t>();
    if (esize == 8)
        k_to_caller<uint64_t><<<g, 256, 0, s>>>(nnz, em, (const uint64_t *)src, tmp.as<uint64_t>());
    else if (esize == 4)
        k_to_caller<uint32_t><<<g, 256, 0, s>>>(nnz, em, (const uint32_t *)src, tmp.as<uint32_t>());
    else
        k_to_caller<uint8_t><<<g, 256, 0, s>>>(nnz, em, (const uint8_t *)src, tmp.as<uint8_t>());
    LB_LAUNCH_CHECK();
    LB_CUDA(cudaMemcpyAsync(dst_host, tmp.ptr, (size_t)esize * nnz, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
}

void vcs_structure(const Problem &p, const VcsLevel &lv, int64_t *ptr_host, int32_t *col_host, cudaStream_t s) {
    const int64_t n = p.n;
    if (ptr_host) {
        std::vector<int64_t> iptr((size_t)n + 1);
        LB_CUDA(cudaMemcpyAsync(iptr.data(), lv.ptr.ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
        ptr_host[0] = 0;
        if (!p.permuted) {
            std::copy(iptr.begin(), iptr.end(), ptr_host);
        } else {
            for (int64_t i = 0; i < n; i++) {
                const int64_t k = p.inv_h[i];
                ptr_host[i + 1] = ptr_host[i] + (iptr[k + 1] - iptr[k]);
            }
        }
    }
    if (col_host) vcs_entries_to_caller(p, lv, lv.col.ptr, col_host, 4, s);
}

}  // namespace lb
