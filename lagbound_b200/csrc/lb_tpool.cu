// Triangle pool on the device: the incidence records of a pool, and the solver's pool round (alm_vcs.py:1735-1756):
// purge the triangles with lam = 0, separate (when there is room), merge the candidates, rebuild the incidences.
//
// The pool is p.tri (int32 T x 3, internal row ids) with p.lam; the reference's keys (a n + b) n + c are formed on
// caller ids in wrapping int64 arithmetic, as numpy forms them.  Merge (alm_vcs.py:1745-1753): the one-edge-arm
// family keeps its tri1_add best by value and joins the edge-arm family, whose values are raised by 10; candidates
// already in the pool are dropped, repeated keys keep their first occurrence (np.unique's return_index, in key
// order), and the best min(tri_add + tri1_add, room) by value join with lam 0.  Sorts here are stable, so value ties
// keep key order (numpy's default argsort leaves the order of ties unspecified).
//
// Incidence records (alm_vcs.py:94-104): per vertex, the triangles ascending, record (o1, o2, t | role << 30) with
// role 0 (a): o1 = c, o2 = b; role 1 (b): o1 = a, o2 = c; role 2 (c): o1 = a, o2 = b.  Built as a stable radix sort
// of the 3T (vertex, 3t + role) pairs by vertex.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "lb_internal.cuh"

namespace lb {
namespace {

unsigned grid_of(int64_t m) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((m + 255) / 256, 1 << 20)); }

int bits_for(uint64_t x) {   // bits needed for values in [0, x)
    int b = 1;
    while (b < 64 && (((uint64_t)1 << b) < x)) b++;
    return b;
}

#define GRID_LOOP(i, m) for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (m); i += (int64_t)gridDim.x * blockDim.x)

__device__ __forceinline__ int64_t tri_key(int64_t a, int64_t b, int64_t c, int64_t n) {
    const uint64_t k = ((uint64_t)a * (uint64_t)n + (uint64_t)b) * (uint64_t)n + (uint64_t)c;
    return (int64_t)k;                                    // int64 wrap, as numpy's int64 arithmetic
}

__global__ void k_inc_pairs(int64_t T, const int *__restrict__ tri, int *__restrict__ vkey, unsigned *__restrict__ rec) {
    GRID_LOOP(j, 3 * T) {
        vkey[j] = tri[j];
        rec[j] = (unsigned)j;                             // 3 t + role
    }
}

// tptr[v] = first sorted position of vertex v (v in [0, n])
__global__ void k_tptr(int64_t n, int64_t m, const int *__restrict__ skey, int64_t *__restrict__ tptr) {
    GRID_LOOP(v, n + 1) {
        int64_t lo = 0, hi = m;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (skey[mid] < v) lo = mid + 1;
            else hi = mid;
        }
        tptr[v] = lo;
    }
}

__global__ void k_inc_fill(int64_t m, const unsigned *__restrict__ srec, const int *__restrict__ tri,
                           int *__restrict__ tinc) {
    GRID_LOOP(k, m) {
        const unsigned r = srec[k], t = r / 3u, role = r % 3u;
        const int a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
        tinc[3 * k] = role == 0 ? c : a;
        tinc[3 * k + 1] = role == 1 ? c : b;
        tinc[3 * k + 2] = (int)(t | (role << 30));
    }
}

__global__ void k_pos_flags(int64_t T, const double *__restrict__ lam, uint8_t *__restrict__ flag) {
    GRID_LOOP(t, T) flag[t] = lam[t] > 0.0 ? 1 : 0;
}

__global__ void k_iota(int64_t m, int64_t *__restrict__ x) {
    GRID_LOOP(i, m) x[i] = i;
}

__global__ void k_gather_pool(int64_t m, const int64_t *__restrict__ sel, const int *__restrict__ tri,
                              const double *__restrict__ lam, int *__restrict__ tri_out, double *__restrict__ lam_out) {
    GRID_LOOP(i, m) {
        const int64_t t = sel[i];
        tri_out[3 * i] = tri[3 * t];
        tri_out[3 * i + 1] = tri[3 * t + 1];
        tri_out[3 * i + 2] = tri[3 * t + 2];
        lam_out[i] = lam[t];
    }
}

// keys of the pool triangles on caller ids (order: internal -> caller, null for the identity)
__global__ void k_pool_keys(int64_t T, const int *__restrict__ tri, const int *__restrict__ order, int64_t n,
                            int64_t *__restrict__ key) {
    GRID_LOOP(t, T) {
        int64_t a = tri[3 * t], b = tri[3 * t + 1], c = tri[3 * t + 2];
        if (order) {
            a = order[a];
            b = order[b];
            c = order[c];
        }
        key[t] = tri_key(a, b, c, n);
    }
}

__global__ void k_cand_keys(int64_t m, const int64_t *__restrict__ cand, int64_t n, int64_t *__restrict__ key) {
    GRID_LOOP(i, m) key[i] = tri_key(cand[3 * i], cand[3 * i + 1], cand[3 * i + 2], n);
}

// fresh[i] = key i is not in the sorted pool keys
__global__ void k_fresh(int64_t m, const int64_t *__restrict__ key, const int64_t *__restrict__ pooled, int64_t T,
                        uint8_t *__restrict__ fresh) {
    GRID_LOOP(i, m) {
        const int64_t k = key[i];
        int64_t lo = 0, hi = T;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (pooled[mid] < k) lo = mid + 1;
            else hi = mid;
        }
        fresh[i] = (lo < T && pooled[lo] == k) ? 0 : 1;
    }
}

__global__ void k_gather_i64(int64_t m, const int64_t *__restrict__ sel, const int64_t *__restrict__ src,
                             int64_t *__restrict__ dst) {
    GRID_LOOP(i, m) dst[i] = src[sel[i]];
}

__global__ void k_gather_f64(int64_t m, const int64_t *__restrict__ sel, const double *__restrict__ src,
                             double *__restrict__ dst) {
    GRID_LOOP(i, m) dst[i] = src[sel[i]];
}

// first of each run of equal sorted keys
__global__ void k_run_first(int64_t m, const int64_t *__restrict__ skey, uint8_t *__restrict__ flag) {
    GRID_LOOP(i, m) flag[i] = (i == 0 || skey[i] != skey[i - 1]) ? 1 : 0;
}

// append candidates cand[sel[i]] (caller ids -> internal) with lam 0 after the kept pool
__global__ void k_append(int64_t m, const int64_t *__restrict__ sel, const int64_t *__restrict__ cand,
                         const int *__restrict__ inv, int *__restrict__ tri_out, double *__restrict__ lam_out) {
    GRID_LOOP(i, m) {
        const int64_t c = sel[i];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            const int64_t v = cand[3 * c + r];
            tri_out[3 * i + r] = inv ? inv[v] : (int)v;
        }
        lam_out[i] = 0.0;
    }
}

// DeviceSelect::Flagged over the indices [0, m)
int64_t select_flagged(Problem &p, int64_t m, const uint8_t *flag, int64_t *out, cudaStream_t s) {
    DBuf &iota = p.scratch("lb_tpool:153:iota"), &cnt = p.scratch("lb_tpool:153:cnt"),
         &tmp = p.scratch("lb_tpool:153:tmp");
    iota.alloc(sizeof(int64_t) * std::max<int64_t>(m, 1));
    cnt.alloc(sizeof(int64_t));
    k_iota<<<grid_of(m), 256, 0, s>>>(m, iota.as<int64_t>());
    LB_LAUNCH_CHECK();
    size_t tb = 0;
    LB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, iota.as<int64_t>(), flag, out, cnt.as<int64_t>(), (int)m, s));
    tmp.alloc(tb);
    LB_CUDA(cub::DeviceSelect::Flagged(tmp.ptr, tb, iota.as<int64_t>(), flag, out, cnt.as<int64_t>(), (int)m, s));
    int64_t k = 0;
    LB_CUDA(cudaMemcpyAsync(&k, cnt.ptr, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    return k;
}

void swap_buf(DBuf &a, DBuf &b) {
    std::swap(a.ptr, b.ptr);
    std::swap(a.owner, b.owner);
    std::swap(a.bytes, b.bytes);
}

}  // namespace

void tri_rebuild_incidence(Problem &p, cudaStream_t s) {
    const int64_t T = p.T, n = p.n, m = 3 * T;
    LB_CHECK(m < ((int64_t)1 << 31), LB_ERR_INVALID, "triangle pool too large (3 T must be below 2^31)");
    p.pt.alloc(sizeof(double) * std::max<int64_t>(T, 1));
    p.gt.alloc(sizeof(double) * std::max<int64_t>(T, 1));
    p.tptr.alloc(sizeof(int64_t) * (n + 1));
    p.tinc.alloc(sizeof(int) * 3 * std::max<int64_t>(m, 1));
    if (m) {
        DBuf &vk = p.scratch("lb_tpool:183:vk"), &rc = p.scratch("lb_tpool:183:rc"),
             &vk2 = p.scratch("lb_tpool:183:vk2"), &rc2 = p.scratch("lb_tpool:183:rc2"),
             &tmp = p.scratch("lb_tpool:183:tmp");
        vk.alloc(sizeof(int) * m);
        rc.alloc(sizeof(unsigned) * m);
        vk2.alloc(sizeof(int) * m);
        rc2.alloc(sizeof(unsigned) * m);
        k_inc_pairs<<<grid_of(m), 256, 0, s>>>(T, p.tri.as<int>(), vk.as<int>(), rc.as<unsigned>());
        LB_LAUNCH_CHECK();
        size_t tb = 0;
        const int eb = bits_for((uint64_t)n);
        LB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, vk.as<int>(), vk2.as<int>(), rc.as<unsigned>(),
                                                rc2.as<unsigned>(), (int)m, 0, eb, s));
        tmp.alloc(tb);
        LB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, vk.as<int>(), vk2.as<int>(), rc.as<unsigned>(),
                                                rc2.as<unsigned>(), (int)m, 0, eb, s));
        k_tptr<<<grid_of(n + 1), 256, 0, s>>>(n, m, vk2.as<int>(), p.tptr.as<int64_t>());
        LB_LAUNCH_CHECK();
        k_inc_fill<<<grid_of(m), 256, 0, s>>>(m, rc2.as<unsigned>(), p.tri.as<int>(), p.tinc.as<int>());
        LB_LAUNCH_CHECK();
        p.tptr_h.resize((size_t)n + 1);
        LB_CUDA(cudaMemcpyAsync(p.tptr_h.data(), p.tptr.ptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
        p.launches += 3;
    } else {
        LB_CUDA(cudaMemsetAsync(p.tptr.ptr, 0, sizeof(int64_t) * (n + 1), s));
        p.tptr_h.assign((size_t)n + 1, 0);
    }
    build_heavy(p, s);
    LB_CUDA(cudaStreamSynchronize(s));
    p.have_eval = false;
}

void tri_pool_round(Problem &p, SepParams sp, int64_t tri_add, int64_t tri1_add, int64_t tri_max, int64_t *counts,
                    cudaStream_t s) {
    const int64_t n = p.n, T0 = p.T;
    // --- purge (alm_vcs.py:1738): keep lam > 0, in pool order
    DBuf &flag = p.scratch("lb_tpool:218:flag"), &kept = p.scratch("lb_tpool:218:kept"),
         &tri_k = p.scratch("lb_tpool:218:tri_k"), &lam_k = p.scratch("lb_tpool:218:lam_k");
    flag.alloc(std::max<int64_t>(T0, 1));
    kept.alloc(sizeof(int64_t) * std::max<int64_t>(T0, 1));
    int64_t Tk = 0;
    if (T0) {
        k_pos_flags<<<grid_of(T0), 256, 0, s>>>(T0, p.lam.as<double>(), flag.as<uint8_t>());
        LB_LAUNCH_CHECK();
        Tk = select_flagged(p, T0, flag.as<uint8_t>(), kept.as<int64_t>(), s);
    }
    const int64_t room = std::max<int64_t>(0, tri_max - Tk);
    // --- separation (alm_vcs.py:1740-1745) and the candidate list
    int64_t k = 0;
    std::vector<int64_t> cand_h;
    std::vector<double> val_h;
    if (room) {
        sp.cap0 = (int64_t)((double)std::min(tri_add, room) * 1.3) + 10;
        sp.cap1 = tri1_add ? (int64_t)((double)tri1_add * 1.3) + 10 : 0;
        sp.want0 = true;
        sp.want1 = tri1_add > 0;
        separate_run(p, sp, s);
        const std::vector<int64_t> &t0v = p.sep_tri[0];
        const std::vector<double> &v0 = p.sep_val[0];
        cand_h = t0v;
        val_h = v0;
        if (tri1_add && !p.sep_val[1].empty()) {
            // np.argsort(-v1)[:tri1_add], ties in candidate order; the edge-arm values are raised by 10
            const std::vector<double> &v1 = p.sep_val[1];
            std::vector<int64_t> o1(v1.size());
            for (size_t i = 0; i < o1.size(); i++) o1[i] = (int64_t)i;
            std::stable_sort(o1.begin(), o1.end(), [&](int64_t x, int64_t y) { return v1[x] > v1[y]; });
            o1.resize(std::min<size_t>(o1.size(), (size_t)tri1_add));
            for (double &v : val_h) v += 10.0;
            for (int64_t i : o1) {
                for (int r = 0; r < 3; r++) cand_h.push_back(p.sep_tri[1][3 * i + r]);
                val_h.push_back(v1[i]);
            }
        }
    }
    const int64_t mc = (int64_t)val_h.size();
    DBuf &cand = p.scratch("lb_tpool:257:cand"), &cval = p.scratch("lb_tpool:257:cval"),
         &sel = p.scratch("lb_tpool:257:sel");
    if (mc) {
        upload(cand, cand_h, s);
        upload(cval, val_h, s);
        // pool keys (kept triangles, caller ids), sorted
        DBuf &pk = p.scratch("lb_tpool:262:pk"), &pks = p.scratch("lb_tpool:262:pks"),
             &ck = p.scratch("lb_tpool:262:ck"), &fr = p.scratch("lb_tpool:262:fr"),
             &fsel = p.scratch("lb_tpool:262:fsel"), &fk = p.scratch("lb_tpool:262:fk"),
             &fks = p.scratch("lb_tpool:262:fks"), &fidx = p.scratch("lb_tpool:262:fidx"),
             &fidx2 = p.scratch("lb_tpool:262:fidx2"), &tmp = p.scratch("lb_tpool:262:tmp");
        const int *ord = p.permuted ? p.order_d.as<int>() : nullptr;
        pk.alloc(sizeof(int64_t) * std::max<int64_t>(Tk, 1));
        pks.alloc(sizeof(int64_t) * std::max<int64_t>(Tk, 1));
        if (Tk) {
            tri_k.alloc(sizeof(int) * 3 * Tk);
            lam_k.alloc(sizeof(double) * Tk);
            k_gather_pool<<<grid_of(Tk), 256, 0, s>>>(Tk, kept.as<int64_t>(), p.tri.as<int>(), p.lam.as<double>(),
                                                      tri_k.as<int>(), lam_k.as<double>());
            LB_LAUNCH_CHECK();
            k_pool_keys<<<grid_of(Tk), 256, 0, s>>>(Tk, tri_k.as<int>(), ord, n, pk.as<int64_t>());
            LB_LAUNCH_CHECK();
            size_t tb = 0;
            LB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, pk.as<int64_t>(), pks.as<int64_t>(), (int)Tk, 0, 64, s));
            tmp.alloc(tb);
            LB_CUDA(cub::DeviceRadixSort::SortKeys(tmp.ptr, tb, pk.as<int64_t>(), pks.as<int64_t>(), (int)Tk, 0, 64, s));
        }
        // candidates not in the pool
        ck.alloc(sizeof(int64_t) * mc);
        fr.alloc(mc);
        fsel.alloc(sizeof(int64_t) * mc);
        k_cand_keys<<<grid_of(mc), 256, 0, s>>>(mc, cand.as<int64_t>(), n, ck.as<int64_t>());
        LB_LAUNCH_CHECK();
        k_fresh<<<grid_of(mc), 256, 0, s>>>(mc, ck.as<int64_t>(), pks.as<int64_t>(), Tk, fr.as<uint8_t>());
        LB_LAUNCH_CHECK();
        const int64_t mf = select_flagged(p, mc, fr.as<uint8_t>(), fsel.as<int64_t>(), s);
        if (mf) {
            // first occurrence of each key, in key order (stable sort of (key, candidate index))
            fk.alloc(sizeof(int64_t) * mf);
            fks.alloc(sizeof(int64_t) * mf);
            fidx2.alloc(sizeof(int64_t) * mf);
            k_gather_i64<<<grid_of(mf), 256, 0, s>>>(mf, fsel.as<int64_t>(), ck.as<int64_t>(), fk.as<int64_t>());
            LB_LAUNCH_CHECK();
            size_t tb = 0;
            LB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, fk.as<int64_t>(), fks.as<int64_t>(),
                                                    fsel.as<int64_t>(), fidx2.as<int64_t>(), (int)mf, 0, 64, s));
            tmp.alloc(tb);
            LB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.ptr, tb, fk.as<int64_t>(), fks.as<int64_t>(),
                                                    fsel.as<int64_t>(), fidx2.as<int64_t>(), (int)mf, 0, 64, s));
            DBuf &rf = p.scratch("lb_tpool:301:rf"), &upos = p.scratch("lb_tpool:301:upos");
            rf.alloc(mf);
            upos.alloc(sizeof(int64_t) * mf);
            k_run_first<<<grid_of(mf), 256, 0, s>>>(mf, fks.as<int64_t>(), rf.as<uint8_t>());
            LB_LAUNCH_CHECK();
            const int64_t mu = select_flagged(p, mf, rf.as<uint8_t>(), upos.as<int64_t>(), s);
            // unique candidates (candidate index), key order; then by value descending, stable
            DBuf &uidx = p.scratch("lb_tpool:308:uidx"), &uval = p.scratch("lb_tpool:308:uval"),
                 &uval2 = p.scratch("lb_tpool:308:uval2"), &uidx2 = p.scratch("lb_tpool:308:uidx2");
            uidx.alloc(sizeof(int64_t) * mu);
            uval.alloc(sizeof(double) * mu);
            uval2.alloc(sizeof(double) * mu);
            uidx2.alloc(sizeof(int64_t) * mu);
            k_gather_i64<<<grid_of(mu), 256, 0, s>>>(mu, upos.as<int64_t>(), fidx2.as<int64_t>(), uidx.as<int64_t>());
            LB_LAUNCH_CHECK();
            k_gather_f64<<<grid_of(mu), 256, 0, s>>>(mu, uidx.as<int64_t>(), cval.as<double>(), uval.as<double>());
            LB_LAUNCH_CHECK();
            tb = 0;
            LB_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, uval.as<double>(), uval2.as<double>(),
                                                              uidx.as<int64_t>(), uidx2.as<int64_t>(), (int)mu, 0,
                                                              64, s));
            tmp.alloc(tb);
            LB_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.ptr, tb, uval.as<double>(), uval2.as<double>(),
                                                              uidx.as<int64_t>(), uidx2.as<int64_t>(), (int)mu, 0,
                                                              64, s));
            k = std::min<int64_t>({tri_add + tri1_add, room, mu});
            sel.alloc(sizeof(int64_t) * std::max<int64_t>(k, 1));
            if (k)
                LB_CUDA(cudaMemcpyAsync(sel.ptr, uidx2.ptr, sizeof(int64_t) * k, cudaMemcpyDeviceToDevice, s));
            LB_CUDA(cudaStreamSynchronize(s));
            p.launches += 5;
        }
        p.launches += 4;
    }
    // --- the new pool: kept triangles, then the k new ones with lam 0
    const int64_t T1 = Tk + k;
    LB_CHECK(T1 < ((int64_t)1 << 30), LB_ERR_INVALID, "triangle pool too large (2^30)");
    DBuf &tri_n = p.scratch("lb_tpool:337:tri_n"), &lam_n = p.scratch("lb_tpool:337:lam_n");
    tri_n.alloc(sizeof(int) * 3 * std::max<int64_t>(T1, 1));
    lam_n.alloc(sizeof(double) * std::max<int64_t>(T1, 1));
    if (Tk) {
        if (!mc) {
            k_gather_pool<<<grid_of(Tk), 256, 0, s>>>(Tk, kept.as<int64_t>(), p.tri.as<int>(), p.lam.as<double>(),
                                                      tri_n.as<int>(), lam_n.as<double>());
            LB_LAUNCH_CHECK();
        } else {
            LB_CUDA(cudaMemcpyAsync(tri_n.ptr, tri_k.ptr, sizeof(int) * 3 * Tk, cudaMemcpyDeviceToDevice, s));
            LB_CUDA(cudaMemcpyAsync(lam_n.ptr, lam_k.ptr, sizeof(double) * Tk, cudaMemcpyDeviceToDevice, s));
        }
    }
    if (k) {
        if (p.permuted && p.inv_d.bytes < sizeof(int) * (size_t)n) {
            std::vector<int> inv(n);
            for (int64_t i = 0; i < n; i++) inv[i] = (int)p.inv_h[i];
            upload(p.inv_d, inv, s);
        }
        k_append<<<grid_of(k), 256, 0, s>>>(k, sel.as<int64_t>(), cand.as<int64_t>(),
                                            p.permuted ? p.inv_d.as<int>() : nullptr, tri_n.as<int>() + 3 * Tk,
                                            lam_n.as<double>() + Tk);
        LB_LAUNCH_CHECK();
    }
    swap_buf(p.tri, tri_n);
    swap_buf(p.lam, lam_n);
    p.T = T1;
    tri_rebuild_incidence(p, s);
    if (counts) {
        counts[0] = T0 - Tk;
        counts[1] = k;
        counts[2] = T1;
    }
}

void tri_pool_get(const Problem &p, int64_t *tri, cudaStream_t s) {
    if (!tri || p.T == 0) return;
    std::vector<int> t32((size_t)p.T * 3);
    LB_CUDA(cudaMemcpyAsync(t32.data(), p.tri.ptr, sizeof(int) * 3 * p.T, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    for (size_t j = 0; j < t32.size(); j++) tri[j] = p.permuted ? p.order_h[t32[j]] : t32[j];
}

}  // namespace lb
