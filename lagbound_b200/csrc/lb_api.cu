// C ABI of lagbound_b200 (declared in include/lagbound_b200.h): contexts, problem setup (host-side preprocessing of
// the CSR, cluster member lists, VCS column views and triangle incidence records), evaluation entry points.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cstdio>

#include "lb_internal.cuh"

#include <mutex>

namespace lb {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }

// Pinned host slots for problems' scalar results, from slabs kept for the life of the process: freeing pinned memory
// synchronises the device, which would stall the other problems' streams each time a problem is destroyed.
static std::mutex g_pin_mu;
static std::vector<lb_eval_out *> g_pin_free;
static lb_eval_out *pinned_slot_get() {
    std::lock_guard<std::mutex> lock(g_pin_mu);
    if (g_pin_free.empty()) {
        constexpr int SLAB = 256;
        lb_eval_out *slab = nullptr;
        LB_CUDA(cudaMallocHost(&slab, sizeof(lb_eval_out) * SLAB));
        for (int k = SLAB - 1; k >= 0; k--) g_pin_free.push_back(slab + k);
    }
    lb_eval_out *q = g_pin_free.back();
    g_pin_free.pop_back();
    return q;
}
static void pinned_slot_put(lb_eval_out *q) {
    std::lock_guard<std::mutex> lock(g_pin_mu);
    g_pin_free.push_back(q);
}

cudaStream_t &alloc_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}

Problem::~Problem() {
    for (auto *l : plev) delete l;
    for (auto *l : vlev) delete l;
    if (scal_host) pinned_slot_put(scal_host);
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (lobpcg) lobpcg_state_free(lobpcg);
}

Problem::HostPipe::~HostPipe() {
    if (!ready) return;
    cudaStreamSynchronize(cin);
    cudaStreamSynchronize(cout);
    for (int k = 0; k < 2; k++) {
        cudaEventDestroy(in[k]);
        cudaEventDestroy(conv[k]);
        cudaEventDestroy(comp[k]);
        cudaEventDestroy(out[k]);
        if (scal[k]) cudaFreeHost(scal[k]);
    }
    cudaStreamDestroy(cin);
    cudaStreamDestroy(cout);
}

cudaEvent_t Problem::next_event() {
    if (ev_used == ev_pool.size()) {
        cudaEvent_t e;
        LB_CUDA(cudaEventCreate(&e));
        ev_pool.push_back(e);
    }
    return ev_pool[ev_used++];
}

template <typename F> static int guard(F &&f) {
    struct Clear {
        ~Clear() { alloc_stream() = nullptr; }      // the call's allocation stream ends with the call
    } clear;
    try {
        f();
        return LB_OK;
    } catch (const Err &e) {
        return e.code;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return LB_ERR_NOMEM;
    } catch (...) {
        set_error("unexpected exception");
        return LB_ERR_INVALID;
    }
}

static cudaStream_t stream_of(const Problem &p) { return p.ctx->c.stream; }

static void set_device(const Problem &p) {
    LB_CUDA(cudaSetDevice(p.ctx->c.device));
    alloc_stream() = p.ctx->c.stream;
}

// rows sorted by label (stable counting sort): member list + offsets
static void members_of(const std::vector<int> &lab, int32_t P, std::vector<int> &mem, std::vector<int64_t> &ptr) {
    ptr.assign((size_t)P + 1, 0);
    for (int l : lab) ptr[(size_t)l + 1]++;
    for (int32_t q = 0; q < P; q++) ptr[q + 1] += ptr[q];
    std::vector<int64_t> pos(ptr.begin(), ptr.end() - 1);
    mem.resize(lab.size());
    for (size_t i = 0; i < lab.size(); i++) mem[pos[lab[i]]++] = (int)i;
}

// labels given in the caller's row order -> internal order
static std::vector<int> check_labels(const Problem &p, const int64_t *lab, int32_t P) {
    LB_CHECK(lab != nullptr && P > 0, LB_ERR_INVALID, "labels: null pointer or P <= 0");
    std::vector<int> out((size_t)p.n);
    for (int64_t k = 0; k < p.n; k++) {
        const int64_t i = p.permuted ? p.order_h[k] : k;
        LB_CHECK(lab[i] >= 0 && lab[i] < P, LB_ERR_INVALID,
                 "label out of range at row " + std::to_string(i) + ": " + std::to_string(lab[i]));
        out[k] = (int)lab[i];
    }
    return out;
}

static void fetch_scalars(Problem &p, lb_eval_out *out) {
    cudaStream_t s = stream_of(p);
    LB_CUDA(cudaMemcpyAsync(p.scal_host, p.scal.ptr, sizeof(lb_eval_out), cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    if (out) *out = *p.scal_host;
}

// device per-entry array of a VCS level -> host, in the caller's entry order
template <typename E> static void get_entries(const Problem &p, const VcsLevel &lv, const DBuf &src, E *dst) {
    vcs_entries_to_caller(p, lv, src.ptr, dst, (int)sizeof(E), stream_of(p));
}

}  // namespace lb

using namespace lb;

extern "C" {

const char *lb_version(void) { return "lagbound_b200 0.1 (sm_100a)"; }
const char *lb_last_error(void) { return g_err.c_str(); }

static int ctx_create(int device, cudaStream_t stream, bool own, lb_ctx **out) {
    return guard([&] {
        LB_CHECK(out != nullptr, LB_ERR_INVALID, "out is null");
        int ndev = 0;
        LB_CUDA(cudaGetDeviceCount(&ndev));
        LB_CHECK(device >= 0 && device < ndev, LB_ERR_INVALID, "no such CUDA device");
        LB_CUDA(cudaSetDevice(device));
        cudaDeviceProp prop;
        LB_CUDA(cudaGetDeviceProperties(&prop, device));
        LB_CHECK(prop.major >= 10, LB_ERR_INVALID,
                 std::string("this library is built for sm_100a (B200); device is ") + prop.name);
        auto *c = new lb_ctx();
        c->c.device = device;
        c->c.num_sms = prop.multiProcessorCount;
        if (own)
            LB_CUDA(cudaStreamCreateWithFlags(&c->c.stream, cudaStreamNonBlocking));
        else
            c->c.stream = stream;
        c->c.own_stream = own;
        // the device's default memory pool (stream-ordered buffers) keeps freed memory for reuse instead of
        // returning it at every synchronisation
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
        c->c.persist_max = (size_t)prop.persistingL2CacheMaxSize;
        c->c.window_max = (size_t)prop.accessPolicyMaxWindowSize;
        LB_CUDA(cudaEventCreate(&c->c.t0));
        LB_CUDA(cudaEventCreate(&c->c.t1));
        *out = c;
    });
}

int lb_ctx_create(int device, lb_ctx **out) { return ctx_create(device, nullptr, true, out); }

int lb_ctx_create_on_stream(int device, void *stream, lb_ctx **out) {
    return ctx_create(device, (cudaStream_t)stream, false, out);
}

int lb_ctx_destroy(lb_ctx *ctx) {
    if (!ctx) return LB_OK;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    cudaEventDestroy(ctx->c.t0);
    cudaEventDestroy(ctx->c.t1);
    if (ctx->c.own_stream) cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return LB_OK;
}

int lb_ctx_capture_begin(lb_ctx *ctx) {
    return guard([&] {
        LB_CHECK(ctx, LB_ERR_INVALID, "null context");
        LB_CUDA(cudaSetDevice(ctx->c.device));
        LB_CUDA(cudaStreamBeginCapture(ctx->c.stream, cudaStreamCaptureModeRelaxed));
    });
}

int lb_ctx_capture_end(lb_ctx *ctx, lb_cuda_graph **out) {
    return guard([&] {
        LB_CHECK(ctx && out, LB_ERR_INVALID, "null argument");
        LB_CUDA(cudaSetDevice(ctx->c.device));
        cudaGraph_t g = nullptr;
        LB_CUDA(cudaStreamEndCapture(ctx->c.stream, &g));
        auto *cg = new lb_cuda_graph();
        cg->graph = g;
        cg->device = ctx->c.device;
        cg->stream = ctx->c.stream;
        size_t nn = 0;
        cudaError_t e = cudaGraphGetNodes(g, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
        for (size_t k = 0; e == cudaSuccess && k < nn; k++) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) cg->kernels++;
        }
        e = e == cudaSuccess ? cudaGraphInstantiate(&cg->exec, g, 0) : e;
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            delete cg;
            LB_CUDA(e);
        }
        *out = cg;
    });
}

int lb_cuda_graph_launch(lb_cuda_graph *g) {
    return guard([&] {
        LB_CHECK(g, LB_ERR_INVALID, "null graph");
        LB_CUDA(cudaSetDevice(g->device));
        LB_CUDA(cudaGraphLaunch(g->exec, g->stream));
    });
}

int lb_cuda_graph_kernels(const lb_cuda_graph *g, int64_t *kernels) {
    return guard([&] {
        LB_CHECK(g && kernels, LB_ERR_INVALID, "null argument");
        *kernels = g->kernels;
    });
}

int lb_cuda_graph_destroy(lb_cuda_graph *g) {
    if (!g) return LB_OK;
    cudaSetDevice(g->device);
    cudaStreamSynchronize(g->stream);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return LB_OK;
}

int lb_ctx_set_cache(lb_ctx *ctx, int l2_fetch_bytes, double v_persist_fraction) {
    return guard([&] {
        LB_CHECK(ctx, LB_ERR_INVALID, "null context");
        LB_CHECK(l2_fetch_bytes == 0 || l2_fetch_bytes == 32 || l2_fetch_bytes == 64 || l2_fetch_bytes == 128,
                 LB_ERR_INVALID, "l2_fetch_bytes must be 0, 32, 64 or 128");
        LB_CHECK(v_persist_fraction >= 0.0 && v_persist_fraction <= 1.0, LB_ERR_INVALID,
                 "v_persist_fraction must be in [0, 1]");
        LB_CUDA(cudaSetDevice(ctx->c.device));
        if (l2_fetch_bytes) LB_CUDA(cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, (size_t)l2_fetch_bytes));
        ctx->c.v_persist = v_persist_fraction;
        if (v_persist_fraction > 0 && ctx->c.persist_max)
            LB_CUDA(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, ctx->c.persist_max));
        if (v_persist_fraction == 0) {
            cudaStreamAttrValue v{};
            v.accessPolicyWindow.num_bytes = 0;
            LB_CUDA(cudaStreamSetAttribute(ctx->c.stream, cudaStreamAttributeAccessPolicyWindow, &v));
        }
    });
}

int lb_ctx_synchronize(lb_ctx *ctx) {
    return guard([&] {
        LB_CHECK(ctx, LB_ERR_INVALID, "null context");
        LB_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}

int lb_ctx_timer(lb_ctx *ctx, int stop, float *ms) {
    return guard([&] {
        LB_CHECK(ctx, LB_ERR_INVALID, "null context");
        if (!stop) {
            LB_CUDA(cudaEventRecord(ctx->c.t0, ctx->c.stream));
        } else {
            LB_CUDA(cudaEventRecord(ctx->c.t1, ctx->c.stream));
            LB_CUDA(cudaEventSynchronize(ctx->c.t1));
            float t = 0.f;
            LB_CUDA(cudaEventElapsedTime(&t, ctx->c.t0, ctx->c.t1));
            if (ms) *ms = t;
        }
    });
}

int lb_problem_create_ordered(lb_ctx *ctx, int64_t n, const int64_t *indptr, const int64_t *indices,
                              const double *weights, const double *d, double L, double C0, int32_t r,
                              lb_dtype vdtype, const int64_t *order, lb_problem **out) {
    lb_problem *h = nullptr;
    int rc = guard([&] {
        LB_CHECK(ctx && out && indptr && indices && d, LB_ERR_INVALID, "null argument");
        LB_CHECK(n > 0 && n < (int64_t)1 << 31, LB_ERR_INVALID, "n must be in [1, 2^31)");
        LB_CHECK(vdtype == LB_F64 || vdtype == LB_F32 || vdtype == LB_BF16, LB_ERR_INVALID, "unknown dtype");
        LB_CHECK(r >= 1 && (int64_t)pad_ld(r, vdtype) * (int64_t)dtype_size(vdtype) <= 512, LB_ERR_INVALID,
                 "rank r out of range (row must fit 512 bytes)");
        LB_CHECK(L > 0 && isfinite(L) && isfinite(C0), LB_ERR_INVALID, "L must be positive and finite");
        LB_CHECK(indptr[0] == 0, LB_ERR_INVALID, "indptr[0] != 0");
        const int64_t nnz = indptr[n];
        LB_CHECK(nnz >= 0 && nnz < ((int64_t)1 << 31), LB_ERR_INVALID, "nnz must be < 2^31");
        for (int64_t i = 0; i < n; i++) {
            LB_CHECK(indptr[i + 1] >= indptr[i], LB_ERR_INVALID, "indptr is not monotone");
            LB_CHECK(isfinite(d[i]) && d[i] >= 0, LB_ERR_INVALID, "volumes d must be finite and >= 0");
        }
        LB_CUDA(cudaSetDevice(ctx->c.device));
        h = new lb_problem();
        Problem &p = h->p;
        p.ctx = ctx;
        p.n = n;
        p.nnz = nnz;
        p.r = r;
        p.vdtype = vdtype;
        p.ld = pad_ld(r, vdtype);
        p.L = L;
        p.C0 = C0;
        cudaStream_t s = stream_of(p);
        alloc_stream() = s;
        if (order) {
            p.order_h.assign(order, order + n);
            p.inv_h.assign((size_t)n, -1);
            for (int64_t k = 0; k < n; k++) {
                LB_CHECK(order[k] >= 0 && order[k] < n && p.inv_h[order[k]] < 0, LB_ERR_INVALID,
                         "order is not a permutation of 0..n-1");
                p.inv_h[order[k]] = k;
            }
            p.permuted = true;
            for (int64_t k = 0; k < n && p.permuted; k++) p.permuted = order[k] != k;
        }
        // internal CSR: row k = caller row order[k], columns renumbered and sorted
        std::vector<int> idx32((size_t)nnz);
        std::vector<float> w32(weights ? (size_t)nnz : 0);
        p.indptr_h.assign((size_t)n + 1, 0);
        p.d_h.resize((size_t)n);
        bool weighted = false;
        std::vector<std::pair<int, float>> rowbuf;
        for (int64_t k = 0; k < n; k++) {
            const int64_t i = p.permuted ? p.order_h[k] : k;
            const int64_t a = indptr[i], b = indptr[i + 1], o = p.indptr_h[k];
            p.indptr_h[k + 1] = o + (b - a);
            p.d_h[k] = d[i];
            rowbuf.clear();
            for (int64_t e = a; e < b; e++) {
                LB_CHECK(indices[e] >= 0 && indices[e] < n, LB_ERR_INVALID,
                         "column index out of range at edge " + std::to_string(e));
                float f = 1.0f;
                if (weights) {
                    f = (float)weights[e];
                    LB_CHECK((double)f == weights[e] && isfinite(weights[e]), LB_ERR_INVALID,
                             "edge weights must be finite and exactly representable in FP32 (edge multiplicities)");
                    if (f != 1.0f) weighted = true;
                }
                const int j = (int)(p.permuted ? p.inv_h[indices[e]] : indices[e]);
                rowbuf.emplace_back(j, f);
            }
            if (p.permuted) std::sort(rowbuf.begin(), rowbuf.end());
            for (size_t q = 0; q < rowbuf.size(); q++) {
                idx32[o + q] = rowbuf[q].first;
                if (weights) w32[o + q] = rowbuf[q].second;
            }
        }
        p.weighted = weighted;
        upload(p.indptr, p.indptr_h, s);
        upload(p.indices, idx32, s);
        if (weighted) upload(p.weights, w32, s);
        upload(p.d, p.d_h, s);
        if (p.permuted) {
            std::vector<int> o32(p.order_h.begin(), p.order_h.end());
            upload(p.order_d, o32, s);
        }
        build_heavy(p, s);
        p.V.alloc(dtype_size(vdtype) * (size_t)n * p.ld);
        LB_CUDA(cudaMemsetAsync(p.V.ptr, 0, p.V.bytes, s));
        p.G.alloc((vdtype == LB_F64 ? 8 : 4) * (size_t)n * p.ld);
        p.z.alloc(sizeof(double) * p.ld);
        p.scal.alloc(sizeof(lb_eval_out));
        p.scal_host = pinned_slot_get();
        p.zplan.build({0, n}, s);
        LB_CUDA(cudaStreamSynchronize(s));
        *out = h;
    });
    if (rc != LB_OK && h) delete h;
    return rc;
}

int lb_problem_create(lb_ctx *ctx, int64_t n, const int64_t *indptr, const int64_t *indices, const double *weights,
                      const double *d, double L, double C0, int32_t r, lb_dtype vdtype, lb_problem **out) {
    return lb_problem_create_ordered(ctx, n, indptr, indices, weights, d, L, C0, r, vdtype, nullptr, out);
}

int lb_problem_create_batched(lb_ctx *ctx, int32_t ngraphs, const int64_t *row_ptr, int64_t n,
                              const int64_t *indptr, const int64_t *indices, const double *weights, const double *d,
                              const double *L, const double *C0, int32_t r, lb_dtype vdtype, const int64_t *order,
                              lb_problem **out) {
    lb_problem *h = nullptr;
    int rc = guard([&] {
        LB_CHECK(ctx && out && row_ptr && indptr && indices && L && C0, LB_ERR_INVALID, "null argument");
        LB_CHECK(ngraphs >= 1 && row_ptr[0] == 0 && row_ptr[ngraphs] == n, LB_ERR_INVALID,
                 "row_ptr must run from 0 to n over ngraphs >= 1 graphs");
        double Lsum = 0.0, C0sum = 0.0;
        for (int32_t g = 0; g < ngraphs; g++) {
            LB_CHECK(row_ptr[g + 1] > row_ptr[g], LB_ERR_INVALID, "every graph needs at least one row");
            LB_CHECK(L[g] > 0 && isfinite(L[g]) && isfinite(C0[g]), LB_ERR_INVALID, "L must be positive and finite");
            Lsum += L[g];
            C0sum += C0[g];
            for (int64_t i = row_ptr[g]; i < row_ptr[g + 1]; i++) {
                if (order) LB_CHECK(order[i] >= row_ptr[g] && order[i] < row_ptr[g + 1], LB_ERR_INVALID,
                                    "batched problem: order must keep every graph's rows in the graph's range");
                for (int64_t e = indptr[i]; e < indptr[i + 1]; e++)
                    LB_CHECK(indices[e] >= row_ptr[g] && indices[e] < row_ptr[g + 1], LB_ERR_INVALID,
                             "batched problem: an edge joins two graphs (the CSR must be block diagonal)");
            }
        }
        int rc2 = lb_problem_create_ordered(ctx, n, indptr, indices, weights, d, Lsum, C0sum, r, vdtype, order, &h);
        if (rc2 != LB_OK) throw Err{rc2};
        Problem &p = h->p;
        cudaStream_t s = stream_of(p);
        p.ngraphs = ngraphs;
        p.gptr_h.assign(row_ptr, row_ptr + ngraphs + 1);
        p.gtptr_h.assign((size_t)ngraphs + 1, 0);
        std::vector<int> gid((size_t)n);
        std::vector<double> gL(L, L + ngraphs), ginvL(ngraphs), gC0(C0, C0 + ngraphs);
        for (int32_t g = 0; g < ngraphs; g++) {
            ginvL[g] = 1.0 / L[g];
            for (int64_t i = row_ptr[g]; i < row_ptr[g + 1]; i++) gid[i] = g;
        }
        upload(p.gid, gid, s);
        upload(p.gL, gL, s);
        upload(p.ginvL, ginvL, s);
        upload(p.gC0, gC0, s);
        upload(p.gptr, p.gptr_h, s);
        upload(p.gtptr, p.gtptr_h, s);
        p.gout.alloc(sizeof(double) * 5 * (size_t)ngraphs);
        p.gsum.alloc(sizeof(double) * 2);
        p.z.alloc(sizeof(double) * (size_t)ngraphs * p.ld);
        p.zplan.build(p.gptr_h, s);
        LB_CUDA(cudaStreamSynchronize(s));
        *out = h;
    });
    if (rc != LB_OK && h) {
        lb_problem_destroy(h);
        h = nullptr;
    }
    return rc;
}

int lb_eval_graphs(lb_problem *h, double *out) {
    return guard([&] {
        LB_CHECK(h && out, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(p.ngraphs > 0, LB_ERR_INVALID, "not a batched problem");
        set_device(p);
        cudaStream_t s = stream_of(p);
        LB_CUDA(cudaMemcpyAsync(out, p.gout.ptr, sizeof(double) * 5 * p.ngraphs, cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
    });
}

int lb_problem_destroy(lb_problem *h) {
    if (!h) return LB_OK;
    cudaSetDevice(h->p.ctx->c.device);
    cudaStreamSynchronize(h->p.ctx->c.stream);
    delete h;
    return LB_OK;
}

int lb_problem_info(const lb_problem *h, int32_t *ld, int64_t *heavy_rows, int64_t *device_bytes) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        const Problem &p = h->p;
        if (ld) *ld = p.ld;
        if (heavy_rows) *heavy_rows = p.n_heavy;
        if (device_bytes) {
            size_t b = p.indptr.bytes + p.indices.bytes + p.weights.bytes + p.d.bytes + p.V.bytes + p.G.bytes +
                       p.heavy_items.bytes + p.heavy_part.bytes + p.tri.bytes + p.lam.bytes + p.pt.bytes +
                       p.gt.bytes + p.tptr.bytes + p.tinc.bytes + p.partials.bytes;
            for (auto *l : p.plev) b += l->sig.bytes + l->pp.bytes + l->Y.bytes + l->M.bytes + l->lab.bytes;
            for (auto *l : p.vlev)
                b += l->ptr.bytes + l->col.bytes + l->sig.bytes + l->ppv.bytes + l->stn.bytes + l->stZ.bytes +
                     l->age.bytes + l->slack.bytes + l->crow.bytes + l->cent.bytes + l->Y.bytes + l->Z.bytes +
                     l->items.bytes + l->SY.bytes + l->SYpart.bytes;
            b += p.row_quad.bytes + p.sched.bytes + p.nlight.bytes + p.scratch_bytes();
            b += p.sw_Vnew.bytes + p.sw_Vold.bytes + p.sw_DD.bytes + p.sw_GX.bytes + p.sw_KX.bytes + p.sw_mpart.bytes;
            *device_bytes = (int64_t)b;
        }
    });
}

int lb_set_V(lb_problem *h, const double *V) {
    return guard([&] {
        LB_CHECK(h && V, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        set_device(p);
        cudaStream_t s = stream_of(p);
        DBuf tmp;
        upload(tmp, V, (size_t)p.n * p.r, s);
        convert_V_from_f64(p, tmp.as<double>(), s);
        LB_CUDA(cudaStreamSynchronize(s));
    });
}

int lb_set_V_raw(lb_problem *h, const void *V, lb_dtype dtype) {
    return guard([&] {
        LB_CHECK(h && V, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(dtype == p.vdtype, LB_ERR_INVALID, "raw V must be in the problem's storage dtype");
        set_device(p);
        cudaStream_t s = stream_of(p);
        const size_t bytes = dtype_size(p.vdtype) * (size_t)p.n * p.r;
        if (p.r == p.ld && !p.permuted) {
            LB_CUDA(cudaMemcpyAsync(p.V.ptr, V, bytes, cudaMemcpyHostToDevice, s));
        } else {
            p.staging.alloc(bytes);
            LB_CUDA(cudaMemcpyAsync(p.staging.ptr, V, bytes, cudaMemcpyHostToDevice, s));
            convert_V_raw(p, p.staging.ptr, s);
        }
    });
}

int lb_get_V(lb_problem *h, double *V) {
    return guard([&] {
        LB_CHECK(h && V, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        set_device(p);
        cudaStream_t s = stream_of(p);
        DBuf tmp;
        tmp.alloc(sizeof(double) * (size_t)p.n * p.r);
        convert_V_to_f64(p, tmp.as<double>(), s);
        LB_CUDA(cudaMemcpyAsync(V, tmp.ptr, tmp.bytes, cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
    });
}

int lb_pair_level_add(lb_problem *h, int32_t P, const int64_t *lab, double w, int32_t *level) {
    return guard([&] {
        LB_CHECK(h && h->p.ngraphs == 0, LB_ERR_INVALID, "levels are not supported on batched problems");
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK((int)p.plev.size() < MAX_LEVELS, LB_ERR_INVALID, "too many pair levels (max 4)");
        LB_CHECK(P <= 24576, LB_ERR_INVALID, "pair levels hold at most 24576 clusters (the reference caps them with "
                                             "--max_clusters, 6000 in production)");
        set_device(p);
        cudaStream_t s = stream_of(p);
        std::vector<int> lb32 = check_labels(p, lab, P);
        const std::vector<double> &dh = p.d_h;
        // rq = |Q| / max(vol_Q, 1)^2, dsq = sum d^2 (alm_vcs.py:1181-1184, aggops.py:61)
        std::vector<double> cnt(P, 0.0), vol(P, 0.0), dsq(P, 0.0), rq(P);
        for (int64_t i = 0; i < p.n; i++) {
            cnt[lb32[i]] += 1.0;
            vol[lb32[i]] += dh[i];
            dsq[lb32[i]] += dh[i] * dh[i];
        }
        for (int32_t q = 0; q < P; q++) {
            const double v = std::max(vol[q], 1.0);
            rq[q] = cnt[q] / (v * v);
        }
        auto *lv = new PairLevel();
        lv->P = P;
        lv->w = w;
        upload(lv->lab, lb32, s);
        upload(lv->rq, rq, s);
        upload(lv->dsq, dsq, s);
        lv->sig.alloc(sizeof(double) * (size_t)P * P);
        LB_CUDA(cudaMemsetAsync(lv->sig.ptr, 0, lv->sig.bytes, s));
        lv->pp.alloc(sizeof(double) * (size_t)P * P);
        lv->Y.alloc(sizeof(double) * (size_t)P * p.ld);
        lv->M.alloc(sizeof(double) * (size_t)P * p.ld);
        lv->pdiag.alloc(sizeof(double) * P);
        lv->kq.alloc(sizeof(double) * P);
        std::vector<int> mem;
        members_of(lb32, P, mem, lv->member_ptr_h);
        upload(lv->members, mem, s);
        upload(lv->member_ptr, lv->member_ptr_h, s);
        lv->plan.build(lv->member_ptr_h, s);
        LB_CUDA(cudaStreamSynchronize(s));
        p.plev.push_back(lv);
        if (level) *level = (int32_t)p.plev.size() - 1;
    });
}

int lb_pair_level_set_sigma(lb_problem *h, int32_t level, const double *sig) {
    return guard([&] {
        LB_CHECK(h && sig, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.plev.size(), LB_ERR_INVALID, "no such pair level");
        auto *lv = p.plev[level];
        const size_t cnt = (size_t)lv->P * lv->P;
        for (size_t k = 0; k < cnt; k++)
            LB_CHECK(sig[k] >= 0 && isfinite(sig[k]), LB_ERR_INVALID, "pair multipliers must be finite and >= 0");
        set_device(p);
        upload(lv->sig, sig, cnt, stream_of(p));
        LB_CUDA(cudaStreamSynchronize(stream_of(p)));
        p.have_eval = false;
    });
}

int lb_pair_level_get_sigma(lb_problem *h, int32_t level, double *sig) {
    return guard([&] {
        LB_CHECK(h && sig, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.plev.size(), LB_ERR_INVALID, "no such pair level");
        auto *lv = p.plev[level];
        set_device(p);
        LB_CUDA(cudaMemcpyAsync(sig, lv->sig.ptr, sizeof(double) * (size_t)lv->P * lv->P, cudaMemcpyDeviceToHost,
                                stream_of(p)));
        LB_CUDA(cudaStreamSynchronize(stream_of(p)));
    });
}

int lb_set_pair_weight(lb_problem *h, double w, double vc_weight) {
    return guard([&] {
        LB_CHECK(h && isfinite(w) && w > 0, LB_ERR_INVALID, "pair weight must be positive");
        for (auto *lv : h->p.plev) lv->w = w;
        for (auto *lv : h->p.vlev) lv->wv = vc_weight * w;
    });
}

int lb_vcs_level_add(lb_problem *h, int32_t P, const int64_t *lab, double wv, int32_t *level) {
    return guard([&] {
        LB_CHECK(h && h->p.ngraphs == 0, LB_ERR_INVALID, "levels are not supported on batched problems");
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK((int)p.vlev.size() < MAX_LEVELS, LB_ERR_INVALID, "too many VCS levels (max 4)");
        set_device(p);
        cudaStream_t s = stream_of(p);
        std::vector<int> lb32 = check_labels(p, lab, P);
        const std::vector<double> &dh = p.d_h;
        // vcsops.py:33-44: vol = max(bincount(lab, d), 1), rq = |R| / vol^2
        std::vector<double> cnt(P, 0.0), vol(P, 0.0), rq(P);
        for (int64_t i = 0; i < p.n; i++) {
            cnt[lb32[i]] += 1.0;
            vol[lb32[i]] += dh[i];
        }
        for (int32_t q = 0; q < P; q++) {
            vol[q] = std::max(vol[q], 1.0);
            rq[q] = cnt[q] / (vol[q] * vol[q]);
        }
        auto *lv = new VcsLevel();
        lv->P = P;
        lv->wv = wv;
        upload(lv->lab, lb32, s);
        upload(lv->rq, rq, s);
        upload(lv->vol, vol, s);
        std::vector<int64_t> zp((size_t)p.n + 1, 0);
        upload(lv->ptr, zp, s);
        std::vector<int64_t> own((size_t)p.n, -1);
        upload(lv->own, own, s);
        lv->Y.alloc(sizeof(double) * (size_t)P * p.ld);
        lv->Z.alloc(sizeof(double) * (size_t)P * p.ld);
        lv->cnt.alloc(sizeof(double) * P);
        std::vector<int> mem;
        members_of(lb32, P, mem, lv->member_ptr_h);
        upload(lv->members, mem, s);
        lv->yplan.build(lv->member_ptr_h, s);
        std::vector<int64_t> cptr((size_t)P + 1, 0);
        upload(lv->cptr, cptr, s);
        lv->zplan.build(cptr, s);
        LB_CUDA(cudaStreamSynchronize(s));
        p.vlev.push_back(lv);
        if (level) *level = (int32_t)p.vlev.size() - 1;
    });
}

int lb_vcs_set_ws(lb_problem *h, int32_t level, int64_t nnz, const int64_t *ptr, const int32_t *col, const double *sig,
                  const uint8_t *age) {
    return guard([&] {
        LB_CHECK(h && ptr, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        auto *lv = p.vlev[level];
        LB_CHECK(ptr[0] == 0 && ptr[p.n] == nnz && nnz >= 0, LB_ERR_INVALID, "working-set ptr inconsistent with nnz");
        LB_CHECK(nnz == 0 || (col && sig), LB_ERR_INVALID, "null col/sig");
        set_device(p);
        cudaStream_t s = stream_of(p);
        // internal working set: internal row k = caller row order[k]; entries keep their order within a row
        std::vector<int64_t> iptr((size_t)p.n + 1, 0);
        std::vector<int> icol((size_t)nnz);
        std::vector<double> isig((size_t)nnz);
        std::vector<uint8_t> iage((size_t)nnz, 0);
        for (int64_t k = 0; k < p.n; k++) {
            const int64_t i = p.permuted ? p.order_h[k] : k;
            LB_CHECK(ptr[i + 1] >= ptr[i], LB_ERR_INVALID, "working-set ptr not monotone");
            int64_t o = iptr[k];
            for (int64_t e = ptr[i]; e < ptr[i + 1]; e++, o++) {
                LB_CHECK(col[e] >= 0 && col[e] < lv->P, LB_ERR_INVALID, "working-set column out of range");
                LB_CHECK(e == ptr[i] || col[e] > col[e - 1], LB_ERR_INVALID, "working-set columns not sorted/unique");
                LB_CHECK(sig[e] >= 0 && isfinite(sig[e]), LB_ERR_INVALID, "VCS multipliers must be finite and >= 0");
                icol[o] = col[e];
                isig[o] = sig[e];
                if (age) iage[o] = age[e];
            }
            iptr[k + 1] = o;
        }
        lv->nnz = nnz;
        upload(lv->ptr, iptr, s);
        upload(lv->col, icol, s);
        upload(lv->sig, isig, s);
        lv->age.alloc(std::max<int64_t>(nnz, 1));
        if (nnz) LB_CUDA(cudaMemcpyAsync(lv->age.ptr, iage.data(), (size_t)nnz, cudaMemcpyHostToDevice, s));
        // entry of (i, lab_i), column view (entries sorted by column, rows ascending: the order of
        // vcsops.py:216-235 vcs_zinit_rows) and the caller's entry order, built on the device
        vcs_rebuild_views(p, *lv, s);
        p.have_eval = false;
    });
}

int lb_vcs_get_ws(lb_problem *h, int32_t level, double *sig, uint8_t *age) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        auto *lv = p.vlev[level];
        set_device(p);
        get_entries(p, *lv, lv->sig, sig);
        get_entries(p, *lv, lv->age, age);
    });
}

int lb_tri_set(lb_problem *h, int64_t T, const int64_t *tri, const double *lam) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(T >= 0 && 3 * T < ((int64_t)1 << 31), LB_ERR_INVALID, "T must be in [0, 2^31 / 3)");
        LB_CHECK(T == 0 || (tri && lam), LB_ERR_INVALID, "null triangle arrays");
        set_device(p);
        cudaStream_t s = stream_of(p);
        std::vector<int> t32((size_t)T * 3);
        for (int64_t t = 0; t < T; t++) {
            for (int r = 0; r < 3; r++) {
                int64_t v = tri[3 * t + r];
                LB_CHECK(v >= 0 && v < p.n, LB_ERR_INVALID, "triangle vertex out of range");
                if (p.permuted) v = p.inv_h[v];
                t32[3 * t + r] = (int)v;
            }
            LB_CHECK(lam[t] >= 0 && isfinite(lam[t]), LB_ERR_INVALID, "triangle multipliers must be finite and >= 0");
        }
        if (p.ngraphs) {
            // batched: every triangle inside one graph, triangles grouped by graph in graph order
            p.gtptr_h.assign((size_t)p.ngraphs + 1, 0);
            int64_t gprev = 0;
            for (int64_t t = 0; t < T; t++) {
                int64_t gt = -1;
                for (int r = 0; r < 3; r++) {
                    const int64_t v = t32[3 * t + r];
                    const int64_t g = std::upper_bound(p.gptr_h.begin(), p.gptr_h.end(), v) - p.gptr_h.begin() - 1;
                    LB_CHECK(gt < 0 || g == gt, LB_ERR_INVALID, "batched problem: a triangle spans two graphs");
                    gt = g;
                }
                LB_CHECK(gt >= gprev, LB_ERR_INVALID, "batched problem: triangles must be grouped by graph in order");
                gprev = gt;
                p.gtptr_h[(size_t)gt + 1]++;
            }
            for (int32_t g = 0; g < p.ngraphs; g++) p.gtptr_h[g + 1] += p.gtptr_h[g];
            upload(p.gtptr, p.gtptr_h, s);
        }
        p.T = T;
        upload(p.tri, t32, s);
        upload(p.lam, lam, (size_t)T, s);
        // incidence records in the reference's incidence order (alm_vcs.py:94-104), built on the device:
        // role 0 (a): +h (v_c - v_b); role 1 (b): -h (v_a + v_c); role 2 (c): +h (v_a - v_b)  (tri_apply 106-120)
        tri_rebuild_incidence(p, s);
    });
}

int lb_tri_pool_round(lb_problem *h, double thresh, int32_t maxh, int32_t maxk, int32_t hub2, int32_t cap2,
                      double vtol, int32_t nchunk, int32_t nbins, int64_t tri_add, int64_t tri1_add, int64_t tri_max,
                      int64_t *counts) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        LB_CHECK(maxh >= 1 && maxk >= 1 && hub2 >= 0 && cap2 >= 0 && nchunk >= 1 && nbins >= 1 && isfinite(thresh) &&
                     isfinite(vtol) && vtol < 2.0 && tri_add >= 0 && tri1_add >= 0 && tri_max >= 0,
                 LB_ERR_INVALID, "invalid triangle pool parameters");
        LB_CHECK(tri_max < ((int64_t)1 << 29), LB_ERR_INVALID, "tri_max must be below 2^29");
        Problem &p = h->p;
        set_device(p);
        LB_CHECK(p.ngraphs == 0, LB_ERR_INVALID, "the pool round is not supported on batched problems");
        SepParams sp{thresh, vtol, maxh, maxk, hub2, cap2, nchunk, nbins, 0, 0, true, false};
        tri_pool_round(p, sp, tri_add, tri1_add, tri_max, counts, stream_of(p));
    });
}

int lb_tri_get(lb_problem *h, int64_t *tri) {
    return guard([&] {
        LB_CHECK(h && (tri || h->p.T == 0), LB_ERR_INVALID, "null argument");
        set_device(h->p);
        tri_pool_get(h->p, tri, stream_of(h->p));
    });
}

int lb_tri_count(const lb_problem *h, int64_t *T) {
    return guard([&] {
        LB_CHECK(h && T, LB_ERR_INVALID, "null argument");
        *T = h->p.T;
    });
}

int lb_tri_get_lam(lb_problem *h, double *lam) {
    return guard([&] {
        LB_CHECK(h && (lam || h->p.T == 0), LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        set_device(p);
        if (p.T) {
            LB_CUDA(cudaMemcpyAsync(lam, p.lam.ptr, sizeof(double) * p.T, cudaMemcpyDeviceToHost, stream_of(p)));
            LB_CUDA(cudaStreamSynchronize(stream_of(p)));
        }
    });
}

static void check_eval_args(const Problem &p, double rho, double tri_weight, int flags) {
    const bool fixed = flags & LB_EVAL_FIXED;
    LB_CHECK((flags & ~(LB_EVAL_GRAD | LB_EVAL_FIXED | LB_EVAL_TIMING)) == 0, LB_ERR_INVALID, "unknown eval flags");
    if (!fixed) {
        LB_CHECK(isfinite(rho) && rho > 0, LB_ERR_INVALID, "rho must be positive (the PHR terms divide by rho r)");
        LB_CHECK(p.T == 0 || (isfinite(tri_weight) && tri_weight > 0), LB_ERR_INVALID,
                 "tri_weight must be positive");
    }
}

int lb_eval_async(lb_problem *h, double rho, double tri_weight, int flags) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        check_eval_args(p, rho, tri_weight, flags);
        set_device(p);
        eval_run(p, rho, tri_weight, flags, stream_of(p));
    });
}

int lb_eval_fetch(lb_problem *h, lb_eval_out *out) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(p.have_eval, LB_ERR_STATE, "no evaluation to fetch");
        set_device(p);
        fetch_scalars(p, out);
    });
}

int lb_eval(lb_problem *h, double rho, double tri_weight, int flags, lb_eval_out *out) {
    int rc = lb_eval_async(h, rho, tri_weight, flags);
    if (rc != LB_OK) return rc;
    return lb_eval_fetch(h, out);
}

int lb_eval_host(lb_problem *h, const void *V_host, double rho, double tri_weight, int flags, lb_eval_out *out) {
    int rc = lb_set_V_raw(h, V_host, h ? h->p.vdtype : LB_F64);
    if (rc != LB_OK) return rc;
    return lb_eval(h, rho, tri_weight, flags, out);
}

static int set_V_device(lb_problem *h, const double *X, bool wait) {
    return guard([&] {
        LB_CHECK(h && X, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        set_device(p);
        cudaPointerAttributes at{};
        LB_CUDA(cudaPointerGetAttributes(&at, X));
        LB_CHECK(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged, LB_ERR_INVALID,
                 "X must be device memory");
        cudaStream_t s = stream_of(p);
        convert_V_from_f64(p, X, s);
        if (wait) LB_CUDA(cudaStreamSynchronize(s));
    });
}
int lb_set_V_device(lb_problem *h, const double *X) { return set_V_device(h, X, true); }
int lb_set_V_device_async(lb_problem *h, const double *X) { return set_V_device(h, X, false); }

static int get_G_device(lb_problem *h, double *G, bool wait) {
    return guard([&] {
        LB_CHECK(h && G, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(p.have_eval && (p.last_flags & LB_EVAL_GRAD), LB_ERR_STATE, "no gradient evaluated");
        set_device(p);
        cudaPointerAttributes at{};
        LB_CUDA(cudaPointerGetAttributes(&at, G));
        LB_CHECK(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged, LB_ERR_INVALID,
                 "G must be device memory");
        cudaStream_t s = stream_of(p);
        G_to_f64(p, G, s);
        if (wait) LB_CUDA(cudaStreamSynchronize(s));
    });
}
int lb_get_G_device(lb_problem *h, double *G) { return get_G_device(h, G, true); }
int lb_get_G_device_async(lb_problem *h, double *G) { return get_G_device(h, G, false); }

int lb_get_G(lb_problem *h, double *G) {
    return guard([&] {
        LB_CHECK(h && G, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(p.have_eval && (p.last_flags & LB_EVAL_GRAD), LB_ERR_STATE, "no gradient evaluated");
        set_device(p);
        cudaStream_t s = stream_of(p);
        DBuf tmp;
        tmp.alloc(sizeof(double) * (size_t)p.n * p.r);
        G_to_f64(p, tmp.as<double>(), s);
        LB_CUDA(cudaMemcpyAsync(G, tmp.ptr, tmp.bytes, cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
    });
}

int lb_get_G_raw(lb_problem *h, void *G) {
    return guard([&] {
        LB_CHECK(h && G, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(p.have_eval && (p.last_flags & LB_EVAL_GRAD), LB_ERR_STATE, "no gradient evaluated");
        set_device(p);
        cudaStream_t s = stream_of(p);
        const size_t bytes = (p.vdtype == LB_F64 ? 8 : 4) * (size_t)p.n * p.r;
        if (p.r == p.ld && !p.permuted) {
            LB_CUDA(cudaMemcpyAsync(G, p.G.ptr, bytes, cudaMemcpyDeviceToHost, s));
        } else {
            p.staging.alloc(bytes);
            G_raw(p, p.staging.ptr, s);
            LB_CUDA(cudaMemcpyAsync(G, p.staging.ptr, bytes, cudaMemcpyDeviceToHost, s));
        }
        LB_CUDA(cudaStreamSynchronize(s));
    });
}

int lb_eval_host_pipelined(lb_problem *h, int32_t nsteps, const void *const *V_hosts, void *const *G_hosts,
                            double rho, double tri_weight, int flags, lb_eval_out *outs) {
    return guard([&] {
        LB_CHECK(h && V_hosts && nsteps >= 0, LB_ERR_INVALID, "null argument or nsteps < 0");
        Problem &p = h->p;
        check_eval_args(p, rho, tri_weight, flags);
        LB_CHECK(!(flags & LB_EVAL_TIMING), LB_ERR_INVALID, "phase timing is not available in pipelined evaluations");
        LB_CHECK(!G_hosts || (flags & LB_EVAL_GRAD), LB_ERR_INVALID, "G_hosts needs LB_EVAL_GRAD");
        for (int32_t k = 0; k < nsteps; k++) LB_CHECK(V_hosts[k], LB_ERR_INVALID, "null V_hosts entry");
        if (nsteps == 0) return;
        set_device(p);
        cudaStream_t s = stream_of(p);
        auto &q = p.pipe;
        if (!q.ready) {
            LB_CUDA(cudaStreamCreateWithFlags(&q.cin, cudaStreamNonBlocking));
            LB_CUDA(cudaStreamCreateWithFlags(&q.cout, cudaStreamNonBlocking));
            for (int k = 0; k < 2; k++) {
                LB_CUDA(cudaEventCreateWithFlags(&q.in[k], cudaEventDisableTiming));
                LB_CUDA(cudaEventCreateWithFlags(&q.conv[k], cudaEventDisableTiming));
                LB_CUDA(cudaEventCreateWithFlags(&q.comp[k], cudaEventDisableTiming));
                LB_CUDA(cudaEventCreateWithFlags(&q.out[k], cudaEventDisableTiming));
                LB_CUDA(cudaMallocHost(&q.scal[k], sizeof(lb_eval_out)));
            }
            q.ready = true;
        }
        const size_t vbytes = dtype_size(p.vdtype) * (size_t)p.n * p.r;
        const size_t gbytes = (p.vdtype == LB_F64 ? 8 : 4) * (size_t)p.n * p.r;
        // every slot starts free: its events recorded on streams with no pending work of this call
        for (int k = 0; k < 2; k++) {
            q.vst[k].alloc(vbytes);
            if (G_hosts) q.gst[k].alloc(gbytes);
            LB_CUDA(cudaEventRecord(q.conv[k], s));
            LB_CUDA(cudaEventRecord(q.comp[k], s));
            LB_CUDA(cudaEventRecord(q.out[k], q.cout));
        }
        auto take_scalars = [&](int32_t k) {
            LB_CUDA(cudaEventSynchronize(q.comp[k & 1]));
            if (outs) outs[k] = *q.scal[k & 1];
        };
        // on an error part-way, the copies already queued still read and write the caller's buffers: let them finish
        // before the call returns
        struct Drain {
            cudaStream_t a, b, c;
            bool armed = true;
            ~Drain() {
                if (!armed) return;
                cudaStreamSynchronize(a);
                cudaStreamSynchronize(b);
                cudaStreamSynchronize(c);
            }
        } drain{q.cin, q.cout, s};
        for (int32_t k = 0; k < nsteps; k++) {
            const int sl = k & 1;
            if (k >= 2) take_scalars(k - 2);     // step k - 2 used this slot's pinned scalars
            // copy-in: once step k - 2 has converted this slot's staged V
            LB_CUDA(cudaStreamWaitEvent(q.cin, q.conv[sl], 0));
            LB_CUDA(cudaMemcpyAsync(q.vst[sl].ptr, V_hosts[k], vbytes, cudaMemcpyHostToDevice, q.cin));
            LB_CUDA(cudaEventRecord(q.in[sl], q.cin));
            // compute: V from the staged copy, the evaluation, the raw G into this slot (once step k - 2's copy-out
            // has read it), the scalars to pinned memory
            LB_CUDA(cudaStreamWaitEvent(s, q.in[sl], 0));
            convert_V_raw(p, q.vst[sl].ptr, s);
            LB_CUDA(cudaEventRecord(q.conv[sl], s));
            eval_run(p, rho, tri_weight, flags, s);
            if (G_hosts && G_hosts[k]) {
                LB_CUDA(cudaStreamWaitEvent(s, q.out[sl], 0));
                G_raw(p, q.gst[sl].ptr, s);
            }
            LB_CUDA(cudaMemcpyAsync(q.scal[sl], p.scal.ptr, sizeof(lb_eval_out), cudaMemcpyDeviceToHost, s));
            LB_CUDA(cudaEventRecord(q.comp[sl], s));
            // copy-out
            if (G_hosts && G_hosts[k]) {
                LB_CUDA(cudaStreamWaitEvent(q.cout, q.comp[sl], 0));
                LB_CUDA(cudaMemcpyAsync(G_hosts[k], q.gst[sl].ptr, gbytes, cudaMemcpyDeviceToHost, q.cout));
                LB_CUDA(cudaEventRecord(q.out[sl], q.cout));
            }
        }
        for (int32_t k = std::max(0, nsteps - 2); k < nsteps; k++) take_scalars(k);
        drain.armed = false;
        LB_CUDA(cudaStreamSynchronize(q.cout));
        LB_CUDA(cudaStreamSynchronize(q.cin));
        LB_CUDA(cudaStreamSynchronize(s));
    });
}

int lb_get_pair_pp(lb_problem *h, int32_t level, double *pp) {
    return guard([&] {
        LB_CHECK(h && pp, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(p.have_eval, LB_ERR_STATE, "no evaluation");
        LB_CHECK(level >= 0 && level < (int)p.plev.size(), LB_ERR_INVALID, "no such pair level");
        auto *lv = p.plev[level];
        set_device(p);
        LB_CUDA(cudaMemcpyAsync(pp, lv->pp.ptr, sizeof(double) * (size_t)lv->P * lv->P, cudaMemcpyDeviceToHost,
                                stream_of(p)));
        LB_CUDA(cudaStreamSynchronize(stream_of(p)));
    });
}

int lb_get_tri_pt(lb_problem *h, double *pt, double *gt) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(p.have_eval, LB_ERR_STATE, "no evaluation");
        set_device(p);
        if (p.T) {
            if (pt) LB_CUDA(cudaMemcpyAsync(pt, p.pt.ptr, sizeof(double) * p.T, cudaMemcpyDeviceToHost, stream_of(p)));
            if (gt && !(p.last_flags & LB_EVAL_FIXED))
                LB_CUDA(cudaMemcpyAsync(gt, p.gt.ptr, sizeof(double) * p.T, cudaMemcpyDeviceToHost, stream_of(p)));
        }
        LB_CUDA(cudaStreamSynchronize(stream_of(p)));
    });
}

int lb_get_vcs_ppv(lb_problem *h, int32_t level, double *ppv, uint8_t *slack, double *stn) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(p.have_eval, LB_ERR_STATE, "no evaluation");
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        auto *lv = p.vlev[level];
        set_device(p);
        get_entries(p, *lv, lv->ppv, ppv);
        get_entries(p, *lv, lv->slack, slack);
        get_entries(p, *lv, lv->stn, stn);
    });
}

int lb_sweeps(lb_problem *h, int32_t nsweeps, double rho, double rt, double damp, int32_t nbatch,
              const int64_t *perms, double kap2) {
    return guard([&] {
        LB_CHECK(h && perms, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(nsweeps >= 0 && nbatch >= 1 && nbatch <= p.n, LB_ERR_INVALID, "need nsweeps >= 0, 1 <= nbatch <= n");
        LB_CHECK(p.ngraphs == 0, LB_ERR_INVALID, "sweeps are not supported on batched problems");
        LB_CHECK(isfinite(rho) && rho >= 0 && isfinite(rt) && rt >= 0 && isfinite(damp) && damp >= 0,
                 LB_ERR_INVALID, "rho, rt and damp must be finite and >= 0");
        if (nsweeps == 0) return;
        set_device(p);
        cudaStream_t s = stream_of(p);
        // permutations in the caller's row ids -> internal rows (int32), validated
        std::vector<int> perm32((size_t)nsweeps * p.n);
        std::vector<char> seen((size_t)p.n);
        for (int32_t w = 0; w < nsweeps; w++) {
            std::fill(seen.begin(), seen.end(), 0);
            for (int64_t k = 0; k < p.n; k++) {
                const int64_t v = perms[(int64_t)w * p.n + k];
                LB_CHECK(v >= 0 && v < p.n && !seen[v], LB_ERR_INVALID, "perms must hold permutations of 0..n-1");
                seen[v] = 1;
                perm32[(size_t)w * p.n + k] = (int)(p.permuted ? p.inv_h[v] : v);
            }
        }
        upload(p.sw_perm, perm32, s);
        sweeps_run(p, nsweeps, rho, rt, damp, nbatch, p.sw_perm.as<int>(), kap2, s);
        LB_CUDA(cudaStreamSynchronize(s));
        p.have_eval = false;
    });
}

int lb_separate(lb_problem *h, double thresh, int32_t maxh, int32_t maxk, int32_t hub2, int32_t cap2, double vtol,
                int64_t cap0, int64_t cap1, int32_t nchunk, int32_t nbins, int32_t families, int64_t *n0,
                int64_t *n1) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        LB_CHECK(maxh >= 1 && maxk >= 1 && hub2 >= 0 && cap2 >= 0 && nchunk >= 1 && nbins >= 1 && cap0 >= 0 &&
                     cap1 >= 0 && isfinite(thresh) && isfinite(vtol) && vtol < 2.0,
                 LB_ERR_INVALID, "invalid separation parameters");
        Problem &p = h->p;
        set_device(p);
        SepParams sp{thresh, vtol, maxh, maxk, hub2, cap2, nchunk, nbins, cap0, cap1, (families & 1) != 0,
                     (families & 2) != 0};
        separate_run(p, sp, stream_of(p));
        if (n0) *n0 = (int64_t)p.sep_val[0].size();
        if (n1) *n1 = (int64_t)p.sep_val[1].size();
    });
}

int lb_separate_get(lb_problem *h, int32_t family, int64_t *tri, double *val) {
    return guard([&] {
        LB_CHECK(h && (family == 0 || family == 1), LB_ERR_INVALID, "family must be 0 or 1");
        const Problem &p = h->p;
        if (tri) std::copy(p.sep_tri[family].begin(), p.sep_tri[family].end(), tri);
        if (val) std::copy(p.sep_val[family].begin(), p.sep_val[family].end(), val);
    });
}

int lb_vcs_separate(lb_problem *h, int32_t level, int64_t nadd, double tol, int32_t mode, int64_t *count,
                    double *stats) {
    return guard([&] {
        LB_CHECK(h && count, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        LB_CHECK(nadd >= 0 && nadd < ((int64_t)1 << 31), LB_ERR_INVALID, "nadd must be in [0, 2^31)");
        LB_CHECK(mode >= 0 && mode <= 2 && isfinite(tol), LB_ERR_INVALID, "mode must be 0 (pen), 1 (mean) or 2 (mass)");
        set_device(p);
        vcs_separate_run(p, level, nadd, tol, mode, count, stats, stream_of(p));
    });
}

int lb_vcs_grow(lb_problem *h, int32_t level, int64_t nadd, double tol, int32_t mode, int32_t drop_age,
                int64_t max_nnz, double *stats, int64_t *counts) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        LB_CHECK(nadd >= 0 && nadd < ((int64_t)1 << 31), LB_ERR_INVALID, "nadd must be in [0, 2^31)");
        LB_CHECK(mode >= 0 && mode <= 2 && isfinite(tol), LB_ERR_INVALID, "mode must be 0 (pen), 1 (mean) or 2 (mass)");
        LB_CHECK(drop_age <= 255, LB_ERR_INVALID, "drop_age must be <= 255 (ages are 8-bit)");
        LB_CHECK(max_nnz >= 0, LB_ERR_INVALID, "max_nnz must be >= 0");
        set_device(p);
        vcs_grow_run(p, level, nadd, tol, mode, drop_age, max_nnz, stats, counts, stream_of(p));
    });
}

int lb_vcs_get_structure(lb_problem *h, int32_t level, int64_t *ptr, int32_t *col) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        set_device(p);
        vcs_structure(p, *p.vlev[level], ptr, col, stream_of(p));
    });
}

int lb_vcs_nnz(const lb_problem *h, int32_t level, int64_t *nnz) {
    return guard([&] {
        LB_CHECK(h && nnz, LB_ERR_INVALID, "null argument");
        LB_CHECK(level >= 0 && level < (int)h->p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        *nnz = h->p.vlev[level]->nnz;
    });
}

int lb_vcs_sig_stats(lb_problem *h, int32_t level, double *sig_sum, int64_t *active) {
    return guard([&] {
        LB_CHECK(h && sig_sum && active, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(level >= 0 && level < (int)p.vlev.size(), LB_ERR_INVALID, "no such VCS level");
        set_device(p);
        vcs_sig_stats_run(p, level, sig_sum, active, stream_of(p));
    });
}

int lb_vcs_separate_get(lb_problem *h, int64_t *rows, int32_t *cols, double *scores) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        const Problem &p = h->p;
        const int64_t P = std::max<int32_t>(p.vsep_P, 1);
        for (size_t k = 0; k < p.vsep_idx.size(); k++) {
            const int64_t i = p.vsep_idx[k] / P, R = p.vsep_idx[k] % P;
            if (rows) rows[k] = p.permuted ? p.order_h[i] : i;
            if (cols) cols[k] = (int32_t)R;
            if (scores) scores[k] = p.vsep_score[k];
        }
    });
}

int lb_timing_collect(lb_problem *h, double *ms, int64_t *count) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        set_device(p);
        LB_CUDA(cudaStreamSynchronize(stream_of(p)));
        constexpr int NE = LB_NPHASES + 1;
        double acc[LB_NPHASES] = {0};
        const size_t nrec = p.ev_used / NE;
        for (size_t r = 0; r < nrec; r++)
            for (int ph = 0; ph < LB_NPHASES; ph++) {
                float t = 0.f;
                LB_CUDA(cudaEventElapsedTime(&t, p.ev_pool[r * NE + ph], p.ev_pool[r * NE + ph + 1]));
                acc[ph] += t;
            }
        if (ms)
            for (int ph = 0; ph < LB_NPHASES; ph++) ms[ph] = acc[ph];
        if (count) *count = (int64_t)nrec;
        p.ev_used = 0;
    });
}

int lb_set_light_threshold(lb_problem *h, int32_t work) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        int li = -1;
        for (int k = 0; k < N_LIGHT; k++)
            if (LIGHT_WORK[k] == work) li = k;
        LB_CHECK(work == -1 || li >= 0, LB_ERR_INVALID, "light threshold must be -1 (autotune), 0, 64, 128, 256, 512 or 1024");
        h->p.light_idx = li;
    });
}

int lb_get_light_threshold(const lb_problem *h, int32_t *work, float *tune_ms) {
    return guard([&] {
        LB_CHECK(h && work, LB_ERR_INVALID, "null argument");
        *work = h->p.light_idx < 0 ? -1 : LIGHT_WORK[h->p.light_idx];
        if (tune_ms)
            for (int k = 0; k < N_LIGHT; k++) tune_ms[k] = h->p.tune_ms[k];
    });
}

int lb_launch_count(const lb_problem *h, int64_t *launches) {
    return guard([&] {
        LB_CHECK(h && launches, LB_ERR_INVALID, "null argument");
        *launches = h->p.launches;
    });
}

// Pointers the multiplier update swaps (sig <-> pp, sig <-> ppv, lam <-> pt), saved so that a capture that fails
// part-way can put them back (the swaps it made never ran on the device).
struct SwapState {
    std::vector<std::pair<void *, void *>> pl, vl;
    void *lam = nullptr, *pt = nullptr;
    explicit SwapState(Problem &p) {
        for (auto *lv : p.plev) pl.emplace_back(lv->sig.ptr, lv->pp.ptr);
        for (auto *lv : p.vlev) vl.emplace_back(lv->sig.ptr, lv->ppv.ptr);
        lam = p.lam.ptr;
        pt = p.pt.ptr;
    }
    void restore(Problem &p) const {
        for (size_t k = 0; k < pl.size(); k++) {
            if (p.plev[k]->sig.ptr != pl[k].first) {
                std::swap(p.plev[k]->sig.ptr, p.plev[k]->pp.ptr);
                std::swap(p.plev[k]->sig.owner, p.plev[k]->pp.owner);
                std::swap(p.plev[k]->sig.bytes, p.plev[k]->pp.bytes);
            }
        }
        for (size_t k = 0; k < vl.size(); k++) {
            if (p.vlev[k]->sig.ptr != vl[k].first) {
                std::swap(p.vlev[k]->sig.ptr, p.vlev[k]->ppv.ptr);
                std::swap(p.vlev[k]->sig.owner, p.vlev[k]->ppv.owner);
                std::swap(p.vlev[k]->sig.bytes, p.vlev[k]->ppv.bytes);
            }
        }
        if (p.lam.ptr != lam) {
            std::swap(p.lam.ptr, p.pt.ptr);
            std::swap(p.lam.owner, p.pt.owner);
            std::swap(p.lam.bytes, p.pt.bytes);
        }
    }
};

int lb_outer_loop(lb_problem *h, int32_t iters, const int64_t *perms, int32_t nperm, double rho, double tri_weight,
                  double damp, int32_t nbatch, double kap2, int32_t use_graph, int64_t *graph_kernels) {
    return guard([&] {
        LB_CHECK(h && perms, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(iters >= 0 && nperm >= 1, LB_ERR_INVALID, "need iters >= 0 and nperm >= 1");
        LB_CHECK(nbatch >= 1 && nbatch <= p.n, LB_ERR_INVALID, "need 1 <= nbatch <= n");
        LB_CHECK(p.ngraphs == 0, LB_ERR_INVALID, "outer loops are not supported on batched problems");
        LB_CHECK(isfinite(damp) && damp >= 0, LB_ERR_INVALID, "damp must be finite and >= 0");
        check_eval_args(p, rho, tri_weight, 0);
        if (graph_kernels) *graph_kernels = 0;
        if (iters == 0) return;
        set_device(p);
        cudaStream_t s = stream_of(p);
        // row orders in the caller's ids -> internal rows (int32), validated as lb_sweeps does
        std::vector<int> perm32((size_t)nperm * p.n);
        std::vector<char> seen((size_t)p.n);
        for (int32_t w = 0; w < nperm; w++) {
            std::fill(seen.begin(), seen.end(), 0);
            for (int64_t k = 0; k < p.n; k++) {
                const int64_t v = perms[(int64_t)w * p.n + k];
                LB_CHECK(v >= 0 && v < p.n && !seen[v], LB_ERR_INVALID, "perms must hold permutations of 0..n-1");
                seen[v] = 1;
                perm32[(size_t)w * p.n + k] = (int)(p.permuted ? p.inv_h[v] : v);
            }
        }
        upload(p.sw_perm_pool, perm32, s);
        p.sw_nperm = nperm;
        p.sw_perm_cur.alloc(sizeof(int) * (size_t)p.n);
        p.sw_perm_ctr.alloc(sizeof(unsigned long long));
        LB_CUDA(cudaMemsetAsync(p.sw_perm_ctr.ptr, 0, sizeof(unsigned long long), s));
        const double rt = rho * tri_weight;
        // one outer iteration (alm_vcs.py:1384-1436 sweep, 1496-1533 evaluation, 1704-1723 multiplier update)
        auto one = [&]() {
            perm_pick(p, s);
            sweeps_run(p, 1, rho, rt, damp, nbatch, p.sw_perm_cur.as<int>(), kap2, s);
            eval_run(p, rho, tri_weight, 0, s);
            multiplier_update(p, s);
        };
        int32_t done = 0;
        one();          // eager: buffers reach their sizes, the row kernel's light threshold is tuned
        done = 1;
        if (use_graph && iters - done >= 4) {
            // two iterations per graph: the multiplier update swaps buffers, two swaps restore the pointers the
            // graph's kernels were captured with
            const SwapState before(p);
            const int64_t launches0 = p.launches;
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ex = nullptr;
            LB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
            bool ok = true;
            try {
                one();
                one();
            } catch (...) {
                ok = false;
            }
            cudaError_t e = cudaStreamEndCapture(s, &g);
            if (!ok || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                before.restore(p);   // nothing captured ran: continue eagerly below
                g = nullptr;
            }
            p.launches = launches0;
            if (g) {
                size_t nn = 0;
                int64_t kern = 0;
                LB_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
                std::vector<cudaGraphNode_t> nodes(nn);
                if (nn) LB_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
                for (size_t k = 0; k < nn; k++) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nodes[k], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) kern++;
                }
                e = cudaGraphInstantiate(&ex, g, 0);
                if (e != cudaSuccess) {
                    cudaGraphDestroy(g);
                    LB_CUDA(e);
                }
                const int32_t reps = (iters - done) / 2;
                for (int32_t r = 0; r < reps && e == cudaSuccess; r++) e = cudaGraphLaunch(ex, s);
                const cudaError_t e2 = cudaStreamSynchronize(s);
                cudaGraphExecDestroy(ex);
                cudaGraphDestroy(g);
                LB_CUDA(e);
                LB_CUDA(e2);
                done += 2 * reps;
                p.launches += kern * reps;
                if (graph_kernels) *graph_kernels = kern;
            }
        }
        while (done < iters) {
            one();
            done++;
        }
        LB_CUDA(cudaStreamSynchronize(s));
        p.have_eval = false;
    });
}

int lb_multiplier_update(lb_problem *h) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null problem");
        Problem &p = h->p;
        LB_CHECK(p.have_eval && !(p.last_flags & LB_EVAL_FIXED), LB_ERR_STATE,
                 "multiplier update needs a preceding penalised evaluation");
        set_device(p);
        multiplier_update(p, stream_of(p));
        LB_CUDA(cudaStreamSynchronize(stream_of(p)));
        p.have_eval = false;
    });
}

// ------------------------------------------------------------------------------------------------ exact reduction
// labels in [0, P) with P = max + 1 (the reference's bincount length)
static int64_t label_count(const int64_t *lab, int64_t n) {
    int64_t mx = -1;
    for (int64_t i = 0; i < n; i++) {
        LB_CHECK(lab[i] >= 0 && lab[i] < ((int64_t)1 << 31), LB_ERR_INVALID, "labels must lie in [0, 2^31)");
        mx = std::max(mx, lab[i]);
    }
    return mx + 1;
}

int lb_reduce_exact(lb_ctx *ctx, int64_t n, int64_t m, const int64_t *keys, lb_reduction **out) {
    return guard([&] {
        LB_CHECK(ctx && out && (keys || m == 0), LB_ERR_INVALID, "null argument");
        LB_CHECK(n >= 1 && n < ((int64_t)1 << 31) && m >= 0 && m < ((int64_t)1 << 30), LB_ERR_INVALID,
                 "need 1 <= n < 2^31 and 0 <= m < 2^30");
        for (int64_t e = 0; e < m; e++)
            LB_CHECK(keys[e] >= 0 && keys[e] < n * n && keys[e] / n != keys[e] % n, LB_ERR_INVALID,
                     "edge keys must be u * n + v with u != v in [0, n)");
        LB_CUDA(cudaSetDevice(ctx->c.device));
        auto *h = new lb_reduction();
        h->r.ctx = &ctx->c;
        h->r.n = n;
        h->r.m = m;
        try {
            reduce_run(h->r, keys);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int lb_reduce_info(const lb_reduction *h, int64_t *info) {
    return guard([&] {
        LB_CHECK(h && info, LB_ERR_INVALID, "null argument");
        const Reduction &r = h->r;
        const int64_t v[7] = {r.N, r.M, 2 * r.m, r.inside, r.leaf_unions, r.twin_unions, r.n};
        std::copy(v, v + 7, info);
    });
}

int lb_reduce_get(const lb_reduction *h, int64_t *keys, double *weights, int64_t *vol, int64_t *group_of) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null reduction");
        LB_CUDA(cudaSetDevice(h->r.ctx->device));
        reduce_get(h->r, keys, weights, vol, group_of);
    });
}

int lb_reduce_labels(lb_reduction *h, const int64_t *lab, int64_t *lab_red, int64_t *counts) {
    return guard([&] {
        LB_CHECK(h && lab && counts, LB_ERR_INVALID, "null argument");
        Reduction &r = h->r;
        const int64_t P = label_count(lab, r.n);
        LB_CUDA(cudaSetDevice(r.ctx->device));
        reduce_labels(r, lab, P, lab_red, counts);
    });
}

int lb_reduce_destroy(lb_reduction *h) {
    if (!h) return LB_OK;
    cudaSetDevice(h->r.ctx->device);
    cudaStreamSynchronize(h->r.ctx->stream);
    delete h;
    return LB_OK;
}

int lb_simple_graph(lb_ctx *ctx, int64_t m, const int64_t *pairs, int64_t n_names, lb_graph **out) {
    return guard([&] {
        LB_CHECK(ctx && pairs && out, LB_ERR_INVALID, "null argument");
        LB_CHECK(m >= 1 && m < ((int64_t)1 << 30), LB_ERR_INVALID, "need 1 <= m < 2^30 node pairs");
        LB_CHECK(n_names < ((int64_t)1 << 31), LB_ERR_INVALID, "need n_names < 2^31");
        if (n_names >= 0)
            for (int64_t i = 0; i < 2 * m; i++)
                LB_CHECK(pairs[i] >= 0 && pairs[i] < n_names, LB_ERR_INVALID, "node index outside [0, n_names)");
        LB_CUDA(cudaSetDevice(ctx->c.device));
        auto *h = new lb_graph();
        h->g.ctx = &ctx->c;
        try {
            simple_graph_run(h->g, pairs, m, n_names);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int lb_graph_info(const lb_graph *h, int64_t *info) {
    return guard([&] {
        LB_CHECK(h && info, LB_ERR_INVALID, "null argument");
        const SimpleGraph &g = h->g;
        const int64_t v[5] = {g.n, g.m, g.n_names - g.n, g.self_loops, g.n_names};
        std::copy(v, v + 5, info);
    });
}

int lb_graph_get(const lb_graph *h, int64_t *u, int64_t *v, int64_t *kept, int64_t *isolated) {
    return guard([&] {
        LB_CHECK(h, LB_ERR_INVALID, "null graph");
        LB_CUDA(cudaSetDevice(h->g.ctx->device));
        simple_graph_get(h->g, u, v, kept, isolated);
    });
}

int lb_graph_destroy(lb_graph *h) {
    if (!h) return LB_OK;
    cudaSetDevice(h->g.ctx->device);
    cudaStreamSynchronize(h->g.ctx->stream);
    delete h;
    return LB_OK;
}

int lb_modularity_counts(lb_ctx *ctx, int64_t n, int64_t m, const int64_t *u, const int64_t *v, const int64_t *lab,
                         int64_t *inside, int64_t *sum_vol2) {
    return guard([&] {
        LB_CHECK(ctx && lab && inside && sum_vol2 && ((u && v) || m == 0), LB_ERR_INVALID, "null argument");
        LB_CHECK(n >= 1 && n < ((int64_t)1 << 31) && m >= 0 && m < ((int64_t)1 << 31), LB_ERR_INVALID,
                 "need 1 <= n < 2^31 and 0 <= m < 2^31");
        for (int64_t e = 0; e < m; e++)
            LB_CHECK(u[e] >= 0 && u[e] < n && v[e] >= 0 && v[e] < n, LB_ERR_INVALID, "endpoint outside [0, n)");
        const int64_t P = label_count(lab, n);
        LB_CUDA(cudaSetDevice(ctx->c.device));
        modularity_counts_run(ctx->c, n, m, u, v, lab, P, inside, sum_vol2);
    });
}

}  // extern "C"
