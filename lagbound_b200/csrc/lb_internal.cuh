// Internal declarations of the lagbound_b200 library (device structures, vector-load traits, launchers).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/lagbound_b200.h"

namespace lb {

// ------------------------------------------------------------------------------------------------ errors
void set_error(const std::string &msg);
struct Err {
    int code;
};
#define LB_CUDA(call)                                                                                       \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) {                                                                            \
            ::lb::set_error(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ":" +   \
                            std::to_string(__LINE__) + ")");                                                \
            throw ::lb::Err{LB_ERR_CUDA};                                                                   \
        }                                                                                                   \
    } while (0)
#define LB_CHECK(cond, code, msg)                                                                           \
    do {                                                                                                    \
        if (!(cond)) {                                                                                      \
            ::lb::set_error(msg);                                                                           \
            throw ::lb::Err{code};                                                                          \
        }                                                                                                   \
    } while (0)
#define LB_LAUNCH_CHECK() LB_CUDA(cudaGetLastError())

// ------------------------------------------------------------------------------------------------ device buffers
// The stream on which the current library call of a problem orders its buffer allocations and frees (set by the
// entry points that work for a problem, cleared when they return; nullptr: synchronous cudaMalloc / cudaFree).
// Stream-ordered allocation keeps a buffer's growth or release from synchronising the whole device, which would
// stall every other problem's stream (the bound server runs many at once).
cudaStream_t &alloc_stream();

struct DBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t owner = nullptr;   // the stream it was allocated on (freed there, after the work queued before)
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (ptr) {
            if (owner)
                cudaFreeAsync(ptr, owner);
            else
                cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
        owner = nullptr;
    }
    void alloc(size_t b) {
        if (b <= bytes && ptr) return;
        release();
        if (b == 0) b = 16;
        cudaStream_t s = alloc_stream();
        cudaError_t e = s ? cudaMallocAsync(&ptr, b, s) : cudaMalloc(&ptr, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            set_error("cudaMalloc(" + std::to_string(b) + " bytes): " + cudaGetErrorString(e));
            throw Err{LB_ERR_NOMEM};
        }
        bytes = b;
        owner = s;
    }
    template <typename T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

template <typename T> void upload(DBuf &b, const T *host, size_t count, cudaStream_t s) {
    b.alloc(sizeof(T) * count);
    if (count) LB_CUDA(cudaMemcpyAsync(b.ptr, host, sizeof(T) * count, cudaMemcpyHostToDevice, s));
}
template <typename T> void upload(DBuf &b, const std::vector<T> &v, cudaStream_t s) {
    upload(b, v.data(), v.size(), s);
}

// ------------------------------------------------------------------------------------------------ vector traits
// One "chunk" = 16 bytes of a V row; a lane group of NCH lanes covers a row of NCH chunks.
template <typename T> struct VT;
template <> struct VT<double> {
    using Acc = double;
    static constexpr int EPL = 2;
    __device__ __forceinline__ static void load(const double *p, double (&x)[2]) {
        const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
        x[0] = v.x;
        x[1] = v.y;
    }
};
template <> struct VT<float> {
    using Acc = float;
    static constexpr int EPL = 4;
    __device__ __forceinline__ static void load(const float *p, float (&x)[4]) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
        x[0] = v.x;
        x[1] = v.y;
        x[2] = v.z;
        x[3] = v.w;
    }
};
template <> struct VT<__nv_bfloat16> {
    using Acc = float;
    static constexpr int EPL = 8;
    __device__ __forceinline__ static void load(const __nv_bfloat16 *p, float (&x)[8]) {
        const uint4 u = __ldg(reinterpret_cast<const uint4 *>(p));
        const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float2 f = __bfloat1622float2(h[k]);
            x[2 * k] = f.x;
            x[2 * k + 1] = f.y;
        }
    }
};

// A row chunk kept as its raw 16 bytes while the load is in flight, unpacked when it is consumed (holding eight
// chunks unpacked would cost four times the registers in BF16).
__device__ __forceinline__ uint4 ld_chunk(const void *p) { return __ldg(reinterpret_cast<const uint4 *>(p)); }
template <typename T> struct Unpack;
template <> struct Unpack<double> {
    __device__ __forceinline__ static void run(const uint4 &u, double (&x)[2]) {
        x[0] = __hiloint2double((int)u.y, (int)u.x);
        x[1] = __hiloint2double((int)u.w, (int)u.z);
    }
};
template <> struct Unpack<float> {
    __device__ __forceinline__ static void run(const uint4 &u, float (&x)[4]) {
        x[0] = __uint_as_float(u.x);
        x[1] = __uint_as_float(u.y);
        x[2] = __uint_as_float(u.z);
        x[3] = __uint_as_float(u.w);
    }
};
// BF16 is the upper half of an FP32: the element in the low half of a word moves up, the high one is masked
template <> struct Unpack<__nv_bfloat16> {
    __device__ __forceinline__ static void run(const uint4 &u, float (&x)[8]) {
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            x[2 * k] = __uint_as_float(w[k] << 16);
            x[2 * k + 1] = __uint_as_float(w[k] & 0xffff0000u);
        }
    }
};

// acc[k] += x[k] for a raw chunk, in the accumulation type, without unpacking to registers first: BF16 elements
// through the mixed-precision add (FP32 result and addend, BF16 operand, exact conversion), FP32 pairs through the
// packed FP32x2 add; both round exactly as the scalar FP32 add of the unpacked values.
template <typename T> struct Accum;
template <> struct Accum<double> {
    __device__ __forceinline__ static void add(double (&acc)[2], const uint4 &u) {
        double x[2];
        Unpack<double>::run(u, x);
        acc[0] += x[0];
        acc[1] += x[1];
    }
};
template <> struct Accum<float> {
    __device__ __forceinline__ static void add(float (&acc)[4], const uint4 &u) {
        asm("{\n\t.reg .b64 a, x;\n\tmov.b64 a, {%0, %1};\n\tmov.b64 x, {%2, %3};\n\tadd.rn.f32x2 a, a, x;\n\t"
            "mov.b64 {%0, %1}, a;\n\t}"
            : "+f"(acc[0]), "+f"(acc[1])
            : "r"(u.x), "r"(u.y));
        asm("{\n\t.reg .b64 a, x;\n\tmov.b64 a, {%0, %1};\n\tmov.b64 x, {%2, %3};\n\tadd.rn.f32x2 a, a, x;\n\t"
            "mov.b64 {%0, %1}, a;\n\t}"
            : "+f"(acc[2]), "+f"(acc[3])
            : "r"(u.z), "r"(u.w));
    }
};
template <> struct Accum<__nv_bfloat16> {
    __device__ __forceinline__ static void add(float (&acc)[8], const uint4 &u) {
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int k = 0; k < 4; k++)
            asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\tadd.rn.f32.bf16 %0, lo, %0;\n\t"
                "add.rn.f32.bf16 %1, hi, %1;\n\t}"
                : "+f"(acc[2 * k]), "+f"(acc[2 * k + 1])
                : "r"(w[k]));
    }
};

// Load EPL elements of a row chunk into double precision.
template <typename T> __device__ __forceinline__ void load_d(const T *p, double (&x)[VT<T>::EPL]) {
    typename VT<T>::Acc t[VT<T>::EPL];
    VT<T>::load(p, t);
#pragma unroll
    for (int k = 0; k < VT<T>::EPL; k++) x[k] = (double)t[k];
}

template <typename T> struct Store;
template <> struct Store<double> {
    __device__ __forceinline__ static void st(double *p, const double *x, int cnt) {
        for (int k = 0; k < cnt; k += 2) *reinterpret_cast<double2 *>(p + k) = make_double2(x[k], x[k + 1]);
    }
    // streaming store (written once, not read again by this kernel)
    __device__ __forceinline__ static void st_cs(double *p, const double *x, int cnt) {
        for (int k = 0; k < cnt; k += 2) __stcs(reinterpret_cast<double2 *>(p + k), make_double2(x[k], x[k + 1]));
    }
};
template <> struct Store<float> {
    __device__ __forceinline__ static void st(float *p, const float *x, int cnt) {
        for (int k = 0; k < cnt; k += 4) *reinterpret_cast<float4 *>(p + k) = make_float4(x[k], x[k + 1], x[k + 2], x[k + 3]);
    }
    __device__ __forceinline__ static void st_cs(float *p, const float *x, int cnt) {
        for (int k = 0; k < cnt; k += 4)
            __stcs(reinterpret_cast<float4 *>(p + k), make_float4(x[k], x[k + 1], x[k + 2], x[k + 3]));
    }
};

// ------------------------------------------------------------------------------------------------ problem state
constexpr int MAX_LEVELS = 4;       // pair levels and VCS levels per problem (production uses 1-2 of each)
constexpr int HEAVY_DEG = 2048;     // rows with more edges, or more than HEAVY_TRI triangle incidences, are split:
constexpr int SEG_EDGES = 1024;     //   edges into segments of SEG_EDGES and incidences into segments of SEG_TRI,
constexpr int HEAVY_TRI = 512;      //   one warp per segment, partials summed in segment order
constexpr int SEG_TRI = 256;
// light-row thresholds of the row kernel (work = edges + 2 x triangle incidences): rows at or below the chosen one run
// one per lane group, the others one per warp; the autotuner picks one per problem
constexpr int N_LIGHT = 6;
constexpr int LIGHT_WORK[N_LIGHT] = {0, 64, 128, 256, 512, 1024};
constexpr int SEGSUM_CHUNK = 256;   // entries per work item of the deterministic segmented sums
constexpr int VSEG = 64;            // VCS working-set entries per evaluation item (a row with more is split)

// Work items of a deterministic segmented sum: item t covers entries [e0, e1) of segment seg.
// Segments with more than SEGSUM_GROUP items are combined in two levels: groups of SEGSUM_GROUP consecutive items,
// then the groups of each segment (both in a fixed order).
constexpr int SEGSUM_GROUP = 64;
struct SegPlan {
    int64_t nseg = 0, nitems = 0, ngroups = 0;   // ngroups = 0: one level
    DBuf item_seg, item_e0, item_e1;   // int32 seg, int64 ranges
    DBuf seg_item_ptr;                 // int64 nseg+1: items of each segment are contiguous
    DBuf group_item_ptr, seg_group_ptr;   // int64 ngroups+1, nseg+1 (two-level plans)
    void build(const std::vector<int64_t> &seg_ptr, cudaStream_t s);
    int64_t scratch_rows() const { return nitems + ngroups; }   // partial rows (of ld doubles) segsum_run needs
};

struct PairLevel {
    int32_t P = 0;
    double w = 1.0;
    DBuf lab;          // int32 n
    DBuf rq, dsq;      // f64 P
    DBuf sig, pp;      // f64 P x P (pp = effective multipliers of the last evaluation)
    DBuf Y, M;         // f64 P x ld
    DBuf pdiag, kq;    // f64 P
    DBuf members, member_ptr;   // int32 n (rows sorted by label, stable), int64 P+1
    SegPlan plan;
    std::vector<int64_t> member_ptr_h;
};

struct VcsLevel {
    int32_t P = 0;
    double wv = 1.0;
    int64_t nnz = 0;
    DBuf lab;                       // int32 n
    DBuf rq, vol;                   // f64 P
    DBuf ptr;                       // int64 n+1
    DBuf col;                       // int32 nnz
    DBuf sig, ppv, stn, stZ;        // f64 nnz
    DBuf age, slack;                // uint8 nnz
    DBuf own;                       // int64 n: entry (i, lab_i) or -1
    DBuf crow, cent;                // column view: row (int32) and entry (int64) of the entries sorted by column
    DBuf Y, Z, cnt;                 // f64 P x ld, P x ld, P
    DBuf cptr;                      // int64 P+1: column view offsets
    SegPlan yplan, zplan;
    DBuf members;                   // int32 n rows sorted by label
    std::vector<int64_t> member_ptr_h;
    DBuf ent_map;                   // int64 nnz: internal entry -> caller entry (locality order only)
    // evaluation items: (row, e0, e1, slot) with at most VSEG entries of one row each; rows split into several items
    // sum their items' partial rows (slots) in k_vcs_sy_combine
    DBuf items;                     // int4 nitems
    DBuf SY, SYpart;                // f64 n x ld: sum over the row's entries of ppv_e Y_R; f64 nslots x ld
    DBuf inv2a;                     // f64 P: 1 / (2 rho wv rq_R) of the last evaluation
    DBuf multi_rows, multi_slot_ptr;   // int32 nmulti, int32 nmulti+1
    int64_t nitems = 0, nmulti = 0, nslots = 0;
};

struct LobpcgState;                       // lb_lobpcg.cu
void lobpcg_state_free(LobpcgState *st);

struct Problem {
    lb_ctx *ctx = nullptr;
    int64_t n = 0, nnz = 0;
    int32_t r = 0, ld = 0;
    lb_dtype vdtype = LB_F64;
    double L = 1.0, C0 = 0.0;
    bool weighted = false;
    DBuf indptr, indices, weights, d;     // int64 n+1, int32 nnz, f32 nnz (weighted only), f64 n
    DBuf V, G;                            // vdtype n x ld, (f64 | f32) n x ld
    DBuf heavy_items;                     // int64 x4 per item: row, kind (0 edges, 1 incidences), e0, e1
    DBuf heavy_rows, heavy_item_ptr;      // int32 heavy row ids, int64 item ranges per heavy row
    int64_t n_heavy = 0, n_heavy_items = 0;
    DBuf heavy_part;                      // acc-type partial row sums, n_heavy_items x ld
    DBuf z;                               // f64 ld
    SegPlan zplan;
    DBuf all_rows;                        // int32 0..n-1 (rows of the z segment)
    // locality order: internal row k holds the caller's row order[k]; V, G, labels, working sets and triangles are
    // given and returned in the caller's order
    bool permuted = false;
    std::vector<int64_t> order_h, inv_h;
    DBuf order_d;                         // int32 n
    std::vector<int64_t> indptr_h, tptr_h;
    std::vector<double> d_h;              // internal order
    // triangle separation: caller-numbered CSR (kept when a locality order is used) and the last results
    DBuf cindptr, cindices, inv_d;
    std::vector<int64_t> cindptr_h;
    std::vector<int64_t> sep_tri[2];
    std::vector<int64_t> vsep_idx;        // VCS separation result: internal row * P + cluster, best first
    std::vector<double> vsep_score;
    int32_t vsep_P = 0;
    DBuf vsep_dev;                        // the same selection kept on the device (vcs_grow_run)
    int64_t vsep_dev_count = 0;
    std::vector<double> sep_val[2];
    std::vector<PairLevel *> plev;
    std::vector<VcsLevel *> vlev;
    // triangles
    int64_t T = 0;
    DBuf tri, lam, pt, gt;                // int32 T x 3, f64 T
    DBuf tptr, tinc;                      // int64 n+1, int32 x3 per incidence (o1, o2, t | role << 30)
    // reductions
    DBuf partials;                        // f64 scratch for per-block partial sums
    DBuf row_counter;                     // work counter of k_rows' dynamic row scheduling
    DBuf row_quad;                        // f64 n: v_i . (A V)_i of the last evaluation
    // batched problems: several graphs in one block-diagonal CSR; internal rows of graph g are
    // [gptr_h[g], gptr_h[g + 1]) and its triangles [gtptr_h[g], gtptr_h[g + 1])
    int32_t ngraphs = 0;
    std::vector<int64_t> gptr_h, gtptr_h;
    DBuf gid;                             // int32 n: graph of each internal row
    DBuf gL, ginvL, gC0;                  // f64 per graph
    DBuf gptr, gtptr;                     // int64 G+1
    DBuf gout;                            // f64 G x 5: value, primal, quadA, zz, tri_tot of the last evaluation
    DBuf gsum;                            // f64 2: sum of zz_g and of zz_g / L_g
    DBuf gpart;                           // f64 G x slices x 2: per-graph partial sums
    int light_idx = -1;                   // light-row threshold of k_rows (index into LIGHT_WORK; -1: autotune)
    float tune_ms[N_LIGHT] = {0, 0, 0, 0, 0, 0};  // autotuner timings by threshold
    DBuf sched, nlight;                   // k_rows schedule: rows by work inside each chunk, light rows per chunk
    DBuf staging;                         // host-buffer uploads of V (lb_set_V_raw with a locality order)
    // sweep scratch (lb_sweeps)
    DBuf sw_Vnew, sw_Vold, sw_DD, sw_GX, sw_KX, sw_mark, sw_list, sw_count, sw_perm;
    // outer loops (lb_outer_loop): the row orders of its sweeps (int32 nperm x n, internal rows), the order of the
    // current sweep (int32 n) and the device counter of sweeps taken, which picks the next order
    DBuf sw_perm_pool, sw_perm_cur, sw_perm_ctr;
    int32_t sw_nperm = 0;
    DBuf sw_mpart;                        // f64 partial pair rows: touched cluster x R split x ld
    DBuf scal;                            // device lb_eval_out
    lb_eval_out *scal_host = nullptr;     // pinned
    LobpcgState *lobpcg = nullptr;        // handles and buffers of lb_lobpcg (created on first use)
    // pipelined host evaluations (lb_eval_host_pipelined): copy-in and copy-out streams beside the context's stream,
    // two slots of V staging, raw-G staging and pinned scalars, and the events that hand each slot between them
    struct HostPipe {
        cudaStream_t cin = nullptr, cout = nullptr;
        cudaEvent_t in[2] = {}, conv[2] = {}, comp[2] = {}, out[2] = {};
        lb_eval_out *scal[2] = {nullptr, nullptr};
        DBuf vst[2], gst[2];
        bool ready = false;
        ~HostPipe();
    } pipe;
    bool have_eval = false;
    int last_flags = 0;
    int64_t launches = 0;                 // kernels launched for this problem
    // scratch of the working-set, triangle-pool and separation rounds, one buffer per use site, kept and grown
    // across rounds: once the sizes have been reached the main loop makes no cudaMalloc / cudaFree calls (which
    // synchronise the device and fragment memory under a serving loop's HBM budget)
    std::unordered_map<std::string, std::unique_ptr<DBuf>> scratch_bufs;
    DBuf &scratch(const char *site) {
        auto &b = scratch_bufs[site];
        if (!b) b.reset(new DBuf());
        return *b;
    }
    size_t scratch_bytes() const {
        size_t t = 0;
        for (auto &kv : scratch_bufs) t += kv.second->bytes;
        return t;
    }
    std::vector<cudaEvent_t> ev_pool;     // LB_EVAL_TIMING: 7 events per recorded evaluation
    size_t ev_used = 0;
    cudaEvent_t next_event();
    ~Problem();
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;       // false: the caller's stream (lb_ctx_create_on_stream)
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    int num_sms = 148;
    double v_persist = 0.0;       // share of V kept persisting in L2 during evaluations (0 = off)
    size_t persist_max = 0, window_max = 0;
};
void apply_l2_window(Problem &p, cudaStream_t s);

// ------------------------------------------------------------------------------------------------ launchers
// eval pipeline (lb_eval.cu)
void eval_run(Problem &p, double rho, double tri_weight, int flags, cudaStream_t s);
void build_heavy(Problem &p, cudaStream_t s);
struct SepParams {
    double thresh, vtol;
    int maxh, maxk, hub2, cap2, nchunk, nbins;
    int64_t cap0, cap1;
    bool want0, want1;
};
void separate_run(Problem &p, const SepParams &sp, cudaStream_t s);
// triangle pool on the device (lb_tpool.cu)
void tri_rebuild_incidence(Problem &p, cudaStream_t s);
void tri_pool_round(Problem &p, SepParams sp, int64_t tri_add, int64_t tri1_add, int64_t tri_max, int64_t *counts,
                    cudaStream_t s);
void tri_pool_get(const Problem &p, int64_t *tri, cudaStream_t s);
void sweeps_run(Problem &p, int nsw, double rho, double rt, double damp, int nbatch, const int *perms_dev, double kap2,
                cudaStream_t s);
void convert_V_from_f64(Problem &p, const double *dV_f64_n_r, cudaStream_t s);   // device n x r f64 -> V
void convert_V_to_f64(const Problem &p, double *dout_n_r, cudaStream_t s);
void convert_V_raw(Problem &p, const void *dsrc_n_r, cudaStream_t s);            // device n x r storage dtype -> V
void G_to_f64(const Problem &p, double *dout_n_r, cudaStream_t s);
void G_raw(const Problem &p, void *dout_n_r, cudaStream_t s);                      // G -> n x r in its own dtype
void multiplier_update(Problem &p, cudaStream_t s);
// the next row order of an outer loop: sw_perm_cur = pool[counter % nperm], then counter + 1 (two kernels)
void perm_pick(Problem &p, cudaStream_t s);
void vcs_cluster_sums(Problem &p, VcsLevel &lv, cudaStream_t s);                 // lb_eval.cu
void vcs_separate_run(Problem &p, int level, int64_t nadd, double tol, int mode, int64_t *count, double *stats,
                      cudaStream_t s, bool to_host = true);                      // lb_vsep.cu
// working sets on the device (lb_vgrow.cu)
void vcs_rebuild_views(Problem &p, VcsLevel &lv, cudaStream_t s);
void vcs_build_items(Problem &p, VcsLevel &lv, cudaStream_t s);                   // lb_eval.cu
void vcs_grow_run(Problem &p, int level, int64_t nadd, double tol, int mode, int drop_age, int64_t max_nnz,
                  double *stats, int64_t *counts, cudaStream_t s);
void vcs_entries_to_caller(const Problem &p, const VcsLevel &lv, const void *src, void *dst_host, int esize,
                           cudaStream_t s);
void vcs_structure(const Problem &p, const VcsLevel &lv, int64_t *ptr_host, int32_t *col_host, cudaStream_t s);
void vcs_sig_stats_run(Problem &p, int level, double *sum, int64_t *active, cudaStream_t s);

// exact reduction and modularity counts (lb_reduce.cu)
struct Reduction {
    Ctx *ctx = nullptr;
    int64_t n = 0, m = 0;                      // original graph
    int64_t N = 0, M = 0;                      // groups, reduced edges
    int64_t inside = 0, leaf_unions = 0, twin_unions = 0;
    DBuf eu, ev, deg;                          // int64 m, int64 m, u64 n
    DBuf label, rank, grp, vol;                // int32 n (component root), int32 n (root rank), int64 n, u64 N
    DBuf rkeys, ru, rv, rw;                    // int64 M (a * N + b), int64 M, int64 M, u64 M (edge counts)
};
void reduce_run(Reduction &r, const int64_t *keys_h);
void reduce_get(const Reduction &r, int64_t *keys, double *weights, int64_t *vol, int64_t *group_of);
void reduce_labels(Reduction &r, const int64_t *lab_h, int64_t P, int64_t *lr_out, int64_t *counts);
struct SimpleGraph {
    Ctx *ctx = nullptr;
    int64_t n_names = 0, n = 0, m = 0, self_loops = 0;
    DBuf u, v, kept, isolated;                 // int64 m, m, n, n_names - n
};
void simple_graph_run(SimpleGraph &g, const int64_t *pairs_h, int64_t m_in, int64_t n_names);
void simple_graph_get(const SimpleGraph &g, int64_t *u, int64_t *v, int64_t *kept, int64_t *isolated);
void modularity_counts_run(Ctx &c, int64_t n, int64_t m, const int64_t *u_h, const int64_t *v_h,
                           const int64_t *lab_h, int64_t P, int64_t *inside, int64_t *sum_vol2);

inline int pad_ld(int32_t r, lb_dtype dt) {
    const int esz = dt == LB_F64 ? 8 : dt == LB_F32 ? 4 : 2;
    int ld = 16 / esz;                  // at least one 16-byte chunk
    while (ld < r) ld *= 2;
    return ld;
}
inline size_t dtype_size(lb_dtype dt) { return dt == LB_F64 ? 8 : dt == LB_F32 ? 4 : 2; }

}  // namespace lb

struct lb_ctx {
    lb::Ctx c;
};
struct lb_problem {
    lb::Problem p;
};
struct lb_reduction {
    lb::Reduction r;
};
struct lb_graph {
    lb::SimpleGraph g;
};
struct lb_cuda_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t kernels = 0;
};
