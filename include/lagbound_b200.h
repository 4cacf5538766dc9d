/*
 * lagbound_b200.h -- C ABI of the B200 (sm_100a) augmented-Lagrangian inner loop of lagbound ("Atris").
 *
 * The reference (Yahiahu/Lagbound) has no in-process plugin interface for this path: its API launches the stage
 * scripts src/lagbound/_core/alm_vcs.py and est_dual_vcs.py as subprocesses (src/lagbound/pipeline.py:58-76,
 * 105-136, 156-170) and hands data over through files.  These entry points are what a drop-in replacement of those
 * scripts binds (lagbound_b200/_capi.py through ctypes); each comment names the reference code it replaces.
 *
 * Conventions
 *   - Every function returns LB_OK (0) or a negative LB_ERR_* code; nothing is thrown across the ABI.  The message
 *     of the last failure on the calling host thread is returned by lb_last_error().
 *   - Host arrays are read (or written) during the call only; the library keeps its own device copies.  Index
 *     arrays use the reference's int64 layout (CSR indptr/indices, labels, triangle triples); VCS working-set
 *     columns are int32 as in vcsops.py.
 *   - All work of a problem is ordered on its context's CUDA stream.  Calls that return host results synchronise
 *     that stream; the others are asynchronous.  One context per host thread.
 *   - A problem's device buffers are stream-ordered (cudaMallocAsync / cudaFreeAsync on its context's stream, from
 *     the device's default memory pool, whose release threshold lb_ctx_create raises so that freed memory stays
 *     reserved for reuse); growing or destroying a problem does not synchronise the device.  lb_bv_noalloc is the
 *     entry point for hosts that must do all device allocation themselves.
 *   - All reductions (d^T V, cluster sums, the Lagrangian value and its terms, dual residuals, candidate-bound sums)
 *     are accumulated in FP64 in a fixed order, so results are reproducible run to run.
 *   - V is stored in the problem's dtype (FP64, FP32 or BF16) with rows padded to a power-of-two width of at least
 *     16 bytes; gradients are written in FP64 for the FP64 form and FP32 otherwise.
 */
#ifndef LAGBOUND_B200_H
#define LAGBOUND_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LB_OK 0
#define LB_ERR_INVALID (-1)     /* bad argument (size, index out of range, unsupported combination) */
#define LB_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define LB_ERR_NOMEM (-3)       /* device or host allocation failed */
#define LB_ERR_STATE (-4)       /* call out of order (e.g. multiplier update before an evaluation) */
#define LB_ERR_TIMEOUT (-5)     /* a bounded device-side wait gave up */
#define LB_ERR_NUMERIC (-6)     /* non-finite input or result */

typedef enum { LB_F64 = 0, LB_F32 = 1, LB_BF16 = 2 } lb_dtype;

typedef struct lb_ctx lb_ctx;
typedef struct lb_problem lb_problem;
typedef struct lb_reduction lb_reduction;
typedef struct lb_graph lb_graph;
typedef struct lb_cuda_graph lb_cuda_graph;

/* Scalars of one augmented-Lagrangian evaluation (alm_vcs.py:1496-1533 augmented()). */
typedef struct {
    double value;      /* C0 + <B,X> - sum of the PHR terms of all levels, triangles and VCS levels (Lc) */
    double primal;     /* C0 + <B,X> = C0 + quadA - |d^T V|^2 / L (prim) */
    double quadA;      /* sum_ij A_ij v_i.v_j (quadA, alm_vcs.py:463-474) */
    double zz;         /* |d^T V|^2 */
    double level_tot;  /* sum over pair levels of sum (pp^2 - sig^2)/(2 rho r) (level_aug) */
    double tri_tot;    /* sum (pt^2 - lam^2)/(2 rt) (tri_aug) */
    double vcs_tot;    /* sum over VCS levels of the working-set PHR term (vcs_aug) */
    double gmin;       /* min over stored triangles of 1 - tau (+inf without triangles) */
    int64_t nviol;     /* pair levels: #(h < -1e-9) summed over levels */
    int64_t vcs_nviol; /* VCS levels: #(g < -1e-9) */
    double lam_sum;    /* sum of the stored triangle multipliers */
    double reserved[5];
} lb_eval_out;

/* lb_eval flags */
#define LB_EVAL_GRAD 1          /* also write G = C(y_eff) V (alm_vcs.py:1299-1312 CV at the effective multipliers) */
#define LB_EVAL_FIXED 2         /* fixed multipliers (rho ignored): pp = sig, pt = lam, ppv = sig; no PHR terms
                                   (est_dual_vcs.py:227-242 CV) */
#define LB_EVAL_TIMING 4        /* record CUDA events around every phase on the problem's stream (lb_timing_collect) */

/* Phases of one evaluation, in launch order (the index into lb_timing_collect's output). */
#define LB_PHASE_AGGREGATES 0   /* d^T V and cluster sums Y (segmented sums) */
#define LB_PHASE_PAIR 1         /* pair levels: h, pp, M, PHR terms */
#define LB_PHASE_VCS 2          /* VCS entries and Z */
#define LB_PHASE_TRI 3          /* triangles: tau, pt, PHR term */
#define LB_PHASE_ROWS 4         /* rows: A V, fused epilogue, G (the dominant kernel) */
#define LB_PHASE_FINAL 5        /* FP64 reduction of the partials */
#define LB_NPHASES 6

/* ------------------------------------------------------------------------------------------------ context */
const char *lb_version(void);
const char *lb_last_error(void);
int lb_ctx_create(int device, lb_ctx **out);
/* A context whose work goes on the caller's CUDA stream (a cudaStream_t, e.g. torch's current stream; not destroyed
 * with the context): the library's kernels are then ordered with the caller's own work on that stream, and
 * device-resident inputs and outputs need no synchronisation between the two (lb_set_V_device_async,
 * lb_eval_async, lb_get_G_device_async). */
int lb_ctx_create_on_stream(int device, void *stream, lb_ctx **out);
int lb_ctx_destroy(lb_ctx *ctx);
int lb_ctx_synchronize(lb_ctx *ctx);
/* Record elapsed device time: lb_ctx_timer(ctx, 0) starts, lb_ctx_timer(ctx, 1) stops and returns ms in *ms. */
int lb_ctx_timer(lb_ctx *ctx, int stop, float *ms);

/* CUDA-graph capture of the context's stream: between lb_ctx_capture_begin and lb_ctx_capture_end only
 * asynchronous entry points may be called (lb_eval_async, lb_set_V_device_async); calls that return host results
 * synchronise and end the capture with an error.  Every problem captured must have been evaluated once before (the
 * first evaluation autotunes and allocates).  The graph replays the captured work with the same buffers and
 * arguments (V read as it is at replay time); lb_cuda_graph_kernels gives its number of kernel launches. */
int lb_ctx_capture_begin(lb_ctx *ctx);
int lb_ctx_capture_end(lb_ctx *ctx, lb_cuda_graph **out);
int lb_cuda_graph_launch(lb_cuda_graph *g);
int lb_cuda_graph_kernels(const lb_cuda_graph *g, int64_t *kernels);
int lb_cuda_graph_destroy(lb_cuda_graph *g);

/* Cache controls of the context (they last as long as the context, nothing outlasts the process):
 * l2_fetch_bytes: maximum L2 fetch granularity for the device (cudaLimitMaxL2FetchGranularity: 0 = leave as is,
 * else 32, 64 or 128); v_persist_fraction: share of the V rows of the problem being evaluated kept as persisting in
 * L2 through an access-policy window on the context's stream (0 = off). */
int lb_ctx_set_cache(lb_ctx *ctx, int l2_fetch_bytes, double v_persist_fraction);

/* Random row-gather probe (measurement only): ngather gathers of whole rows of row_bytes (64 or 128) picked uniformly
 * at random from a table of footprint_bytes, by lane groups of 16-byte loads with eight rows in flight per lane;
 * ms_per_launch receives the mean device time of `reps` launches after two untimed ones.  The rate against the
 * footprint is the ceiling of a row-gather kernel on the device (row indices come from a hash, so only the table
 * passes through the caches). */
int lb_gather_probe(lb_ctx *ctx, int64_t footprint_bytes, int32_t row_bytes, int64_t ngather, int32_t reps,
                    float *ms_per_launch);

/* ------------------------------------------------------------------------------------------------ problem */
/* Instance load + CSR (alm_vcs.py:1103-1117): symmetric CSR with sorted column indices, edge weights
 * (NULL = unit weights; reduced instances carry integer multiplicities), volumes d, L = 2 m_orig, C0.
 * r = embedding rank (alm_vcs.py --k), vdtype = storage type of V. */
int lb_problem_create(lb_ctx *ctx, int64_t n, const int64_t *indptr, const int64_t *indices, const double *weights,
                      const double *d, double L, double C0, int32_t r, lb_dtype vdtype, lb_problem **out);
/* Same with a locality order: order[k] = the caller's row placed at internal row k (a permutation of 0..n-1;
 * NULL = identity).  Rows of one community placed together let the gathers of neighbour rows hit L1/L2.  Every
 * other entry point keeps taking and returning V, G, labels, working sets and triangles in the caller's order. */
int lb_problem_create_ordered(lb_ctx *ctx, int64_t n, const int64_t *indptr, const int64_t *indices,
                              const double *weights, const double *d, double L, double C0, int32_t r,
                              lb_dtype vdtype, const int64_t *order, lb_problem **out);
/* Batched problem: ngraphs independent graphs in one block-diagonal CSR (graph g holds rows [row_ptr[g],
 * row_ptr[g + 1]); no edge joins two graphs), each with its own L[g] and C0[g], one rank r and dtype for all.  One
 * evaluation runs every graph in the same launches (the row kernel's degree correction takes each row's graph's
 * d^T V and L).  order (optional) must keep every graph's rows inside the graph's range.  Triangles (lb_tri_set)
 * must lie inside one graph each and come grouped by graph in graph order.  Pair and VCS levels, sweeps and the pool
 * round are not available on batched problems.  lb_eval_out then holds the sums over the graphs. */
int lb_problem_create_batched(lb_ctx *ctx, int32_t ngraphs, const int64_t *row_ptr, int64_t n,
                              const int64_t *indptr, const int64_t *indices, const double *weights, const double *d,
                              const double *L, const double *C0, int32_t r, lb_dtype vdtype, const int64_t *order,
                              lb_problem **out);
/* Per-graph results of the last evaluation of a batched problem: out[5 g + (0..4)] = value, primal, quadA, zz,
 * tri_tot of graph g (as in lb_eval_out, each summed in a fixed order). */
int lb_eval_graphs(lb_problem *p, double *out);
int lb_problem_destroy(lb_problem *p);
/* Row width (elements) of the stored V and G, and the number of heavy rows split across warps. */
int lb_problem_info(const lb_problem *p, int32_t *ld, int64_t *heavy_rows, int64_t *device_bytes);

/* V (alm_vcs.py:1187-1216 init, 1576-1589 save): host n x r FP64, converted to the storage type. */
int lb_set_V(lb_problem *p, const double *V);
int lb_get_V(lb_problem *p, double *V);
/* Same from host data already in the storage type (n x r, row-major): the end-to-end path (copy included). */
int lb_set_V_raw(lb_problem *p, const void *V, lb_dtype dtype);

/* Pair level (aggops.py:51-68 PairLevel; rq, dsq per alm_vcs.py:1181-1184): labels 0..P-1 (n), pair weight w. */
int lb_pair_level_add(lb_problem *p, int32_t P, const int64_t *lab, double w, int32_t *level);
int lb_pair_level_set_sigma(lb_problem *p, int32_t level, const double *sig);   /* P x P */
int lb_pair_level_get_sigma(lb_problem *p, int32_t level, double *sig);
/* set_pair_weight (alm_vcs.py:1270-1275): w on every pair level and wv = vc_weight * w on every VCS level. */
int lb_set_pair_weight(lb_problem *p, double w, double vc_weight);

/* Sparse vertex-cluster level (vcsops.py:31-71 VCSLevel): labels (n), wv = vc_weight * pair weight. */
int lb_vcs_level_add(lb_problem *p, int32_t P, const int64_t *lab, double wv, int32_t *level);
/* Working set as row CSR (vcsops.py set_ws): ptr (n+1) int64, col int32 sorted in each row, sig FP64, age uint8
 * (NULL = zeros). */
int lb_vcs_set_ws(lb_problem *p, int32_t level, int64_t nnz, const int64_t *ptr, const int32_t *col,
                  const double *sig, const uint8_t *age);
int lb_vcs_get_ws(lb_problem *p, int32_t level, double *sig, uint8_t *age);

/* Triangle pool (alm_vcs.py:1186-1196, 1228): T x 3 int64 (a, b = centre, c), multipliers lam (FP64). */
int lb_tri_set(lb_problem *p, int64_t T, const int64_t *tri, const double *lam);
int lb_tri_get_lam(lb_problem *p, double *lam);
/* The solver's triangle-pool round on the device (alm_vcs.py:1735-1756): triangles with lam = 0 are purged,
 * room = max(0, tri_max - kept); with room, the separation of lb_separate runs with cap0 = int(min(tri_add, room)
 * * 1.3) + 10 and (tri1_add > 0) cap1 = int(tri1_add * 1.3) + 10, the one-edge-arm family keeps its tri1_add best
 * and joins the edge-arm family (values + 10), pooled and repeated candidates are dropped (first occurrence kept)
 * and the best min(tri_add + tri1_add, room) by value join with lam 0; the incidence records are rebuilt.  Value
 * ties keep key order (numpy's argsort leaves them unspecified).  counts[3] (may be NULL) = (purged, added, T). */
int lb_tri_pool_round(lb_problem *p, double thresh, int32_t maxh, int32_t maxk, int32_t hub2, int32_t cap2,
                      double vtol, int32_t nchunk, int32_t nbins, int64_t tri_add, int64_t tri1_add, int64_t tri_max,
                      int64_t *counts);
/* The pool's triangles, T x 3 caller vertex ids in pool order, and their number. */
int lb_tri_get(lb_problem *p, int64_t *tri);
int lb_tri_count(const lb_problem *p, int64_t *T);

/* ------------------------------------------------------------------------------------------------ evaluation */
/* One evaluation at the current V and multipliers: augmented() (alm_vcs.py:1496-1533) and, with LB_EVAL_GRAD,
 * the half-gradient G = C(y_eff) V with y_eff the effective multipliers pp, pt, ppv at V (alm_vcs.py:1299-1312).
 * Writes *out (synchronises). */
int lb_eval(lb_problem *p, double rho, double tri_weight, int flags, lb_eval_out *out);
/* Same, asynchronous: scalars stay on the device until lb_eval_fetch. Used for device-timed loops. */
int lb_eval_async(lb_problem *p, double rho, double tri_weight, int flags);
int lb_eval_fetch(lb_problem *p, lb_eval_out *out);
/* End to end from host data: copy V (n x r in the storage dtype) in, evaluate, copy the scalars out. */
int lb_eval_host(lb_problem *p, const void *V_host, double rho, double tri_weight, int flags, lb_eval_out *out);
/* The gradient of the last evaluation in its own dtype (FP64 for the FP64 form, FP32 otherwise), n x r row-major in
 * the caller's row order, into host memory (pinned memory makes the copy run at full speed): with lb_eval_host the
 * end-to-end path of one evaluation, V in and G out (CV at the effective multipliers, alm_vcs.py:1299-1312). */
int lb_get_G_raw(lb_problem *p, void *G_host);
/* nsteps evaluations from host buffers with the copies overlapped: step k uploads V_hosts[k] (n x r in the storage
 * dtype, as lb_set_V_raw takes it), evaluates with `flags`, and downloads its scalars to outs[k] (may be NULL) and,
 * when G_hosts is given (flags must then hold LB_EVAL_GRAD) and G_hosts[k] is not NULL, its raw G (as lb_get_G_raw
 * gives it) to G_hosts[k].  Copy-in, compute and copy-out run on three streams with two staging slots each way, so
 * step k's G download and step k + 1's V upload overlap the evaluations; results equal the call-by-call sequence
 * lb_eval_host + lb_get_G_raw bit for bit.  Host buffers should be pinned (pageable ones are copied without
 * overlap).  A host buffer may appear at several steps.  Returns when every step is done; afterwards V and G hold
 * the last step's. */
int lb_eval_host_pipelined(lb_problem *p, int32_t nsteps, const void *const *V_hosts, void *const *G_hosts,
                           double rho, double tri_weight, int flags, lb_eval_out *outs);
/* G of the last LB_EVAL_GRAD evaluation to host, n x r FP64. */
int lb_get_G(lb_problem *p, double *G);
/* Device-resident blocks, for callers that keep their vectors on the GPU (the estimate's eigensolver and polish):
 * X is device memory with n x r FP64 in the caller's row order, complete when the call is made (the library's
 * stream does not wait on other streams); it is converted into V and the call returns when that is done.
 * lb_get_G_device writes G of the last gradient evaluation as n x r FP64 in the caller's row order into device memory
 * and returns when the copy is complete.  Host pointers are rejected.  The _async forms return once the work is
 * queued on the context's stream (with lb_ctx_create_on_stream: ordered with the caller's work on that stream). */
int lb_set_V_device(lb_problem *p, const double *X);
int lb_get_G_device(lb_problem *p, double *G);
int lb_set_V_device_async(lb_problem *p, const double *X);
/* Block LOBPCG for the smallest eigenpairs of the pencil (Diag(g) - C(y), Diag(s)) with C(y) the problem's
 * fixed-multiplier evaluation (est_dual_vcs.py eig_round's eigensolver): X is k columns of device memory, n x k FP64
 * row-major in the caller's row order (the start block in, the Ritz vectors out); g, s > 0 and the Jacobi
 * preconditioner prec are n device FP64; maxiter iterations of Rayleigh-Ritz on [X, W, P] (W the preconditioned
 * residuals B-orthogonalised against X, P the last update, dropped for an iteration when it makes the Gram matrix
 * indefinite; the iteration stops early when the residual block is numerically dependent).  theta (host, k, may be
 * NULL) receives the Ritz values ascending, iters_done (may be NULL) the iterations taken.  Needs an FP64 problem
 * with r >= k (its V and G are overwritten) and n >= 3 k; runs on the context's stream (cuBLAS and cuSOLVER). */
int lb_lobpcg(lb_problem *p, int32_t k, double *X, const double *g, const double *s, const double *prec,
              int32_t maxiter, double *theta, int32_t *iters_done);
int lb_get_G_device_async(lb_problem *p, double *G);
/* Effective multipliers of the last evaluation: pair level pp (P x P), triangles pt (T), VCS ppv (nnz). */
int lb_get_pair_pp(lb_problem *p, int32_t level, double *pp);
int lb_get_tri_pt(lb_problem *p, double *pt, double *gt);
int lb_get_vcs_ppv(lb_problem *p, int32_t level, double *ppv, uint8_t *slack, double *stn);

/* Device time per phase summed over the LB_EVAL_TIMING evaluations since the last collect (synchronises):
 * ms[LB_NPHASES], *count = number of evaluations recorded. */
int lb_timing_collect(lb_problem *p, double *ms, int64_t *count);
/* Light-row threshold of the row kernel (work = edges + 2 x triangle incidences): rows at or below it run one per
 * lane group, heavier ones one per warp.  -1 = autotune on the next evaluation (0, 64, 128, 256, 512 and 1024 are
 * each timed once on that evaluation's inputs and the fastest kept), or one of those values.  lb_get_light_threshold
 * returns the value in use (-1 before tuning) and the autotuner's timings in ms for the six values (0 = not timed). */
int lb_set_light_threshold(lb_problem *p, int32_t work);
int lb_get_light_threshold(const lb_problem *p, int32_t *work, float *tune_ms);
/* Number of kernels this library has launched for the problem since it was created. */
int lb_launch_count(const lb_problem *p, int64_t *launches);

/* Batched Gauss-Seidel sweeps of the inner loop (alm_vcs.py:1360-1436 sweeps(), row step batch_step6 256-351):
 * for every sweep, perms[sweep * n ...] is the row order (a permutation of the caller's row ids, as
 * rng.permutation(n) in the reference), split into nbatch batches like np.array_split; every batch steps its rows
 * from the pre-batch V (Jacobi within a batch), then updates d^T V, the cluster sums and the VCS state.
 * rho = 0 gives plain mixing at fixed multipliers (the estimator's polishing); rt = rho * tri_weight; kap2 = VCS
 * transposed-curvature factor (alm_vcs.py --vc_kap2, 1).  Synchronises. */
int lb_sweeps(lb_problem *p, int32_t nsweeps, double rho, double rt, double damp, int32_t nbatch,
              const int64_t *perms, double kap2);

/* AL outer iterations without returning to the caller (alm_vcs.py:1360-1436 sweep, 1496-1533 evaluation,
 * 1704-1723 multiplier update, repeated): iteration k sweeps once in the row order perms[(k mod nperm) n ...]
 * (permutations of the caller's row ids, as lb_sweeps takes them) with rt = rho tri_weight, evaluates without the
 * gradient and updates the multipliers, exactly as the calls lb_sweeps(1 sweep) + lb_eval(flags 0) +
 * lb_multiplier_update would, but with no host synchronisation in between.  With use_graph != 0 the first
 * iteration runs directly (buffers sized, row kernel tuned), the next two are captured as one CUDA graph (two, so
 * that the multiplier update's buffer swaps come back to the captured pointers) and replayed, the last odd one runs
 * directly; a launch-bound loop of small problems then costs one graph launch per two iterations instead of
 * hundreds of kernel launches.  graph_kernels (may be NULL) receives the captured graph's kernel count (0: no
 * graph).  A failed capture falls back to direct launches. */
int lb_outer_loop(lb_problem *p, int32_t iters, const int64_t *perms, int32_t nperm, double rho, double tri_weight,
                  double damp, int32_t nbatch, double kap2, int32_t use_graph, int64_t *graph_kernels);

/* Triangle separation at the current V (alm_vcs.py:938-984 separate / separate_both with separate_ref semantics):
 * family 0 (edge arms: neighbours i of a centre j with X_ij > thresh, the top maxh by value when more) and family 1
 * (one-edge arms: 2-hop vertices through the first hub2 arms, first cap2 neighbours each, not adjacent to j,
 * X_jk > thresh, sorted by id or the top maxk by value); violations vm = X_aj + X_jc - X_ac - 1 > vtol histogrammed
 * in nbins bins over nchunk chunks of centres, the threshold bin chosen so at most cap0 (cap1) candidates remain,
 * collected in generation order with the per-chunk caps.  families: bit 0 = family 0, bit 1 = family 1.  Outputs
 * the candidate counts; lb_separate_get copies (min(a,c), j, max(a,c)) triples (caller vertex ids) and values.
 * Indices are identical to the reference's for the same V (FP64 sequential dot products without FMA). */
int lb_separate(lb_problem *p, double thresh, int32_t maxh, int32_t maxk, int32_t hub2, int32_t cap2, double vtol,
                int64_t cap0, int64_t cap1, int32_t nchunk, int32_t nbins, int32_t families, int64_t *n0,
                int64_t *n1);
int lb_separate_get(lb_problem *p, int32_t family, int64_t *tri, double *val);

/* VCS working-set separation (vcsops.py:364-414 separate) of one VCS level at the current V: the entries (i, R)
 * outside the working set with mean violation xbar = s / vol(R minus i) < -tol, s = v_i.Y_R - [R = R(i)] d_i,
 * vol(R minus i) = vol_R - [R = R(i)] d_i > 0, scored by mode 0 pen (wv rq_R s^2), 1 mean (-xbar) or 2 mass
 * (-d_i s); the nadd best are kept (ties: row, then cluster, ascending) and *count is their number.
 * stats[4] (may be NULL) = (#violated entries, their mass sum(-d_i s), #violated in the working set, their mass).
 * The products are FP64 in a fixed order, so the result is reproducible; the reference forms them with BLAS, so a
 * candidate whose score is within rounding of the cut-off may be chosen differently.  Synchronises. */
int lb_vcs_separate(lb_problem *p, int32_t level, int64_t nadd, double tol, int32_t mode, int64_t *count,
                    double *stats);
/* The last separation's entries, best first: caller rows, clusters, scores (each may be NULL). */
int lb_vcs_separate_get(lb_problem *p, int64_t *rows, int32_t *cols, double *scores);
/* Sum of the working-set multipliers of a VCS level and the number of positive ones (the vcssig / act figures of
 * the main loop's log line, alm_vcs.py:1760-1762). */
int lb_vcs_sig_stats(lb_problem *p, int32_t level, double *sig_sum, int64_t *active);
/* The solver's working-set round on the device (alm_vcs.py:1713-1720 with vcsops.py:457-464 update_ws): entries
 * with age >= drop_age are dropped (drop_age <= 0 keeps all), room = max(0, max_nnz - kept), the separation above
 * picks max(1, min(nadd, room)) entries, which join (none when room is 0) with sig 0 and age 0; rows stay sorted by
 * cluster.  The same working set as lb_vcs_separate + update_ws on the host + lb_vcs_set_ws, without the host round
 * trip.  stats[4] as lb_vcs_separate (may be NULL); counts[3] (may be NULL) = (dropped, added, new nnz).
 * Synchronises. */
int lb_vcs_grow(lb_problem *p, int32_t level, int64_t nadd, double tol, int32_t mode, int32_t drop_age,
                int64_t max_nnz, double *stats, int64_t *counts);
/* Working-set structure in the caller's row order: ptr (n+1) and col (nnz) (each may be NULL; vcsops.py
 * VCSLevel.ptr / .col, the checkpoint's vcsptr / vcscol). */
int lb_vcs_get_structure(lb_problem *p, int32_t level, int64_t *ptr, int32_t *col);
/* Number of working-set entries of a VCS level. */
int lb_vcs_nnz(const lb_problem *p, int32_t level, int64_t *nnz);

/* PHR multiplier update of the main loop (alm_vcs.py:1704-1723): sig <- pp for every pair level, lam <- pt,
 * VCS sig <- ppv with age_update (vcsops.py:300-305) from the slack flags.  Requires a preceding evaluation. */
int lb_multiplier_update(lb_problem *p);

/* ------------------------------------------------------------------------------------------------ simple graph */
/* The simple undirected graph of a list of node pairs; replaces the body of graph.py:71-100 _from_pairs
 * (src/lagbound/graph.py).  pairs: m x 2 int64.  n_names < 0: names are the sorted distinct ids in pairs (the
 * np.unique of _from_pairs without names) and pairs may hold any int64; n_names >= 0: pairs index a name list of
 * that length.  Self-loops are dropped, reversed and repeated pairs merged, edges sorted by (a, b) with a < b, nodes
 * without edges set aside and the others renumbered in name order. */
int lb_simple_graph(lb_ctx *ctx, int64_t m, const int64_t *pairs, int64_t n_names, lb_graph **out);
/* info[5] = {n (non-isolated nodes), m (edges), n_isolated, self-loop pairs dropped, n_names} */
int lb_graph_info(const lb_graph *g, int64_t *info);
/* u, v (m, u < v, in key order), kept (n: the name id of each node: the raw id without names, else the index into
 * the name list), isolated (n_isolated, same ids, ascending); any pointer may be NULL. */
int lb_graph_get(const lb_graph *g, int64_t *u, int64_t *v, int64_t *kept, int64_t *isolated);
int lb_graph_destroy(lb_graph *g);

/* ------------------------------------------------------------------------------------------------ exact reduction */
/* Exact (optimum-preserving) reduction of a graph for modularity; replaces the body of reduce_exact.py:12-46
 * (src/lagbound/_core/reduce_exact.py).  keys: m distinct edges as u * n + v (u != v, either order).  Leaf edges
 * (an endpoint of degree 1) and true-twin pairs (adjacent, N[u] = N[v], d^2 < 2m, d > 1) are merged; groups are
 * numbered by the rank of their smallest vertex.  The handle keeps the result on the device. */
int lb_reduce_exact(lb_ctx *ctx, int64_t n, int64_t m, const int64_t *keys, lb_reduction **out);
/* info[7] = {n_red, m_red, L_orig = 2m, inside_edges (= meta.json leaf_edges), leaf_unions, twin_unions, n} */
int lb_reduce_info(const lb_reduction *r, int64_t *info);
/* keys.npy (m_red, ascending a * n_red + b, a < b), weights.npy (m_red, edge counts as FP64), vol.npy (n_red),
 * group_of.npy (n); any pointer may be NULL. */
int lb_reduce_get(const lb_reduction *r, int64_t *keys, double *weights, int64_t *vol, int64_t *group_of);
/* Label restriction of reduce_exact.py:51-62: lab (n, in [0, 2^31)) -> lab_red (n_red, the label of each group's
 * smallest member; may be NULL) and the integer counts of the exact identity
 *   counts[0], counts[1]: inside edges and sum of squared volumes of the partition with the rules enforced;
 *   counts[2], counts[3]: the same partition on the reduced graph (weighted inside edges, group volumes);
 *   counts[4], counts[5]: the partition as given.
 * Q = 2 (C0 + inside) / L - sum / L^2 with C0 = 0 for the original graph and C0 = inside_edges for the reduced one. */
int lb_reduce_labels(lb_reduction *r, const int64_t *lab, int64_t *lab_red, int64_t *counts);
int lb_reduce_destroy(lb_reduction *r);

/* Integer counts of the exact modularity of modularity.py:21-33 (src/lagbound/modularity.py) and lbutil.py:41-50
 * Q_exact: inside = #edges (u_e, v_e) with equal labels, sum_vol2 = sum over labels of (sum of endpoint-count
 * degrees)^2; Q = inside/m - sum_vol2/(4 m^2).  Labels in [0, 2^31), endpoints in [0, n). */
int lb_modularity_counts(lb_ctx *ctx, int64_t n, int64_t m, const int64_t *u, const int64_t *v, const int64_t *lab,
                         int64_t *inside, int64_t *sum_vol2);

/* ------------------------------------------------------------------------------------------------ ordering */
/* Nested-dissection fill-reducing ordering of a symmetric pattern (CSR: indptr n+1, indices; self loops and
 * duplicates ignored, the pattern is symmetrised): perm[k] = the vertex eliminated k-th, iperm its inverse (NULL =
 * not wanted).  Replaces pymetis.nested_dissection in the certificate and the verifier
 * (src/lagbound/_core/certify_lifted_vc.py:247-251 nd_order, verify_cert.py:353-356), which accept any symmetric
 * ordering; lagbound_b200/dropin/pymetis binds it under that name.  Host code: multilevel bisection (heavy-edge
 * coarsening, region growing, boundary FM refinement), vertex separators from the edge cuts, minimum degree on the
 * leaves; deterministic for a given pattern. */
int lb_nd_order(int64_t n, const int64_t *indptr, const int64_t *indices, int64_t *perm, int64_t *iperm);
/* Nonzeros of the Cholesky factor (diagonal included) of the symmetric pattern under the ordering perm (symbolic:
 * elimination tree and row subtrees); *nnz_L = -1 once the count passes cap (cap <= 0: no cap). */
int lb_chol_fill(int64_t n, const int64_t *indptr, const int64_t *indices, const int64_t *perm, int64_t cap,
                 int64_t *nnz_L);

/* ------------------------------------------------------------------------------------------------ no allocation */
/* lb_bv_noalloc -- G = A V - d (d^T V) / L (the modularity part of C(y) V) with out[0] = quadA = sum_ij A_ij v_i.v_j,
 * out[1] = |d^T V|^2, out[2] = quadA - |d^T V|^2 / L + C0, out[3] = number of column indices outside [0, n), which
 * are skipped, out[4] = number of rows whose edge range [indptr[i], indptr[i+1]) was not inside [0, nnz] or was
 * decreasing (clamped to it, so a malformed indptr never reads past indices or weights).  This entry point has no
 * counterpart in the reference.
 * It is for callers that cannot allocate device memory: a host that owns every device byte through its own pool
 * (a serving loop that admits requests against an HBM budget, or a runtime that accounts for all device memory)
 * cannot let a library call cudaMalloc, which synchronises the device and escapes the pool's accounting.
 * Every pointer is a device pointer owned by the caller: indptr int64 (n+1, meant to be non-decreasing from 0 to
 * nnz), indices int32 and weights FP32 or NULL (unit weights), both nnz long, d FP64 (n), V n x ld in dtype,
 * G n x ld (FP64 for LB_F64 V, FP32 otherwise), out 5 doubles; stream may be NULL (the default stream).  V and G
 * must be 16-byte aligned, indptr, d and out 8-byte aligned, indices and weights 4-byte aligned; a misaligned
 * pointer returns LB_ERR_INVALID before anything is launched.
 * Limits: ld at most 64 elements with ld * element size a power of two of at least 16 bytes (columns past the rank
 * must be zero), n < 2^31; other sizes return LB_ERR_INVALID.  Rows are not split across warps.
 * Scratch: one fixed file-scope device array of 541 KB (no cudaMalloc, cudaFree or allocating library call); every
 * GPU that loads the library holds it until the process exits.  The first call on a device resolves the array's
 * device address (cudaGetSymbolAddress, with that device current) and keeps it for the rest of the process; make
 * that first call before any stream capture, and do not call this entry point again after the device's primary
 * context has been destroyed (cudaDeviceReset) in the same process.
 * All calls share the array and it keeps the last call's contents: every slot a call reads was written earlier in
 * the same call, so nothing needs clearing, but calls whose work overlaps on the GPU (two streams, or two host
 * threads) race on it. */
int lb_bv_noalloc(int64_t n, int64_t nnz, const int64_t *indptr, const int32_t *indices, const float *weights,
                  const double *d, double L, double C0, const void *V, lb_dtype dtype, int32_t ld, void *G,
                  double *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
