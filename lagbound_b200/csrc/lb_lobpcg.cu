// Block LOBPCG for the candidate bound's pencil, in native code: the smallest eigenpairs of (Diag(g) - C(y)) x =
// theta Diag(s) x, C(y) applied by the problem's fixed-multiplier evaluation (est_dual_vcs.py:276-389 eig_round's
// eigensolver; the same iteration as lagbound_b200/estimator_gpu.py lobpcg: Rayleigh-Ritz on span[X, W, P] with W
// the Jacobi-preconditioned residuals B-orthogonalised against X and P the previous update, a soft restart without
// P when the Gram matrix is not positive definite).  Tall blocks are column-major n x k with leading dimension n and
// sit side by side in one buffer, so [X, W, P] needs no copies; the small Gram matrices are factored and
// diagonalised by cuSOLVER on the problem's stream.  One host synchronisation per factorisation reads its status.
#include "lb_internal.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include <cublas_v2.h>
#include <cusolverDn.h>

namespace lb {

#define LB_BLAS(x)                                                                                                 \
    do {                                                                                                           \
        const cublasStatus_t st_ = (x);                                                                            \
        if (st_ != CUBLAS_STATUS_SUCCESS) {                                                                        \
            set_error(std::string("cuBLAS error ") + std::to_string((int)st_) + " at " #x);                         \
            throw Err{LB_ERR_CUDA};                                                                                \
        }                                                                                                          \
    } while (0)
#define LB_SOLVER(x)                                                                                               \
    do {                                                                                                           \
        const cusolverStatus_t st_ = (x);                                                                          \
        if (st_ != CUSOLVER_STATUS_SUCCESS) {                                                                      \
            set_error(std::string("cuSOLVER error ") + std::to_string((int)st_) + " at " #x);                       \
            throw Err{LB_ERR_CUDA};                                                                                \
        }                                                                                                          \
    } while (0)

static inline unsigned nb256(int64_t work) { return (unsigned)((work + 255) / 256); }

// out = s .* Y (rows scaled), column-major n x k
__global__ void k_lo_scale(int64_t n, int k, const double *__restrict__ s, const double *__restrict__ Y,
                           double *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n * k) out[t] = s[t % n] * Y[t];
}
// W = prec .* (AX - s .* X .* lam_j)
__global__ void k_lo_resid(int64_t n, int k, const double *__restrict__ s, const double *__restrict__ prec,
                           const double *__restrict__ X, const double *__restrict__ AX, const double *__restrict__ lam,
                           double *__restrict__ W) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * k) return;
    const int64_t i = t % n;
    const int j = (int)(t / n);
    W[t] = prec[i] * (AX[t] - s[i] * X[t] * lam[j]);
}
// out = g .* Y - CY
__global__ void k_lo_mop(int64_t n, int k, const double *__restrict__ g, const double *__restrict__ Y,
                         const double *__restrict__ CY, double *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n * k) out[t] = g[t % n] * Y[t] - CY[t];
}
// G = (G + G^T) / 2, m x m
__global__ void k_lo_sym(int m, double *__restrict__ G) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m * m) return;
    const int i = t % m, j = t / m;
    if (i < j) {
        const double v = 0.5 * (G[i + (int64_t)j * m] + G[j + (int64_t)i * m]);
        G[i + (int64_t)j * m] = v;
        G[j + (int64_t)i * m] = v;
    }
}
__global__ void k_lo_eye(int m, double *__restrict__ I) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < m * m) I[t] = (t % m == t / m) ? 1.0 : 0.0;
}

// cuBLAS / cuSOLVER handle pairs per device, reused by the problems that come and go (destroying a handle frees its
// device workspace, which synchronises the device)
static std::mutex g_handle_mu;
static std::map<int, std::vector<std::pair<cublasHandle_t, cusolverDnHandle_t>>> g_handles;

// Handles and buffers of a problem's LOBPCG runs, kept between calls (grown when n or the block grows).
struct LobpcgState {
    int device = -1;
    cublasHandle_t blas = nullptr;
    cusolverDnHandle_t sol = nullptr;
    DBuf S[2], AS[2];            // n x 3k column-major: [X, W, P] and [AX, AW, AP]
    DBuf tmp;                    // n x 3k
    DBuf opin, opout;            // n x r row-major: the operator's input and output in the caller's row order
    DBuf gA, gB, Linv, T1, Cc;   // m x m (m <= 3k)
    DBuf w, lam;                 // m eigenvalues, k Ritz values
    DBuf work, info;
    int lwork = 0;
    ~LobpcgState() {
        if (blas && sol) {
            std::lock_guard<std::mutex> lock(g_handle_mu);
            g_handles[device].emplace_back(blas, sol);
        }
    }
};
void lobpcg_state_free(LobpcgState *st) { delete st; }

namespace {

struct Run {
    Problem &p;
    LobpcgState &st;
    cudaStream_t s;
    int64_t n;
    int k;
    const double *g, *sv, *prec;

    // CY = C(y) Y for Y column-major n x k (the problem's fixed evaluation on the caller-ordered rows)
    void apply_C(const double *Y, double *CY) {
        const double one = 1.0, zero = 0.0;
        const int r = p.r;
        double *in = st.opin.as<double>(), *out = st.opout.as<double>();
        LB_BLAS(cublasDgeam(st.blas, CUBLAS_OP_T, CUBLAS_OP_N, k, (int)n, &one, Y, (int)n, &zero, in, r, in, r));
        convert_V_from_f64(p, in, s);
        eval_run(p, 0.02, 1.0, LB_EVAL_FIXED | LB_EVAL_GRAD, s);   // fixed multipliers: rho is not used
        G_to_f64(p, out, s);
        LB_BLAS(cublasDgeam(st.blas, CUBLAS_OP_T, CUBLAS_OP_N, (int)n, k, &one, out, r, &zero, CY, (int)n, CY, (int)n));
    }
    // AY = Diag(g) Y - C(y) Y
    void mop(const double *Y, double *AY) {
        double *CY = st.tmp.as<double>();
        apply_C(Y, CY);
        k_lo_mop<<<nb256(n * k), 256, 0, s>>>(n, k, g, Y, CY, AY);
        LB_LAUNCH_CHECK();
    }
    // G = Y1^T Y2 (m1 x m2), symmetrised when square
    void gram(const double *Y1, int m1, const double *Y2, int m2, double *G, bool sym) {
        const double one = 1.0, zero = 0.0;
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_T, CUBLAS_OP_N, m1, m2, (int)n, &one, Y1, (int)n, Y2, (int)n, &zero,
                            G, m1));
        if (sym) {
            k_lo_sym<<<nb256((int64_t)m1 * m1), 256, 0, s>>>(m1, G);
            LB_LAUNCH_CHECK();
        }
    }
    // lower Cholesky factor of the m x m matrix G in place; false when it is not positive definite
    bool potrf(double *G, int m) {
        LB_SOLVER(cusolverDnDpotrf(st.sol, CUBLAS_FILL_MODE_LOWER, m, G, m, st.work.as<double>(), st.lwork,
                                   st.info.as<int>()));
        int info = 0;
        LB_CUDA(cudaMemcpyAsync(&info, st.info.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
        return info == 0;
    }
    // eigenvalues (ascending, into w) and eigenvectors (in place) of the symmetric m x m matrix G
    void eigh(double *G, int m) {
        LB_SOLVER(cusolverDnDsyevd(st.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, G, m,
                                   st.w.as<double>(), st.work.as<double>(), st.lwork, st.info.as<int>()));
        int info = 0;
        LB_CUDA(cudaMemcpyAsync(&info, st.info.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
        LB_CUDA(cudaStreamSynchronize(s));
        LB_CHECK(info == 0, LB_ERR_NUMERIC, "LOBPCG: the Rayleigh-Ritz eigensolver did not converge");
    }
    // B-orthonormalise the k columns of Y (B = Diag(s)) by the Cholesky factor of Y^T B Y; AY (if any) follows.
    bool b_orth(double *Y, double *AY) {
        double *sY = st.tmp.as<double>(), *G = st.gB.as<double>();
        k_lo_scale<<<nb256(n * k), 256, 0, s>>>(n, k, sv, Y, sY);
        LB_LAUNCH_CHECK();
        gram(Y, k, sY, k, G, true);
        if (!potrf(G, k)) return false;
        const double one = 1.0;
        LB_BLAS(cublasDtrsm(st.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                            (int)n, k, &one, G, k, Y, (int)n));
        if (AY)
            LB_BLAS(cublasDtrsm(st.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T,
                                CUBLAS_DIAG_NON_UNIT, (int)n, k, &one, G, k, AY, (int)n));
        return true;
    }
};

}  // namespace

// The LOBPCG iteration (estimator_gpu.lobpcg): X (row-major n x k, in and out), Ritz values into theta.
static void lobpcg_run(Problem &p, int k, double *Xrm, const double *g, const double *sv, const double *prec,
                       int maxiter, double *theta, int *iters_done, cudaStream_t s) {
    if (!p.lobpcg) p.lobpcg = new LobpcgState();
    LobpcgState &st = *p.lobpcg;
    const int64_t n = p.n;
    const int mmax = 3 * k;
    if (!st.blas) {
        st.device = p.ctx->c.device;
        {
            std::lock_guard<std::mutex> lock(g_handle_mu);
            auto &v = g_handles[st.device];
            if (!v.empty()) {
                st.blas = v.back().first;
                st.sol = v.back().second;
                v.pop_back();
            }
        }
        if (!st.blas) {
            LB_BLAS(cublasCreate(&st.blas));
            LB_SOLVER(cusolverDnCreate(&st.sol));
        }
    }
    LB_BLAS(cublasSetStream(st.blas, s));
    LB_SOLVER(cusolverDnSetStream(st.sol, s));
    for (int b = 0; b < 2; b++) {
        st.S[b].alloc(sizeof(double) * (size_t)n * mmax);
        st.AS[b].alloc(sizeof(double) * (size_t)n * mmax);
    }
    st.tmp.alloc(sizeof(double) * (size_t)n * mmax);
    st.opin.alloc(sizeof(double) * (size_t)n * p.r);
    st.opout.alloc(sizeof(double) * (size_t)n * p.r);
    LB_CUDA(cudaMemsetAsync(st.opin.ptr, 0, sizeof(double) * (size_t)n * p.r, s));   // padding columns stay zero
    for (DBuf *b : {&st.gA, &st.gB, &st.Linv, &st.T1, &st.Cc}) b->alloc(sizeof(double) * (size_t)mmax * mmax);
    st.w.alloc(sizeof(double) * mmax);
    st.info.alloc(sizeof(int));
    int lw1 = 0, lw2 = 0;
    LB_SOLVER(cusolverDnDpotrf_bufferSize(st.sol, CUBLAS_FILL_MODE_LOWER, mmax, st.gB.as<double>(), mmax, &lw1));
    LB_SOLVER(cusolverDnDsyevd_bufferSize(st.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, mmax,
                                          st.gA.as<double>(), mmax, st.w.as<double>(), &lw2));
    st.lwork = std::max({lw1, lw2, 1});
    st.work.alloc(sizeof(double) * (size_t)st.lwork);
    Run R{p, st, s, n, k, g, sv, prec};
    const double one = 1.0, zero = 0.0, mone = -1.0;
    const int ni = (int)n;
    int cur = 0;
    auto col = [&](DBuf &B, int j) { return B.as<double>() + (int64_t)j * k * n; };   // block j (0 X, 1 W, 2 P)
    double *X = col(st.S[cur], 0), *AX = col(st.AS[cur], 0);
    // X column-major, B-orthonormal; AX; Rayleigh-Ritz on span X
    LB_BLAS(cublasDgeam(st.blas, CUBLAS_OP_T, CUBLAS_OP_N, ni, k, &one, Xrm, k, &zero, X, ni, X, ni));
    LB_CHECK(R.b_orth(X, nullptr), LB_ERR_NUMERIC, "LOBPCG start block is rank deficient");
    R.mop(X, AX);
    double *gA = st.gA.as<double>(), *gB = st.gB.as<double>(), *Linv = st.Linv.as<double>();
    double *T1 = st.T1.as<double>(), *Cc = st.Cc.as<double>(), *tmp = st.tmp.as<double>();
    R.gram(X, k, AX, k, gA, true);
    R.eigh(gA, k);
    LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, k, &one, X, ni, gA, k, &zero, tmp, ni));
    LB_CUDA(cudaMemcpyAsync(X, tmp, sizeof(double) * (size_t)n * k, cudaMemcpyDeviceToDevice, s));
    LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, k, &one, AX, ni, gA, k, &zero, tmp, ni));
    LB_CUDA(cudaMemcpyAsync(AX, tmp, sizeof(double) * (size_t)n * k, cudaMemcpyDeviceToDevice, s));
    double *lam = st.w.as<double>();
    st.lam.alloc(sizeof(double) * k);
    LB_CUDA(cudaMemcpyAsync(st.lam.ptr, lam, sizeof(double) * k, cudaMemcpyDeviceToDevice, s));
    bool hasP = false;
    int it = 0;
    for (; it < maxiter; it++) {
        X = col(st.S[cur], 0);
        AX = col(st.AS[cur], 0);
        double *W = col(st.S[cur], 1), *AW = col(st.AS[cur], 1);
        // W = prec (AX - B X Lambda), B-orthogonalised against X, then B-orthonormalised
        k_lo_resid<<<nb256(n * k), 256, 0, s>>>(n, k, sv, prec, X, AX, st.lam.as<double>(), W);
        LB_LAUNCH_CHECK();
        k_lo_scale<<<nb256(n * k), 256, 0, s>>>(n, k, sv, W, tmp);
        LB_LAUNCH_CHECK();
        R.gram(X, k, tmp, k, T1, false);
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, k, &mone, X, ni, T1, k, &one, W, ni));
        if (!R.b_orth(W, nullptr)) break;
        R.mop(W, AW);
        int m = 2 * k;
        if (hasP && R.b_orth(col(st.S[cur], 2), col(st.AS[cur], 2))) m = 3 * k;
        // Rayleigh-Ritz on the m columns; a soft restart without P when the B-Gram matrix is not positive definite
        bool ok = false;
        for (int attempt = 0; attempt < 2 && !ok; attempt++) {
            double *S0 = col(st.S[cur], 0), *AS0 = col(st.AS[cur], 0);
            k_lo_scale<<<nb256(n * m), 256, 0, s>>>(n, m, sv, S0, tmp);
            LB_LAUNCH_CHECK();
            R.gram(S0, m, tmp, m, gB, true);
            R.gram(S0, m, AS0, m, gA, true);
            ok = R.potrf(gB, m);
            if (!ok) {
                if (m == 3 * k)
                    m = 2 * k;
                else
                    break;
            }
        }
        if (!ok) break;
        // Linv = L^-1; M = Linv gA Linv^T; eigenvectors Y of M; Cc = Linv^T Y[:, :k]
        k_lo_eye<<<nb256((int64_t)m * m), 256, 0, s>>>(m, Linv);
        LB_LAUNCH_CHECK();
        LB_BLAS(cublasDtrsm(st.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m, m,
                            &one, gB, m, Linv, m));
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, &one, Linv, m, gA, m, &zero, T1, m));
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_T, m, m, m, &one, T1, m, Linv, m, &zero, gA, m));
        R.eigh(gA, m);
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_T, CUBLAS_OP_N, m, k, m, &one, Linv, m, gA, m, &zero, Cc, m));
        LB_CUDA(cudaMemcpyAsync(st.lam.ptr, lam, sizeof(double) * k, cudaMemcpyDeviceToDevice, s));
        // next [X, -, P] and [AX, -, AP]
        const int nx = cur ^ 1;
        double *S0 = col(st.S[cur], 0), *AS0 = col(st.AS[cur], 0);
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, m, &one, S0, ni, Cc, m, &zero,
                            col(st.S[nx], 0), ni));
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, m, &one, AS0, ni, Cc, m, &zero,
                            col(st.AS[nx], 0), ni));
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, m - k, &one, col(st.S[cur], 1), ni, Cc + k, m,
                            &zero, col(st.S[nx], 2), ni));
        LB_BLAS(cublasDgemm(st.blas, CUBLAS_OP_N, CUBLAS_OP_N, ni, k, m - k, &one, col(st.AS[cur], 1), ni, Cc + k, m,
                            &zero, col(st.AS[nx], 2), ni));
        cur = nx;
        hasP = true;
    }
    X = col(st.S[cur], 0);
    LB_BLAS(cublasDgeam(st.blas, CUBLAS_OP_T, CUBLAS_OP_N, k, ni, &one, X, ni, &zero, Xrm, k, Xrm, k));
    if (theta) LB_CUDA(cudaMemcpyAsync(theta, st.lam.ptr, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
    LB_CUDA(cudaStreamSynchronize(s));
    if (iters_done) *iters_done = it;
}

}  // namespace lb

using namespace lb;

template <typename F> static int lo_guard(F &&f) {
    struct Clear {
        ~Clear() { alloc_stream() = nullptr; }
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

int lb_lobpcg(lb_problem *h, int32_t k, double *X, const double *g, const double *s, const double *prec,
              int32_t maxiter, double *theta, int32_t *iters_done) {
    return lo_guard([&] {
        LB_CHECK(h && X && g && s && prec, LB_ERR_INVALID, "null argument");
        Problem &p = h->p;
        LB_CHECK(p.vdtype == LB_F64, LB_ERR_INVALID, "LOBPCG needs an FP64 problem");
        LB_CHECK(k >= 1 && k <= p.r && maxiter >= 0, LB_ERR_INVALID, "need 1 <= k <= r and maxiter >= 0");
        LB_CHECK(p.n >= 3 * (int64_t)k && p.n < ((int64_t)1 << 31), LB_ERR_INVALID, "need 3 k <= n < 2^31");
        LB_CHECK(p.ngraphs == 0, LB_ERR_INVALID, "not for batched problems");
        for (const void *q : {(const void *)X, (const void *)g, (const void *)s, (const void *)prec}) {
            cudaPointerAttributes at{};
            LB_CUDA(cudaPointerGetAttributes(&at, q));
            LB_CHECK(at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged, LB_ERR_INVALID,
                     "X, g, s and prec must be device memory");
        }
        LB_CUDA(cudaSetDevice(p.ctx->c.device));
        alloc_stream() = p.ctx->c.stream;
        lobpcg_run(p, k, X, g, s, prec, maxiter, theta, iters_done, p.ctx->c.stream);
    });
}
