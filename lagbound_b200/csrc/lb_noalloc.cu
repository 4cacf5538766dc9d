// lb_bv_noalloc: the degree-corrected SpMM G = A V - d (d^T V) / L with quadA, |d^T V|^2 and the primal value, for
// callers that cannot allocate device memory.  All inputs and outputs are the caller's device buffers; the only
// scratch is the fixed file-scope array below.  The regular entry points (lb_eval, ...) allocate their scratch
// through cudaMalloc and are not used here.
//
// Why some callers can't allocate: a host that owns every device byte through its own pool (a serving loop that
// admits requests against an HBM budget, or a runtime such as PyTorch's caching allocator or a JVM/Go host that
// accounts for all device memory) cannot let a library call cudaMalloc behind its back: the call synchronises the
// device and the memory escapes the pool's accounting, so the admission budget would be wrong.
#include <math.h>

#include <algorithm>
#include <mutex>
#include <type_traits>

#include "lb_internal.cuh"

namespace lb {

// Fixed scratch: per-block partial sums of d^T V (MAX_BLOCKS x MAX_LD), per-block quadA partials, invalid-index
// counts and clamped-row counts (MAX_BLOCKS each), and the reduced d^T V (MAX_LD).  541 KB; every GPU that loads the
// library holds it until the process exits.
constexpr int NOALLOC_MAX_BLOCKS = 1024;
constexpr int NOALLOC_MAX_LD = 64;
constexpr size_t NOALLOC_OFF_Q = (size_t)NOALLOC_MAX_BLOCKS * NOALLOC_MAX_LD;
constexpr size_t NOALLOC_OFF_BAD = NOALLOC_OFF_Q + NOALLOC_MAX_BLOCKS;
constexpr size_t NOALLOC_OFF_CLAMP = NOALLOC_OFF_BAD + NOALLOC_MAX_BLOCKS;
constexpr size_t NOALLOC_OFF_Z = NOALLOC_OFF_CLAMP + NOALLOC_MAX_BLOCKS;
constexpr size_t NOALLOC_DOUBLES = NOALLOC_OFF_Z + NOALLOC_MAX_LD;
static __device__ __align__(256) double lb_noalloc_scratch[NOALLOC_DOUBLES];

namespace {

constexpr unsigned FULLM = 0xffffffffu;

// d^T V partials: block b sums rows [b*chunk, min(n, (b+1)*chunk)) in a fixed order; every slot (b, c < ld) written.
template <typename T, int NCH>
__global__ void __launch_bounds__(256) k_na_z(int64_t n, int ld, int64_t chunk, const T *__restrict__ V,
                                              const double *__restrict__ d, double *__restrict__ scratch) {
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    __shared__ double sh[8][NOALLOC_MAX_LD];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, sub = lane / NCH, ch = lane % NCH;
    const int64_t a = (int64_t)blockIdx.x * chunk, b = min(n, a + chunk);
    double acc[EPL];
#pragma unroll
    for (int k = 0; k < EPL; k++) acc[k] = 0.0;
    for (int64_t i = a + w * NPW + sub; i < b; i += 8 * NPW) {
        double x[EPL];
        load_d<T>(V + i * ld + ch * EPL, x);
        const double di = d[i];
#pragma unroll
        for (int k = 0; k < EPL; k++) acc[k] += di * x[k];
    }
#pragma unroll
    for (int off = NCH; off < 32; off <<= 1)
#pragma unroll
        for (int k = 0; k < EPL; k++) acc[k] += __shfl_xor_sync(FULLM, acc[k], off);
    if (sub == 0)
#pragma unroll
        for (int k = 0; k < EPL; k++) sh[w][ch * EPL + k] = acc[k];
    __syncthreads();
    for (int c = threadIdx.x; c < ld; c += blockDim.x) {
        double s = 0.0;
        for (int k = 0; k < 8; k++) s += sh[k][c];
        scratch[(size_t)blockIdx.x * NOALLOC_MAX_LD + c] = s;
    }
}

__global__ void k_na_zfin(int nb, int ld, double *__restrict__ scratch) {
    for (int c = threadIdx.x; c < ld; c += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nb; b++) s += scratch[(size_t)b * NOALLOC_MAX_LD + c];
        scratch[NOALLOC_OFF_Z + c] = s;
    }
}

// Warp per row (grid-stride over a fixed grid): G_i = (A V)_i - (d_i / L) z, quadA partial v_i.(A V)_i.
// Column indices outside [0, n) are skipped and counted (reported in out[3]).  A row's edge range
// [indptr[i], indptr[i+1]) is clamped to [0, nnz] (an empty range when it decreases); rows whose range had to be
// changed are counted (out[4]), so a malformed indptr never reads past the caller's indices and weights.
template <typename T, int NCH, typename TG>
__global__ void __launch_bounds__(256) k_na_rows(int64_t n, int64_t nnz, int ld, const int64_t *__restrict__ indptr,
                                                 const int *__restrict__ indices, const float *__restrict__ w,
                                                 const T *__restrict__ V, const double *__restrict__ d, double invL,
                                                 TG *__restrict__ G, double *__restrict__ scratch) {
    using Acc = typename VT<T>::Acc;
    constexpr int EPL = VT<T>::EPL, NPW = 32 / NCH;
    __shared__ double shq[8], shb[8], shc[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, sub = lane / NCH, ch = lane % NCH;
    const double *z = scratch + NOALLOC_OFF_Z;
    double quad = 0.0, bad = 0.0, clamped = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * 8 + wid; i < n; i += (int64_t)gridDim.x * 8) {
        Acc acc[EPL];
#pragma unroll
        for (int k = 0; k < EPL; k++) acc[k] = 0;
        const int64_t r0 = indptr[i], r1 = indptr[i + 1];
        const int64_t e0 = min(max(r0, (int64_t)0), nnz), e1 = max(min(r1, nnz), e0);
        if (lane == 0 && (e0 != r0 || e1 != r1)) clamped += 1.0;
        for (int64_t e = e0 + sub; e < e1; e += NPW) {
            const int j = indices[e];
            if ((unsigned)j >= (unsigned)n) {
                if (ch == 0) bad += 1.0;
                continue;
            }
            Acc x[EPL];
            VT<T>::load(V + (int64_t)j * ld + ch * EPL, x);
            const Acc wt = w ? (Acc)w[e] : (Acc)1;
#pragma unroll
            for (int k = 0; k < EPL; k++) acc[k] += wt * x[k];
        }
#pragma unroll
        for (int off = NCH; off < 32; off <<= 1)
#pragma unroll
            for (int k = 0; k < EPL; k++) acc[k] += __shfl_xor_sync(FULLM, acc[k], off);
        Acc vi[EPL];
        VT<T>::load(V + i * ld + ch * EPL, vi);
        double q = 0.0;
#pragma unroll
        for (int k = 0; k < EPL; k++) q += (double)vi[k] * (double)acc[k];
#pragma unroll
        for (int off = 1; off < NCH; off <<= 1) q += __shfl_xor_sync(FULLM, q, off);
        if (lane == 0) quad += q;
        if (sub == 0) {
            const double dl = d[i] * invL;
            TG g[EPL];
#pragma unroll
            for (int k = 0; k < EPL; k++) g[k] = (TG)((Acc)acc[k] - (Acc)(dl * z[ch * EPL + k]));
            Store<TG>::st(G + i * ld + ch * EPL, g, EPL);
        }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) bad += __shfl_xor_sync(FULLM, bad, off);
    if (lane == 0) {
        shq[wid] = quad;
        shb[wid] = bad;
        shc[wid] = clamped;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0, sb = 0.0, sc = 0.0;
        for (int k = 0; k < 8; k++) {
            s += shq[k];
            sb += shb[k];
            sc += shc[k];
        }
        scratch[NOALLOC_OFF_Q + blockIdx.x] = s;
        scratch[NOALLOC_OFF_BAD + blockIdx.x] = sb;
        scratch[NOALLOC_OFF_CLAMP + blockIdx.x] = sc;
    }
}

__global__ void k_na_fin(int nb, int ld, double L, double C0, const double *__restrict__ scratch,
                         double *__restrict__ out) {
    if (threadIdx.x != 0) return;
    double q = 0.0, bad = 0.0, clamped = 0.0, zz = 0.0;
    for (int b = 0; b < nb; b++) {
        q += scratch[NOALLOC_OFF_Q + b];
        bad += scratch[NOALLOC_OFF_BAD + b];
        clamped += scratch[NOALLOC_OFF_CLAMP + b];
    }
    for (int c = 0; c < ld; c++) zz += scratch[NOALLOC_OFF_Z + c] * scratch[NOALLOC_OFF_Z + c];
    out[0] = q;
    out[1] = zz;
    out[2] = q - zz / L + C0;
    out[3] = bad;
    out[4] = clamped;
}

// Device address of the scratch array, resolved once per device (with that device current) and kept for the life of
// the process: the address belongs to the device's primary context, so the library must not be used again after
// that context is destroyed (cudaDeviceReset) in the same process.
std::mutex g_mu;
double *g_addr[64] = {nullptr};

double *scratch_address(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, lb_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(std::string("cudaGetSymbolAddress(lb_noalloc_scratch): ") + cudaGetErrorString(e));
            throw Err{LB_ERR_CUDA};
        }
        g_addr[dev] = (double *)p;
    }
    return g_addr[dev];
}

template <typename T, int NCH>
void run(int64_t n, int64_t nnz, const int64_t *indptr, const int32_t *indices, const float *w, const double *d, double L,
         double C0, const void *V, int32_t ld, void *G, double *out, cudaStream_t s, double *scratch) {
    using TG = typename std::conditional<std::is_same<T, double>::value, double, float>::type;
    const int64_t want = (n + 7) / 8;
    const int nb = (int)std::min<int64_t>(want, NOALLOC_MAX_BLOCKS);
    const int64_t chunk = (n + nb - 1) / nb;
    k_na_z<T, NCH><<<nb, 256, 0, s>>>(n, ld, chunk, (const T *)V, d, scratch);
    LB_LAUNCH_CHECK();
    k_na_zfin<<<1, 64, 0, s>>>(nb, ld, scratch);
    LB_LAUNCH_CHECK();
    k_na_rows<T, NCH, TG><<<nb, 256, 0, s>>>(n, nnz, ld, indptr, indices, w, (const T *)V, d, 1.0 / L, (TG *)G, scratch);
    LB_LAUNCH_CHECK();
    k_na_fin<<<1, 32, 0, s>>>(nb, ld, L, C0, scratch, out);
    LB_LAUNCH_CHECK();
}

}  // namespace
}  // namespace lb

using namespace lb;

extern "C" int lb_bv_noalloc(int64_t n, int64_t nnz, const int64_t *indptr, const int32_t *indices,
                             const float *weights, const double *d, double L, double C0, const void *V, lb_dtype dtype,
                             int32_t ld, void *G, double *out, void *stream) {
    try {
        LB_CHECK(indptr && indices && d && V && G && out, LB_ERR_INVALID, "lb_bv_noalloc: null device pointer");
        LB_CHECK(n >= 1 && n < ((int64_t)1 << 31), LB_ERR_INVALID, "lb_bv_noalloc: n must be in [1, 2^31)");
        LB_CHECK(nnz >= 0, LB_ERR_INVALID, "lb_bv_noalloc: nnz must be non-negative");
        // the kernels read V and write G in 16-byte vectors, the FP64/int64 arrays in 8-byte words: a misaligned
        // pointer (e.g. a view at an odd offset) is refused here, before anything is launched
        auto aligned = [](const void *q, uintptr_t a) { return ((uintptr_t)q & (a - 1)) == 0; };
        LB_CHECK(aligned(V, 16) && aligned(G, 16), LB_ERR_INVALID,
                 "lb_bv_noalloc: V and G must be 16-byte aligned device pointers");
        LB_CHECK(aligned(indptr, 8) && aligned(d, 8) && aligned(out, 8) && aligned(indices, 4) &&
                     aligned(weights, 4),
                 LB_ERR_INVALID, "lb_bv_noalloc: indptr, d and out must be 8-byte aligned, indices and weights 4-byte");
        LB_CHECK(L > 0 && isfinite(L) && isfinite(C0), LB_ERR_INVALID, "lb_bv_noalloc: L must be positive and finite");
        LB_CHECK(dtype == LB_F64 || dtype == LB_F32 || dtype == LB_BF16, LB_ERR_INVALID, "lb_bv_noalloc: unknown dtype");
        const int esz = (int)dtype_size(dtype);
        const int bytes = ld * esz;
        LB_CHECK(ld >= 1 && ld <= NOALLOC_MAX_LD && bytes >= 16 && (bytes & (bytes - 1)) == 0, LB_ERR_INVALID,
                 "lb_bv_noalloc: ld must be at most 64 elements and make a row a power-of-two multiple of 16 bytes "
                 "(the scratch holds 1024 x 64 partial sums)");
        int dev = 0;
        LB_CUDA(cudaGetDevice(&dev));
        LB_CHECK(dev >= 0 && dev < 64, LB_ERR_INVALID, "lb_bv_noalloc: device ordinal above 63");
        double *scratch = scratch_address(dev);
        cudaStream_t s = (cudaStream_t)stream;
        const int nch = bytes / 16;
        switch (dtype) {
        case LB_F64:
            switch (nch) {
            case 1: run<double, 1>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 2: run<double, 2>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 4: run<double, 4>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 8: run<double, 8>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 16: run<double, 16>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 32: run<double, 32>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            }
            break;
        case LB_F32:
            switch (nch) {
            case 1: run<float, 1>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 2: run<float, 2>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 4: run<float, 4>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 8: run<float, 8>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 16: run<float, 16>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            }
            break;
        default:
            switch (nch) {
            case 1: run<__nv_bfloat16, 1>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 2: run<__nv_bfloat16, 2>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 4: run<__nv_bfloat16, 4>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            case 8: run<__nv_bfloat16, 8>(n, nnz, indptr, indices, weights, d, L, C0, V, ld, G, out, s, scratch); break;
            }
        }
        return LB_OK;
    } catch (const Err &e) {
        return e.code;
    } catch (...) {
        set_error("lb_bv_noalloc: unexpected exception");
        return LB_ERR_INVALID;
    }
}
