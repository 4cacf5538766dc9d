// Random row-gather probe: how fast this device serves gathers of whole table rows picked uniformly at random from a
// footprint of a given size, the access pattern of the row kernel's neighbour gathers.  Each lane group of 4 (64-byte
// rows) or 8 (128-byte rows) lanes reads one row per step, 16 bytes a lane, eight rows in flight per lane; the row
// indices come from a hash of the gather's number (SplitMix64's finaliser, Steele, Lea and Flood 2014), so nothing
// but the table goes through the caches.  The measured rate, set against the footprint, is the ceiling a row-gather
// kernel meets on this part (the gathers stay in L2 only while the footprint is a fraction of it).
#include "lb_internal.cuh"

namespace lb {
namespace {

__device__ __forceinline__ uint32_t probe_hash(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return (uint32_t)x;
}

template <int LPR>
__global__ void __launch_bounds__(256) k_gather_probe(const uint4 *__restrict__ table, int64_t ngather, uint32_t frows,
                                                      uint32_t seed, float *__restrict__ out) {
    constexpr int RPW = 32 / LPR;   // rows per warp step
    const int lane = threadIdx.x & 31, g = lane / LPR, c = lane % LPR;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int64_t nw = (int64_t)gridDim.x * blockDim.x / 32;
    float acc = 0.f;
    for (int64_t s = gw * RPW; s < ngather; s += nw * RPW * 8) {
        uint4 r[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            const int64_t t = s + (int64_t)u * nw * RPW + g;
            const uint32_t j = probe_hash((uint64_t)t * 0x9e3779b97f4a7c15ull + seed) % frows;
            r[u] = t < ngather ? __ldg(table + (int64_t)j * LPR + c) : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) acc += __uint_as_float(r[u].x & 0xffff0000u) + __uint_as_float(r[u].w << 16);
    }
    out[(int64_t)blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

}  // namespace
}  // namespace lb

using namespace lb;

int lb_gather_probe(lb_ctx *ctx, int64_t footprint_bytes, int32_t row_bytes, int64_t ngather, int32_t reps,
                    float *ms_per_launch) {
    try {
        LB_CHECK(ctx && ms_per_launch, LB_ERR_INVALID, "null argument");
        LB_CHECK(row_bytes == 64 || row_bytes == 128, LB_ERR_INVALID, "row_bytes must be 64 or 128");
        LB_CHECK(footprint_bytes >= row_bytes && footprint_bytes <= ((int64_t)4 << 30), LB_ERR_INVALID,
                 "footprint must be between one row and 4 GiB");
        LB_CHECK(ngather >= 1 && reps >= 1, LB_ERR_INVALID, "need ngather >= 1 and reps >= 1");
        LB_CUDA(cudaSetDevice(ctx->c.device));
        cudaStream_t s = ctx->c.stream;
        const uint32_t frows = (uint32_t)(footprint_bytes / row_bytes);
        DBuf table, out;
        table.alloc((size_t)frows * row_bytes);
        LB_CUDA(cudaMemsetAsync(table.ptr, 0x3f, table.bytes, s));
        const unsigned grid = (unsigned)ctx->c.num_sms * 8;
        out.alloc(sizeof(float) * (size_t)grid * 256);
        auto launch = [&](uint32_t seed) {
            if (row_bytes == 64)
                k_gather_probe<4><<<grid, 256, 0, s>>>(table.as<uint4>(), ngather, frows, seed, out.as<float>());
            else
                k_gather_probe<8><<<grid, 256, 0, s>>>(table.as<uint4>(), ngather, frows, seed, out.as<float>());
            LB_LAUNCH_CHECK();
        };
        launch(1);
        launch(2);
        LB_CUDA(cudaEventRecord(ctx->c.t0, s));
        for (int32_t k = 0; k < reps; k++) launch(3 + (uint32_t)k);
        LB_CUDA(cudaEventRecord(ctx->c.t1, s));
        LB_CUDA(cudaEventSynchronize(ctx->c.t1));
        float ms = 0.f;
        LB_CUDA(cudaEventElapsedTime(&ms, ctx->c.t0, ctx->c.t1));
        *ms_per_launch = ms / reps;
        LB_CUDA(cudaStreamSynchronize(s));
        return LB_OK;
    } catch (const Err &e) {
        return e.code;
    } catch (...) {
        set_error("unexpected exception");
        return LB_ERR_INVALID;
    }
}
