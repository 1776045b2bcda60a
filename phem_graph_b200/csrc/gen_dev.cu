// gen_dev.cu -- the R-MAT draw stream of gen.cpp, generated on the GPU.
//
// phem_gen_rmat_range_device produces exactly what phem_gen_rmat_range (the
// host generator in gen.cpp) produces for the same arguments: draws
// [first, first + count) of the counter-based R-MAT stream, self-loops dropped,
// draw order kept, packed (lo << 32 | hi).  Every value is a pure function of
// (seed, draw index): SplitMix64 at a counter (Steele, Lea, Flood, OOPSLA 2014)
// and integer quadrant thresholds, so no state crosses threads.  It exists so
// that a graph too large to generate on the host in reasonable time (R-MAT
// scale 28, 8.6 G pairs) can be produced batch by batch on the device and
// copied out.  Input generation only: no solver path calls it.
#include <algorithm>
#include <cmath>

#include "internal.h"

namespace phem {
namespace {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kTagRMAT = 0x524D41542D4544ull;  // "RMAT-ED", the tag gen.cpp uses
constexpr int kGenThreads = 256;
constexpr int kGenPerThread = 16;  // contiguous draws per thread
constexpr uint32_t kGenTile = kGenThreads * kGenPerThread;

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct RmatParams {
    uint32_t scale, words;
    uint64_t base, tA, tAB, tABC;
};

// Draw i: `scale` quadrant choices, two per 64-bit stream value.
__device__ __forceinline__ bool rmat_draw(const RmatParams &p, uint64_t i, uint64_t *packed)
{
    uint32_t u = 0, v = 0;
    for (uint32_t l = 0; l < p.scale; l++) {
        const uint64_t word = mix64(p.base + (i * p.words + l / 2 + 1) * kGamma);
        const uint64_t r = (l & 1) ? (word >> 32) : (word & 0xffffffffu);
        const uint32_t ubit = r >= p.tAB;
        const uint32_t vbit = (r >= p.tA && r < p.tAB) || r >= p.tABC;
        u = (u << 1) | ubit;
        v = (v << 1) | vbit;
    }
    if (u == v)
        return false;
    *packed = ((uint64_t)min(u, v) << 32) | max(u, v);
    return true;
}

// One tile of kGenTile draws per block iteration (tiles taken by ticket, so a
// tile's predecessors are always owned by running blocks); survivors are
// placed by a block scan plus a decoupled look-back over the tiles, staged in
// shared memory and written coalesced.
__global__ void __launch_bounds__(kGenThreads) rmat_range_kernel(RmatParams p, uint64_t first, uint64_t count,
                                                                 unsigned long long *out, uint64_t *status,
                                                                 uint32_t epoch, Ctl *ctl)
{
    __shared__ unsigned long long s_out[kGenTile];
    __shared__ uint32_t s_warp[kWarps + 1];
    __shared__ uint32_t s_tile, s_base;
    const uint64_t ntiles = (count + kGenTile - 1) / kGenTile;
    for (;;) {
        if (threadIdx.x == 0)
            s_tile = atomicAdd(&ctl->ticket[0], 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles)
            break;
        const uint64_t d0 = (uint64_t)t * kGenTile + (uint64_t)threadIdx.x * kGenPerThread;
        uint64_t vals[kGenPerThread];
        uint32_t keep = 0, c = 0;
#pragma unroll
        for (int j = 0; j < kGenPerThread; j++) {
            vals[j] = 0;
            if (d0 + j < count && rmat_draw(p, first + d0 + j, &vals[j])) {
                keep |= 1u << j;
                c++;
            }
        }
        uint32_t total;
        uint32_t off = block_exclusive_scan(c, &total, s_warp);
        if (threadIdx.x < 32) {
            const uint32_t ex = lookback_exclusive(status, t, total, epoch, &ctl->err);
            if (threadIdx.x == 0) {
                s_base = ex;
                if (t == ntiles - 1)
                    ctl->misc[4] = (unsigned long long)ex + total;
            }
        }
#pragma unroll
        for (int j = 0; j < kGenPerThread; j++)
            if (keep & (1u << j))
                s_out[off++] = vals[j];
        __syncthreads();
        const uint32_t base = s_base;
        for (uint32_t i = threadIdx.x; i < total; i += kGenThreads)
            out[(uint64_t)base + i] = s_out[i];
        __syncthreads();  // s_out, s_tile and s_base are reused
    }
}

}  // namespace
}  // namespace phem

using namespace phem;

extern "C" phem_status phem_gen_rmat_range_device(phem_context *ctx, uint32_t scale, uint64_t first, uint64_t count,
                                                  double a, double b, double c, uint64_t seed, uint64_t *d_out,
                                                  uint64_t *out_m)
{
    PHEM_TRY(check_ctx(ctx));
    if (scale < 1 || scale > 31 || !out_m || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 ||
        (count > 0 && !d_out) || count >= (1ull << 40)) {
        set_error("gen_rmat_range_device: need 1 <= scale <= 31, a, b, c >= 0 with a + b + c <= 1, "
                  "count < 2^40, device output and out_m");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    if (count > 0 && !is_device_ptr_on(d_out, ctx->device)) {
        set_error("gen_rmat_range_device: the output must be device memory of the context's device %d",
                  ctx->device);
        return PHEM_ERR_INVALID;
    }
    *out_m = 0;
    if (count == 0)
        return PHEM_OK;
    // the same thresholds and stream base as gen.cpp's RmatDraw
    const double two32 = 4294967296.0;
    RmatParams p;
    p.scale = scale;
    p.words = (scale + 1) / 2;
    p.base = mix64(seed * kGamma + kTagRMAT);
    p.tA = (uint64_t)std::floor(a * two32);
    p.tAB = (uint64_t)std::floor((a + b) * two32);
    p.tABC = (uint64_t)std::floor((a + b + c) * two32);
    const uint64_t tiles = (count + kGenTile - 1) / kGenTile;
    if (tiles >= (1ull << 32)) {
        set_error("gen_rmat_range_device: too many draws for one call");
        return PHEM_ERR_INVALID;
    }
    PHEM_TRY(status_reserve(ctx, tiles + 2));
    const uint32_t epoch = (uint32_t)next_epochs(ctx, 1);
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), ctx->stream));
    int per_sm = 0;
    PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rmat_range_kernel, kGenThreads, 0));
    const uint64_t grid = std::min<uint64_t>(tiles, (uint64_t)ctx->sm_count * std::max(1, per_sm));
    rmat_range_kernel<<<(unsigned)grid, kGenThreads, 0, ctx->stream>>>(
        p, first, count, reinterpret_cast<unsigned long long *>(d_out), ctx->status, epoch, ctx->ctl);
    PHEM_CUDA_TRY(cudaGetLastError());
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(ctl_status(ctx->h_ctl->err, "gen_rmat_range_device"));
    *out_m = ctx->h_ctl->misc[4];
    return PHEM_OK;
}
