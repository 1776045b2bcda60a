// cc.cu -- union-find connected components + spanning forest on sm_100a.
//
// Arithmetic follows the reference GPU kernels (CC/ExternalSpanningTree.cu:27-116,
// CC/GPUSpanningTree.cu:24-140): for every packed edge (u << 32 | v) with u < v
// the two roots are found, the larger root is hooked under the smaller with a
// CAS, and the forest slot of the hooked root records the edge; afterwards
// label[i] = root(i), which is the smallest id of i's component because hooks
// always point to smaller ids.
//
// Differences that are B200 choices, not semantics:
//   * edges are read four at a time with 128-bit streaming loads
//     (evict-first), so the 8 B/edge stream does not push the parent array
//     out of L2;
//   * a union first compares the endpoints' parents (two loads settle most
//     edges once trees are flat), then walks both roots in lockstep so the
//     two walks' loads overlap, stopping early where the walks meet; the
//     first walk reads through L1, a walk after a failed CAS through L2,
//     continuing from the parent the CAS returned;
//   * path halving writes are atomic mins: ids fall towards the root, so a
//     walk working from a stale parent never undoes another walk's shortcut;
//   * phem_cc_solve unites a prefix of about one edge per vertex, points
//     every vertex at its root, then unites the rest (cc.sample_per_vertex);
//   * every loop is bounded; a bound that trips sets a status bit instead of
//     hanging the GPU.
#include <algorithm>

#include "internal.h"
#include "uf.cuh"

namespace phem {
namespace {

__global__ void __launch_bounds__(kBlock) cc_init_kernel(int32_t n, int32_t *parent, int32_t *label,
                                                         unsigned long long *forest)
{
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        parent[i] = i;
        if (label)
            label[i] = i;
        if (forest)
            forest[i] = kForestEmpty;
    }
}

__global__ void __launch_bounds__(kBlock) cc_unite_kernel(const unsigned long long *edges, int64_t m, int32_t n,
                                                          int32_t *parent, unsigned long long *forest,
                                                          uint32_t *err)
{
    const int64_t groups = m / 2;  // uint4 = two packed edges
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const uint4 *q = reinterpret_cast<const uint4 *>(edges);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < groups; g += stride) {
        const uint4 a = __ldcs(q + g);
        unite_packed(parent, forest, ((unsigned long long)a.y << 32) | a.x, n, err);
        unite_packed(parent, forest, ((unsigned long long)a.w << 32) | a.z, n, err);
    }
    if ((m & 1) && blockIdx.x == 0 && threadIdx.x == 0)
        unite_packed(parent, forest, __ldcs(edges + m - 1), n, err);
}

// gpu_spanning_tree's candidate pass (CC/GPUSpanningTree.cu:74-96): slots
// [0, n) of fa then [0, n) of fb; empty slots and u >= v are skipped.
__global__ void __launch_bounds__(kBlock) cc_merge_kernel(const unsigned long long *fa,
                                                          const unsigned long long *fb, int32_t n,
                                                          int32_t *parent, unsigned long long *forest,
                                                          uint32_t *err)
{
    const int64_t total = fb ? 2 * (int64_t)n : (int64_t)n;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        const unsigned long long e = i < n ? __ldcs(fa + i) : __ldcs(fb + (i - n));
        if (e == kForestEmpty)
            continue;
        unite_packed(parent, forest, e, n, err);
    }
}

// label[i] = root(i); the path of i is compressed to the root (cc,
// CC/GPUSpanningTree.cu:122-128 with compress at :24-40).
__global__ void __launch_bounds__(kBlock) cc_label_kernel(int32_t n, int32_t *parent, int32_t *label,
                                                          uint32_t *err)
{
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int32_t r = uf_find<true>(parent, i, n, err);
        label[i] = r;
        if (parent[i] != r)
            parent[i] = r;
    }
}

// parent[i] = root(i) for every vertex (no labels): after it every later
// union's first two loads already compare roots.  Here and in the label pass
// the walks read through L1: no union runs, so roots are final, L1 starts
// each launch without lines of earlier launches, and a value that misses a
// concurrent halving write is still an ancestor.
__global__ void __launch_bounds__(kBlock) cc_compress_kernel(int32_t n, int32_t *parent, uint32_t *err)
{
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int32_t r = uf_find<true>(parent, i, n, err);
        if (parent[i] != r)
            parent[i] = r;
    }
}

__device__ __forceinline__ uint32_t plain_root(const uint32_t *parent, uint32_t x, uint32_t n, uint32_t *err)
{
    for (uint32_t steps = 0; steps <= n; steps++) {
        const uint32_t p = parent[x];
        if (p == x)
            return x;
        x = p;
    }
    set_err(err, kErrChase);
    return x;
}

__global__ void __launch_bounds__(kBlock) minid_scatter_kernel(int32_t n, const uint32_t *parent, uint32_t *minid,
                                                               uint32_t *err)
{
    // Lanes of a warp hold consecutive vertices, so among the lanes that share
    // a root the lowest lane has the smallest id: only it reads the guard
    // (through L1: a stale value is never below the true minimum) and
    // offers.  A giant component's vertices no longer all hit one word.
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += stride) {
        const int32_t i = i0 + (int32_t)threadIdx.x;
        const bool in = i < n;
        const uint32_t r = in ? plain_root(parent, (uint32_t)i, (uint32_t)n, err) : 0xffffffffu;
        const unsigned peers = __match_any_sync(0xffffffffu, r);
        if (in && (int)lane_id() == __ffs(peers) - 1 && (uint32_t)i < __ldca(minid + r))
            atomicMin(minid + r, (uint32_t)i);
    }
}

__global__ void __launch_bounds__(kBlock) minid_label_kernel(int32_t n, const uint32_t *parent,
                                                             const uint32_t *minid, int32_t *label, uint32_t *err)
{
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        label[i] = (int32_t)minid[plain_root(parent, (uint32_t)i, (uint32_t)n, err)];
}

// Counts roots (label[i] == i) and filled forest slots into ctl->misc[0..1].
__global__ void __launch_bounds__(kBlock) cc_count_kernel(int32_t n, const int32_t *label,
                                                          const unsigned long long *forest, Ctl *ctl)
{
    // per-thread counts, then one atomic per warp and counter: every warp
    // adding to the same two words once per 32 vertices serialised on them
    __shared__ unsigned long long s_cnt[2];
    if (threadIdx.x < 2)
        s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int32_t stride = gridDim.x * blockDim.x;
    uint32_t roots = 0, slots = 0;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        roots += label[i] == i;
        slots += forest && forest[i] != kForestEmpty;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        roots += __shfl_xor_sync(0xffffffffu, roots, d);
        slots += __shfl_xor_sync(0xffffffffu, slots, d);
    }
    if (lane_id() == 0) {
        if (roots)
            atomicAdd(&s_cnt[0], (unsigned long long)roots);
        if (slots)
            atomicAdd(&s_cnt[1], (unsigned long long)slots);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_cnt[0])
            atomicAdd(&ctl->misc[0], s_cnt[0]);
        if (s_cnt[1])
            atomicAdd(&ctl->misc[1], s_cnt[1]);
    }
}

int grid_for(phem_context *ctx, int64_t work, int per_sm)
{
    int64_t b = (work + kBlock - 1) / kBlock;
    int64_t cap = (int64_t)ctx->sm_count * per_sm;
    return (int)std::max<int64_t>(1, std::min(b, cap));
}

}  // namespace

phem_status cc_launch_init(phem_context *ctx, int32_t n, int32_t *parent, int32_t *label, uint64_t *forest)
{
    KernelScope k(ctx, kKCcInit);
    cc_init_kernel<<<grid_for(ctx, n, 8), kBlock, 0, ctx->stream>>>(n, parent, label,
                                                                    reinterpret_cast<unsigned long long *>(forest));
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status cc_launch_unite(phem_context *ctx, const uint64_t *edges, int64_t m, int32_t n, int32_t *parent,
                            uint64_t *forest)
{
    if (m <= 0)
        return PHEM_OK;
    KernelScope k(ctx, kKCcUnite);
    cc_unite_kernel<<<grid_for(ctx, (m + 1) / 2, 8), kBlock, 0, ctx->stream>>>(
        reinterpret_cast<const unsigned long long *>(edges), m, n, parent,
        reinterpret_cast<unsigned long long *>(forest), &ctx->ctl->err);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status cc_launch_compress(phem_context *ctx, int32_t n, int32_t *parent)
{
    KernelScope k(ctx, kKCcLabel);
    cc_compress_kernel<<<grid_for(ctx, n, 8), kBlock, 0, ctx->stream>>>(n, parent, &ctx->ctl->err);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status cc_launch_label(phem_context *ctx, int32_t n, int32_t *parent, int32_t *label)
{
    KernelScope k(ctx, kKCcLabel);
    cc_label_kernel<<<grid_for(ctx, n, 8), kBlock, 0, ctx->stream>>>(n, parent, label, &ctx->ctl->err);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status cc_launch_merge(phem_context *ctx, const uint64_t *fa, const uint64_t *fb, int32_t n, int32_t *parent,
                            uint64_t *forest_out)
{
    KernelScope k(ctx, kKCcMerge);
    cc_merge_kernel<<<grid_for(ctx, fb ? 2 * (int64_t)n : n, 8), kBlock, 0, ctx->stream>>>(
        reinterpret_cast<const unsigned long long *>(fa), reinterpret_cast<const unsigned long long *>(fb), n,
        parent, reinterpret_cast<unsigned long long *>(forest_out), &ctx->ctl->err);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status cc_launch_minid_labels(phem_context *ctx, int32_t n, uint32_t *parent, uint32_t *minid, int32_t *label)
{
    PHEM_CUDA_TRY(cudaMemsetAsync(minid, 0xff, sizeof(uint32_t) * (size_t)n, ctx->stream));
    const int g = grid_for(ctx, n, 8);
    {
        KernelScope k(ctx, kKMinid);
        minid_scatter_kernel<<<g, kBlock, 0, ctx->stream>>>(n, parent, minid, &ctx->ctl->err);
    }
    {
        KernelScope k(ctx, kKMinid);
        minid_label_kernel<<<g, kBlock, 0, ctx->stream>>>(n, parent, minid, label, &ctx->ctl->err);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status cc_launch_count(phem_context *ctx, int32_t n, const int32_t *label, const uint64_t *forest)
{
    KernelScope k(ctx, kKCcCount);
    cc_count_kernel<<<grid_for(ctx, n, 8), kBlock, 0, ctx->stream>>>(
        n, label, reinterpret_cast<const unsigned long long *>(forest), ctx->ctl);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

}  // namespace phem
