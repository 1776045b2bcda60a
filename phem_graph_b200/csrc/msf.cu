// msf.cu -- Boruvka minimum spanning forest on sm_100a.
//
// Same arithmetic as the reference's device_boruvka (MST/src/kernels.cu:507-689):
// per round every component takes its minimum (weight, edge id) edge, a
// mutual pair keeps the lower id as root and every other chooser hooks onto
// the far component (new_grafting_edges, :73-134), hooks are jumped to roots
// (new_shortcutting_step, :254-271) and edges inside a component are dropped
// (relabelling_step / filtering_step / remove_if, :273-321, :641-649).
//
// Layout and kernels are B200-first rather than a translation:
//   * round 0 reads the 12-byte {u,v,w} input with 128-bit streaming loads and
//     reduces (w << 32 | id) keys per endpoint inside each warp before one
//     guarded 64-bit atomicMin per distinct endpoint;
//   * rounds >= 1 run ONE streaming pass per round over the live edges: it
//     relabels both endpoints to their roots, drops internal edges, writes the
//     survivors as 16-byte {root_u, root_v, w, id} records with a stable
//     single-pass compaction (decoupled look-back) and offers each survivor's
//     key to both roots in the same pass.  Because the compaction is stable the
//     survivor's position orders like its id, so the key carries the position
//     and the hook step finds the record directly;
//   * the vertex steps (hook, pointer jumping) only visit the components that
//     were roots at the start of the round, kept in a compacted list;
//   * MSF membership is a bitmap over edge ids; one final ordered gather writes
//     the MSF records ascending by id with the uint64 total.
// Every kernel reads the round number and the continue flag from the device
// control block, so the host can queue rounds ahead without reading anything
// back; a round queued after convergence exits at once.
#include <algorithm>
#include <cstring>

#include "internal.h"

namespace phem {
namespace {

struct RoundArgs {
    const void *e0;
    uint64_t m;
    uint32_t n;
    uint32_t epoch_base;
    uint32_t *parent;
    unsigned long long *best;
    uint32_t *cand0, *cand1;
    uint32_t *bitmap;
    uint4 *wl0, *wl1;
    uint64_t *status;
    unsigned long long *forest;
    Ctl *ctl;
};

// ---- input record access --------------------------------------------------

// Four consecutive input records starting at index `base` (a multiple of 4).
// ok[j] is false past the end of the input.
template <int KIND>
__device__ __forceinline__ void load4_e0(const void *e0, uint64_t base, uint64_t m, uint32_t (&u)[4],
                                         uint32_t (&v)[4], uint32_t (&w)[4], bool (&ok)[4])
{
    if (KIND == kKindMsf) {
        const uint32_t *p = reinterpret_cast<const uint32_t *>(e0) + base * 3;
        if (base + 4 <= m) {
            const uint4 *q = reinterpret_cast<const uint4 *>(p);
            uint4 a = __ldcs(q), b = __ldcs(q + 1), c = __ldcs(q + 2);
            u[0] = a.x; v[0] = a.y; w[0] = a.z;
            u[1] = a.w; v[1] = b.x; w[1] = b.y;
            u[2] = b.z; v[2] = b.w; w[2] = c.x;
            u[3] = c.y; v[3] = c.z; w[3] = c.w;
#pragma unroll
            for (int j = 0; j < 4; j++)
                ok[j] = true;
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                ok[j] = base + j < m;
                u[j] = ok[j] ? __ldcs(p + 3 * j) : 0;
                v[j] = ok[j] ? __ldcs(p + 3 * j + 1) : 0;
                w[j] = ok[j] ? __ldcs(p + 3 * j + 2) : 0;
            }
        }
    } else {
        const unsigned long long *p = reinterpret_cast<const unsigned long long *>(e0) + base;
        if (base + 4 <= m) {
            const uint4 *q = reinterpret_cast<const uint4 *>(p);
            uint4 a = __ldcs(q), b = __ldcs(q + 1);
            v[0] = a.x; u[0] = a.y; v[1] = a.z; u[1] = a.w;
            v[2] = b.x; u[2] = b.y; v[3] = b.z; u[3] = b.w;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                ok[j] = true;
                w[j] = 0;
            }
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                ok[j] = base + j < m;
                unsigned long long e = ok[j] ? __ldcs(p + j) : 0ull;
                u[j] = (uint32_t)(e >> 32);
                v[j] = (uint32_t)e;
                w[j] = 0;
            }
        }
    }
}

// An input record takes part in the forest: self-loops never do; packed CC
// edges follow union_find_gpu_COO and only count when u < v
// (CC/ExternalSpanningTree.cu:82).
template <int KIND>
__device__ __forceinline__ bool e0_live(uint32_t u, uint32_t v)
{
    return KIND == kKindMsf ? (u != v) : (u < v);
}

template <int KIND>
__device__ __forceinline__ void e0_endpoints(const void *e0, uint32_t id, uint32_t &u, uint32_t &v)
{
    if (KIND == kKindMsf) {
        const uint32_t *p = reinterpret_cast<const uint32_t *>(e0) + (uint64_t)id * 3;
        u = __ldg(p);
        v = __ldg(p + 1);
    } else {
        unsigned long long e = __ldg(reinterpret_cast<const unsigned long long *>(e0) + id);
        u = (uint32_t)(e >> 32);
        v = (uint32_t)e;
    }
}

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long x, unsigned long long *s)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, d);
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 0)
        s[warp] = x;
    __syncthreads();
    unsigned long long t = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kWarps; i++)
            t += s[i];
    return t;  // valid in thread 0
}

// ---- kernels -----------------------------------------------------------------

__global__ void __launch_bounds__(kBlock) init_kernel(RoundArgs a)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < a.n; x += stride) {
        a.parent[x] = x;
        a.best[x] = kKeyNone;
        if (a.forest)
            a.forest[x] = kForestEmpty;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.ctl->go = 1;
        a.ctl->round = 0;
    }
}

// Round 0: every vertex is its own component; best[x] = min key over incident
// live edges, key = (w << 32 | input index).  Also counts m_0.
template <int KIND>
__global__ void __launch_bounds__(kBlock) round0_kernel(RoundArgs a)
{
    __shared__ unsigned long long s_red[kWarps];
    const uint64_t groups = (a.m + 3) / 4;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long live = 0;
    for (uint64_t g0 = (uint64_t)blockIdx.x * blockDim.x; g0 < groups; g0 += stride) {
        const uint64_t g = g0 + threadIdx.x;
        uint32_t u[4], v[4], w[4];
        bool ok[4];
        if (g < groups) {
            load4_e0<KIND>(a.e0, g * 4, a.m, u, v, w, ok);
        } else {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                ok[j] = false;
                u[j] = v[j] = w[j] = 0;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; j++) {
            bool valid = ok[j] && e0_live<KIND>(u[j], v[j]);
            if (valid && (u[j] >= a.n || v[j] >= a.n)) {
                set_err(&a.ctl->err, kErrRange);
                valid = false;
            }
            live += valid;
            const uint64_t key = ((uint64_t)w[j] << 32) | (uint32_t)(g * 4 + j);
            warp_min_to(a.best, u[j], key, valid);
            warp_min_to(a.best, v[j], key, valid);
        }
    }
    const unsigned long long t = block_sum_u64(live, s_red);
    if (threadIdx.x == 0 && t)
        atomicAdd(&a.ctl->m_r[0], t);
}

// Rounds >= 1: relabel + filter + stable compaction + per-root minimum, one pass.
template <int KIND>
__global__ void __launch_bounds__(kBlock) edge_pass_kernel(RoundArgs a)
{
    __shared__ uint32_t s_tile, s_base;
    __shared__ uint32_t s_warp[kWarps + 1];
    Ctl *ctl = a.ctl;
    if (!*(volatile uint32_t *)&ctl->go)
        return;
    const uint32_t r = *(volatile uint32_t *)&ctl->round;
    const bool from_e0 = (r == 1);
    const uint64_t count = from_e0 ? a.m : ctl->m_r[r - 1];
    const uint4 *in = (r & 1) ? a.wl0 : a.wl1;  // WL[(r - 1) & 1]
    uint4 *out = (r & 1) ? a.wl1 : a.wl0;       // WL[r & 1]
    const uint32_t ntiles = (uint32_t)((count + kTile - 1) / kTile);
    const uint32_t epoch = a.epoch_base + r;
    for (;;) {
        if (threadIdx.x == 0)
            s_tile = atomicAdd(&ctl->ticket[r], 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles)
            break;
        const uint64_t base = (uint64_t)t * kTile + (uint64_t)threadIdx.x * kItems;
        uint32_t ra[4], rb[4], w[4], id[4];
        bool keep[4];
        if (from_e0) {
            uint32_t u[4], v[4];
            bool ok[4];
            load4_e0<KIND>(a.e0, base, count, u, v, w, ok);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                keep[j] = ok[j] && e0_live<KIND>(u[j], v[j]) && u[j] < a.n && v[j] < a.n;
                ra[j] = u[j];
                rb[j] = v[j];
                id[j] = (uint32_t)(base + j);
            }
        } else {
            const uint4 *q = in + base;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                keep[j] = base + j < count;
                uint4 rec = keep[j] ? __ldcs(q + j) : make_uint4(0, 0, 0, 0);
                ra[j] = rec.x;
                rb[j] = rec.y;
                w[j] = rec.z;
                id[j] = rec.w;
            }
        }
        uint32_t c = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (keep[j]) {
                ra[j] = __ldg(a.parent + ra[j]);
                rb[j] = __ldg(a.parent + rb[j]);
                keep[j] = ra[j] != rb[j];
            }
            c += keep[j];
        }
        uint32_t total;
        const uint32_t off = block_exclusive_scan(c, &total, s_warp);
        if (threadIdx.x < 32) {
            const uint32_t ex = lookback_exclusive(a.status, t, total, epoch, &ctl->err);
            if (threadIdx.x == 0) {
                s_base = ex;
                if (t == ntiles - 1)
                    ctl->m_r[r] = (unsigned long long)ex + total;
            }
        }
        __syncthreads();
        uint32_t pos = s_base + off;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            if (keep[j])
                out[pos] = make_uint4(ra[j], rb[j], w[j], id[j]);
            const uint64_t key = ((uint64_t)w[j] << 32) | pos;
            warp_min_to(a.best, ra[j], key, keep[j]);
            warp_min_to(a.best, rb[j], key, keep[j]);
            pos += keep[j];
        }
        __syncthreads();
    }
}

// Hook: each component that found an edge either stays root (lower id of a
// mutual pair) or points at the far component and marks its edge.
template <int KIND>
__global__ void __launch_bounds__(kBlock) hook_kernel(RoundArgs a)
{
    Ctl *ctl = a.ctl;
    if (!*(volatile uint32_t *)&ctl->go)
        return;
    const uint32_t r = *(volatile uint32_t *)&ctl->round;
    const uint32_t count = (r == 0) ? a.n : ctl->roots[r];
    const uint32_t *cand = (r & 1) ? a.cand1 : a.cand0;
    const uint4 *wl = (r & 1) ? a.wl1 : a.wl0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < count; i0 += stride) {
        const uint32_t i = i0 + threadIdx.x;
        const bool in = i < count;
        const uint32_t x = in ? (r == 0 ? i : cand[i]) : 0;
        const unsigned long long bk = in ? a.best[x] : kKeyNone;
        const bool active = bk != kKeyNone;
        warp_count(&ctl->n_r[r], active);
        if (!active)
            continue;
        const uint32_t pos = (uint32_t)bk;
        uint32_t ea, eb, id;
        if (r == 0) {
            e0_endpoints<KIND>(a.e0, pos, ea, eb);
            id = pos;
        } else {
            const uint4 rec = wl[pos];
            ea = rec.x;
            eb = rec.y;
            id = rec.w;
        }
        if (ea != x && eb != x) {
            set_err(&ctl->err, kErrChase);
            continue;
        }
        const uint32_t other = (ea == x) ? eb : ea;
        const bool mutual = a.best[other] == bk;
        if (mutual && x < other)
            continue;  // stays root; the partner hooks and marks the edge
        a.parent[x] = other;
        atomicOr(a.bitmap + (id >> 5), 1u << (id & 31));
        if (KIND == kKindPacked && a.forest)
            a.forest[x] = __ldg(reinterpret_cast<const unsigned long long *>(a.e0) + id);
    }
}

// Pointer jumping over this round's components; roots that remain are
// collected (in any order) as the next round's candidates.  Also resets best.
__global__ void __launch_bounds__(kBlock) compress_kernel(RoundArgs a)
{
    Ctl *ctl = a.ctl;
    if (!*(volatile uint32_t *)&ctl->go)
        return;
    const uint32_t r = *(volatile uint32_t *)&ctl->round;
    const uint32_t count = (r == 0) ? a.n : ctl->roots[r];
    const uint32_t *cand = (r & 1) ? a.cand1 : a.cand0;
    uint32_t *next = (r & 1) ? a.cand0 : a.cand1;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < count; i0 += stride) {
        const uint32_t i = i0 + threadIdx.x;
        const bool in = i < count;
        const uint32_t x = in ? (r == 0 ? i : cand[i]) : 0;
        const bool active = in && a.best[x] != kKeyNone;
        bool stays = false;
        if (active) {
            uint32_t y = a.parent[x];
            uint32_t steps = 0;
            for (;;) {
                const uint32_t p = a.parent[y];
                if (p == y)
                    break;
                y = p;
                if (++steps > a.n) {
                    set_err(&ctl->err, kErrChase);
                    break;
                }
            }
            a.parent[x] = y;
            a.best[x] = kKeyNone;
            stays = (y == x);
        }
        const unsigned b = __ballot_sync(0xffffffffu, stays);
        uint32_t slot = 0;
        if (lane_id() == 0 && b)
            slot = atomicAdd(&ctl->roots[r + 1], (uint32_t)__popc(b));
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (stays)
            next[slot + __popc(b & ((1u << lane_id()) - 1))] = x;
    }
}

// Ends a round: another one is needed while this round still had live edges.
__global__ void advance_kernel(Ctl *ctl)
{
    if (!ctl->go)
        return;
    const uint32_t r = ctl->round;
    bool again = ctl->m_r[r] > 0;
    if (again && r + 1 >= PHEM_MAX_ROUNDS) {
        ctl->err |= kErrRounds;
        again = false;
    }
    ctl->round = r + 1;
    ctl->go = again ? 1u : 0u;
}

// Ordered gather: MSF records ascending by id from the bitmap, plus count and
// uint64 total weight.
__global__ void __launch_bounds__(kBlock) gather_kernel(RoundArgs a, phem_edge *out)
{
    __shared__ uint32_t s_tile, s_base;
    __shared__ uint32_t s_warp[kWarps + 1];
    __shared__ unsigned long long s_red[kWarps];
    Ctl *ctl = a.ctl;
    const uint64_t words = (a.m + 31) / 32;
    const uint32_t ntiles = (uint32_t)((words + kTile - 1) / kTile);
    const uint32_t epoch = a.epoch_base + PHEM_MAX_ROUNDS + 2;
    const uint32_t *E = reinterpret_cast<const uint32_t *>(a.e0);
    for (;;) {
        if (threadIdx.x == 0)
            s_tile = atomicAdd(&ctl->out_ticket, 1u);
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles)
            break;
        const uint64_t wbase = (uint64_t)t * kTile + (uint64_t)threadIdx.x * kItems;
        uint32_t bits[4];
        uint32_t c = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            bits[j] = (wbase + j < words) ? a.bitmap[wbase + j] : 0u;
            c += __popc(bits[j]);
        }
        uint32_t total;
        const uint32_t off = block_exclusive_scan(c, &total, s_warp);
        if (threadIdx.x < 32) {
            const uint32_t ex = lookback_exclusive(a.status, t, total, epoch, &ctl->err);
            if (threadIdx.x == 0) {
                s_base = ex;
                if (t == ntiles - 1)
                    ctl->msf_count = (unsigned long long)ex + total;
            }
        }
        __syncthreads();
        uint32_t pos = s_base + off;
        unsigned long long wsum = 0;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            uint32_t b = bits[j];
            while (b) {
                const int k = __ffs(b) - 1;
                b &= b - 1;
                const uint64_t id = (wbase + j) * 32 + k;
                phem_edge e;
                e.u = __ldg(E + id * 3);
                e.v = __ldg(E + id * 3 + 1);
                e.w = __ldg(E + id * 3 + 2);
                if (out)
                    out[pos] = e;
                pos++;
                wsum += e.w;
            }
        }
        const unsigned long long bs = block_sum_u64(wsum, s_red);
        if (threadIdx.x == 0 && bs)
            atomicAdd(&ctl->msf_total, bs);
        __syncthreads();
    }
}

RoundArgs make_args(phem_context *ctx, const MsfPlan &p)
{
    RoundArgs a;
    a.e0 = p.e0;
    a.m = p.m;
    a.n = p.n;
    a.epoch_base = (uint32_t)p.epoch_base;
    a.parent = p.parent;
    a.best = p.best;
    a.cand0 = p.cand[0];
    a.cand1 = p.cand[1];
    a.bitmap = p.bitmap;
    a.wl0 = p.wl[0];
    a.wl1 = p.wl[1];
    a.status = p.status;
    a.forest = reinterpret_cast<unsigned long long *>(p.forest);
    a.ctl = ctx->ctl;
    return a;
}

int vertex_blocks(phem_context *ctx, uint64_t count)
{
    uint64_t b = (count + kBlock - 1) / kBlock;
    uint64_t cap = (uint64_t)ctx->sm_count * 8;
    return (int)std::max<uint64_t>(1, std::min(b, cap));
}

template <int KIND>
phem_status queue_round(phem_context *ctx, const RoundArgs &a)
{
    const int vb = vertex_blocks(ctx, a.n);
    {
        KernelScope k(ctx, kKEdgePass);
        edge_pass_kernel<KIND><<<ctx->edge_pass_blocks, kBlock, 0, ctx->stream>>>(a);
    }
    {
        KernelScope k(ctx, kKHook);
        hook_kernel<KIND><<<vb, kBlock, 0, ctx->stream>>>(a);
    }
    {
        KernelScope k(ctx, kKCompress);
        compress_kernel<<<vb, kBlock, 0, ctx->stream>>>(a);
    }
    {
        KernelScope k(ctx, kKAdvance);
        advance_kernel<<<1, 1, 0, ctx->stream>>>(a.ctl);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

template <int KIND>
phem_status run_impl(phem_context *ctx, MsfPlan &plan, uint32_t *rounds_out)
{
    cudaStream_t s = ctx->stream;
    if (!ctx->edge_pass_blocks) {
        int per_sm = 0;
        PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, edge_pass_kernel<KIND>, kBlock, 0));
        ctx->edge_pass_blocks = ctx->sm_count * std::max(1, per_sm);
        PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gather_kernel, kBlock, 0));
        ctx->gather_blocks = ctx->sm_count * std::max(1, per_sm);
        PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, round0_kernel<KIND>, kBlock, 0));
        ctx->round0_blocks = ctx->sm_count * std::max(1, per_sm);
    }
    const RoundArgs a = make_args(ctx, plan);
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), s));
    PHEM_CUDA_TRY(cudaMemsetAsync(plan.bitmap, 0, ((plan.m + 31) / 32) * sizeof(uint32_t), s));
    {
        KernelScope k(ctx, kKInit);
        init_kernel<<<vertex_blocks(ctx, plan.n), kBlock, 0, s>>>(a);
    }
    const uint64_t groups = (plan.m + 3) / 4;
    const int r0_blocks = (int)std::max<uint64_t>(
        1, std::min<uint64_t>((groups + kBlock - 1) / kBlock, (uint64_t)ctx->round0_blocks));
    {
        KernelScope k(ctx, kKRound0);
        round0_kernel<KIND><<<r0_blocks, kBlock, 0, s>>>(a);
    }
    const int vb = vertex_blocks(ctx, plan.n);
    {
        KernelScope k(ctx, kKHook);
        hook_kernel<KIND><<<vb, kBlock, 0, s>>>(a);
    }
    {
        KernelScope k(ctx, kKCompress);
        compress_kernel<<<vb, kBlock, 0, s>>>(a);
    }
    {
        KernelScope k(ctx, kKAdvance);
        advance_kernel<<<1, 1, 0, s>>>(a.ctl);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    // Rounds are queued in batches; the host reads the continue flag between
    // batches.  Rounds queued after convergence return immediately.
    int queued = 1;
    int batch = 3;
    while (queued < PHEM_MAX_ROUNDS) {
        for (int k = 0; k < batch && queued < PHEM_MAX_ROUNDS; k++, queued++)
            PHEM_TRY(queue_round<KIND>(ctx, a));
        PHEM_CUDA_TRY(cudaMemcpyAsync(&ctx->h_ctl->go, &ctx->ctl->go, sizeof(uint32_t) * 2,
                                      cudaMemcpyDeviceToHost, s));
        PHEM_TRY(stream_wait(ctx));
        if (!*(volatile uint32_t *)&ctx->h_ctl->go)
            break;
        batch = 2;
    }
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    PHEM_TRY(stream_wait(ctx));
    const Ctl &h = *ctx->h_ctl;
    if (h.go)
        return ctl_status(h.err | kErrRounds, "msf");
    uint32_t rounds = 0;
    while (rounds < PHEM_MAX_ROUNDS && h.m_r[rounds] > 0)
        rounds++;
    if (rounds_out)
        *rounds_out = rounds;
    return ctl_status(h.err, "msf");
}

}  // namespace

size_t msf_workspace_bytes(uint64_t m, uint32_t n)
{
    Carve c;
    c.take<uint32_t>(n);
    c.take<unsigned long long>(n);
    c.take<uint32_t>(n);
    c.take<uint32_t>(n);
    c.take<uint32_t>((m + 31) / 32 + 4);
    c.take<uint4>(m);
    c.take<uint4>(m);
    return c.off;
}

phem_status msf_plan(phem_context *ctx, int kind, const void *d_e0, uint64_t m, uint32_t n, size_t extra_bytes,
                     MsfPlan *plan, size_t *extra_off)
{
    const size_t core = msf_workspace_bytes(m, n);
    Carve c;
    c.off = core;
    const size_t extra_at = c.take<uint8_t>(extra_bytes);
    PHEM_TRY(ws_reserve(ctx, c.off));
    PHEM_TRY(status_reserve(ctx, (m + kTile - 1) / kTile + 2));
    char *base = static_cast<char *>(ctx->ws);
    Carve k;
    plan->status = ctx->status;
    plan->parent = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(n));
    plan->best = reinterpret_cast<unsigned long long *>(base + k.take<unsigned long long>(n));
    plan->cand[0] = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(n));
    plan->cand[1] = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(n));
    plan->bitmap = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>((m + 31) / 32 + 4));
    plan->wl[0] = reinterpret_cast<uint4 *>(base + k.take<uint4>(m));
    plan->wl[1] = reinterpret_cast<uint4 *>(base + k.take<uint4>(m));
    plan->e0 = d_e0;
    plan->m = m;
    plan->n = n;
    plan->forest = nullptr;
    plan->epoch_base = next_epochs(ctx, PHEM_MAX_ROUNDS + 4);
    (void)kind;
    if (extra_off)
        *extra_off = extra_at;
    return PHEM_OK;
}

phem_status msf_run(phem_context *ctx, int kind, MsfPlan &plan, uint32_t *rounds_out)
{
    if (kind == kKindMsf)
        return run_impl<kKindMsf>(ctx, plan, rounds_out);
    return run_impl<kKindPacked>(ctx, plan, rounds_out);
}

phem_status msf_gather(phem_context *ctx, MsfPlan &plan, phem_edge *d_out)
{
    const RoundArgs a = make_args(ctx, plan);
    const uint64_t words = (plan.m + 31) / 32;
    const uint64_t tiles = (words + kTile - 1) / kTile;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)ctx->gather_blocks));
    KernelScope k(ctx, kKGather);
    gather_kernel<<<blocks, kBlock, 0, ctx->stream>>>(a, d_out);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

}  // namespace phem
