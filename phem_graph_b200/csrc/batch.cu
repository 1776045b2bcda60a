// batch.cu -- thousands of small graphs (MSF or CC each) in one persistent launch.
//
// The reference solves one graph per call (boruvka_for_edge_array,
// MST/src/new_boruvka.cu:40-179; SpanningTree, CC/ExternalSpanningTree.cu:133-218),
// paying ~10 launches and several host synchronisations per Boruvka round.
// Small graphs are then pure launch overhead.  Here every CTA of one
// persistent grid takes whole graphs from a device work queue (largest
// first) and solves each to completion on its own, with __syncthreads as the
// only barrier:
//
//   round 0   stream the graph's 12-byte input records once; self-loops are
//             dropped, every other edge offers its key to both endpoints
//             (atomicMin on per-vertex best keys) and is written, compacted,
//             to a 16-byte survivor list {root_u, root_v, w, id};
//   hook      every component with an offer takes its minimum edge; a mutual
//             pair keeps the lower root (new_grafting_edges,
//             MST/src/kernels.cu:73-134); the edge is marked in a bitmap;
//   compress  every live root is jumped to its new root (new_shortcutting_step,
//             MST/src/kernels.cu:254-271), best is reset and the roots that
//             still hold edges form the next round's list;
//   relabel   the survivor list is relabelled to roots; internal edges die
//             (relabelling_step/filtering_step, MST/src/kernels.cu:273-321);
//             the list is compacted in place when enough records died.
//
// Keys are (w << 32 | id) for MSF graphs and id alone for CC graphs, so a CC
// graph's forest is the canonical one (the MSF under edge index order) and
// its labels are the minimum vertex id of each component.  The per-vertex
// state (best key, parent, scratch, live-root list: 20 bytes a vertex) lives
// in dynamic shared memory when the graph fits, else in a global region of
// the graph's own.  After the first round a round touches only the roots
// still holding edges, so its vertex work shrinks with the components.
//
// Tuning: block size B and records per thread I are template parameters, the
// compaction threshold is a run-time ratio; the autotuner in batch_api.cu
// picks all three.
#include "batch.h"

namespace phem {
namespace {

constexpr unsigned long long kKeyInf = ~0ull;
constexpr uint32_t kBatchMaxRounds = 64;
constexpr uint32_t kNoVertex = 0xffffffffu;

template <int B>
struct ScanSmem {
    uint32_t part[2][B / 32 + 1];  // double-buffered warp partials
};

// Exclusive block scan of x; *total gets the block sum.  `parity` selects
// the scratch half so two scans in a row need only the barriers inside.
template <int B>
__device__ __forceinline__ uint32_t block_scan(uint32_t x, ScanSmem<B> &s, int parity, uint32_t *total)
{
    constexpr int NW = B / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d)
            inc += y;
    }
    if (lane == 31)
        s.part[parity][warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t v = lane < NW ? s.part[parity][lane] : 0;
        uint32_t vi = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, vi, d);
            if (lane >= d)
                vi += y;
        }
        if (lane < NW)
            s.part[parity][lane] = vi - v;
        if (lane == NW - 1)
            s.part[parity][NW] = vi;
    }
    __syncthreads();
    *total = s.part[parity][NW];
    return s.part[parity][warp] + inc - x;
}

__device__ __forceinline__ unsigned long long graph_key(uint32_t kind, uint32_t w, uint32_t id)
{
    return kind == PHEM_BATCH_MSF ? (((unsigned long long)w << 32) | id) : (unsigned long long)id;
}

__device__ __forceinline__ void offer(unsigned long long *best, uint32_t t, unsigned long long key)
{
    if (key < best[t])  // a stale (higher) value only lets a redundant atomic through
        atomicMin(best + t, key);
}

// Input record i of a graph: {u, v, w} records, or packed CC pairs
// (u << 32 | v) when p0 is set; a pair with u >= v is skipped, as the
// reference's union kernel skips it (CC/ExternalSpanningTree.cu:82), by
// turning it into a self-loop.
__device__ __forceinline__ void load_edge(const phem_edge *e0, const unsigned long long *p0, uint32_t i, uint32_t &u,
                                          uint32_t &v, uint32_t &w)
{
    if (p0) {
        const unsigned long long p = __ldg(p0 + i);
        u = (uint32_t)(p >> 32);
        v = (uint32_t)p;
        w = 0;
        if (u >= v)
            u = v = 0;  // skipped whatever its range, as the reference skips it
    } else {
        u = __ldg(&e0[i].u);
        v = __ldg(&e0[i].v);
        w = __ldg(&e0[i].w);
    }
}

template <int B>
struct BatchSmem {
    ScanSmem<B> scan;
    unsigned long long red[B / 32];
    uint32_t item;
    uint32_t err;
};

// Root of x by path halving over the graph's parent array (shared or global
// memory), bounded by n + 1 steps.  Concurrent halving writes point vertices
// at ancestors, so walks that overlap them stay correct.  Plain loads: only
// this CTA writes its graph's parent array, and it does so with plain stores
// from this SM, so even a load served by L1 sees every write that its
// barriers order before it (and a value missing a concurrent halving write
// is still an ancestor).
__device__ __forceinline__ uint32_t g_find(uint32_t *parent, uint32_t x, uint32_t n, uint32_t *err)
{
    for (uint32_t steps = 0; steps <= n; steps++) {
        const uint32_t p = parent[x];
        if (p == x)
            return x;
        const uint32_t gp = parent[p];
        if (gp == p)
            return p;
        parent[x] = gp;
        x = gp;
    }
    atomicOr(err, kErrChase);
    return x;
}

// One relabel/filter pass over the graph's edges.  FIRST reads the input
// records (ids = positions) and always compacts into the survivor list;
// later passes read the list and compact in place when `compact` is set
// (writes never overtake reads: an iteration's survivors land below the end
// of its own slots, and all its reads precede the scan barrier).  `fresh`
// lists were written by the previous pass, so their endpoints are roots the
// last compress pointed straight at the current roots: one load relabels
// them; older records walk with g_find.  Returns the survivor count;
// *len_out gets the new list length.
template <int B, int I, bool FIRST>
__device__ __forceinline__ uint32_t relabel_pass(const phem_edge *e0, const unsigned long long *p0, uint4 *wl, uint32_t len,
                                 bool compact, bool fresh, uint32_t n, uint32_t kind, uint32_t *parent,
                                 unsigned long long *best, BatchSmem<B> &sm, uint32_t *len_out)
{
    uint32_t out = 0, live = 0;
    int parity = 0;
    for (uint32_t base = 0; base < len; base += B * I) {
        uint4 rec[I];
        bool keep[I];
#pragma unroll
        for (int j = 0; j < I; j++) {
            const uint32_t i = base + j * B + threadIdx.x;
            keep[j] = false;
            rec[j] = make_uint4(0, 0, 0, 0);
            if (i < len) {
                if (FIRST) {
                    uint32_t u, v, w;
                    load_edge(e0, p0, i, u, v, w);
                    if (u >= n || v >= n) {
                        atomicOr(&sm.err, kErrRange);
                    } else if (u != v) {
                        rec[j] = make_uint4(u, v, w, i);
                        keep[j] = true;
                    }
                } else {
                    rec[j] = wl[i];
                }
            }
        }
        if (!FIRST) {
#pragma unroll
            for (int j = 0; j < I; j++)
                if (base + j * B + threadIdx.x < len) {
                    if (fresh) {
                        rec[j].x = parent[rec[j].x];
                        rec[j].y = parent[rec[j].y];
                    } else {
                        rec[j].x = g_find(parent, rec[j].x, n, &sm.err);
                        rec[j].y = g_find(parent, rec[j].y, n, &sm.err);
                    }
                    keep[j] = rec[j].x != rec[j].y;
                }
        }
#pragma unroll
        for (int j = 0; j < I; j++)
            if (keep[j]) {
                const unsigned long long key = graph_key(kind, rec[j].z, rec[j].w);
                offer(best, rec[j].x, key);
                offer(best, rec[j].y, key);
            }
        uint32_t cnt = 0;
#pragma unroll
        for (int j = 0; j < I; j++)
            cnt += keep[j];
        uint32_t total = 0;
        uint32_t pos = block_scan<B>(cnt, sm.scan, parity, &total);
        parity ^= 1;
        if (FIRST || compact) {
#pragma unroll
            for (int j = 0; j < I; j++)
                if (keep[j])
                    wl[out + pos++] = rec[j];
            out += total;
        }
        live += total;
    }
    *len_out = (FIRST || compact) ? out : len;
    return live;
}

// Per-graph vertex state: best key (8 bytes), parent, aux (the chosen
// edge's far root during a round, min-id labels at the end) and the list of
// live roots (4 bytes each) -- 20 bytes a vertex.
struct GraphState {
    unsigned long long *best;
    uint32_t *parent, *aux, *roots;
};

// SMEM: the vertex state lives in the CTA's dynamic shared memory (graphs of
// at most smem_vertices vertices), else in the graph's global region.  The
// two are separate instantiations, inlined into the kernel, so every state
// access is a plain shared- or global-memory access, never a generic one.
template <int B, int I, bool SMEM>
__device__ __forceinline__ void solve_graph(const BatchArgs &a, const BatchItem &it, BatchSmem<B> &sm,
                                            unsigned char *dyn)
{
    const uint32_t n = it.n, m = it.m;
    const phem_edge *e0 = a.edges + it.e_off;
    const unsigned long long *p0 = it.kind == kBatchPairs ? a.pairs + it.e_off : nullptr;
    uint4 *wl = a.wl + it.wl_off;
    uint32_t *bm = a.bitmap + it.bm_off;
    GraphState g;
    if (SMEM) {
        const size_t S = a.smem_vertices;
        g.best = reinterpret_cast<unsigned long long *>(dyn);
        g.parent = reinterpret_cast<uint32_t *>(dyn + 8 * S);
        g.aux = reinterpret_cast<uint32_t *>(dyn + 12 * S);
        g.roots = reinterpret_cast<uint32_t *>(dyn + 16 * S);
    } else {
        g.best = a.g_best + it.v_off;
        g.parent = a.g_parent + it.v_off;
        g.aux = a.g_aux + it.v_off;
        g.roots = a.g_roots + it.v_off;
    }
    const uint32_t nwords = (m + 31) / 32;

    for (uint32_t x = threadIdx.x; x < n; x += B) {
        g.parent[x] = x;
        g.roots[x] = x;
        g.best[x] = kKeyInf;
    }
    for (uint32_t w = threadIdx.x; w < nwords; w += B)
        bm[w] = 0;
    __syncthreads();

    uint32_t len = 0;
    uint32_t live = relabel_pass<B, I, true>(e0, p0, wl, m, true, true, n, it.kind, g.parent, g.best, sm, &len);
    bool fresh = true;
    uint32_t nroots = n;  // roots that may hold an offer
    uint32_t rounds = 0;
    while (live > 0) {
        if (++rounds > kBatchMaxRounds) {
            if (threadIdx.x == 0)
                atomicOr(&sm.err, kErrRounds);
            break;
        }
        __syncthreads();  // offers complete
        // A: the far root of each component's chosen edge, before any hook
        for (uint32_t i = threadIdx.x; i < nroots; i += B) {
            const uint32_t x = g.roots[i];
            const unsigned long long k = g.best[x];
            if (k == kKeyInf)
                continue;
            uint32_t eu, ev, ew;
            load_edge(e0, p0, (uint32_t)k, eu, ev, ew);
            const uint32_t ru = g_find(g.parent, eu, n, &sm.err), rv = g_find(g.parent, ev, n, &sm.err);
            g.aux[x] = ru == x ? rv : ru;
        }
        __syncthreads();
        // B: hook; a mutual pair keeps the lower root
        for (uint32_t i = threadIdx.x; i < nroots; i += B) {
            const uint32_t x = g.roots[i];
            const unsigned long long k = g.best[x];
            if (k == kKeyInf)
                continue;
            const uint32_t other = g.aux[x];
            if (g.best[other] == k && x < other)
                continue;
            g.parent[x] = other;
            const uint32_t id = (uint32_t)k;
            atomicOr(bm + (id >> 5), 1u << (id & 31));
        }
        __syncthreads();
        // C: point every listed root at its new root, reset best, and keep the
        // roots that had an offer and are still roots (the others are done)
        uint32_t kept = 0;
        int parity = 0;
        for (uint32_t i0 = 0; i0 < nroots; i0 += B) {
            const uint32_t i = i0 + threadIdx.x;
            bool keep = false;
            uint32_t x = 0;
            if (i < nroots) {
                x = g.roots[i];
                const bool had = g.best[x] != kKeyInf;
                const uint32_t r = g_find(g.parent, x, n, &sm.err);
                if (r != x)
                    g.parent[x] = r;
                g.best[x] = kKeyInf;
                keep = had && r == x;
            }
            uint32_t total = 0;
            const uint32_t pos = block_scan<B>(keep ? 1u : 0u, sm.scan, parity, &total);
            parity ^= 1;
            if (keep)
                g.roots[kept + pos] = x;
            kept += total;
        }
        nroots = kept;
        __syncthreads();
        const bool compact = (float)live <= a.compact_ratio * (float)len;
        live = relabel_pass<B, I, false>(e0, p0, wl, len, compact, fresh, n, it.kind, g.parent, g.best, sm, &len);
        fresh = compact;
    }
    __syncthreads();

    // labels: minimum vertex id of each component
    for (uint32_t x = threadIdx.x; x < n; x += B) {
        g.roots[x] = g_find(g.parent, x, n, &sm.err);
        g.aux[x] = kNoVertex;
    }
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < n; x += B)
        atomicMin(g.aux + g.roots[x], x);
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < n; x += B)
        a.labels[it.v_off + x] = (int32_t)g.aux[g.roots[x]];

    // forest edges ascending by id, and the total weight
    uint32_t out = 0;
    unsigned long long wsum = 0;
    int parity = 0;
    for (uint32_t w0 = 0; w0 < nwords; w0 += B) {
        const uint32_t wi = w0 + threadIdx.x;
        uint32_t word = wi < nwords ? bm[wi] : 0u;
        uint32_t total = 0;
        uint32_t pos = block_scan<B>((uint32_t)__popc(word), sm.scan, parity, &total);
        parity ^= 1;
        while (word) {
            const uint32_t b = __ffs(word) - 1;
            word &= word - 1;
            const uint32_t id = wi * 32 + b;
            if (out + pos < n)  // a forest has at most n - 1 edges
                a.msf_ids[it.v_off + out + pos] = id;
            else
                atomicOr(&sm.err, kErrCapacity);
            pos++;
            if (it.kind == PHEM_BATCH_MSF)
                wsum += __ldg(&e0[id].w);
        }
        out += total;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        wsum += __shfl_xor_sync(0xffffffffu, wsum, d);
    if ((threadIdx.x & 31) == 0)
        sm.red[threadIdx.x >> 5] = wsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int i = 0; i < B / 32; i++)
            t += sm.red[i];
        a.msf_count[it.index] = out;
        a.msf_total[it.index] = t;
        a.status[it.index] = sm.err;
        if (a.rounds)
            a.rounds[it.index] = rounds;
    }
}

template <int B, int I>
__global__ void __launch_bounds__(B) batch_kernel(BatchArgs a)
{
    __shared__ BatchSmem<B> sm;
    extern __shared__ __align__(16) unsigned char dyn[];
    const uint32_t G = *a.num_graphs;
    for (;;) {
        if (threadIdx.x == 0) {
            sm.item = atomicAdd(a.queue, 1u);
            sm.err = 0;
        }
        __syncthreads();
        const uint32_t q = sm.item;
        if (q >= G)
            break;
        const BatchItem it = a.items[q];
        if (it.n <= a.smem_vertices)
            solve_graph<B, I, true>(a, it, sm, dyn);
        else
            solve_graph<B, I, false>(a, it, sm, dyn);
        __syncthreads();  // sm.item, sm.err and the shared state are free again
    }
}

template <int B, int I>
const void *kernel_ptr()
{
    return reinterpret_cast<const void *>(&batch_kernel<B, I>);
}

const void *select_kernel(int block, int items)
{
#define PHEM_BATCH_CASE(b, i)         \
    if (block == b && items == i)     \
        return kernel_ptr<b, i>();
    PHEM_BATCH_CASE(256, 1) PHEM_BATCH_CASE(256, 2) PHEM_BATCH_CASE(256, 4)
    PHEM_BATCH_CASE(512, 1) PHEM_BATCH_CASE(512, 2) PHEM_BATCH_CASE(512, 4)
    PHEM_BATCH_CASE(1024, 1) PHEM_BATCH_CASE(1024, 2) PHEM_BATCH_CASE(1024, 4)
#undef PHEM_BATCH_CASE
    return nullptr;
}

}  // namespace

phem_status batch_launch_config(int device, int sm_count, int block, int items, BatchLaunch *out)
{
    const void *k = select_kernel(block, items);
    if (!k) {
        set_error("batch: no kernel for block %d, items %d (blocks 256/512/1024, items 1/2/4)", block, items);
        return PHEM_ERR_INVALID;
    }
    int per_sm_smem = 0, optin = 0;
    PHEM_CUDA_TRY(cudaDeviceGetAttribute(&per_sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    PHEM_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa;
    PHEM_CUDA_TRY(cudaFuncGetAttributes(&fa, k));
    // aim for the thread-limited number of CTAs per SM; each gets an equal
    // share of shared memory for its vertex state (16 bytes a vertex)
    const int want = 2048 / block;
    size_t dyn = (size_t)per_sm_smem / want;
    dyn = dyn > 1024 + fa.sharedSizeBytes ? dyn - 1024 - fa.sharedSizeBytes : 0;
    if (dyn > (size_t)optin - fa.sharedSizeBytes)
        dyn = (size_t)optin - fa.sharedSizeBytes;
    dyn &= ~size_t(15);
    PHEM_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    int occ = 0;
    PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, block, dyn));
    if (occ < 1) {
        set_error("batch: kernel (block %d, items %d) does not fit on an SM", block, items);
        return PHEM_ERR_UNSUPPORTED;
    }
    out->kernel = k;
    out->block = block;
    out->items = items;
    out->dyn_smem = dyn;
    out->smem_vertices = (uint32_t)(dyn / 20);
    out->grid = sm_count * occ;
    return PHEM_OK;
}

phem_status batch_launch(cudaStream_t stream, const BatchLaunch &l, BatchArgs args)
{
    args.smem_vertices = l.smem_vertices;
    void *params[] = {&args};
    PHEM_CUDA_TRY(cudaLaunchKernel(l.kernel, dim3(l.grid), dim3(l.block), params, l.dyn_smem, stream));
    return PHEM_OK;
}

}  // namespace phem
