// batch_api.cu -- entry points of the batched engine: one-shot solve,
// replayable plans (CUDA graph capture) and the autotuner.
#include <algorithm>
#include <numeric>
#include <vector>

#include "batch.h"

namespace phem {

phem_status build_items(const phem_batch_graph *graphs, uint32_t G, uint64_t total_edges, uint32_t total_vertices,
                        BatchLayout *L)
{
    if (G && !graphs) {
        set_error("batch: null graph array");
        return PHEM_ERR_INVALID;
    }
    if (G && is_device_ptr(graphs)) {
        set_error("batch: the graph array must be host memory");
        return PHEM_ERR_INVALID;
    }
    std::vector<uint32_t> by_vertex;
    by_vertex.reserve(G);
    for (uint32_t g = 0; g < G; g++) {
        const phem_batch_graph &x = graphs[g];
        if (x.kind != PHEM_BATCH_MSF && x.kind != PHEM_BATCH_CC) {
            set_error("batch: graph %u has kind %u (PHEM_BATCH_MSF or PHEM_BATCH_CC)", g, x.kind);
            return PHEM_ERR_INVALID;
        }
        if (x.edge_offset > total_edges || x.num_edges > total_edges - x.edge_offset) {
            set_error("batch: graph %u edges [%llu, +%u) exceed the %llu edges", g,
                      (unsigned long long)x.edge_offset, x.num_edges, (unsigned long long)total_edges);
            return PHEM_ERR_INVALID;
        }
        if ((uint64_t)x.vertex_offset + x.num_vertices > total_vertices) {
            set_error("batch: graph %u vertices [%u, +%u) exceed the %u vertices", g, x.vertex_offset,
                      x.num_vertices, total_vertices);
            return PHEM_ERR_INVALID;
        }
        if (x.num_vertices)
            by_vertex.push_back(g);
    }
    std::sort(by_vertex.begin(), by_vertex.end(),
              [&](uint32_t a, uint32_t b) { return graphs[a].vertex_offset < graphs[b].vertex_offset; });
    for (size_t i = 1; i < by_vertex.size(); i++) {
        const phem_batch_graph &p = graphs[by_vertex[i - 1]], &q = graphs[by_vertex[i]];
        if ((uint64_t)p.vertex_offset + p.num_vertices > q.vertex_offset) {
            set_error("batch: vertex ranges of graphs %u and %u overlap", by_vertex[i - 1], by_vertex[i]);
            return PHEM_ERR_INVALID;
        }
    }
    std::vector<uint32_t> order(G);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
        return (uint64_t)graphs[a].num_edges + graphs[a].num_vertices >
               (uint64_t)graphs[b].num_edges + graphs[b].num_vertices;
    });
    L->items.resize(G);
    uint64_t wl = 0, bm = 0;
    for (uint32_t q = 0; q < G; q++) {
        const uint32_t g = order[q];
        const phem_batch_graph &x = graphs[g];
        BatchItem &it = L->items[q];
        it.e_off = x.edge_offset;
        it.wl_off = wl;
        it.m = x.num_edges;
        it.n = x.num_vertices;
        it.v_off = x.vertex_offset;
        it.kind = x.kind;
        it.bm_off = (uint32_t)bm;
        it.index = g;
        wl += x.num_edges;
        bm += (x.num_edges + 31u) / 32u;
    }
    if (bm >= (1ull << 32)) {
        set_error("batch: too many edges for one batch");
        return PHEM_ERR_INVALID;
    }
    L->wl_records = wl;
    L->bm_words = bm;
    return PHEM_OK;
}

// Carves every buffer for the given capacities out of `base` (null: sizing
// only); returns the bytes needed.  `edges_inline` is false when the
// caller's device edges are used in place.
size_t batch_carve(uint32_t G, uint64_t E, uint64_t wl, uint64_t bm, uint32_t V, bool edges_inline, char *base,
                   BatchBuffers *b)
{
    Carve c;
    const uint32_t g1 = G ? G : 1, v1 = V ? V : 1;
    // num_graphs: the batch size, then the sizes of an overlapped batch's launches
    const size_t o_items = c.take<BatchItem>(g1), o_ng = c.take<uint32_t>(1 + kBatchGroups),
                 o_q = c.take<uint32_t>(1);
    const size_t o_e = edges_inline ? c.take<phem_edge>(E ? E : 1) : 0;
    const size_t o_wl = c.take<uint4>(wl ? wl : 1), o_bm = c.take<uint32_t>(bm ? bm : 1);
    const size_t o_gp = c.take<uint32_t>(v1), o_gc = c.take<uint32_t>(v1), o_gr = c.take<uint32_t>(v1);
    const size_t o_gb = c.take<unsigned long long>(v1);
    const size_t o_ids = c.take<uint32_t>(v1), o_cnt = c.take<uint32_t>(g1);
    const size_t o_tot = c.take<unsigned long long>(g1), o_lab = c.take<int32_t>(v1);
    const size_t o_st = c.take<uint32_t>(g1), o_rd = c.take<uint32_t>(g1);
    if (base) {
        b->items = reinterpret_cast<BatchItem *>(base + o_items);
        b->num_graphs = reinterpret_cast<uint32_t *>(base + o_ng);
        b->queue = reinterpret_cast<uint32_t *>(base + o_q);
        b->edges = edges_inline ? reinterpret_cast<phem_edge *>(base + o_e) : nullptr;
        b->wl = reinterpret_cast<uint4 *>(base + o_wl);
        b->bitmap = reinterpret_cast<uint32_t *>(base + o_bm);
        b->g_parent = reinterpret_cast<uint32_t *>(base + o_gp);
        b->g_aux = reinterpret_cast<uint32_t *>(base + o_gc);
        b->g_roots = reinterpret_cast<uint32_t *>(base + o_gr);
        b->g_best = reinterpret_cast<unsigned long long *>(base + o_gb);
        b->msf_ids = reinterpret_cast<uint32_t *>(base + o_ids);
        b->msf_count = reinterpret_cast<uint32_t *>(base + o_cnt);
        b->msf_total = reinterpret_cast<unsigned long long *>(base + o_tot);
        b->labels = reinterpret_cast<int32_t *>(base + o_lab);
        b->status = reinterpret_cast<uint32_t *>(base + o_st);
        b->rounds = reinterpret_cast<uint32_t *>(base + o_rd);
    }
    return c.off;
}

BatchArgs make_args(const BatchBuffers &b, const phem_edge *edges, float ratio)
{
    BatchArgs a{};
    a.items = b.items;
    a.num_graphs = b.num_graphs;
    a.queue = b.queue;
    a.edges = edges;
    a.wl = b.wl;
    a.bitmap = b.bitmap;
    a.g_parent = b.g_parent;
    a.g_aux = b.g_aux;
    a.g_roots = b.g_roots;
    a.g_best = b.g_best;
    a.msf_ids = b.msf_ids;
    a.msf_count = b.msf_count;
    a.msf_total = b.msf_total;
    a.labels = b.labels;
    a.status = b.status;
    a.rounds = b.rounds;
    a.compact_ratio = ratio;
    return a;
}

namespace {

phem_status batch_status(const uint32_t *status, uint32_t G)
{
    uint32_t err = 0;
    for (uint32_t g = 0; g < G; g++)
        err |= status[g];
    return ctl_status(err, "batch");
}

// Stages a batch into the context workspace: items, batch size, edges.  With
// `grp`, a large batch of host edges is instead grouped for overlapped
// launches (grp->k > 0): the items are reordered by the chunk that completes
// each graph's edges (queue order kept within a group) and the edges are
// left for launch_overlapped to copy.
phem_status batch_stage(phem_context *ctx, const phem_batch_graph *graphs, uint32_t G, const phem_edge *edges,
                        uint64_t E, uint32_t V, BatchLayout *L, BatchBuffers *b, const phem_edge **d_edges,
                        BatchGroups *grp = nullptr)
{
    PHEM_TRY(build_items(graphs, G, E, V, L));
    if (E && !edges) {
        set_error("batch: null edge array");
        return PHEM_ERR_INVALID;
    }
    const bool dev_edges = E && is_device_ptr(edges) && ((uintptr_t)edges & 3) == 0;
    const size_t bytes = batch_carve(G, E, L->wl_records, L->bm_words, V, !dev_edges, nullptr, nullptr);
    PHEM_TRY(ws_reserve(ctx, bytes));
    batch_carve(G, E, L->wl_records, L->bm_words, V, !dev_edges, static_cast<char *>(ctx->ws), b);
    uint32_t nums[1 + kBatchGroups] = {G};
    if (grp && !dev_edges && E >= kBatchOverlapMinEdges && G >= 2) {
        grp->k = kBatchGroups;
        for (int k = 0; k <= kBatchGroups; k++)
            grp->bound[k] = E * (uint64_t)k / kBatchGroups;
        std::vector<BatchItem> by_group;
        by_group.reserve(G);
        for (int k = 0; k < kBatchGroups; k++) {
            grp->start[k] = (uint32_t)by_group.size();
            for (const BatchItem &it : L->items) {
                const uint64_t end = it.e_off + it.m;
                int g = 0;
                while (g + 1 < kBatchGroups && end > grp->bound[g + 1])
                    g++;
                if (g == k)
                    by_group.push_back(it);
            }
            grp->count[k] = (uint32_t)by_group.size() - grp->start[k];
            nums[1 + k] = grp->count[k];
        }
        L->items.swap(by_group);
    } else if (grp) {
        grp->k = 0;
    }
    if (G)
        PHEM_CUDA_TRY(cudaMemcpyAsync(b->items, L->items.data(), sizeof(BatchItem) * G, cudaMemcpyHostToDevice,
                                      ctx->stream));
    PHEM_CUDA_TRY(cudaMemcpyAsync(b->num_graphs, nums, sizeof(nums), cudaMemcpyHostToDevice, ctx->stream));
    if (dev_edges) {
        *d_edges = edges;
    } else {
        if (E && !(grp && grp->k))
            PHEM_CUDA_TRY(cudaMemcpyAsync(b->edges, edges, sizeof(phem_edge) * E, cudaMemcpyDefault, ctx->stream));
        *d_edges = b->edges;
    }
    if (G)
        PHEM_CUDA_TRY(cudaMemsetAsync(b->rounds, 0, sizeof(uint32_t) * G, ctx->stream));
    return PHEM_OK;
}

phem_status launch_once(phem_context *ctx, const BatchLaunch &l, const BatchArgs &args)
{
    PHEM_CUDA_TRY(cudaMemsetAsync(args.queue, 0, sizeof(uint32_t), ctx->stream));
    KernelScope k(ctx, kKBatch);
    return batch_launch(ctx->stream, l, args);
}

// The launches of an overlapped batch: chunk k of the host edges is copied on
// the copy stream, and launch k (the graphs complete after chunk k) waits
// only for it.
phem_status launch_overlapped(phem_context *ctx, const BatchLaunch &l, const BatchArgs &args,
                              const BatchGroups &grp, const phem_edge *h_edges, phem_edge *d_edges,
                              const BatchBuffers &b)
{
    cudaEvent_t ev[kBatchGroups + 1] = {};
    phem_status st = PHEM_OK;
    for (auto &e : ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            e = nullptr;
            set_error("batch: cannot create copy events");
            st = PHEM_ERR_CUDA;
        }
    // the first copy waits for earlier work on the context stream, which may
    // still read the workspace
    if (st == PHEM_OK && (cudaEventRecord(ev[kBatchGroups], ctx->stream) != cudaSuccess ||
                          cudaStreamWaitEvent(ctx->copy_stream, ev[kBatchGroups], 0) != cudaSuccess)) {
        set_error("batch: cannot order the copy stream");
        st = PHEM_ERR_CUDA;
    }
    for (int k = 0; st == PHEM_OK && k < grp.k; k++) {
        const uint64_t lo = grp.bound[k], cnt = grp.bound[k + 1] - lo;
        if ((cnt && cudaMemcpyAsync(d_edges + lo, h_edges + lo, sizeof(phem_edge) * cnt, cudaMemcpyDefault,
                                    ctx->copy_stream) != cudaSuccess) ||
            cudaEventRecord(ev[k], ctx->copy_stream) != cudaSuccess ||
            cudaStreamWaitEvent(ctx->stream, ev[k], 0) != cudaSuccess) {
            set_error("batch: chunk copy failed: %s", cudaGetErrorString(cudaGetLastError()));
            st = PHEM_ERR_CUDA;
            break;
        }
        if (grp.count[k]) {
            BatchArgs a = args;
            a.items = args.items + grp.start[k];
            a.num_graphs = b.num_graphs + 1 + k;
            st = launch_once(ctx, l, a);
        }
    }
    if (st != PHEM_OK)
        cudaStreamSynchronize(ctx->copy_stream);  // no copy may still land in the workspace
    for (auto e : ev)
        if (e)
            cudaEventDestroy(e);
    return st;
}

void fill_stats(phem_batch_stats *st, const BatchLaunch &l, float ratio, float ms, uint32_t max_rounds)
{
    if (!st)
        return;
    st->max_rounds = max_rounds;
    st->block_size = (uint32_t)l.block;
    st->items = (uint32_t)l.items;
    st->compact_ratio = ratio;
    st->grid = (uint32_t)l.grid;
    st->smem_vertices = l.smem_vertices;
    st->device_ms = ms;
}

}  // namespace
}  // namespace phem

using namespace phem;

namespace phem {

// (Re)captures a plan's launch -- queue reset + persistent kernel -- into its
// CUDA graph, with `pairs` as the input of kBatchPairs graphs.
phem_status batch_plan_capture(phem_batch_plan *p, const unsigned long long *pairs)
{
    if (p->exec) {
        cudaGraphExecDestroy(p->exec);
        p->exec = nullptr;
    }
    if (p->graph) {
        cudaGraphDestroy(p->graph);
        p->graph = nullptr;
    }
    *p->h_num = 0;
    cudaStream_t s = p->ctx->stream;
    cudaError_t e = cudaMemcpyAsync(p->buf.num_graphs, p->h_num, sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e == cudaSuccess)
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        const cudaError_t e1 = cudaMemsetAsync(p->buf.queue, 0, sizeof(uint32_t), s);
        BatchArgs a = make_args(p->buf, p->buf.edges, p->ratio);
        a.pairs = pairs;
        a.smem_vertices = p->launch.smem_vertices;
        void *params[] = {&a};
        const cudaError_t e2 = cudaLaunchKernel(p->launch.kernel, dim3(p->launch.grid), dim3(p->launch.block),
                                                params, p->launch.dyn_smem, s);
        e = cudaStreamEndCapture(s, &p->graph);
        if (e == cudaSuccess)
            e = e1 != cudaSuccess ? e1 : e2;
    }
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    if (e != cudaSuccess) {
        set_error("batch plan: graph capture failed: %s", cudaGetErrorString(e));
        cudaGetLastError();
        return PHEM_ERR_CUDA;
    }
    return PHEM_OK;
}

}  // namespace phem

extern "C" {

phem_status phem_batch_solve(phem_context *ctx, const phem_batch_graph *graphs, uint32_t num_graphs,
                             const phem_edge *edges, uint64_t total_edges, uint32_t total_vertices, uint32_t *msf_ids,
                             uint32_t *msf_count, uint64_t *msf_total, int32_t *labels, phem_batch_stats *stats)
{
    PHEM_TRY(check_ctx(ctx));
    if (!msf_count || !msf_total) {
        set_error("batch_solve: msf_count and msf_total are required");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard guard(ctx->device);
    BatchLayout L;
    BatchBuffers b{};
    const phem_edge *d_edges = nullptr;
    BatchGroups grp;
    PHEM_TRY(batch_stage(ctx, graphs, num_graphs, edges, total_edges, total_vertices, &L, &b, &d_edges, &grp));
    BatchLaunch l;
    PHEM_TRY(batch_launch_config(ctx->device, ctx->sm_count, ctx->tune_batch_block, ctx->tune_batch_items, &l));
    const float ratio = (float)ctx->tune_batch_compact;
    const BatchArgs args = make_args(b, d_edges, ratio);
    float ms = 0.f;
    {
        Timed timer(ctx);
        if (grp.k)
            PHEM_TRY(launch_overlapped(ctx, l, args, grp, edges, b.edges, b));
        else
            PHEM_TRY(launch_once(ctx, l, args));
        ms = timer.stop();
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    std::vector<uint32_t> status(num_graphs), rounds(num_graphs);
    const size_t vb = sizeof(uint32_t) * (size_t)total_vertices;
    if (msf_ids && vb)
        PHEM_CUDA_TRY(cudaMemcpyAsync(msf_ids, b.msf_ids, vb, cudaMemcpyDefault, ctx->stream));
    if (labels && vb)
        PHEM_CUDA_TRY(cudaMemcpyAsync(labels, b.labels, vb, cudaMemcpyDefault, ctx->stream));
    if (num_graphs) {
        PHEM_CUDA_TRY(cudaMemcpyAsync(msf_count, b.msf_count, sizeof(uint32_t) * num_graphs, cudaMemcpyDefault,
                                      ctx->stream));
        PHEM_CUDA_TRY(cudaMemcpyAsync(msf_total, b.msf_total, sizeof(uint64_t) * num_graphs, cudaMemcpyDefault,
                                      ctx->stream));
        PHEM_CUDA_TRY(cudaMemcpyAsync(status.data(), b.status, sizeof(uint32_t) * num_graphs,
                                      cudaMemcpyDeviceToHost, ctx->stream));
        PHEM_CUDA_TRY(cudaMemcpyAsync(rounds.data(), b.rounds, sizeof(uint32_t) * num_graphs,
                                      cudaMemcpyDeviceToHost, ctx->stream));
    }
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(batch_status(status.data(), num_graphs));
    fill_stats(stats, l, ratio, ms, num_graphs ? *std::max_element(rounds.begin(), rounds.end()) : 0);
    return PHEM_OK;
}

phem_status phem_batch_autotune(phem_context *ctx, const phem_batch_graph *graphs, uint32_t num_graphs,
                                const phem_edge *edges, uint64_t total_edges, uint32_t total_vertices, uint32_t reps,
                                phem_batch_stats *best)
{
    PHEM_TRY(check_ctx(ctx));
    if (reps == 0 || reps > 1000) {
        set_error("batch_autotune: reps must be in [1, 1000]");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard guard(ctx->device);
    BatchLayout L;
    BatchBuffers b{};
    const phem_edge *d_edges = nullptr;
    PHEM_TRY(batch_stage(ctx, graphs, num_graphs, edges, total_edges, total_vertices, &L, &b, &d_edges));
    static const int kBlocks[] = {256, 512, 1024};
    static const int kItems[] = {1, 2, 4};
    static const float kRatios[] = {0.25f, 0.5f, 1.0f};
    float best_ms = -1.f;
    BatchLaunch best_l;
    float best_ratio = 0.5f;
    for (int blk : kBlocks)
        for (int it : kItems) {
            BatchLaunch l;
            if (batch_launch_config(ctx->device, ctx->sm_count, blk, it, &l) != PHEM_OK)
                continue;  // this configuration does not fit; the others still compete
            for (float ratio : kRatios) {
                const BatchArgs args = make_args(b, d_edges, ratio);
                PHEM_TRY(launch_once(ctx, l, args));  // warm-up
                Timed timer(ctx);
                for (uint32_t r = 0; r < reps; r++)
                    PHEM_TRY(launch_once(ctx, l, args));
                const float ms = timer.stop() / (float)reps;
                PHEM_CUDA_TRY(cudaGetLastError());
                if (best_ms < 0.f || ms < best_ms) {
                    best_ms = ms;
                    best_l = l;
                    best_ratio = ratio;
                }
            }
        }
    if (best_ms < 0.f) {
        set_error("batch_autotune: no kernel configuration fits this device");
        return PHEM_ERR_UNSUPPORTED;
    }
    std::vector<uint32_t> status(num_graphs);
    if (num_graphs)
        PHEM_CUDA_TRY(cudaMemcpyAsync(status.data(), b.status, sizeof(uint32_t) * num_graphs, cudaMemcpyDeviceToHost,
                                      ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(batch_status(status.data(), num_graphs));
    ctx->tune_batch_block = best_l.block;
    ctx->tune_batch_items = best_l.items;
    ctx->tune_batch_compact = best_ratio;
    fill_stats(best, best_l, best_ratio, best_ms, 0);
    return PHEM_OK;
}

void phem_batch_plan_destroy(phem_batch_plan *p)
{
    if (!p)
        return;
    DeviceGuard guard(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    if (p->exec)
        cudaGraphExecDestroy(p->exec);
    if (p->graph)
        cudaGraphDestroy(p->graph);
    if (p->staged)
        cudaEventDestroy(p->staged);
    if (p->h_items)
        cudaFreeHost(p->h_items);
    if (p->h_num)
        cudaFreeHost(p->h_num);
    if (p->h_status)
        cudaFreeHost(p->h_status);
    if (p->mem)
        cudaFree(p->mem);
    delete p;
}

phem_status phem_batch_plan_create(phem_context *ctx, uint32_t max_graphs, uint64_t max_edges, uint32_t max_vertices,
                                   phem_batch_plan **out)
{
    PHEM_TRY(check_ctx(ctx));
    if (!out || max_graphs == 0) {
        set_error("batch_plan_create: need an output pointer and max_graphs > 0");
        return PHEM_ERR_INVALID;
    }
    *out = nullptr;
    if (!ctx->stream) {
        set_error("batch_plan_create: the context stream must not be the legacy default stream");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard guard(ctx->device);
    auto *p = new phem_batch_plan();
    p->ctx = ctx;
    p->max_graphs = max_graphs;
    p->max_edges = max_edges;
    p->max_vertices = max_vertices;
    p->max_wl = max_edges;
    p->max_bm = max_edges / 32 + max_graphs;
    p->ratio = (float)ctx->tune_batch_compact;
    phem_status st = batch_launch_config(ctx->device, ctx->sm_count, ctx->tune_batch_block, ctx->tune_batch_items,
                                         &p->launch);
    const size_t bytes = batch_carve(max_graphs, max_edges, p->max_wl, p->max_bm, max_vertices, true, nullptr,
                                     nullptr);
    if (st == PHEM_OK && cudaMalloc(&p->mem, bytes) != cudaSuccess) {
        cudaGetLastError();
        p->mem = nullptr;
        set_error("batch_plan_create: cannot allocate %zu bytes", bytes);
        st = PHEM_ERR_NOMEM;
    }
    if (st == PHEM_OK && (cudaMallocHost(&p->h_items, sizeof(BatchItem) * max_graphs) != cudaSuccess ||
                          cudaMallocHost(&p->h_num, sizeof(uint32_t)) != cudaSuccess ||
                          cudaMallocHost(&p->h_status, sizeof(uint32_t) * max_graphs) != cudaSuccess ||
                          cudaEventCreateWithFlags(&p->staged, cudaEventDisableTiming) != cudaSuccess)) {
        cudaGetLastError();
        set_error("batch_plan_create: cannot allocate pinned staging");
        st = PHEM_ERR_NOMEM;
    }
    if (st == PHEM_OK) {
        batch_carve(max_graphs, max_edges, p->max_wl, p->max_bm, max_vertices, true, static_cast<char *>(p->mem),
                    &p->buf);
        st = phem::batch_plan_capture(p, nullptr);
    }
    if (st != PHEM_OK) {
        phem_batch_plan_destroy(p);
        return st;
    }
    *out = p;
    return PHEM_OK;
}

phem_status phem_batch_plan_upload(phem_batch_plan *p, const phem_batch_graph *graphs, uint32_t num_graphs,
                                   const phem_edge *edges, uint64_t total_edges, uint32_t total_vertices)
{
    if (!p) {
        set_error("batch_plan_upload: null plan");
        return PHEM_ERR_INVALID;
    }
    if (num_graphs > p->max_graphs || total_edges > p->max_edges || total_vertices > p->max_vertices) {
        set_error("batch_plan_upload: batch (%u graphs, %llu edges, %u vertices) exceeds the plan (%u, %llu, %u)",
                  num_graphs, (unsigned long long)total_edges, total_vertices, p->max_graphs,
                  (unsigned long long)p->max_edges, p->max_vertices);
        return PHEM_ERR_INVALID;
    }
    if (total_edges && !edges) {
        set_error("batch_plan_upload: null edge array");
        return PHEM_ERR_INVALID;
    }
    BatchLayout L;
    PHEM_TRY(build_items(graphs, num_graphs, total_edges, total_vertices, &L));
    DeviceGuard guard(p->ctx->device);
    cudaStream_t s = p->ctx->stream;
    PHEM_CUDA_TRY(cudaEventSynchronize(p->staged));  // the previous upload's staging was consumed
    std::copy(L.items.begin(), L.items.end(), p->h_items);
    *p->h_num = num_graphs;
    if (num_graphs)
        PHEM_CUDA_TRY(cudaMemcpyAsync(p->buf.items, p->h_items, sizeof(BatchItem) * num_graphs,
                                      cudaMemcpyHostToDevice, s));
    PHEM_CUDA_TRY(cudaMemcpyAsync(p->buf.num_graphs, p->h_num, sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    PHEM_CUDA_TRY(cudaEventRecord(p->staged, s));
    if (total_edges)
        PHEM_CUDA_TRY(cudaMemcpyAsync(p->buf.edges, edges, sizeof(phem_edge) * total_edges, cudaMemcpyDefault, s));
    p->num_graphs = num_graphs;
    p->total_vertices = total_vertices;
    return PHEM_OK;
}

phem_status phem_batch_plan_run(phem_batch_plan *p)
{
    if (!p) {
        set_error("batch_plan_run: null plan");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard guard(p->ctx->device);
    p->ctx->launches[kKBatch]++;
    PHEM_CUDA_TRY(cudaGraphLaunch(p->exec, p->ctx->stream));
    return PHEM_OK;
}

phem_status phem_batch_plan_download(phem_batch_plan *p, uint32_t *msf_ids, uint32_t *msf_count, uint64_t *msf_total,
                                     int32_t *labels)
{
    if (!p) {
        set_error("batch_plan_download: null plan");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard guard(p->ctx->device);
    cudaStream_t s = p->ctx->stream;
    const size_t vb = sizeof(uint32_t) * (size_t)p->total_vertices, G = p->num_graphs;
    if (msf_ids && vb)
        PHEM_CUDA_TRY(cudaMemcpyAsync(msf_ids, p->buf.msf_ids, vb, cudaMemcpyDefault, s));
    if (labels && vb)
        PHEM_CUDA_TRY(cudaMemcpyAsync(labels, p->buf.labels, vb, cudaMemcpyDefault, s));
    if (G) {
        if (msf_count)
            PHEM_CUDA_TRY(cudaMemcpyAsync(msf_count, p->buf.msf_count, sizeof(uint32_t) * G, cudaMemcpyDefault, s));
        if (msf_total)
            PHEM_CUDA_TRY(cudaMemcpyAsync(msf_total, p->buf.msf_total, sizeof(uint64_t) * G, cudaMemcpyDefault, s));
        PHEM_CUDA_TRY(cudaMemcpyAsync(p->h_status, p->buf.status, sizeof(uint32_t) * G, cudaMemcpyDeviceToHost, s));
    }
    PHEM_TRY(stream_wait(p->ctx));
    return batch_status(p->h_status, (uint32_t)G);
}

phem_status phem_batch_plan_device(phem_batch_plan *p, phem_edge **edges, uint32_t **msf_ids, uint32_t **msf_count,
                                   uint64_t **msf_total, int32_t **labels)
{
    if (!p) {
        set_error("batch_plan_device: null plan");
        return PHEM_ERR_INVALID;
    }
    if (edges)
        *edges = p->buf.edges;
    if (msf_ids)
        *msf_ids = p->buf.msf_ids;
    if (msf_count)
        *msf_count = p->buf.msf_count;
    if (msf_total)
        *msf_total = reinterpret_cast<uint64_t *>(p->buf.msf_total);
    if (labels)
        *labels = p->buf.labels;
    return PHEM_OK;
}

}  // extern "C"
