// server.cu -- serving loop: continuous batching of MSF / CC requests.
//
// Requests of mixed sizes arrive from any host thread.  Small ones (at most
// `large_edges` edges) are packed into batched persistent launches (batch.cu);
// `slots` of them are in flight at once on their own streams, so requests
// that arrive while a batch runs form the next batch and are admitted as soon
// as a slot and its memory are free; their work overlaps on the device.
// Large requests run on the device-wide engines (phem_msf_solve,
// phem_cc_solve) in `large_workers` threads, each with its own context and
// stream, concurrently with the batches.  Device memory is fixed at creation
// and bounded by the budget: slot arenas are allocated up front, and each
// device-wide worker may grow its workspace to its share of the budget;
// a request that fits nowhere is refused at submission.
//
// Every request gets the result it would get alone: MSF requests the unique
// forest under (w, edge index), CC requests min-id labels (and the forest
// size), whichever path serves them.  There is no reference counterpart: the
// reference runs one solve per process invocation (CC/main.cu, MST/main.cu).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"

namespace {

using phem::BatchLayout;

uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Pending {
    uint64_t ticket = 0;
    phem_request req{};
    phem_request_result res{};
    bool done = false;
};

// One batched launch in flight: its context (stream), plan and the requests
// it carries.
struct Slot {
    phem_context *ctx = nullptr;
    phem_batch_plan *plan = nullptr;
    unsigned long long *d_pairs = nullptr;  // CC requests' packed pairs
    cudaEvent_t done = nullptr;
    uint32_t *h_ids = nullptr, *h_count = nullptr;  // pinned results
    uint64_t *h_total = nullptr;
    int32_t *h_labels = nullptr;
    std::vector<phem_batch_graph> graphs;
    std::vector<Pending *> reqs;
    uint64_t edges = 0;
    uint32_t vertices = 0;
    bool busy = false;
};

// Device bytes a device-wide solve of this request may need (workspace
// growth included), an upper estimate used for admission.
uint64_t large_bytes(const phem_request &r)
{
    const uint64_t m = r.num_edges, n = r.num_vertices;
    if (r.kind == PHEM_BATCH_CC)
        return 8 * m + 16 * n + (1u << 20);
    return phem::msf_workspace_bytes(m, (uint32_t)n, 148) + 12 * m + 12 * n + (1u << 20);
}

}  // namespace

struct phem_server {
    int device = 0;
    phem_server_config cfg{};
    uint64_t slot_edges = 0;  // per-slot capacity
    uint32_t slot_vertices = 0;
    uint64_t large_share = 0;  // device bytes per device-wide worker
    std::vector<Slot> slots;
    std::vector<phem_context *> large_ctx;

    std::mutex mu;
    std::condition_variable cv_work, cv_large, cv_done;
    std::deque<Pending *> small_q, large_q;
    std::unordered_map<uint64_t, Pending *> live;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::vector<std::thread> threads;

    phem_status fatal = PHEM_OK;  // a CUDA failure in a worker: every later request fails with it

    void complete(Pending *p, phem_status st)
    {
        p->res.status = st;
        p->res.done_ns = now_ns();
        {
            std::lock_guard<std::mutex> lk(mu);
            p->done = true;
        }
        cv_done.notify_all();
    }

    // Copies one admitted batch to a free slot and replays its launch.
    phem_status launch(Slot &s)
    {
        phem_edge *d_edges = nullptr;
        PHEM_TRY(phem_batch_plan_device(s.plan, &d_edges, nullptr, nullptr, nullptr, nullptr));
        cudaStream_t st = static_cast<cudaStream_t>(phem_context_stream(s.ctx));
        const uint64_t t0 = now_ns();
        for (size_t i = 0; i < s.reqs.size(); i++) {
            const phem_request &r = s.reqs[i]->req;
            const phem_batch_graph &g = s.graphs[i];
            s.reqs[i]->res.start_ns = t0;
            if (!r.num_edges)
                continue;
            if (r.kind == PHEM_BATCH_CC)
                PHEM_CUDA_TRY(cudaMemcpyAsync(s.d_pairs + g.edge_offset, r.pairs, 8 * r.num_edges,
                                              cudaMemcpyHostToDevice, st));
            else
                PHEM_CUDA_TRY(cudaMemcpyAsync(d_edges + g.edge_offset, r.edges, 12 * r.num_edges,
                                              cudaMemcpyHostToDevice, st));
        }
        BatchLayout L;
        PHEM_TRY(phem::build_items(s.graphs.data(), (uint32_t)s.graphs.size(), s.edges, s.vertices, &L));
        for (auto &it : L.items)
            if (it.kind == PHEM_BATCH_CC)
                it.kind = phem::kBatchPairs;
        phem_batch_plan *p = s.plan;
        PHEM_CUDA_TRY(cudaEventSynchronize(p->staged));
        std::copy(L.items.begin(), L.items.end(), p->h_items);
        *p->h_num = (uint32_t)L.items.size();
        PHEM_CUDA_TRY(cudaMemcpyAsync(p->buf.items, p->h_items, sizeof(phem::BatchItem) * L.items.size(),
                                      cudaMemcpyHostToDevice, st));
        PHEM_CUDA_TRY(cudaMemcpyAsync(p->buf.num_graphs, p->h_num, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        PHEM_CUDA_TRY(cudaEventRecord(p->staged, st));
        p->num_graphs = (uint32_t)L.items.size();
        p->total_vertices = s.vertices;
        PHEM_TRY(phem_batch_plan_run(p));
        PHEM_CUDA_TRY(cudaEventRecord(s.done, st));
        s.busy = true;
        return PHEM_OK;
    }

    // Results of a finished slot back to its requests.  Writing a request's
    // result (the forest records gathered from its edges by the batch's ids,
    // or its labels) is host work proportional to the result, so the requests
    // of a large batch are split over a few threads: on one thread it capped
    // the batched path at about 40 k small requests per second.
    static constexpr size_t kRetireThreads = 8;
    static constexpr size_t kRetireSerialBelow = 64;  // requests; fewer are finished on this thread

    void retire_range(Slot &s, phem_status st, bool cuda_ok, size_t lo, size_t hi)
    {
        for (size_t i = lo; i < hi; i++) {
            Pending *p = s.reqs[i];
            const phem_batch_graph &g = s.graphs[i];
            phem_status rs = cuda_ok ? phem::ctl_status(s.plan->h_status[i], "serve") : st;
            p->res.path = PHEM_PATH_BATCHED;
            p->res.forest_edges = s.h_count[i];
            p->res.total_weight = p->req.kind == PHEM_BATCH_MSF ? s.h_total[i] : 0;
            if (rs == PHEM_OK) {
                if (p->req.kind == PHEM_BATCH_MSF && p->req.forest) {
                    const uint32_t *ids = s.h_ids + g.vertex_offset;
                    for (uint32_t k = 0; k < s.h_count[i]; k++)
                        p->req.forest[k] = p->req.edges[ids[k]];
                }
                if (p->req.kind == PHEM_BATCH_CC && p->req.labels)
                    std::memcpy(p->req.labels, s.h_labels + g.vertex_offset, 4 * (size_t)g.num_vertices);
            }
            complete(p, rs);
        }
    }

    void retire(Slot &s)
    {
        phem_status st = phem_batch_plan_download(s.plan, s.h_ids, s.h_count, s.h_total, s.h_labels);
        const bool cuda_ok = st == PHEM_OK || st == PHEM_ERR_INVALID || st == PHEM_ERR_NONCONVERGED;
        if (!cuda_ok)
            fatal = st;
        const size_t n = s.reqs.size();
        if (n < kRetireSerialBelow) {
            retire_range(s, st, cuda_ok, 0, n);
        } else {
            std::thread helpers[kRetireThreads - 1];
            for (size_t t = 1; t < kRetireThreads; t++)
                helpers[t - 1] = std::thread([&, t] { retire_range(s, st, cuda_ok, n * t / kRetireThreads,
                                                                   n * (t + 1) / kRetireThreads); });
            retire_range(s, st, cuda_ok, 0, n / kRetireThreads);
            for (auto &h : helpers)
                h.join();
        }
        s.reqs.clear();
        s.graphs.clear();
        s.busy = false;
    }

    void batch_loop()
    {
        DeviceGuardLite dg(device);
        for (;;) {
            bool progressed = false;
            for (auto &s : slots)
                if (s.busy && cudaEventQuery(s.done) != cudaErrorNotReady) {
                    retire(s);
                    progressed = true;
                }
            for (auto &s : slots) {
                if (s.busy)
                    continue;
                {
                    std::lock_guard<std::mutex> lk(mu);
                    // admit in arrival order while the request fits this slot
                    s.edges = 0;
                    s.vertices = 0;
                    while (!small_q.empty() && s.reqs.size() < cfg.max_batch_graphs) {
                        Pending *p = small_q.front();
                        if (s.edges + p->req.num_edges > slot_edges ||
                            (uint64_t)s.vertices + p->req.num_vertices > slot_vertices)
                            break;
                        small_q.pop_front();
                        phem_batch_graph g{};
                        g.edge_offset = s.edges;
                        g.num_edges = (uint32_t)p->req.num_edges;
                        g.num_vertices = p->req.num_vertices;
                        g.vertex_offset = s.vertices;
                        g.kind = p->req.kind;
                        s.graphs.push_back(g);
                        s.reqs.push_back(p);
                        s.edges += p->req.num_edges;
                        s.vertices += p->req.num_vertices;
                    }
                }
                if (s.reqs.empty())
                    continue;
                progressed = true;
                phem_status st = fatal != PHEM_OK ? fatal : launch(s);
                if (st != PHEM_OK) {
                    if (st == PHEM_ERR_CUDA)
                        fatal = st;
                    for (Pending *p : s.reqs)
                        complete(p, st);
                    s.reqs.clear();
                    s.graphs.clear();
                    s.busy = false;
                }
            }
            if (progressed)
                continue;
            std::unique_lock<std::mutex> lk(mu);
            const bool any_busy = std::any_of(slots.begin(), slots.end(), [](const Slot &s) { return s.busy; });
            if (stop && !any_busy && small_q.empty())
                return;
            if (any_busy)
                cv_work.wait_for(lk, std::chrono::microseconds(20));
            else
                cv_work.wait(lk, [&] { return stop || !small_q.empty(); });
        }
    }

    void large_loop(phem_context *ctx)
    {
        DeviceGuardLite dg(device);
        for (;;) {
            Pending *p = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_large.wait(lk, [&] { return stop || !large_q.empty(); });
                if (large_q.empty())
                    return;
                p = large_q.front();
                large_q.pop_front();
            }
            p->res.start_ns = now_ns();
            p->res.path = PHEM_PATH_DEVICE;
            const phem_request &r = p->req;
            phem_status st;
            if (r.kind == PHEM_BATCH_MSF) {
                uint64_t count = 0, total = 0;
                st = phem_msf_solve(ctx, r.edges, r.num_edges, r.num_vertices, r.forest, &count, &total, nullptr);
                p->res.forest_edges = count;
                p->res.total_weight = total;
            } else {
                std::vector<int32_t> scratch;
                int32_t *labels = r.labels;
                if (!labels) {
                    scratch.resize(r.num_vertices);
                    labels = scratch.data();
                }
                phem_cc_stats cs{};
                st = phem_cc_solve(ctx, r.pairs, (int64_t)r.num_edges, (int32_t)r.num_vertices, labels, nullptr,
                                   PHEM_CC_DEFAULT, &cs);
                p->res.forest_edges = cs.forest_edges;
            }
            complete(p, st);
        }
    }

    // Makes the server's device current in a worker thread.
    struct DeviceGuardLite {
        explicit DeviceGuardLite(int dev) { cudaSetDevice(dev); }
    };
};

namespace {

void server_free(phem_server *s)
{
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    s->cv_large.notify_all();
    for (auto &t : s->threads)
        t.join();
    cudaSetDevice(s->device);
    for (auto &sl : s->slots) {
        if (sl.plan)
            phem_batch_plan_destroy(sl.plan);
        if (sl.d_pairs)
            cudaFree(sl.d_pairs);
        if (sl.done)
            cudaEventDestroy(sl.done);
        if (sl.h_ids)
            cudaFreeHost(sl.h_ids);
        if (sl.h_count)
            cudaFreeHost(sl.h_count);
        if (sl.h_total)
            cudaFreeHost(sl.h_total);
        if (sl.h_labels)
            cudaFreeHost(sl.h_labels);
        if (sl.ctx)
            phem_context_destroy(sl.ctx);
    }
    for (auto *c : s->large_ctx)
        phem_context_destroy(c);
    for (auto &kv : s->live)
        delete kv.second;
    delete s;
}

}  // namespace

extern "C" {

phem_status phem_server_create(int device, const phem_server_config *cfg, phem_server **out)
{
    if (!cfg || !out) {
        phem::set_error("server_create: null argument");
        return PHEM_ERR_INVALID;
    }
    *out = nullptr;
    if (cfg->slots < 1 || cfg->slots > 8 || cfg->large_workers < 1 || cfg->large_workers > 8 ||
        cfg->max_batch_graphs < 1 || cfg->large_edges < 1 || cfg->large_edges >= (1ull << 32)) {
        phem::set_error("server_create: need 1..8 slots, 1..8 large workers, max_batch_graphs >= 1, "
                        "1 <= large_edges < 2^32");
        return PHEM_ERR_INVALID;
    }
    auto *s = new phem_server();
    s->device = device;
    s->cfg = *cfg;
    // half of the budget for the batch slots: per edge 12 B input + 8 B pairs
    // + 16 B list + bitmap; per vertex 20 B state + 8 B outputs, sized with
    // one vertex per edge
    const uint64_t per_edge = 12 + 8 + 16 + 1 + 28;
    uint64_t e = cfg->memory_budget / 2 / cfg->slots / per_edge;
    e = std::min<uint64_t>(e, 1ull << 26);
    s->slot_edges = std::max<uint64_t>(e, cfg->large_edges);
    s->slot_vertices = (uint32_t)std::min<uint64_t>(s->slot_edges, 0xffffffffu);
    const uint64_t slot_bytes = per_edge * s->slot_edges * cfg->slots;
    if (slot_bytes > cfg->memory_budget) {
        phem::set_error("server_create: budget of %llu bytes cannot hold %u slots of large_edges = %llu",
                        (unsigned long long)cfg->memory_budget, cfg->slots, (unsigned long long)cfg->large_edges);
        delete s;
        return PHEM_ERR_INVALID;
    }
    s->large_share = (cfg->memory_budget - slot_bytes) / cfg->large_workers;
    phem_status st = PHEM_OK;
    s->slots.resize(cfg->slots);
    for (auto &sl : s->slots) {
        if (st == PHEM_OK)
            st = phem_context_create(device, &sl.ctx);
        if (st == PHEM_OK)
            st = phem_batch_plan_create(sl.ctx, cfg->max_batch_graphs, s->slot_edges, s->slot_vertices, &sl.plan);
        if (st == PHEM_OK && (cudaMalloc(&sl.d_pairs, 8 * s->slot_edges) != cudaSuccess ||
                              cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
                              cudaMallocHost(&sl.h_ids, 4 * (size_t)s->slot_vertices) != cudaSuccess ||
                              cudaMallocHost(&sl.h_labels, 4 * (size_t)s->slot_vertices) != cudaSuccess ||
                              cudaMallocHost(&sl.h_count, 4 * (size_t)cfg->max_batch_graphs) != cudaSuccess ||
                              cudaMallocHost(&sl.h_total, 8 * (size_t)cfg->max_batch_graphs) != cudaSuccess)) {
            cudaGetLastError();
            phem::set_error("server_create: cannot allocate slot buffers");
            st = PHEM_ERR_NOMEM;
        }
    }
    for (uint32_t k = 0; st == PHEM_OK && k < cfg->large_workers; k++) {
        phem_context *c = nullptr;
        st = phem_context_create(device, &c);
        if (st == PHEM_OK)
            s->large_ctx.push_back(c);
    }
    // re-capture every slot's launch with its CC pairs buffer wired in
    for (auto &sl : s->slots) {
        if (st != PHEM_OK)
            break;
        st = phem::batch_plan_capture(sl.plan, sl.d_pairs);
    }
    if (st != PHEM_OK) {
        server_free(s);
        return st;
    }
    s->threads.emplace_back([s] { s->batch_loop(); });
    for (auto *c : s->large_ctx)
        s->threads.emplace_back([s, c] { s->large_loop(c); });
    *out = s;
    return PHEM_OK;
}

void phem_server_destroy(phem_server *s)
{
    if (s)
        server_free(s);
}

phem_status phem_server_submit(phem_server *s, const phem_request *req, uint64_t *ticket)
{
    if (!s || !req || !ticket) {
        phem::set_error("server_submit: null argument");
        return PHEM_ERR_INVALID;
    }
    const phem_request &r = *req;
    if ((r.kind != PHEM_BATCH_MSF && r.kind != PHEM_BATCH_CC) || r.num_vertices == 0 ||
        r.num_vertices > 0x7fffffffu || r.num_edges >= (1ull << 32) - (1ull << 24) ||
        (r.num_edges && r.kind == PHEM_BATCH_MSF && !r.edges) || (r.num_edges && r.kind == PHEM_BATCH_CC && !r.pairs)) {
        phem::set_error("server_submit: bad request (kind, 0 < n < 2^31, m < 2^32 - 2^24, input array)");
        return PHEM_ERR_INVALID;
    }
    const bool small = r.num_edges <= s->cfg.large_edges && r.num_edges <= s->slot_edges &&
                       r.num_vertices <= s->slot_vertices;
    if (!small && large_bytes(r) > s->large_share) {
        phem::set_error("server_submit: request (n = %u, m = %llu) needs more than the %llu device bytes a "
                        "worker may hold",
                        r.num_vertices, (unsigned long long)r.num_edges, (unsigned long long)s->large_share);
        return PHEM_ERR_NOMEM;
    }
    auto *p = new Pending();
    p->req = r;
    p->res.submit_ns = now_ns();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        p->ticket = s->next_ticket++;
        s->live[p->ticket] = p;
        (small ? s->small_q : s->large_q).push_back(p);
    }
    (small ? s->cv_work : s->cv_large).notify_one();
    *ticket = p->ticket;
    return PHEM_OK;
}

phem_status phem_server_wait(phem_server *s, uint64_t ticket, uint32_t timeout_ms, phem_request_result *res)
{
    if (!s || !res) {
        phem::set_error("server_wait: null argument");
        return PHEM_ERR_INVALID;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->live.find(ticket);
    if (it == s->live.end()) {
        phem::set_error("server_wait: unknown ticket %llu", (unsigned long long)ticket);
        return PHEM_ERR_INVALID;
    }
    Pending *p = it->second;
    auto ready = [&] { return p->done; };
    if (timeout_ms == 0)
        s->cv_done.wait(lk, ready);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        phem::set_error("server_wait: request %llu not done after %u ms", (unsigned long long)ticket, timeout_ms);
        return PHEM_ERR_TIMEOUT;
    }
    *res = p->res;
    s->live.erase(it);
    lk.unlock();
    delete p;
    return PHEM_OK;
}

phem_status phem_server_replay(phem_server *s, const phem_request *reqs, const uint64_t *arrival_ns, uint32_t count,
                               phem_request_result *results)
{
    if (!s || (count && (!reqs || !arrival_ns || !results))) {
        phem::set_error("server_replay: null argument");
        return PHEM_ERR_INVALID;
    }
    std::vector<uint64_t> tickets(count, 0);
    std::vector<phem_status> sub(count, PHEM_OK);
    const uint64_t t0 = now_ns();
    for (uint32_t i = 0; i < count; i++) {
        const uint64_t due = t0 + arrival_ns[i];
        for (;;) {  // open-loop arrivals: sleep while far, spin when close
            const uint64_t t = now_ns();
            if (t >= due)
                break;
            if (due - t > 200000)
                std::this_thread::sleep_for(std::chrono::nanoseconds(due - t - 100000));
        }
        sub[i] = phem_server_submit(s, &reqs[i], &tickets[i]);
    }
    phem_status first = PHEM_OK;
    for (uint32_t i = 0; i < count; i++) {
        if (sub[i] != PHEM_OK) {
            results[i] = phem_request_result{};
            results[i].status = sub[i];
            if (first == PHEM_OK)
                first = sub[i];
            continue;
        }
        PHEM_TRY(phem_server_wait(s, tickets[i], 0, &results[i]));
    }
    return first;
}

}  // extern "C"
