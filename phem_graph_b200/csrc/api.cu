// api.cu -- the C ABI of libphem.so (include/phem.h).
//
// Host orchestration only: argument checks, the context (stream, grow-only
// workspace, control block), staging of host arrays through the workspace,
// and the mapping of device status bits to phem_status.  No graph arithmetic
// happens here and there is no CPU path: without a usable sm_100 device every
// solve fails with PHEM_ERR_NO_DEVICE.
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <thread>

#include "internal.h"

namespace phem {

namespace {
thread_local char g_last_error[512] = "";

}  // namespace

const char *const kKernelNames[kKernelCount] = {
    "msf_init", "msf_select", "msf_edge_pass", "msf_hook", "msf_compress", "msf_advance", "msf_gather",
    "cc_init", "cc_unite", "cc_merge", "cc_label", "cc_minid", "cc_count", "csr_to_coo", "batch_solve"};

constexpr size_t kLaunchLogCap = 1u << 16;

static cudaEvent_t pool_get(phem_context *ctx)
{
    if (!ctx->event_pool.empty()) {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

KernelScope::KernelScope(phem_context *c, int k) : ctx(c), kernel(k)
{
    ctx->launches[k]++;
    if (ctx->profiling) {
        start = pool_get(ctx);
        if (start)
            cudaEventRecord(start, ctx->stream);
    }
}

KernelScope::~KernelScope()
{
    if (!start)
        return;
    cudaEvent_t stop = pool_get(ctx);
    if (!stop) {
        ctx->event_pool.push_back(start);
        return;
    }
    cudaEventRecord(stop, ctx->stream);
    ctx->pending.push_back({kernel, start, stop});
}

void resolve_timings(phem_context *ctx)
{
    for (auto &p : ctx->pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.stop) == cudaSuccess && cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
            ctx->kernel_ms[p.kernel] += ms;
            ctx->timed_launches[p.kernel]++;
            if (ctx->launch_log.size() < kLaunchLogCap)
                ctx->launch_log.emplace_back(p.kernel, ms);
        }
        ctx->event_pool.push_back(p.start);
        ctx->event_pool.push_back(p.stop);
    }
    ctx->pending.clear();
}

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

bool is_device_ptr(const void *p)
{
    if (!p)
        return false;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();  // clear the sticky-free error from an unknown pointer
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

bool is_device_ptr_on(const void *p, int dev)
{
    if (!p)
        return false;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) && attr.device == dev;
}

uint64_t next_epochs(phem_context *ctx, uint32_t count)
{
    // Epochs are stored in 30 bits of a status word.  Before they wrap the
    // status array is cleared so that no word from an old launch can match.
    if (((ctx->epoch + count) >> 30) != (ctx->epoch >> 30) || ctx->epoch + count >= (1ull << 30)) {
        if (ctx->status && ctx->status_words)
            cudaMemsetAsync(ctx->status, 0, ctx->status_words * sizeof(uint64_t), ctx->stream);
        ctx->epoch = 1;
    }
    const uint64_t e = ctx->epoch;
    ctx->epoch += count;
    return e;
}

// Grows a grow-only device buffer to at least `bytes` (contents are not kept).
static phem_status grow_buffer(phem_context *ctx, void **buf, size_t *have, size_t bytes, const char *what)
{
    if (bytes <= *have)
        return PHEM_OK;
    PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (*buf) {
        cudaFree(*buf);
        *buf = nullptr;
        *have = 0;
    }
    const size_t want = bytes + bytes / 8;  // some headroom against small growth steps
    if (cudaMalloc(buf, want) != cudaSuccess) {
        cudaGetLastError();
        if (cudaMalloc(buf, bytes) != cudaSuccess) {
            cudaGetLastError();
            *buf = nullptr;
            set_error("%s: cannot allocate %zu bytes", what, bytes);
            return PHEM_ERR_NOMEM;
        }
        *have = bytes;
        return PHEM_OK;
    }
    *have = want;
    return PHEM_OK;
}

phem_status ws_reserve(phem_context *ctx, size_t bytes)
{
    return grow_buffer(ctx, &ctx->ws, &ctx->ws_bytes, bytes, "workspace");
}

phem_status input_reserve(phem_context *ctx, size_t bytes)
{
    return grow_buffer(ctx, &ctx->input, &ctx->input_bytes, bytes, "converted input");
}

phem_status status_reserve(phem_context *ctx, size_t words)
{
    if (words <= ctx->status_words)
        return PHEM_OK;
    PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->status)
        cudaFree(ctx->status);
    ctx->status = nullptr;
    ctx->status_words = 0;
    const size_t want = words + words / 8 + 64;
    if (cudaMalloc(&ctx->status, want * sizeof(uint64_t)) != cudaSuccess) {
        cudaGetLastError();
        ctx->status = nullptr;
        set_error("look-back status: cannot allocate %zu words", want);
        return PHEM_ERR_NOMEM;
    }
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->status, 0, want * sizeof(uint64_t), ctx->stream));
    ctx->status_words = want;
    return PHEM_OK;
}

phem_status stream_wait(phem_context *ctx)
{
    if (!ctx->timeout_ms) {
        PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        resolve_timings(ctx);
        return PHEM_OK;
    }
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(ctx->timeout_ms);
    for (;;) {
        cudaError_t e = cudaStreamQuery(ctx->stream);
        if (e == cudaSuccess) {
            resolve_timings(ctx);
            return PHEM_OK;
        }
        if (e != cudaErrorNotReady) {
            set_error("stream: %s", cudaGetErrorString(e));
            return PHEM_ERR_CUDA;
        }
        if (std::chrono::steady_clock::now() > deadline) {
            set_error("watchdog: work not finished after %u ms", ctx->timeout_ms);
            return PHEM_ERR_TIMEOUT;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

phem_status ctl_status(uint32_t err, const char *what)
{
    if (!err)
        return PHEM_OK;
    if (err & kErrRange) {
        set_error("%s: an edge endpoint is >= n", what);
        return PHEM_ERR_INVALID;
    }
    set_error("%s: device loop bound reached (status bits 0x%x)", what, err);
    return PHEM_ERR_NONCONVERGED;
}

namespace {

// Edge ids and survivor-list positions are 32-bit; a survivor list holds the
// edges plus up to 2^24 records of padding.
constexpr uint64_t kMaxEdges = (1ull << 32) - (1ull << 24);

}  // namespace
}  // namespace phem

using namespace phem;

extern "C" {

int phem_version(void) { return PHEM_VERSION; }

const char *phem_last_error(void) { return g_last_error; }

const char *phem_status_string(phem_status s)
{
    switch (s) {
    case PHEM_OK: return "ok";
    case PHEM_ERR_INVALID: return "invalid argument";
    case PHEM_ERR_CUDA: return "CUDA error";
    case PHEM_ERR_NOMEM: return "out of memory";
    case PHEM_ERR_NONCONVERGED: return "device loop bound reached";
    case PHEM_ERR_TIMEOUT: return "watchdog timeout";
    case PHEM_ERR_UNSUPPORTED: return "unsupported";
    case PHEM_ERR_NO_DEVICE: return "no sm_100 device";
    }
    return "unknown status";
}

phem_status phem_context_create(int device, phem_context **out)
{
    if (!out) {
        set_error("null output pointer");
        return PHEM_ERR_INVALID;
    }
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        set_error("device %d not available (%d CUDA devices)", device, count);
        return PHEM_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    PHEM_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return PHEM_ERR_NO_DEVICE;
    }
    DeviceGuard g(device);
    phem_context *c = new phem_context();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    auto fail = [&](const char *what) {
        set_error("context: %s failed: %s", what, cudaGetErrorString(cudaGetLastError()));
        phem_context_destroy(c);
        return PHEM_ERR_CUDA;
    };
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail("stream");
    if (cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail("copy stream");
    c->stream = c->own_stream;
    if (cudaMalloc(&c->ctl, sizeof(Ctl)) != cudaSuccess)
        return fail("control block");
    if (cudaMallocHost(&c->h_ctl, sizeof(Ctl)) != cudaSuccess)
        return fail("pinned control block");
    if (cudaEventCreate(&c->ev_start) != cudaSuccess || cudaEventCreate(&c->ev_stop) != cudaSuccess)
        return fail("events");
    if (cudaMemset(c->ctl, 0, sizeof(Ctl)) != cudaSuccess)
        return fail("control block init");
    *out = c;
    return PHEM_OK;
}

void phem_context_destroy(phem_context *ctx)
{
    if (!ctx)
        return;
    DeviceGuard g(ctx->device);
    if (ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    for (auto &e : ctx->msf_exec)
        if (e)
            cudaGraphExecDestroy(e);
    if (ctx->ws)
        cudaFree(ctx->ws);
    if (ctx->input)
        cudaFree(ctx->input);
    if (ctx->status)
        cudaFree(ctx->status);
    if (ctx->ctl)
        cudaFree(ctx->ctl);
    if (ctx->h_ctl)
        cudaFreeHost(ctx->h_ctl);
    if (ctx->ev_start)
        cudaEventDestroy(ctx->ev_start);
    if (ctx->ev_stop)
        cudaEventDestroy(ctx->ev_stop);
    for (auto &p : ctx->pending) {
        cudaEventDestroy(p.start);
        cudaEventDestroy(p.stop);
    }
    for (auto e : ctx->event_pool)
        cudaEventDestroy(e);
    if (ctx->copy_stream)
        cudaStreamSynchronize(ctx->copy_stream);
    for (int b = 0; b < 2; b++) {
        if (ctx->ccs.buf[b])
            cudaFree(ctx->ccs.buf[b]);
        if (ctx->ccs.copied[b])
            cudaEventDestroy(ctx->ccs.copied[b]);
        if (ctx->ccs.freed[b])
            cudaEventDestroy(ctx->ccs.freed[b]);
    }
    if (ctx->ccs.t0)
        cudaEventDestroy(ctx->ccs.t0);
    if (ctx->ccs.t1)
        cudaEventDestroy(ctx->ccs.t1);
    if (ctx->copy_stream)
        cudaStreamDestroy(ctx->copy_stream);
    if (ctx->own_stream)
        cudaStreamDestroy(ctx->own_stream);
    delete ctx;
}

phem_status phem_context_set_stream(phem_context *ctx, void *stream)
{
    PHEM_TRY(check_ctx(ctx));
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return PHEM_OK;
}

void *phem_context_stream(phem_context *ctx) { return ctx ? ctx->stream : nullptr; }

phem_status phem_context_set_timeout_ms(phem_context *ctx, uint32_t ms)
{
    PHEM_TRY(check_ctx(ctx));
    ctx->timeout_ms = ms;
    return PHEM_OK;
}

phem_status phem_context_set_profiling(phem_context *ctx, int on)
{
    PHEM_TRY(check_ctx(ctx));
    ctx->profiling = on != 0;
    return PHEM_OK;
}

phem_status phem_context_profile(phem_context *ctx, phem_kernel_profile *out, uint32_t max, uint32_t *count)
{
    PHEM_TRY(check_ctx(ctx));
    DeviceGuard g(ctx->device);
    PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    resolve_timings(ctx);
    uint32_t k = 0;
    for (int i = 0; i < kKernelCount; i++) {
        if (!ctx->launches[i])
            continue;
        if (out && k < max) {
            std::memset(&out[k], 0, sizeof(out[k]));
            std::snprintf(out[k].name, sizeof(out[k].name), "%s", kKernelNames[i]);
            out[k].launches = ctx->launches[i];
            out[k].timed_launches = ctx->timed_launches[i];
            out[k].total_ms = ctx->kernel_ms[i];
        }
        k++;
    }
    if (count)
        *count = k;
    return PHEM_OK;
}

phem_status phem_context_profile_reset(phem_context *ctx)
{
    PHEM_TRY(check_ctx(ctx));
    DeviceGuard g(ctx->device);
    PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    resolve_timings(ctx);
    for (int i = 0; i < kKernelCount; i++) {
        ctx->launches[i] = 0;
        ctx->timed_launches[i] = 0;
        ctx->kernel_ms[i] = 0;
    }
    ctx->launch_log.clear();
    return PHEM_OK;
}

phem_status phem_context_launch_log(phem_context *ctx, phem_launch_record *out, uint32_t max, uint32_t *count)
{
    PHEM_TRY(check_ctx(ctx));
    DeviceGuard g(ctx->device);
    PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    resolve_timings(ctx);
    const uint32_t n = (uint32_t)ctx->launch_log.size();
    for (uint32_t i = 0; out && i < n && i < max; i++) {
        std::memset(&out[i], 0, sizeof(out[i]));
        std::snprintf(out[i].name, sizeof(out[i].name), "%s", kKernelNames[ctx->launch_log[i].first]);
        out[i].ms = ctx->launch_log[i].second;
    }
    if (count)
        *count = n;
    return PHEM_OK;
}

phem_status phem_context_set_tuning(phem_context *ctx, const char *key, double value)
{
    PHEM_TRY(check_ctx(ctx));
    if (!key) {
        set_error("set_tuning: null key");
        return PHEM_ERR_INVALID;
    }
    const std::string k(key);
    if (k == "msf.light_per_vertex" && value >= 0 && value < 1e6) {
        ctx->tune_light_per_vertex = value;
    } else if (k == "msf.filter_min_ratio" && value >= 1.0 && value < 1e6) {
        ctx->tune_filter_min_ratio = value;
    } else if (k == "msf.first_batch" && value >= 1 && value <= PHEM_MAX_ROUNDS) {
        ctx->tune_first_batch = (int)value;
    } else if (k == "msf.next_batch" && value >= 1 && value <= PHEM_MAX_ROUNDS) {
        ctx->tune_next_batch = (int)value;
    } else if (k == "msf.graph" && (value == 0 || value == 1)) {
        ctx->tune_graph = (int)value;
    } else if (k == "msf.edge_ctas_per_sm" && value >= 1 && value <= 4 && value == (int)value) {
        ctx->tune_edge_ctas = (int)value;
        ctx->kernels_ready = 0;  // the grid size is recomputed at the next solve
    } else if (k == "cc.canonical_light_per_vertex" && value >= 0 && value < 1e6) {
        ctx->tune_canonical_light = value;
    } else if (k == "cc.sample_per_vertex" && value >= 0.0 && value < 1e6) {
        ctx->tune_cc_sample = value;
    } else if (k == "batch.block_size" && (value == 256 || value == 512 || value == 1024)) {
        ctx->tune_batch_block = (int)value;
    } else if (k == "batch.items" && (value == 1 || value == 2 || value == 4)) {
        ctx->tune_batch_items = (int)value;
    } else if (k == "batch.compact_ratio" && value >= 0.0 && value <= 1.0) {
        ctx->tune_batch_compact = value;
    } else {
        set_error("set_tuning: unknown key or value out of range: %s = %g", key, value);
        return PHEM_ERR_INVALID;
    }
    return PHEM_OK;
}

phem_status phem_context_get_tuning(phem_context *ctx, const char *key, double *value)
{
    PHEM_TRY(check_ctx(ctx));
    if (!key || !value) {
        set_error("get_tuning: null argument");
        return PHEM_ERR_INVALID;
    }
    const std::string k(key);
    if (k == "msf.light_per_vertex")
        *value = ctx->tune_light_per_vertex;
    else if (k == "msf.filter_min_ratio")
        *value = ctx->tune_filter_min_ratio;
    else if (k == "cc.canonical_light_per_vertex")
        *value = ctx->tune_canonical_light;
    else if (k == "msf.first_batch")
        *value = ctx->tune_first_batch;
    else if (k == "msf.next_batch")
        *value = ctx->tune_next_batch;
    else if (k == "msf.graph")
        *value = ctx->tune_graph;
    else if (k == "msf.edge_ctas_per_sm")
        *value = ctx->tune_edge_ctas;
    else if (k == "cc.sample_per_vertex")
        *value = ctx->tune_cc_sample;
    else if (k == "batch.block_size")
        *value = ctx->tune_batch_block;
    else if (k == "batch.items")
        *value = ctx->tune_batch_items;
    else if (k == "batch.compact_ratio")
        *value = ctx->tune_batch_compact;
    else {
        set_error("get_tuning: unknown key %s", key);
        return PHEM_ERR_INVALID;
    }
    return PHEM_OK;
}

phem_status phem_context_trim(phem_context *ctx)
{
    PHEM_TRY(check_ctx(ctx));
    DeviceGuard g(ctx->device);
    PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ctx->ws)
        cudaFree(ctx->ws);
    ctx->ws = nullptr;
    ctx->ws_bytes = 0;
    if (ctx->input)
        cudaFree(ctx->input);
    ctx->input = nullptr;
    ctx->input_bytes = 0;
    return PHEM_OK;
}

// ------------------------------------------------------------------ CC

// Host edges of at least this many are copied in chunks overlapped with the
// unions (smaller inputs: one copy, then the unions).
constexpr int64_t kOverlapMinEdges = 1 << 20;
constexpr int64_t kOverlapChunkEdges = 1 << 21;  // 16 MB per copy

// The default CC schedule (unite [0, s), compress, unite [s, m)) over host
// edges: chunks are copied into d_stage on the copy stream, and each chunk's
// union waits only for its own copy, so the link and the unions overlap.
// Chunk boundaries are even, keeping every chunk 16-byte aligned for the
// union's 128-bit loads.
static phem_status cc_unite_overlapped(phem_context *ctx, const uint64_t *h_edges, uint64_t *d_stage, int64_t m,
                                       int64_t s, int32_t n, int32_t *d_par, uint64_t *d_for)
{
    std::vector<std::pair<int64_t, int64_t>> chunks;  // (offset, count)
    for (int64_t off = 0; off < s; off += kOverlapChunkEdges)
        chunks.emplace_back(off, std::min(kOverlapChunkEdges, s - off));
    const size_t prefix_chunks = chunks.size();
    for (int64_t off = s; off < m; off += kOverlapChunkEdges)
        chunks.emplace_back(off, std::min(kOverlapChunkEdges, m - off));
    std::vector<cudaEvent_t> copied(chunks.size() + 1, nullptr);
    phem_status st = PHEM_OK;
    for (auto &e : copied)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            e = nullptr;
            set_error("cc_solve: cannot create copy events");
            st = PHEM_ERR_CUDA;
        }
    // the first copy waits for earlier work on the context stream, which may
    // still read the staging area
    if (st == PHEM_OK && (cudaEventRecord(copied.back(), ctx->stream) != cudaSuccess ||
                          cudaStreamWaitEvent(ctx->copy_stream, copied.back(), 0) != cudaSuccess)) {
        set_error("cc_solve: cannot order the copy stream");
        st = PHEM_ERR_CUDA;
    }
    for (size_t c = 0; st == PHEM_OK && c < chunks.size(); c++) {
        const int64_t off = chunks[c].first, cnt = chunks[c].second;
        if (cudaMemcpyAsync(d_stage + off, h_edges + off, (size_t)cnt * sizeof(uint64_t), cudaMemcpyDefault,
                            ctx->copy_stream) != cudaSuccess ||
            cudaEventRecord(copied[c], ctx->copy_stream) != cudaSuccess ||
            cudaStreamWaitEvent(ctx->stream, copied[c], 0) != cudaSuccess) {
            set_error("cc_solve: chunk copy failed: %s", cudaGetErrorString(cudaGetLastError()));
            st = PHEM_ERR_CUDA;
            break;
        }
        st = cc_launch_unite(ctx, d_stage + off, cnt, n, d_par, d_for);
        if (st == PHEM_OK && c + 1 == prefix_chunks && s < m)
            st = cc_launch_compress(ctx, n, d_par);
    }
    if (st != PHEM_OK)
        cudaStreamSynchronize(ctx->copy_stream);  // no copy may still land in the workspace
    for (auto e : copied)
        if (e)
            cudaEventDestroy(e);  // released once the work recorded on it completes
    return st;
}

phem_status phem_cc_solve(phem_context *ctx, const uint64_t *edges, int64_t m, int32_t n, int32_t *labels,
                          uint64_t *forest, uint32_t flags, phem_cc_stats *stats)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || m < 0 || (m > 0 && !edges) || !labels) {
        set_error("cc_solve: need n > 0, m >= 0, edges and labels");
        return PHEM_ERR_INVALID;
    }
    const bool canonical = flags & PHEM_CC_CANONICAL;
    if (canonical && (uint64_t)m > kMaxEdges) {
        set_error("cc_solve: canonical forest needs m <= 2^32 - 2^24");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    const size_t eb = (size_t)m * sizeof(uint64_t), lb = (size_t)n * sizeof(int32_t),
                 fb = (size_t)n * sizeof(uint64_t);
    // extra area: staged edges | labels | forest | parent (default path)
    const size_t o_edges = 0, o_lab = align256(eb), o_for = o_lab + align256(lb), o_par = o_for + align256(fb);
    const size_t extra = o_par + align256(lb);
    size_t base = 0;
    MsfPlan plan;
    if (canonical) {
        PHEM_TRY(msf_plan(ctx, kKindPacked, nullptr, (uint64_t)m, (uint32_t)n, extra, &plan, &base));
    } else {
        PHEM_TRY(ws_reserve(ctx, extra));
    }
    Staged se, sl, sf;
    const bool on_device = is_device_ptr(edges);
    const bool aligned_dev = on_device && (((uintptr_t)edges & 15) == 0);
    // large host inputs of the default path are copied in chunks, overlapped
    // with the unions of the chunks before them
    const bool overlap = !canonical && !on_device && m >= kOverlapMinEdges;
    if (aligned_dev) {
        se.dev = const_cast<uint64_t *>(edges);
    } else {
        se.dev = static_cast<char *>(ctx->ws) + base + o_edges;
        if (m && !overlap)
            PHEM_CUDA_TRY(cudaMemcpyAsync(se.dev, edges, eb, cudaMemcpyDefault, ctx->stream));
    }
    stage_out(ctx, labels, lb, base + o_lab, &sl);
    stage_out(ctx, forest, fb, base + o_for, &sf);
    const uint64_t *d_edges = static_cast<const uint64_t *>(se.dev);
    int32_t *d_lab = static_cast<int32_t *>(sl.dev);
    uint64_t *d_for = static_cast<uint64_t *>(sf.dev);

    Timed timer(ctx);
    uint32_t rounds = 0;
    if (canonical) {
        plan.e0 = d_edges;
        plan.forest = d_for;
        PHEM_TRY(msf_run(ctx, kKindPacked, plan, &rounds));
        // plan.best is free after the rounds: reuse it as the per-root min-id array
        PHEM_TRY(cc_launch_minid_labels(ctx, n, plan.parent, reinterpret_cast<uint32_t *>(plan.best), d_lab));
    } else {
        int32_t *d_par = reinterpret_cast<int32_t *>(static_cast<char *>(ctx->ws) + base + o_par);
        PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), ctx->stream));
        PHEM_TRY(cc_launch_init(ctx, n, d_par, nullptr, d_for));
        // a prefix sample of about tune_cc_sample edges per vertex builds the
        // big components, a compress points every vertex at its root, and
        // the remaining edges then mostly settle with two loads
        int64_t s = (int64_t)(ctx->tune_cc_sample * (double)n) & ~int64_t(1);
        if (s <= 0 || s >= m)
            s = m;
        if (overlap) {
            PHEM_TRY(cc_unite_overlapped(ctx, edges, const_cast<uint64_t *>(d_edges), m, s, n, d_par, d_for));
        } else {
            PHEM_TRY(cc_launch_unite(ctx, d_edges, s, n, d_par, d_for));
            if (s < m) {
                PHEM_TRY(cc_launch_compress(ctx, n, d_par));
                PHEM_TRY(cc_launch_unite(ctx, d_edges + s, m - s, n, d_par, d_for));
            }
        }
        PHEM_TRY(cc_launch_label(ctx, n, d_par, d_lab));
    }
    const float ms = timer.stop();
    PHEM_CUDA_TRY(cudaMemsetAsync(&ctx->ctl->misc[0], 0, 2 * sizeof(unsigned long long), ctx->stream));
    PHEM_TRY(cc_launch_count(ctx, n, d_lab, d_for));
    PHEM_TRY(copy_back(ctx, sl, lb));
    PHEM_TRY(copy_back(ctx, sf, fb));
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(ctl_status(ctx->h_ctl->err, "cc_solve"));
    if (stats) {
        stats->components = (uint32_t)ctx->h_ctl->misc[0];
        stats->forest_edges = d_for ? ctx->h_ctl->misc[1] : (uint64_t)n - ctx->h_ctl->misc[0];
        stats->rounds = rounds;
        stats->device_ms = ms;
    }
    return PHEM_OK;
}

phem_status phem_cc_init(phem_context *ctx, int32_t n, int32_t *d_parent, int32_t *d_label, uint64_t *d_forest)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || !d_parent) {
        set_error("cc_init: need n > 0 and a parent array");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    return cc_launch_init(ctx, n, d_parent, d_label, d_forest);
}

phem_status phem_cc_unite(phem_context *ctx, const uint64_t *d_edges, int64_t m, int32_t n, int32_t *d_parent,
                          uint64_t *d_forest)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || m < 0 || !d_parent || (m > 0 && !d_edges) || ((uintptr_t)d_edges & 15)) {
        set_error("cc_unite: need n > 0, m >= 0, 16-byte aligned device edges");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    return cc_launch_unite(ctx, d_edges, m, n, d_parent, d_forest);
}

phem_status phem_cc_label(phem_context *ctx, int32_t n, int32_t *d_parent, int32_t *d_label)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || !d_parent || !d_label) {
        set_error("cc_label: need n > 0, parent and label arrays");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    return cc_launch_label(ctx, n, d_parent, d_label);
}

phem_status phem_cc_stream(phem_context *ctx, const uint64_t *h_edges, int64_t m, int32_t n, int64_t batch,
                           int32_t *d_parent, int32_t *d_label, uint64_t *d_forest, float *ms)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || m < 0 || batch <= 0 || !d_parent || (m > 0 && !h_edges)) {
        set_error("cc_stream: need n > 0, m >= 0, batch > 0, parent array");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    constexpr int kBuffers = 3;
    const size_t bb = align256((size_t)batch * sizeof(uint64_t));
    PHEM_TRY(ws_reserve(ctx, bb * kBuffers));
    cudaEvent_t copied[kBuffers], freed[kBuffers];
    for (int b = 0; b < kBuffers; b++) {
        PHEM_CUDA_TRY(cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming));
        PHEM_CUDA_TRY(cudaEventCreateWithFlags(&freed[b], cudaEventDisableTiming));
    }
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), ctx->stream));
    PHEM_TRY(cc_launch_init(ctx, n, d_parent, d_label, d_forest));
    Timed timer(ctx);
    // Copies run on the copy stream, unions on the context stream.  Buffer b is
    // refilled only after the union that read it has finished (freed[b]; an
    // event that was never recorded does not block), and a union starts only
    // after its copy (copied[b]).  The first copy waits for the timer start.
    PHEM_CUDA_TRY(cudaEventRecord(copied[0], ctx->stream));
    PHEM_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, copied[0], 0));
    int64_t k = 0;
    for (int64_t off = 0; off < m; off += batch, k++) {
        const int b = (int)(k % kBuffers);
        const int64_t cnt = std::min<int64_t>(batch, m - off);
        uint64_t *buf = reinterpret_cast<uint64_t *>(static_cast<char *>(ctx->ws) + bb * b);
        PHEM_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, freed[b], 0));
        PHEM_CUDA_TRY(cudaMemcpyAsync(buf, h_edges + off, (size_t)cnt * sizeof(uint64_t), cudaMemcpyDefault,
                                      ctx->copy_stream));
        PHEM_CUDA_TRY(cudaEventRecord(copied[b], ctx->copy_stream));
        PHEM_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, copied[b], 0));
        PHEM_TRY(cc_launch_unite(ctx, buf, cnt, n, d_parent, d_forest));
        PHEM_CUDA_TRY(cudaEventRecord(freed[b], ctx->stream));
    }
    const float t = timer.stop();
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    phem_status st = stream_wait(ctx);
    for (int b = 0; b < kBuffers; b++) {
        cudaEventDestroy(copied[b]);
        cudaEventDestroy(freed[b]);
    }
    PHEM_TRY(st);
    PHEM_TRY(ctl_status(ctx->h_ctl->err, "cc_stream"));
    if (ms)
        *ms = t;
    return PHEM_OK;
}

// Incremental SpanningTree: the batches of phem_cc_stream, handed over one
// call at a time.  Host batches go through two staging buffers: batch k is
// copied on the copy stream once the union that read its buffer (batch k - 2)
// has finished, the union waits for its copy, and push returns when the copy
// has landed, so the caller may refill its own buffer while the union runs.
phem_status phem_cc_stream_begin(phem_context *ctx, int32_t n, int32_t *d_parent, int32_t *d_label,
                                 uint64_t *d_forest)
{
    PHEM_TRY(check_ctx(ctx));
    if (ctx->ccs.active) {
        set_error("cc_stream_begin: a stream is already open on this context (end it first)");
        return PHEM_ERR_INVALID;
    }
    if (n <= 0 || !d_parent || !is_device_ptr_on(d_parent, ctx->device) ||
        (d_label && !is_device_ptr_on(d_label, ctx->device)) ||
        (d_forest && !is_device_ptr_on(d_forest, ctx->device))) {
        set_error("cc_stream_begin: need n > 0 and parent (label, forest) arrays in device memory of device %d",
                  ctx->device);
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    auto &c = ctx->ccs;
    for (int b = 0; b < 2; b++) {
        if (!c.copied[b])
            PHEM_CUDA_TRY(cudaEventCreateWithFlags(&c.copied[b], cudaEventDisableTiming));
        if (!c.freed[b])
            PHEM_CUDA_TRY(cudaEventCreateWithFlags(&c.freed[b], cudaEventDisableTiming));
    }
    if (!c.t0)
        PHEM_CUDA_TRY(cudaEventCreate(&c.t0));
    if (!c.t1)
        PHEM_CUDA_TRY(cudaEventCreate(&c.t1));
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), ctx->stream));
    PHEM_TRY(cc_launch_init(ctx, n, d_parent, d_label, d_forest));
    PHEM_CUDA_TRY(cudaEventRecord(c.t0, ctx->stream));
    // both buffers free; the first copies wait for the init
    for (int b = 0; b < 2; b++)
        PHEM_CUDA_TRY(cudaEventRecord(c.freed[b], ctx->stream));
    c.active = true;
    c.n = n;
    c.parent = d_parent;
    c.forest = d_forest;
    c.batches = c.edges = 0;
    return PHEM_OK;
}

phem_status phem_cc_stream_push(phem_context *ctx, const uint64_t *edges, int64_t m)
{
    PHEM_TRY(check_ctx(ctx));
    auto &c = ctx->ccs;
    if (!c.active) {
        set_error("cc_stream_push: no stream is open on this context (phem_cc_stream_begin)");
        return PHEM_ERR_INVALID;
    }
    if (m < 0 || (m > 0 && !edges)) {
        set_error("cc_stream_push: need m >= 0 and an edge array");
        return PHEM_ERR_INVALID;
    }
    if (m == 0)
        return PHEM_OK;
    DeviceGuard g(ctx->device);
    const bool dev = is_device_ptr(edges);
    if (dev && !is_device_ptr_on(edges, ctx->device)) {
        set_error("cc_stream_push: device edges must be memory of the context's device %d", ctx->device);
        return PHEM_ERR_INVALID;
    }
    if (dev && ((uintptr_t)edges & 15) == 0) {
        // a device batch is united in place (it stays valid until the next
        // push or the end)
        PHEM_TRY(cc_launch_unite(ctx, edges, m, c.n, c.parent, c.forest));
    } else {
        if ((size_t)m > c.cap) {
            // grow both buffers once every copy and union that uses them is done
            PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
            PHEM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            for (int b = 0; b < 2; b++) {
                if (c.buf[b])
                    cudaFree(c.buf[b]);
                c.buf[b] = nullptr;
            }
            c.cap = 0;
            const size_t cap = std::max<size_t>((size_t)m, 1u << 20);
            for (int b = 0; b < 2; b++)
                if (cudaMalloc(&c.buf[b], cap * sizeof(uint64_t)) != cudaSuccess) {
                    cudaGetLastError();
                    set_error("cc_stream_push: cannot allocate a %zu-edge staging buffer", cap);
                    return PHEM_ERR_CUDA;
                }
            c.cap = cap;
        }
        const int b = (int)(c.batches & 1);
        PHEM_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, c.freed[b], 0));
        PHEM_CUDA_TRY(cudaMemcpyAsync(c.buf[b], edges, (size_t)m * sizeof(uint64_t), cudaMemcpyDefault,
                                      ctx->copy_stream));
        PHEM_CUDA_TRY(cudaEventRecord(c.copied[b], ctx->copy_stream));
        PHEM_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, c.copied[b], 0));
        PHEM_TRY(cc_launch_unite(ctx, c.buf[b], m, c.n, c.parent, c.forest));
        PHEM_CUDA_TRY(cudaEventRecord(c.freed[b], ctx->stream));
        // the caller's buffer is read once the copy has landed
        PHEM_CUDA_TRY(cudaEventSynchronize(c.copied[b]));
    }
    c.batches++;
    c.edges += m;
    return PHEM_OK;
}

phem_status phem_cc_stream_end(phem_context *ctx, float *ms)
{
    PHEM_TRY(check_ctx(ctx));
    auto &c = ctx->ccs;
    if (!c.active) {
        set_error("cc_stream_end: no stream is open on this context (phem_cc_stream_begin)");
        return PHEM_ERR_INVALID;
    }
    c.active = false;
    DeviceGuard g(ctx->device);
    PHEM_CUDA_TRY(cudaEventRecord(c.t1, ctx->stream));
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(ctl_status(ctx->h_ctl->err, "cc_stream"));
    if (ms) {
        *ms = 0.f;
        if (cudaEventElapsedTime(ms, c.t0, c.t1) != cudaSuccess)
            *ms = 0.f;
    }
    return PHEM_OK;
}

phem_status phem_cc_merge(phem_context *ctx, const uint64_t *d_forest_a, const uint64_t *d_forest_b, int32_t n,
                          int32_t *d_parent, int32_t *d_label, uint64_t *d_forest_out, float *ms)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || !d_forest_a || !d_parent || !d_label) {
        set_error("cc_merge: need n > 0, forest_a, parent and label arrays");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), ctx->stream));
    PHEM_TRY(cc_launch_init(ctx, n, d_parent, d_label, d_forest_out));
    Timed timer(ctx);
    PHEM_TRY(cc_launch_merge(ctx, d_forest_a, d_forest_b, n, d_parent, d_forest_out));
    PHEM_TRY(cc_launch_label(ctx, n, d_parent, d_label));
    const float t = timer.stop();
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(ctl_status(ctx->h_ctl->err, "cc_merge"));
    if (ms)
        *ms = t;
    return PHEM_OK;
}

// ------------------------------------------------------------------ MSF

static phem_status msf_common(phem_context *ctx, const phem_edge *edges, uint64_t m, uint32_t n, phem_edge *msf,
                              uint64_t *count, uint64_t *total, phem_msf_stats *stats, uint64_t *d_count_total)
{
    if (n == 0 || n == UINT32_MAX || m > kMaxEdges || (m > 0 && !edges)) {
        set_error("msf: need 0 < n < 2^32 - 1, m <= 2^32 - 2^24 and an edge array");
        return PHEM_ERR_INVALID;
    }
    const bool aligned_dev = is_device_ptr(edges) && (((uintptr_t)edges & 15) == 0);
    const size_t eb = (size_t)m * sizeof(phem_edge), ob = (size_t)n * sizeof(phem_edge);
    const size_t o_edges = 0, o_out = aligned_dev ? 0 : align256(eb);  // edges read in place: no staging area
    size_t base = 0;
    MsfPlan plan;
    PHEM_TRY(msf_plan(ctx, kKindMsf, nullptr, m, n, o_out + align256(ob), &plan, &base));
    Staged se, so;
    if (aligned_dev) {
        se.dev = const_cast<phem_edge *>(edges);
    } else {
        se.dev = static_cast<char *>(ctx->ws) + base + o_edges;
        if (m)
            PHEM_CUDA_TRY(cudaMemcpyAsync(se.dev, edges, eb, cudaMemcpyDefault, ctx->stream));
    }
    stage_out(ctx, msf, ob, base + o_out, &so);
    plan.e0 = se.dev;
    Timed timer(ctx);
    uint32_t rounds = 0;
    // rounds, gather and the count copy are queued back to back; one wait at
    // the end (a host round trip between them would leave the GPU idle)
    PHEM_TRY(msf_run(ctx, kKindMsf, plan, &rounds, true));
    PHEM_TRY(msf_gather(ctx, plan, static_cast<phem_edge *>(so.dev)));
    PHEM_CUDA_TRY(cudaEventRecord(ctx->ev_stop, ctx->stream));
    if (d_count_total)
        PHEM_CUDA_TRY(cudaMemcpyAsync(d_count_total, &ctx->ctl->msf_count, 2 * sizeof(uint64_t),
                                      cudaMemcpyDeviceToDevice, ctx->stream));
    PHEM_TRY(msf_finish(ctx, &rounds));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop) != cudaSuccess)
        ms = 0.f;
    const Ctl &h = *ctx->h_ctl;
    PHEM_TRY(ctl_status(h.err, "msf"));
    if (h.msf_count > (uint64_t)n - 1 + (n == 0)) {
        set_error("msf: %llu forest edges for %u vertices", (unsigned long long)h.msf_count, n);
        return PHEM_ERR_NONCONVERGED;
    }
    if (so.host && h.msf_count)
        PHEM_CUDA_TRY(cudaMemcpy(so.host, so.dev, h.msf_count * sizeof(phem_edge), cudaMemcpyDeviceToHost));
    if (count)
        *count = h.msf_count;
    if (total)
        *total = h.msf_total;
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->rounds = rounds;
        for (uint32_t r = 0; r < rounds && r < PHEM_MAX_ROUNDS; r++) {
            stats->m_r[r] = h.m_r[r];
            stats->n_r[r] = h.n_r[r];
        }
        stats->light_rounds = h.light_rounds;
        stats->threshold = h.threshold;
        stats->msf_edges = h.msf_count;
        stats->total_weight = h.msf_total;
        stats->device_ms = ms;
    }
    return PHEM_OK;
}

static phem_status msf_stream_impl(phem_context *ctx, const phem_edge *h_edges, uint64_t m, uint32_t n,
                                   uint64_t chunk, phem_edge *msf, uint64_t *count, uint64_t *total, float *ms,
                                   phem_msf_stats *last_stats);

// Host MSF inputs of this many edges or more are solved in four chunks while
// the next chunk is copied (see phem_msf_solve).
constexpr uint64_t kMsfOverlapMinEdges = 1ull << 24;

phem_status phem_msf_solve(phem_context *ctx, const phem_edge *edges, uint64_t m, uint32_t n, phem_edge *msf,
                           uint64_t *count, uint64_t *total, phem_msf_stats *stats)
{
    PHEM_TRY(check_ctx(ctx));
    DeviceGuard g(ctx->device);
    // A large host input would otherwise be copied whole before the solve
    // starts.  Solved in four chunks instead -- chunk k with the forest of the
    // chunks before it while chunk k + 1 is copied -- the copy hides every
    // solve but the last, and the forest is the same (the chunked solve is
    // exact, record for record).
    const uint64_t chunk = ((m + 3) / 4 + 3) & ~3ull;
    const uint64_t R = ((uint64_t)n + 2) & ~3ull;
    if (m >= kMsfOverlapMinEdges && edges && !is_device_ptr(edges) && n > 1 && n < UINT32_MAX && R < kMaxEdges &&
        chunk <= kMaxEdges - R && R < chunk)
        return msf_stream_impl(ctx, edges, m, n, chunk, msf, count, total, nullptr, stats);
    return msf_common(ctx, edges, m, n, msf, count, total, stats, nullptr);
}

phem_status phem_msf_solve_device(phem_context *ctx, const phem_edge *d_edges, uint64_t m, uint32_t n,
                                  phem_edge *d_msf, uint64_t *d_count_total, phem_msf_stats *stats)
{
    PHEM_TRY(check_ctx(ctx));
    if (!is_device_ptr_on(d_edges, ctx->device) || (d_msf && !is_device_ptr_on(d_msf, ctx->device)) ||
        (d_count_total && !is_device_ptr_on(d_count_total, ctx->device))) {
        set_error("msf_solve_device: arrays must be device memory of the context's device %d", ctx->device);
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    return msf_common(ctx, d_edges, m, n, d_msf, nullptr, nullptr, stats, d_count_total);
}

// Chunked MSF (streamline_boruvka, MST/src/kernels.cu:849-1154): chunk k is
// solved together with the forest of chunks 0..k-1, since under a strict total
// order MSF(G1 + G2) = MSF(MSF(G1) + G2).  Each solve orders its input by
// (w, position).  The carried forest sits directly before the chunk, ascending
// by global edge index, and every one of its edges precedes every chunk edge
// globally, so position order is global index order and the final forest is
// exactly phem_msf_solve's.  Layout in the context's input buffer: two slots of
// [R forest records | chunk records] and an output area of R records, with
// R = n - 1 rounded up to 4 records so the chunk and every solve input start
// 16-byte aligned; up to 3 zero records (self-loops, ignored) pad the gap
// between the rounded start and the forest.  Chunk k + 1 is copied on the copy
// stream while chunk k is solved.
phem_status phem_msf_stream(phem_context *ctx, const phem_edge *h_edges, uint64_t m, uint32_t n, uint64_t chunk,
                            phem_edge *msf, uint64_t *count, uint64_t *total, float *ms)
{
    return msf_stream_impl(ctx, h_edges, m, n, chunk, msf, count, total, ms, nullptr);
}

// last_stats (may be NULL): the per-round counts of the last chunk's solve,
// with the whole forest's count and total.
static phem_status msf_stream_impl(phem_context *ctx, const phem_edge *h_edges, uint64_t m, uint32_t n,
                                   uint64_t chunk, phem_edge *msf, uint64_t *count, uint64_t *total, float *ms,
                                   phem_msf_stats *last_stats)
{
    PHEM_TRY(check_ctx(ctx));
    const uint64_t R = ((uint64_t)n + 2) & ~3ull;  // n - 1 rounded up to a multiple of 4
    if (n == 0 || n == UINT32_MAX || chunk == 0 || (m > 0 && !h_edges) || R >= kMaxEdges ||
        chunk > kMaxEdges - R) {
        set_error("msf_stream: need 0 < n < 2^32 - 1, 0 < chunk <= 2^32 - 2^24 - (n - 1 rounded up to 4), edges");
        return PHEM_ERR_INVALID;
    }
    if (count)
        *count = 0;
    if (total)
        *total = 0;
    if (ms)
        *ms = 0.f;
    // a device output must be this context's device memory: checked before
    // the stream is solved, not at the final copy
    if (msf && is_device_ptr(msf) && !is_device_ptr_on(msf, ctx->device)) {
        set_error("msf_stream: the output is device memory of another device than the context's %d", ctx->device);
        return PHEM_ERR_INVALID;
    }
    if (m == 0)
        return PHEM_OK;
    DeviceGuard g(ctx->device);
    const uint64_t top = std::min(chunk, m);  // largest chunk
    const size_t slot_bytes = align256((R + top) * sizeof(phem_edge));
    PHEM_TRY(input_reserve(ctx, 2 * slot_bytes + align256(R * sizeof(phem_edge)) + 256));
    {
        // size the solve workspace once for the largest solve (a later growth
        // would free memory, which waits for the copies in flight)
        MsfPlan plan;
        PHEM_TRY(msf_plan(ctx, kKindMsf, nullptr, R + top, n, align256((size_t)n * sizeof(phem_edge)), &plan,
                          nullptr));
    }
    char *b = static_cast<char *>(ctx->input);
    phem_edge *slot[2] = {reinterpret_cast<phem_edge *>(b), reinterpret_cast<phem_edge *>(b + slot_bytes)};
    phem_edge *d_out = reinterpret_cast<phem_edge *>(b + 2 * slot_bytes);
    const uint64_t chunks = (m + chunk - 1) / chunk;
    cudaEvent_t copied[2] = {nullptr, nullptr}, t0 = nullptr, t1 = nullptr;
    phem_status st = PHEM_OK;
    for (auto *e : {&copied[0], &copied[1], &t0, &t1})
        if (cudaEventCreateWithFlags(e, (e == &t0 || e == &t1) ? cudaEventDefault : cudaEventDisableTiming) !=
            cudaSuccess) {
            cudaGetLastError();
            *e = nullptr;
            st = PHEM_ERR_CUDA;
        }
    // the first copy waits for earlier work on the context stream, which may
    // still read the input buffer
    if (st == PHEM_OK && (cudaEventRecord(t0, ctx->stream) != cudaSuccess ||
                          cudaStreamWaitEvent(ctx->copy_stream, t0, 0) != cudaSuccess))
        st = PHEM_ERR_CUDA;
    if (st != PHEM_OK)
        set_error("msf_stream: cannot set up events: %s", cudaGetErrorString(cudaGetLastError()));
    auto issue = [&](uint64_t k) -> phem_status {
        const uint64_t off = k * chunk, len = std::min(chunk, m - off);
        if (cudaMemcpyAsync(slot[k & 1] + R, h_edges + off, len * sizeof(phem_edge), cudaMemcpyDefault,
                            ctx->copy_stream) != cudaSuccess ||
            cudaEventRecord(copied[k & 1], ctx->copy_stream) != cudaSuccess) {
            set_error("msf_stream: chunk copy failed: %s", cudaGetErrorString(cudaGetLastError()));
            return PHEM_ERR_CUDA;
        }
        return PHEM_OK;
    };
    uint64_t carried = 0, weight = 0;  // forest of the chunks solved so far
    if (st == PHEM_OK)
        st = issue(0);
    for (uint64_t k = 0; st == PHEM_OK && k < chunks; k++) {
        // slot (k + 1) & 1 was last read by solve k - 1, which has returned
        if (k + 1 < chunks && (st = issue(k + 1)) != PHEM_OK)
            break;
        phem_edge *cur = slot[k & 1];
        const uint64_t len = std::min(chunk, m - k * chunk);
        const uint64_t start = (R - carried) & ~3ull;
        if (cudaStreamWaitEvent(ctx->stream, copied[k & 1], 0) != cudaSuccess ||
            (R - carried > start && cudaMemsetAsync(cur + start, 0, (R - carried - start) * sizeof(phem_edge),
                                                    ctx->stream) != cudaSuccess)) {
            set_error("msf_stream: cannot queue chunk %llu", (unsigned long long)k);
            st = PHEM_ERR_CUDA;
            break;
        }
        st = msf_common(ctx, cur + start, R - start + len, n, d_out, &carried, &weight,
                        k + 1 == chunks ? last_stats : nullptr, nullptr);
        // the forest goes directly before the next chunk
        if (st == PHEM_OK && k + 1 < chunks && carried &&
            cudaMemcpyAsync(slot[(k + 1) & 1] + R - carried, d_out, carried * sizeof(phem_edge),
                            cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess) {
            set_error("msf_stream: cannot carry the forest");
            st = PHEM_ERR_CUDA;
        }
    }
    float t = 0.f;
    if (st == PHEM_OK && (cudaEventRecord(t1, ctx->stream) != cudaSuccess ||
                          (msf && carried &&
                           cudaMemcpyAsync(msf, d_out, carried * sizeof(phem_edge), cudaMemcpyDefault,
                                           ctx->stream) != cudaSuccess))) {
        set_error("msf_stream: cannot copy the forest out");
        st = PHEM_ERR_CUDA;
    }
    if (st == PHEM_OK)
        st = stream_wait(ctx);
    if (st == PHEM_OK && cudaEventElapsedTime(&t, t0, t1) != cudaSuccess)
        t = 0.f;
    if (st != PHEM_OK)
        cudaStreamSynchronize(ctx->copy_stream);  // no copy may still land in the input buffer
    for (auto e : {copied[0], copied[1], t0, t1})
        if (e)
            cudaEventDestroy(e);
    if (st != PHEM_OK)
        return st;
    if (count)
        *count = carried;
    if (total)
        *total = weight;
    if (ms)
        *ms = t;
    if (last_stats) {
        last_stats->device_ms = t;  // first copy to last solve
        last_stats->msf_edges = carried;
        last_stats->total_weight = weight;
    }
    return PHEM_OK;
}

phem_status phem_msf_solve_csr(phem_context *ctx, const int64_t *offsets, const uint32_t *cols, uint32_t n,
                               const uint32_t *weights, uint64_t m_upper, phem_edge *msf, uint64_t *count,
                               uint64_t *total, phem_msf_stats *stats)
{
    PHEM_TRY(check_ctx(ctx));
    if (n == 0 || n >= (1u << 31) || !offsets || m_upper >= (1ull << 32) || (m_upper > 0 && (!cols || !weights))) {
        set_error("msf_solve_csr: need 0 < n < 2^31, offsets, cols, weights, m_upper < 2^32");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    int64_t nnz = 0;
    PHEM_CUDA_TRY(cudaMemcpyAsync(&nnz, offsets + n, sizeof(int64_t), cudaMemcpyDefault, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    if (nnz < 0 || (uint64_t)nnz >= (1ull << 32)) {
        set_error("msf_solve_csr: offsets[n] = %lld out of range", (long long)nnz);
        return PHEM_ERR_INVALID;
    }
    // The converted edge list lives in the context's grow-only input buffer
    // (not the workspace, which the MSF solve sizes freely).
    const size_t ob = (size_t)(n + 1) * sizeof(int64_t), cb = (size_t)nnz * sizeof(uint32_t),
                 tb = csr_scratch_bytes(nnz), wb = (size_t)m_upper * sizeof(uint32_t),
                 rb = (size_t)m_upper * sizeof(phem_edge);
    const size_t o_off = 0, o_col = align256(ob), o_w = o_col + align256(cb), o_tr = o_w + align256(wb),
                 o_rec = o_tr + tb;
    PHEM_TRY(input_reserve(ctx, o_rec + align256(rb) + 256));
    char *b = static_cast<char *>(ctx->input);
    auto put = [&](const void *src, size_t bytes, size_t off) -> const void * {
        if (is_device_ptr(src))
            return src;
        if (bytes)
            cudaMemcpyAsync(b + off, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
        return b + off;
    };
    const int64_t *d_off = static_cast<const int64_t *>(put(offsets, ob, o_off));
    const uint32_t *d_col = static_cast<const uint32_t *>(put(cols, cb, o_col));
    const uint32_t *d_w = static_cast<const uint32_t *>(put(weights, wb, o_w));
    uint32_t *d_tr = reinterpret_cast<uint32_t *>(b + o_tr);
    phem_edge *d_rec = reinterpret_cast<phem_edge *>(b + o_rec);
    // one pass: kept entry p becomes the record {row, col, weights[p]}
    phem_status st = csr_launch_to_coo(ctx, d_off, d_col, (int32_t)n, nnz, d_tr, nullptr, d_w, d_rec, m_upper);
    // The solve is queued behind the conversion with no host round trip
    // between them; the conversion's count of entries with row < col is kept
    // aside (the solve resets the control block) and checked afterwards.  The
    // conversion writes no record past m_upper, and a short count leaves stale
    // records that the solve range-checks like any input, so a mismatch only
    // discards the solve's result.
    uint64_t *d_kept = reinterpret_cast<uint64_t *>(b + o_rec + align256(rb));
    if (st == PHEM_OK && cudaMemcpyAsync(d_kept, &ctx->ctl->misc[2], sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                                         ctx->stream) != cudaSuccess)
        st = PHEM_ERR_CUDA;
    if (st != PHEM_OK)
        return st;
    const phem_status solved = msf_common(ctx, d_rec, m_upper, n, msf, count, total, stats, nullptr);
    uint64_t kept = 0;
    if (cudaMemcpyAsync(&ctx->h_ctl->misc[2], d_kept, sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream) !=
        cudaSuccess)
        return PHEM_ERR_CUDA;
    PHEM_TRY(stream_wait(ctx));
    kept = ctx->h_ctl->misc[2];
    if (kept != m_upper) {
        set_error("msf_solve_csr: CSR has %llu entries with row < col, m_upper = %llu",
                  (unsigned long long)kept, (unsigned long long)m_upper);
        return PHEM_ERR_INVALID;
    }
    return solved;
}

phem_status phem_csr_to_coo(phem_context *ctx, const int64_t *offsets, const uint32_t *cols, int32_t n,
                            uint64_t *out, int64_t *out_m)
{
    PHEM_TRY(check_ctx(ctx));
    if (n <= 0 || !offsets || !out_m) {
        set_error("csr_to_coo: need n > 0, offsets and out_m");
        return PHEM_ERR_INVALID;
    }
    DeviceGuard g(ctx->device);
    int64_t nnz = 0;
    PHEM_CUDA_TRY(cudaMemcpyAsync(&nnz, offsets + n, sizeof(int64_t), cudaMemcpyDefault, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    if (nnz < 0 || (nnz > 0 && !cols)) {
        set_error("csr_to_coo: bad offsets[n] = %lld", (long long)nnz);
        return PHEM_ERR_INVALID;
    }
    const size_t ob = (size_t)(n + 1) * sizeof(int64_t), cb = (size_t)nnz * sizeof(uint32_t),
                 xb = (size_t)nnz * sizeof(uint64_t);
    const size_t o_off = 0, o_col = align256(ob), o_tr = o_col + align256(cb),
                 o_out = o_tr + csr_scratch_bytes(nnz);
    auto scratch = [&] { return reinterpret_cast<uint32_t *>(static_cast<char *>(ctx->ws) + o_tr); };
    PHEM_TRY(ws_reserve(ctx, o_out + align256(xb / 2 + 16)));
    Staged so, sc, sx;
    PHEM_TRY(stage_in(ctx, offsets, ob, o_off, &so));
    PHEM_TRY(stage_in(ctx, cols, cb, o_col, &sc));
    stage_out(ctx, out, 0, o_out, &sx);
    // a status bit an earlier call left set is not this call's
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), ctx->stream));
    // host output: stage only as much as can be kept (at most nnz / 2 entries have row < col
    // in a symmetric CSR; a non-symmetric one may keep more, so count first in that case)
    if (sx.host) {
        PHEM_TRY(csr_launch_to_coo(ctx, static_cast<const int64_t *>(so.dev), static_cast<const uint32_t *>(sc.dev),
                                   n, nnz, scratch(), nullptr));
        PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
        PHEM_TRY(stream_wait(ctx));
        const uint64_t kept = ctx->h_ctl->misc[2];
        if (kept > xb / 2 / sizeof(uint64_t) + 2) {
            // grow: the workspace is reallocated, so stage the inputs again
            PHEM_TRY(ws_reserve(ctx, o_out + align256(kept * sizeof(uint64_t))));
            PHEM_TRY(stage_in(ctx, offsets, ob, o_off, &so));
            PHEM_TRY(stage_in(ctx, cols, cb, o_col, &sc));
            stage_out(ctx, out, 0, o_out, &sx);
        }
    }
    PHEM_TRY(csr_launch_to_coo(ctx, static_cast<const int64_t *>(so.dev), static_cast<const uint32_t *>(sc.dev), n,
                               nnz, scratch(), static_cast<uint64_t *>(sx.dev)));
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    PHEM_TRY(ctl_status(ctx->h_ctl->err, "csr_to_coo"));
    const uint64_t kept = ctx->h_ctl->misc[2];
    if (sx.host && kept)
        PHEM_CUDA_TRY(cudaMemcpy(sx.host, sx.dev, kept * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    *out_m = (int64_t)kept;
    return PHEM_OK;
}

}  // extern "C"
