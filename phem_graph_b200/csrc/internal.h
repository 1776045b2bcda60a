// internal.h -- host-side internals shared by the library's translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/phem.h"
#include "common.cuh"

namespace phem {
// Kernels the library launches; the profile reports them by these names.
enum KernelId : int {
    kKInit = 0, kKSelect, kKEdgePass, kKHook, kKCompress, kKAdvance, kKGather,
    kKCcInit, kKCcUnite, kKCcMerge, kKCcLabel, kKMinid, kKCcCount, kKCsrCoo, kKBatch,
    kKernelCount
};
extern const char *const kKernelNames[kKernelCount];

struct PendingTiming {
    int kernel;
    cudaEvent_t start, stop;
};
}  // namespace phem

struct phem_context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;     // stream the work is ordered on
    cudaStream_t own_stream = nullptr; // stream created with the context
    cudaStream_t copy_stream = nullptr;// second stream for overlapped host copies
    void *ws = nullptr;                // grow-only device workspace
    size_t ws_bytes = 0;
    void *input = nullptr;             // grow-only buffer for converted inputs (CSR -> records)
    size_t input_bytes = 0;
    uint64_t *status = nullptr;        // look-back status words, only ever written by look-back
    // phem_cc_stream_begin/push/end: the stream in progress (the union-find
    // state is the caller's) and two staging buffers of its own, outside the
    // workspace
    struct CcStream {
        bool active = false;
        int32_t n = 0;
        int32_t *parent = nullptr;
        uint64_t *forest = nullptr;
        uint64_t *buf[2] = {nullptr, nullptr};
        size_t cap = 0;                // edges per staging buffer
        cudaEvent_t copied[2] = {nullptr, nullptr}, freed[2] = {nullptr, nullptr}, t0 = nullptr, t1 = nullptr;
        int64_t batches = 0, edges = 0;
    } ccs;
    size_t status_words = 0;           // (zeroed when grown; epochs keep old words from matching)
    phem::Ctl *ctl = nullptr;          // device control block
    phem::Ctl *h_ctl = nullptr;        // pinned host mirror of the control block
    uint64_t epoch = 1;                // look-back epoch counter
    uint32_t timeout_ms = 0;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    int edge_pass_blocks = 0;          // persistent grid sizes, from the occupancy API
    uint32_t kernels_ready = 0;        // bit k: launch attributes of edge kind k are set
    int gather_blocks = 0;
    int tune_edge_ctas = 4;              // MSF edge pass: CTAs (of 8 independent warps) per SM, 1 to 4
    int tune_graph = 1;                  // MSF rounds as a CUDA graph with a device-driven while-node
    cudaGraphExec_t msf_exec[2] = {nullptr, nullptr};  // cached round-loop graphs, per edge kind
    uint64_t msf_key[2][40] = {};        // what each was built for
    uint64_t msf_seen[2][40] = {};       // the last solve's key (a graph is built when it repeats)
    bool msf_graph_pending = false;      // a graph solve's launches are still to be counted
    bool msf_graph_select = false;       // ... and it had a threshold select
    // tuning knobs (phem_context_set_tuning)
    double tune_light_per_vertex = 0.5;  // light edges per vertex in the MSF filter (0: no filter)
    double tune_canonical_light = 1.5;   // the same for the canonical CC forest (edges by index)
    double tune_filter_min_ratio = 2.0;  // filter only when m >= ratio * light edges
    int tune_first_batch = 12;           // Boruvka rounds queued before the first host check
    int tune_next_batch = 4;             // rounds queued per later check
    int tune_batch_block = 1024;         // batched kernel: threads per CTA
    int tune_batch_items = 4;            // batched kernel: records per thread per step
    double tune_batch_compact = 1.0;     // batched kernel: compaction threshold
    double tune_cc_sample = 1.0;         // CC: edges per vertex united before a compress (0: one pass)
    // launch accounting and optional per-kernel CUDA-event timing
    uint64_t launches[phem::kKernelCount] = {};
    double kernel_ms[phem::kKernelCount] = {};
    uint64_t timed_launches[phem::kKernelCount] = {};
    bool profiling = false;
    std::vector<phem::PendingTiming> pending;
    std::vector<cudaEvent_t> event_pool;
    std::vector<std::pair<int, float>> launch_log;  // (kernel, ms) of timed launches, oldest first
};

namespace phem {

// Thread-local last-error text.
void set_error(const char *fmt, ...);

// CUDA call check: records the failure and returns PHEM_ERR_CUDA.
#define PHEM_CUDA_TRY(call)                                                                 \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            ::phem::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return PHEM_ERR_CUDA;                                                           \
        }                                                                                   \
    } while (0)

#define PHEM_TRY(expr)                       \
    do {                                     \
        phem_status s_ = (expr);             \
        if (s_ != PHEM_OK)                   \
            return s_;                       \
    } while (0)

// Carves 256-byte aligned sub-buffers out of the context workspace.
struct Carve {
    size_t off = 0;
    template <class T>
    size_t take(size_t count)
    {
        size_t at = (off + 255) & ~size_t(255);
        off = at + count * sizeof(T);
        return at;
    }
};

// Ensures ws_bytes >= bytes (contents are not preserved when it grows).
phem_status ws_reserve(phem_context *ctx, size_t bytes);
// Ensures input_bytes >= bytes (the converted-input buffer; contents not preserved).
phem_status input_reserve(phem_context *ctx, size_t bytes);
// Ensures the look-back status array holds >= words entries.
phem_status status_reserve(phem_context *ctx, size_t words);

// Waits for the stream, honouring the context watchdog.
phem_status stream_wait(phem_context *ctx);

// Maps the control block's error bits to a status (and the last-error text).
phem_status ctl_status(uint32_t err, const char *what);

// True when p is device (or managed) memory of the current device.
bool is_device_ptr(const void *p);
// True when p is device (or managed) memory of device `dev`.
bool is_device_ptr_on(const void *p, int dev);

uint64_t next_epochs(phem_context *ctx, uint32_t count);

// Brackets one kernel launch: counts it and, when profiling is on, records a
// pair of events on the context stream around it.
struct KernelScope {
    phem_context *ctx;
    int kernel;
    cudaEvent_t start = nullptr;
    KernelScope(phem_context *c, int k);
    ~KernelScope();
};
// Folds finished event pairs into the per-kernel totals (call after a sync).
void resolve_timings(phem_context *ctx);

// ---- call helpers shared by the entry points ----

// Makes ctx->device current for the duration of a call, restoring the caller's.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
            prev = -1;
        if (prev != dev)
            ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev)
            cudaSetDevice(prev);
    }
};

// A caller array staged through the workspace when it is host memory.
struct Staged {
    void *dev = nullptr;   // pointer the kernels use
    void *host = nullptr;  // caller's host pointer (null when it was already device memory)
    size_t bytes = 0;
};

inline phem_status check_ctx(phem_context *ctx)
{
    if (!ctx) {
        set_error("null context");
        return PHEM_ERR_INVALID;
    }
    return PHEM_OK;
}

// Event-timed region on the context stream.
struct Timed {
    phem_context *ctx;
    explicit Timed(phem_context *c) : ctx(c) { cudaEventRecord(ctx->ev_start, ctx->stream); }
    float stop()
    {
        float ms = 0.f;
        cudaEventRecord(ctx->ev_stop, ctx->stream);
        if (cudaEventSynchronize(ctx->ev_stop) == cudaSuccess)
            cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
        return ms;
    }
};

// Stages `bytes` of a caller input into the workspace at `off` when it is host
// memory (queued on the context stream).
inline phem_status stage_in(phem_context *ctx, const void *p, size_t bytes, size_t off, Staged *st)
{
    st->bytes = bytes;
    if (is_device_ptr(p)) {
        st->dev = const_cast<void *>(p);
        st->host = nullptr;
        return PHEM_OK;
    }
    st->dev = static_cast<char *>(ctx->ws) + off;
    st->host = nullptr;
    if (bytes)
        PHEM_CUDA_TRY(cudaMemcpyAsync(st->dev, p, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return PHEM_OK;
}

// An output: device pointer used directly, host pointer via workspace at `off`.
inline void stage_out(phem_context *ctx, void *p, size_t bytes, size_t off, Staged *st)
{
    st->bytes = bytes;
    if (!p || is_device_ptr(p)) {
        st->dev = p;
        st->host = nullptr;
        return;
    }
    st->dev = static_cast<char *>(ctx->ws) + off;
    st->host = p;
}

inline phem_status copy_back(phem_context *ctx, const Staged &st, size_t bytes)
{
    if (st.host && bytes)
        PHEM_CUDA_TRY(cudaMemcpyAsync(st.host, st.dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return PHEM_OK;
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// ---- MSF engine (msf.cu) ----
enum EdgeKind : int { kKindMsf = 0, kKindPacked = 1 };

struct MsfPlan {
    // device buffers (all inside the context workspace)
    const void *e0;          // input records: phem_edge (kKindMsf) or packed uint64 (kKindPacked)
    uint64_t m;
    uint32_t n;
    uint32_t *parent;        // n
    unsigned long long *best;// n
    uint32_t *cand;          // n: the round's choosers (hook -> compress)
    uint32_t *samples;       // 8192: the threshold select's sampled weights
    uint32_t *bitmap;        // ceil(m / 32)
    uint32_t *chunk_cnt;     // MSF edges per 1024 edge ids, then their offsets (gather)
    uint4 *wl[2];            // m each
    uint64_t *status;        // look-back status (context-owned), >= tiles
    uint64_t epoch_base;
    uint64_t *forest;        // kKindPacked only: forest slot per hooked root (may be null)
};

size_t msf_workspace_bytes(uint64_t m, uint32_t n, int sm_count);
phem_status msf_plan(phem_context *ctx, int kind, const void *d_e0, uint64_t m, uint32_t n, size_t extra_bytes,
                     MsfPlan *plan, size_t *extra_off);
// Queues the whole Boruvka solve; returns after the rounds are done and
// checked (the stream form checks the round flag between batches).  With
// `deferred` the graph form returns once the rounds are queued, and the
// caller queues more work before msf_finish waits and checks.  After the
// rounds the bitmap marks the MSF.
phem_status msf_run(phem_context *ctx, int kind, MsfPlan &plan, uint32_t *rounds_out, bool deferred = false);
// Waits for the queued work and checks the rounds (copies the control block
// to ctx->h_ctl).
phem_status msf_finish(phem_context *ctx, uint32_t *rounds_out);
// Queues the ordered gather of MSF edges (kKindMsf): out[0..count) + count/total into ctl.
phem_status msf_gather(phem_context *ctx, MsfPlan &plan, phem_edge *d_out);

// ---- CC engine (cc.cu) ----
phem_status cc_launch_init(phem_context *ctx, int32_t n, int32_t *parent, int32_t *label, uint64_t *forest);
phem_status cc_launch_unite(phem_context *ctx, const uint64_t *edges, int64_t m, int32_t n, int32_t *parent,
                            uint64_t *forest);
phem_status cc_launch_label(phem_context *ctx, int32_t n, int32_t *parent, int32_t *label);
// parent[i] = root(i) for all i.
phem_status cc_launch_compress(phem_context *ctx, int32_t n, int32_t *parent);
phem_status cc_launch_merge(phem_context *ctx, const uint64_t *fa, const uint64_t *fb, int32_t n, int32_t *parent,
                            uint64_t *forest_out);
// min-id labels from an arbitrary-root parent array (canonical forest path)
phem_status cc_launch_minid_labels(phem_context *ctx, int32_t n, uint32_t *parent, uint32_t *minid,
                                   int32_t *label);
phem_status cc_launch_count(phem_context *ctx, int32_t n, const int32_t *label, const uint64_t *forest);

// ---- CSR (csr.cu) ----
// Device scratch the conversion needs for nnz entries (per-tile rows, counts
// and offsets).
size_t csr_scratch_bytes(int64_t nnz);
// Queues the conversion of a device CSR with nnz entries; the kept count lands
// in ctx->ctl->misc[2].  With records set, the kept entry at position p is
// written as {row, col, w[p]} to records[p] for p < cap (out is ignored);
// otherwise packed pairs go to out, or only the count when out is null.
phem_status csr_launch_to_coo(phem_context *ctx, const int64_t *offsets, const uint32_t *cols, int32_t n,
                              int64_t nnz, uint32_t *scratch, uint64_t *out, const uint32_t *w = nullptr,
                              phem_edge *records = nullptr, uint64_t cap = 0);

}  // namespace phem
