/*
 * phem.h -- C ABI of the B200-native PHEM graph library (libphem.so).
 *
 * Two hot paths of the PHEM reference, rebuilt as sm_100a CUDA kernels:
 *   - union-find connected components + spanning forest
 *       (CC/ExternalSpanningTree.cu, CC/GPUSpanningTree.cu);
 *   - Boruvka minimum spanning forest (MST/src/kernels.cu, MST/src/new_boruvka.cu).
 *
 * The reference exports name-mangled C++ functions that print and exit() on any
 * CUDA error.  This header is the plain C boundary a foreign-function binding
 * attaches to: POD arguments, pointers and sizes, status codes, no exit().
 * Each entry point names the reference function it stands in for.
 *
 * Pointers.  Unless an entry point says "device", every array argument may be
 * host memory (pageable or pinned) or device memory of the context's GPU; the
 * library looks the pointer up and stages host arrays through its own device
 * workspace, copying results back before it returns.  Device-resident inputs
 * are never copied.
 *
 * Streams.  All GPU work of a context is ordered on its stream.  Entry points
 * return after the work is complete unless they say "asynchronous".
 *
 * Errors.  A non-zero phem_status is returned; phem_last_error() gives a
 * one-line description (thread-local).  Device loops are bounded: a loop that
 * hits its cap sets a status word and the call returns PHEM_ERR_NONCONVERGED
 * instead of hanging.
 */
#ifndef PHEM_H
#define PHEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHEM_VERSION 100

typedef enum phem_status {
    PHEM_OK = 0,
    PHEM_ERR_INVALID = 1,        /* bad argument: size, range, null pointer, endpoint >= n */
    PHEM_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    PHEM_ERR_NOMEM = 3,          /* device or pinned allocation failed */
    PHEM_ERR_NONCONVERGED = 4,   /* a bounded device loop reached its cap */
    PHEM_ERR_TIMEOUT = 5,        /* the host watchdog deadline passed */
    PHEM_ERR_UNSUPPORTED = 6,    /* valid request outside what this build supports */
    PHEM_ERR_NO_DEVICE = 7       /* no CUDA device, or the device is not sm_100 */
} phem_status;

/* MSF edge record, MST/src/constants.h:15-19 (`edge`: vertex u, vertex v, weight w;
 * all uint32).  Records are 12 bytes, array of structures. */
typedef struct phem_edge {
    uint32_t u;
    uint32_t v;
    uint32_t w;
} phem_edge;

/* Empty forest slot, INT_MAX held in a uint64 (CC/ExternalSpanningTree.cu:114,
 * CC/GPUSpanningTree.cu:139). */
#define PHEM_FOREST_EMPTY 0x7fffffffULL

/* Upper bound on Boruvka rounds (each round at least halves the live
 * components, so 33 suffice for 2^32 vertices); the reference caps at 100
 * (MST/src/kernels.cu:679-682). */
#define PHEM_MAX_ROUNDS 64

typedef struct phem_context phem_context;

/* ---------------------------------------------------------------- context */

/* Binds a context to CUDA device `device` and creates its stream.  Fails with
 * PHEM_ERR_NO_DEVICE when the device is missing or is not compute capability
 * 10.x (the kernels are built for sm_100a only). */
phem_status phem_context_create(int device, phem_context **out);
void phem_context_destroy(phem_context *ctx);

/* Orders the context's work on `stream` (a cudaStream_t of the same device);
 * NULL restores the context's own stream. */
phem_status phem_context_set_stream(phem_context *ctx, void *stream);
void *phem_context_stream(phem_context *ctx);

/* Host watchdog for the synchronous entry points: when a solve has not
 * finished `ms` milliseconds after it was queued the call returns
 * PHEM_ERR_TIMEOUT (the work itself is left to finish; the device is never
 * reset).  0 disables the watchdog (default). */
phem_status phem_context_set_timeout_ms(phem_context *ctx, uint32_t ms);

/* Per-kernel accounting.  Every kernel launch is counted; with profiling on,
 * each launch is also bracketed by CUDA events on the context stream and its
 * duration added up (for roofline figures measured inside an application). */
typedef struct phem_kernel_profile {
    char name[32];
    uint64_t launches;        /* launches since the last reset */
    uint64_t timed_launches;  /* launches that were event-timed */
    double total_ms;          /* summed event time of the timed launches */
} phem_kernel_profile;

phem_status phem_context_set_profiling(phem_context *ctx, int on);
/* Copies up to `max` entries (kernels launched at least once) and sets *count
 * to the number available.  Synchronises the context stream. */
phem_status phem_context_profile(phem_context *ctx, phem_kernel_profile *out, uint32_t max, uint32_t *count);
phem_status phem_context_profile_reset(phem_context *ctx);

/* Event-timed launches in launch order since the last reset (profiling on). */
typedef struct phem_launch_record {
    char name[32];
    float ms;
} phem_launch_record;
phem_status phem_context_launch_log(phem_context *ctx, phem_launch_record *out, uint32_t max, uint32_t *count);

/* Tuning knobs (defaults suit B200; the autotuner may change them):
 *   "msf.light_per_vertex"  light edges per vertex taken by the MSF filter
 *                           before the heavy pass; 0 disables the filter   [0.5]
 *   "msf.filter_min_ratio"  filter only when m >= ratio * light edges      [2.0]
 *   "msf.first_batch"       Boruvka rounds queued before the first check  [12]
 *   "msf.next_batch"        rounds queued per later check                 [4]
 *   "msf.edge_ctas_per_sm"  CTAs of 8 independent warps per SM in the edge
 *                           pass, 1 to 4                                  [4]
 *   "msf.graph"             1: the Boruvka rounds run as a cached CUDA graph
 *                           whose while-node the device drives; 0: rounds
 *                           queued on the stream in batches (per-launch
 *                           profiling always uses the stream form)        [1]
 *   "cc.canonical_light_per_vertex"  msf.light_per_vertex for the
 *                           PHEM_CC_CANONICAL forest (light = first by index) [1.5]
 *   "cc.sample_per_vertex"  phem_cc_solve unites this many edges per vertex
 *                           (a prefix of the list), compresses, then the
 *                           rest; 0 unites all at once                     [1]
 *   "batch.block_size"      threads per CTA of the batched kernel,
 *                           256, 512 or 1024                               [1024]
 *   "batch.items"           records per thread per step, 1, 2 or 4         [4]
 *   "batch.compact_ratio"   a batched list pass compacts when the live
 *                           records are at most this share of the list     [1.0]
 * None of them changes a result. */
phem_status phem_context_set_tuning(phem_context *ctx, const char *key, double value);
phem_status phem_context_get_tuning(phem_context *ctx, const char *key, double *value);

/* Releases the context's device workspace and converted-input buffer (both
 * grow on demand otherwise). */
phem_status phem_context_trim(phem_context *ctx);

const char *phem_status_string(phem_status s);
const char *phem_last_error(void);
int phem_version(void);

/* ---------------------------------------------------------------- statistics */

typedef struct phem_cc_stats {
    uint64_t forest_edges;  /* edges written to the forest (= n - components) */
    uint32_t components;    /* number of distinct labels */
    uint32_t rounds;        /* Boruvka rounds (canonical forest only, else 0) */
    float device_ms;        /* GPU time of the solve, CUDA events on the stream */
} phem_cc_stats;

typedef struct phem_msf_stats {
    uint32_t rounds;                     /* Boruvka rounds run (light phase + heavy phase) */
    uint32_t light_rounds;               /* rounds of the light phase; round light_rounds
                                            is the pass that filters the heavy edges */
    uint64_t m_r[PHEM_MAX_ROUNDS];       /* live edges found by round r's edge pass */
    uint64_t n_r[PHEM_MAX_ROUNDS];       /* components that chose an edge in round r */
    uint64_t msf_edges;                  /* = n - components */
    uint64_t total_weight;               /* uint64 sum of MSF weights */
    uint64_t threshold;                  /* light edge <=> (w << 32 | id) < threshold
                                            (packed CC edges: id < threshold); all ones = no filter */
    float device_ms;                     /* GPU time of the solve, CUDA events on the stream */
} phem_msf_stats;

/* -------------------------------------------------- connected components / SF */

/* Forest selection for phem_cc_solve. */
#define PHEM_CC_DEFAULT 0u
/* The forest is the minimum spanning forest under edge index order: the edge
 * SET that the reference's CPU path (CC/host_spanning_tree.cu:67-86) produces
 * with one Parlay worker.  Without the flag the forest is whichever edges won
 * the hooking races, as in the reference GPU kernels. */
#define PHEM_CC_CANONICAL 1u

/* One-shot CC + spanning forest over packed edges (u << 32 | v).
 * Replaces init_parent_label_T1edges + union_find_gpu_COO + cc
 * (CC/ExternalSpanningTree.cu:77-116, CC/GPUSpanningTree.cu:122-128).
 *   labels[n]  <- smallest vertex id of each vertex's component;
 *   forest[n]  <- at slot r, the edge whose union hooked root r; other slots
 *                 PHEM_FOREST_EMPTY (forest may be NULL).
 * Edges with u >= v are skipped, as union_find_gpu_COO skips them
 * (CC/ExternalSpanningTree.cu:82).  Endpoints must be < n (else INVALID).
 * PHEM_CC_CANONICAL requires m < 2^32.  stats may be NULL.
 * Host edges (2^20 or more, default forest) are copied in chunks on a second
 * stream, overlapped with the unions of earlier chunks; stats->device_ms then
 * includes the copy. */
phem_status phem_cc_solve(phem_context *ctx, const uint64_t *edges, int64_t m, int32_t n,
                          int32_t *labels, uint64_t *forest, uint32_t flags, phem_cc_stats *stats);

/* Stage-level entry points on DEVICE arrays, asynchronous on the context stream. */

/* parent[i] = label[i] = i, forest[i] = PHEM_FOREST_EMPTY.
 * init_parent_label_T1edges / _T2edges (CC/ExternalSpanningTree.cu:108-116,
 * CC/GPUSpanningTree.cu:132-140).  label or forest may be NULL. */
phem_status phem_cc_init(phem_context *ctx, int32_t n, int32_t *d_parent, int32_t *d_label,
                         uint64_t *d_forest);

/* Unions a batch of packed edges into the resident parent array and records
 * hooks in forest.  union_find_gpu_COO / COO1 (CC/ExternalSpanningTree.cu:77-97). */
phem_status phem_cc_unite(phem_context *ctx, const uint64_t *d_edges, int64_t m, int32_t n,
                          int32_t *d_parent, uint64_t *d_forest);

/* label[i] = find(i) with path compression.  cc (CC/GPUSpanningTree.cu:122-128). */
phem_status phem_cc_label(phem_context *ctx, int32_t n, int32_t *d_parent, int32_t *d_label);

/* Streaming spanning forest over host-resident batches.
 * SpanningTree (CC/ExternalSpanningTree.cu:133-218): initialises the state,
 * streams h_edges[0..m) to the GPU in batches of `batch` edges through
 * double-buffered copies overlapped with the union kernels, and leaves the
 * union-find state in d_parent and the per-batch forest in d_forest (both n
 * entries, device).  d_label is initialised to the identity.  h_edges should
 * be pinned for the copies to overlap.  *ms receives the event time. */
phem_status phem_cc_stream(phem_context *ctx, const uint64_t *h_edges, int64_t m, int32_t n,
                           int64_t batch, int32_t *d_parent, int32_t *d_label, uint64_t *d_forest,
                           float *ms);

/* The same stream, one batch per call, for batches that arrive over time (a
 * producer that reads or receives edges while earlier batches unite).
 *   begin: initialises d_parent and d_forest (n entries, device; d_forest may be
 *          NULL) and d_label (may be NULL) as phem_cc_stream does.
 *   push:  unites edges[0..m) into the state.  A host batch (pinned for the
 *          copy to overlap) is copied into one of two staging buffers of the
 *          context while the previous batch's unions run; push returns when
 *          the copy has landed, so the caller may refill its buffer at once.
 *          A 16-byte aligned device batch is united in place and must stay
 *          valid until the next push or end returns.
 *   end:   waits for every union, reports a failed bound (status codes as
 *          phem_cc_solve) and gives the time from begin to the last union.
 * The state is then what phem_cc_stream leaves (phem_cc_label gives labels).
 * One stream per context at a time; between begin and end the context runs
 * no other solve (they would reset the status word the unions report into). */
phem_status phem_cc_stream_begin(phem_context *ctx, int32_t n, int32_t *d_parent, int32_t *d_label,
                                 uint64_t *d_forest);
phem_status phem_cc_stream_push(phem_context *ctx, const uint64_t *edges, int64_t m);
phem_status phem_cc_stream_end(phem_context *ctx, float *ms);

/* Merge of two forests into final labels and a final forest.
 * gpu_spanning_tree (CC/GPUSpanningTree.cu:169-198): resets the state, unions
 * the 2n candidates d_forest_a[n] ++ d_forest_b[n] (PHEM_FOREST_EMPTY slots and
 * u >= v skipped), writes d_forest_out[n] and d_label[n] (min id).  d_forest_b
 * may be NULL (n empty slots).  *ms receives the event time. */
phem_status phem_cc_merge(phem_context *ctx, const uint64_t *d_forest_a, const uint64_t *d_forest_b,
                          int32_t n, int32_t *d_parent, int32_t *d_label, uint64_t *d_forest_out,
                          float *ms);

/* Largest n that phem_cc_solve_noalloc accepts: its scratch is a fixed
 * file-scope device array of this many parent words (4 MiB). */
#define PHEM_CC_NOALLOC_MAX_VERTICES (1 << 20)

/* CC + spanning forest that allocates nothing.  No counterpart in the
 * reference: it is phem_cc_solve's default path (same labels, a forest of the
 * same kind) for callers that cannot allocate device memory at solve time --
 * a serving process whose memory is committed under a budget, or a loop that
 * cannot afford cudaMalloc/cudaFree stalling the device -- and so takes no
 * context either.  The parent array lives in fixed static device scratch.
 *   d_edges[m]  packed (u << 32 | v), DEVICE memory, 16-byte aligned;
 *   d_labels[n] <- smallest vertex id of each component (DEVICE);
 *   d_forest[n] <- forest slot per hooked root, PHEM_FOREST_EMPTY elsewhere
 *                  (DEVICE, may be NULL);
 *   stream      cudaStream_t the work is queued on (NULL: the default stream).
 * Runs on the current device and returns when the work is complete.
 * n > PHEM_CC_NOALLOC_MAX_VERTICES returns PHEM_ERR_INVALID.  Every call looks
 * the scratch address up in the current CUDA context (no allocation); the first
 * call on a device also loads the library's module there.  All calls on a
 * device share the scratch: calls that overlap
 * in time race and corrupt each other's results. */
phem_status phem_cc_solve_noalloc(const uint64_t *d_edges, int64_t m, int32_t n, int32_t *d_labels,
                                  uint64_t *d_forest, void *stream);

/* ------------------------------------------------------------ minimum spanning forest */

/* Minimum spanning forest of edges[0..m) over vertices [0, n) under the strict
 * order (w, edge index).  Stands in for boruvka_for_edge_array
 * (MST/src/new_boruvka.cu:40-179) and the PBBS mst() (MST/src/utils.cu:794-841):
 *   msf[0..*count) <- the MSF edges, ascending by edge index (the order of the
 *                     PBBS result, utils.cu:837,871-885); msf needs room for
 *                     n - 1 records and may be NULL;
 *   *count, *total <- number of MSF edges and their uint64 total weight.
 * Self-loops are ignored.  Endpoints must be < n.  m < 2^32.  count, total and
 * stats may be NULL.  Host edges of 2^24 or more are solved as phem_msf_stream
 * solves them, in four chunks copied while the chunk before is solved (the
 * forest is the same, record for record); stats then holds the last chunk's
 * per-round counts, the whole forest's count and total, and device_ms from
 * the first copy to the last solve. */
phem_status phem_msf_solve(phem_context *ctx, const phem_edge *edges, uint64_t m, uint32_t n,
                           phem_edge *msf, uint64_t *count, uint64_t *total, phem_msf_stats *stats);

/* Same on DEVICE arrays: d_msf (room for n - 1 records, may be NULL) gets the
 * records and d_count_total[0], d_count_total[1] the count and total weight
 * (may be NULL).  Stands in for device_boruvka (MST/src/kernels.cu:507-689),
 * which works on caller-owned device buffers.  Returns when the solve is done. */
phem_status phem_msf_solve_device(phem_context *ctx, const phem_edge *d_edges, uint64_t m, uint32_t n,
                                  phem_edge *d_msf, uint64_t *d_count_total, phem_msf_stats *stats);

/* Chunked MSF over host-resident edges: streamline_boruvka
 * (MST/src/kernels.cu:849-1154).  h_edges[0..m) is taken in chunks of `chunk`
 * edges; chunk k is solved together with the forest of chunks 0..k-1
 * (MSF(G1 + G2) = MSF(MSF(G1) + G2)), while chunk k + 1 is copied on a second
 * stream.  The result is exactly phem_msf_solve's -- the unique MSF under
 * (w, edge index), ascending by edge index -- but m has no 2^32 limit: each
 * solve holds one chunk plus at most n - 1 forest edges, so device memory
 * scales with chunk + n, not m.
 *   msf (host memory, or device memory of the context's device, room for
 *   n - 1 records, may be NULL; checked before any chunk is solved), *count,
 *   *total as phem_msf_solve; *ms = device time from the first copy to the
 *   last solve.
 * Needs 0 < chunk <= 2^32 - 2^24 - R, with R = n - 1 rounded up to a multiple
 * of 4 (else INVALID).  h_edges may be host (pinned for the copies to overlap)
 * or device memory.  count, total and ms may be NULL. */
phem_status phem_msf_stream(phem_context *ctx, const phem_edge *h_edges, uint64_t m, uint32_t n, uint64_t chunk,
                            phem_edge *msf, uint64_t *count, uint64_t *total, float *ms);

/* MSF of a symmetrised CSR graph (int64 offsets[n + 1], uint32 cols[2m]).
 * Edge i is the i-th entry with row < col in row-major order (the numbering of
 * csr_to_coo, CC/graph.cu:169-187); weights[i] is its weight.  Output as
 * phem_msf_solve.  m_upper must be the number of such entries: the count is
 * checked once the solve has run (no host round trip sits between the
 * conversion and the solve), and a mismatch returns PHEM_ERR_INVALID with the
 * outputs unspecified. */
phem_status phem_msf_solve_csr(phem_context *ctx, const int64_t *offsets, const uint32_t *cols,
                               uint32_t n, const uint32_t *weights, uint64_t m_upper,
                               phem_edge *msf, uint64_t *count, uint64_t *total,
                               phem_msf_stats *stats);

/* CSR -> packed COO (row << 32 | col) for entries with row < col, in row-major
 * order.  csr_to_coo (CC/graph.cu:149-196), on the GPU.  out needs room for
 * the number of such entries (NULL to count only); *out_m receives it. */
phem_status phem_csr_to_coo(phem_context *ctx, const int64_t *offsets, const uint32_t *cols, int32_t n,
                            uint64_t *out, int64_t *out_m);

/* ------------------------------------------------------------ batched small graphs */
/* Many independent graphs solved in ONE persistent kernel launch: CTAs take
 * whole graphs from a device work queue (largest first) and run Boruvka on
 * each to completion.  No reference counterpart: the reference solves one
 * graph per call (boruvka_for_edge_array, MST/src/new_boruvka.cu:40-179),
 * and this is the batch of such calls without their launch overhead.  Every
 * graph gets exactly what the one-graph entry points give it:
 *   PHEM_BATCH_MSF  forest = the unique MSF under (w, edge index), as
 *                   phem_msf_solve; total = its uint64 weight;
 *   PHEM_BATCH_CC   forest = the canonical spanning forest (MSF under edge
 *                   index order, phem_cc_solve with PHEM_CC_CANONICAL);
 *                   total = 0;
 * and labels = smallest vertex id of each vertex's component. */
#define PHEM_BATCH_MSF 0u
#define PHEM_BATCH_CC 1u

/* One graph of a batch.  Its edges are edges[edge_offset, + num_edges) with
 * vertex ids local to the graph (< num_vertices); an edge's id is its
 * position within the graph.  Vertex-indexed outputs of the graph occupy
 * [vertex_offset, + num_vertices); graphs' vertex ranges must not overlap. */
typedef struct phem_batch_graph {
    uint64_t edge_offset;
    uint32_t num_edges;
    uint32_t num_vertices;
    uint32_t vertex_offset;
    uint32_t kind;  /* PHEM_BATCH_MSF or PHEM_BATCH_CC */
} phem_batch_graph;

typedef struct phem_batch_stats {
    uint32_t max_rounds;    /* most Boruvka rounds any graph needed */
    uint32_t block_size;    /* kernel configuration used */
    uint32_t items;
    float compact_ratio;
    uint32_t grid;          /* persistent CTAs launched */
    uint32_t smem_vertices; /* graphs up to this many vertices kept their state in shared memory */
    float device_ms;        /* GPU time of the batched launch (events on the stream) */
} phem_batch_stats;

/* Solves every graph of the batch.
 *   graphs[num_graphs]       HOST array;
 *   edges[total_edges]       host or device;
 *   msf_ids[total_vertices]  <- graph g's forest edge ids, ascending, at
 *                               [vertex_offset, + msf_count[g]) (may be NULL);
 *   msf_count[num_graphs], msf_total[num_graphs] (required);
 *   labels[total_vertices]   <- local min-id labels (may be NULL).
 * Outputs may be host or device memory.  stats may be NULL.
 * Host edges of a large batch (2^22 edges or more) are copied in four chunks
 * on a second stream; the graphs complete after each chunk are solved by
 * their own launch, which waits only for that chunk, so copies and solves
 * overlap (stats->device_ms then includes the copy). */
phem_status phem_batch_solve(phem_context *ctx, const phem_batch_graph *graphs, uint32_t num_graphs,
                             const phem_edge *edges, uint64_t total_edges, uint32_t total_vertices,
                             uint32_t *msf_ids, uint32_t *msf_count, uint64_t *msf_total, int32_t *labels,
                             phem_batch_stats *stats);

/* Replayable batch plan: device buffers sized for a maximum batch plus a
 * captured CUDA graph (queue reset + persistent kernel) that reads the batch
 * size from device memory, so one capture serves every batch that fits.
 * Kernel configuration comes from the context's batch.* tuning at creation;
 * the context stream must not be the legacy default stream. */
typedef struct phem_batch_plan phem_batch_plan;
phem_status phem_batch_plan_create(phem_context *ctx, uint32_t max_graphs, uint64_t max_edges,
                                   uint32_t max_vertices, phem_batch_plan **out);
void phem_batch_plan_destroy(phem_batch_plan *plan);
/* Queues the copies of a batch (host arrays; pinned edges overlap best) into
 * the plan's buffers, asynchronously on the context stream. */
phem_status phem_batch_plan_upload(phem_batch_plan *plan, const phem_batch_graph *graphs, uint32_t num_graphs,
                                   const phem_edge *edges, uint64_t total_edges, uint32_t total_vertices);
/* Replays the captured graph (asynchronous). */
phem_status phem_batch_plan_run(phem_batch_plan *plan);
/* Waits for the batch and copies results to host or device arrays (any may be
 * NULL); returns the first error any graph reported. */
phem_status phem_batch_plan_download(phem_batch_plan *plan, uint32_t *msf_ids, uint32_t *msf_count,
                                     uint64_t *msf_total, int32_t *labels);
/* Device addresses of the plan's buffers (for callers that keep inputs and
 * results on the GPU).  Any pointer argument may be NULL. */
phem_status phem_batch_plan_device(phem_batch_plan *plan, phem_edge **edges, uint32_t **msf_ids,
                                   uint32_t **msf_count, uint64_t **msf_total, int32_t **labels);

/* Autotuner: times every kernel configuration (block 256/512/1024 x items
 * 1/2/4 x compaction ratio 0.25/0.5/1.0) on this batch, `reps` launches each,
 * stores the fastest in the context's batch.* tuning and reports it in
 * *best (whose device_ms is the best mean time).  Results are not returned. */
phem_status phem_batch_autotune(phem_context *ctx, const phem_batch_graph *graphs, uint32_t num_graphs,
                                const phem_edge *edges, uint64_t total_edges, uint32_t total_vertices,
                                uint32_t reps, phem_batch_stats *best);

/* ------------------------------------------------------------------ serving loop */
/* A request loop with continuous batching.  No reference counterpart (the
 * reference solves one graph per process run, CC/main.cu, MST/main.cu).
 * Requests of mixed sizes are submitted from any host thread.  Small ones are
 * packed into batched persistent launches, `slots` of them in flight at once,
 * so requests arriving while a batch runs form the next one and start as
 * soon as a slot frees up; large ones run on the device-wide engines
 * (phem_msf_solve, phem_cc_solve) in `large_workers` threads, concurrently.
 * Device memory is bounded by `memory_budget`: slot arenas are fixed at
 * creation and each device-wide worker grows its workspace at most to its
 * share; a request that fits nowhere is refused at submission with
 * PHEM_ERR_NOMEM.  A request's result is the same whichever path serves it
 * and whatever else is in flight. */
typedef struct phem_server phem_server;

typedef struct phem_server_config {
    uint64_t memory_budget;     /* device bytes the server may hold */
    uint32_t slots;             /* batched launches in flight, 1..8 */
    uint32_t max_batch_graphs;  /* requests per batched launch */
    uint64_t large_edges;       /* requests with more edges use the device-wide engines */
    uint32_t large_workers;     /* concurrent device-wide solves, 1..8 */
    uint32_t reserved;
} phem_server_config;

/* One request.  Arrays are host memory owned by the caller and must stay
 * valid until the request's result has been collected. */
typedef struct phem_request {
    uint32_t kind;             /* PHEM_BATCH_MSF or PHEM_BATCH_CC */
    uint32_t num_vertices;     /* n > 0 */
    uint64_t num_edges;        /* m */
    const phem_edge *edges;    /* MSF input: {u, v, w} records */
    const uint64_t *pairs;     /* CC input: packed (u << 32 | v); pairs with u >= v are skipped */
    phem_edge *forest;         /* MSF output: forest records ascending by edge index
                                  (room for n - 1; may be NULL) */
    int32_t *labels;           /* CC output: min-id labels, n entries (may be NULL) */
} phem_request;

#define PHEM_PATH_BATCHED 0u
#define PHEM_PATH_DEVICE 1u

typedef struct phem_request_result {
    int32_t status;            /* phem_status of this request */
    uint32_t path;             /* PHEM_PATH_BATCHED or PHEM_PATH_DEVICE */
    uint64_t forest_edges;     /* forest size (CC: n - components) */
    uint64_t total_weight;     /* MSF: uint64 forest weight; CC: 0 */
    uint64_t submit_ns;        /* steady-clock times: submitted, work started, result written */
    uint64_t start_ns;
    uint64_t done_ns;
} phem_request_result;

phem_status phem_server_create(int device, const phem_server_config *cfg, phem_server **out);
/* Finishes every submitted request, then releases the server. */
void phem_server_destroy(phem_server *server);
/* Queues a request (thread-safe); *ticket identifies it for phem_server_wait. */
phem_status phem_server_submit(phem_server *server, const phem_request *req, uint64_t *ticket);
/* Waits for a request (timeout_ms 0: no limit) and returns its result; each
 * ticket is collected once. */
phem_status phem_server_wait(phem_server *server, uint64_t ticket, uint32_t timeout_ms, phem_request_result *res);
/* Open-loop load: submits reqs[i] at arrival_ns[i] after the call starts
 * (nanoseconds, non-decreasing), then collects every result in order.
 * Returns the first submission error (results[i].status has each one). */
phem_status phem_server_replay(phem_server *server, const phem_request *reqs, const uint64_t *arrival_ns,
                               uint32_t count, phem_request_result *results);

/* ------------------------------------------------------------------ graph files */
/* The reference drivers' input formats, read on the host (see io.cpp).
 * Errors: PHEM_ERR_INVALID with phem_io_last_error() describing it. */

/* MatrixMarket coordinate file as the MST driver reads it (getGraphInfo +
 * mmapPopulateEdgeArray, MST/src/utils.cu:160-180, 896-1036): *n_out = rows,
 * *m_out = nnz of the size line; out[i] = (min(u, v) - 1, max(u, v) - 1, w)
 * of data line i, w read from the line or, with generate_weights, set to
 * ((u - 1) * (v - 1) mod rows) + 1 in 32-bit arithmetic.  A missing or empty
 * line gives {0, 0, 0}.  out == NULL queries the sizes. */
phem_status phem_read_mtx(const char *path, int generate_weights, phem_edge *out, uint64_t capacity,
                          uint32_t *n_out, uint64_t *m_out);

/* ECL binary CSR as the CC driver reads it (readECLgraph, CC/graph.cu:90-121):
 * int64 n, int64 nnz, int64 offsets[n + 1], int32 cols[nnz].  offsets or
 * cols NULL queries the sizes. */
phem_status phem_read_ecl(const char *path, int64_t *offsets, uint32_t *cols, uint64_t cols_capacity,
                          uint32_t *n_out, uint64_t *nnz_out);

/* The CC driver's input as packed pairs (u << 32 | v), u < v, in file order
 * (undirected_graph, CC/graph.cu:13-196): ".edges", ".eg2" and ".txt" files
 * are text edge lists ("n m" then m lines "u v"), any other name is ECL
 * binary CSR converted in row-major order.  pairs NULL counts. */
phem_status phem_read_graph_pairs(const char *path, uint64_t *pairs, uint64_t capacity, uint32_t *n_out,
                                  uint64_t *m_out);

/* Description of the last reader error of this thread. */
const char *phem_io_last_error(void);

/* --------------------------------------------------------- synthetic inputs (host) */
/* Seeded generators for tests and benchmarks (no reference counterpart: the
 * reference reads graph files).  Deterministic for any thread count. */

/* SplitMix64 value i of stream `tag` under `seed`. */
uint64_t phem_gen_mix64(uint64_t seed, uint64_t tag, uint64_t i);

/* Erdos-Renyi: `draws` uniform pairs over [0, n); self-loops dropped,
 * duplicates kept, packed (min << 32 | max) in draw order.  out needs `draws`
 * entries (NULL to count); *out_m receives the number kept. */
phem_status phem_gen_er(uint32_t n, uint64_t draws, uint64_t seed, uint64_t *out, uint64_t *out_m);

/* R-MAT (Chakrabarti, Zhan, Faloutsos 2004) on 2^scale vertices with quadrant
 * probabilities a, b, c (d = 1 - a - b - c), no vertex permutation; self-loops
 * dropped, duplicates kept; pairs packed (min << 32 | max) and sorted, i.e. the
 * upper triangle of the symmetrised CSR in row-major order.  out needs `draws`
 * entries (NULL to count). */
phem_status phem_gen_rmat(uint32_t scale, uint64_t draws, double a, double b, double c, uint64_t seed,
                          uint64_t *out, uint64_t *out_m);

/* Draws [first, first + count) of the phem_gen_rmat stream, unsorted, packed
 * (min << 32 | max), self-loops dropped, draw order kept (for generating a
 * huge graph batch by batch).  out needs `count` entries (NULL to count). */
phem_status phem_gen_rmat_range(uint32_t scale, uint64_t first, uint64_t count, double a, double b, double c,
                                uint64_t seed, uint64_t *out, uint64_t *out_m);

/* phem_gen_rmat_range on the GPU: the identical draws, in the identical order,
 * written to d_out (device memory of the context's device, room for `count`
 * entries); *out_m receives the number written.  Returns when done.  Input
 * generation for graphs too large to generate on the host (no reference
 * counterpart; the reference reads its graphs from files). */
phem_status phem_gen_rmat_range_device(phem_context *ctx, uint32_t scale, uint64_t first, uint64_t count,
                                       double a, double b, double c, uint64_t seed, uint64_t *d_out,
                                       uint64_t *out_m);

/* w[i] = 1 + (SplitMix64 value i & (2^bits - 1)), i.e. uniform in [1, 2^bits]. */
phem_status phem_gen_weights(uint64_t m, uint64_t seed, uint32_t bits, uint32_t *w);

/* {u, v, w} records from packed pairs and weights (w may be NULL: zero). */
phem_status phem_pack_msf_edges(const uint64_t *pairs, const uint32_t *w, uint64_t m, phem_edge *out);

/* Symmetrised CSR from pairs sorted by (u, v) with u < v. */
phem_status phem_csr_from_sorted_pairs(const uint64_t *pairs, uint64_t m, uint32_t n, int64_t *offsets,
                                       uint32_t *cols);

/* 2-D random geometric graph: n points uniform in the unit square, each
 * linked to its k nearest neighbours (ties by lower index), every pair once,
 * sorted and packed (min << 32 | max); w[e] = floor(distance * 2^24) computed
 * in double precision.  out and w need n * k entries (either may be NULL). */
phem_status phem_gen_rgg(uint32_t n, uint32_t k, uint64_t seed, uint64_t *out, uint32_t *w, uint64_t *out_m);

#ifdef __cplusplus
}
#endif

#endif /* PHEM_H */
