// batch.h -- device layout and launch plumbing of the batched engine.
#pragma once

#include <vector>

#include "internal.h"

namespace phem {

// Internal kind: a CC graph whose edges are packed pairs (u << 32 | v) in
// BatchArgs::pairs at e_off (the serving loop's CC requests).
constexpr uint32_t kBatchPairs = 2;

// One graph as the kernel sees it, in queue order (largest first).  Scratch
// offsets are the host's exclusive prefix sums, so graphs whose caller edge
// ranges overlap or leave gaps still get private scratch.
struct BatchItem {
    uint64_t e_off;   // first input record (caller's edge_offset)
    uint64_t wl_off;  // first survivor-list record (prefix sum of m)
    uint32_t m, n;
    uint32_t v_off;   // caller's vertex_offset: outputs and global vertex state
    uint32_t kind;    // PHEM_BATCH_MSF, PHEM_BATCH_CC or kBatchPairs
    uint32_t bm_off;  // first word of the graph's forest bitmap (prefix sum of ceil(m / 32))
    uint32_t index;   // caller's graph index: per-graph outputs
};
static_assert(sizeof(BatchItem) == 40, "BatchItem layout");

struct BatchArgs {
    const BatchItem *items;
    const uint32_t *num_graphs;  // device word, so one captured launch serves any batch size
    uint32_t *queue;             // next item to take (zeroed before each launch)
    const phem_edge *edges;
    const unsigned long long *pairs;  // kBatchPairs graphs' input (may be null otherwise)
    uint4 *wl;                   // sum of m records
    uint32_t *bitmap;            // sum of ceil(m / 32) words
    unsigned long long *g_best;  // vertex state of graphs too large for shared memory
    uint32_t *g_parent;
    uint32_t *g_aux;
    uint32_t *g_roots;
    uint32_t *msf_ids;           // vertex-indexed: graph g's forest at [vertex_offset, + count)
    uint32_t *msf_count;         // per graph
    unsigned long long *msf_total;
    int32_t *labels;             // vertex-indexed
    uint32_t *status;            // per graph error bits
    uint32_t *rounds;            // per graph Boruvka rounds (may be null)
    uint32_t smem_vertices;      // set by batch_launch
    float compact_ratio;         // compact a list pass when live <= ratio * length
};

struct BatchLaunch {
    const void *kernel = nullptr;
    int block = 0, items = 0, grid = 0;
    size_t dyn_smem = 0;
    uint32_t smem_vertices = 0;
};

// Device buffers of one batch (context workspace or plan memory).
struct BatchBuffers {
    BatchItem *items;
    uint32_t *num_graphs, *queue;
    phem_edge *edges;
    uint4 *wl;
    uint32_t *bitmap, *g_parent, *g_aux, *g_roots;
    unsigned long long *g_best;
    uint32_t *msf_ids, *msf_count;
    unsigned long long *msf_total;
    int32_t *labels;
    uint32_t *status, *rounds;
};

// A large batch whose edges are in host memory is copied in kBatchGroups
// chunks on the copy stream; the graphs whose edges are complete after chunk
// k form launch k, which waits only for that chunk's copy, so the copies and
// the solves overlap.
constexpr int kBatchGroups = 4;
constexpr uint64_t kBatchOverlapMinEdges = 1ull << 22;
struct BatchGroups {
    int k = 0;                           // launches; 0: one launch after one copy
    uint64_t bound[kBatchGroups + 1];    // edge chunk boundaries
    uint32_t start[kBatchGroups] = {};   // first item of each launch (queue order)
    uint32_t count[kBatchGroups] = {};   // items of each launch
};

// Validated work items in queue order (largest graphs first, so the longest
// solves start early and the persistent grid finishes together), with the
// private scratch offsets of every graph.
struct BatchLayout {
    std::vector<BatchItem> items;
    uint64_t wl_records = 0;
    uint64_t bm_words = 0;
};

// Validates caller graphs (ranges, kinds, non-overlapping vertex ranges) and
// builds the queue-ordered items with private scratch offsets.
phem_status build_items(const phem_batch_graph *graphs, uint32_t G, uint64_t total_edges, uint32_t total_vertices,
                        BatchLayout *L);
// Carves every buffer for the given capacities out of `base` (null: sizing
// only); returns the bytes needed.
size_t batch_carve(uint32_t G, uint64_t E, uint64_t wl, uint64_t bm, uint32_t V, bool edges_inline, char *base,
                   BatchBuffers *b);
BatchArgs make_args(const BatchBuffers &b, const phem_edge *edges, float ratio);

// Resolves the kernel for (block, items), sets its shared-memory attribute and
// sizes the persistent grid from the occupancy API.
phem_status batch_launch_config(int device, int sm_count, int block, int items, BatchLaunch *out);
phem_status batch_launch(cudaStream_t stream, const BatchLaunch &l, BatchArgs args);

}  // namespace phem

struct phem_batch_plan {
    phem_context *ctx = nullptr;
    uint32_t max_graphs = 0, max_vertices = 0;
    uint64_t max_edges = 0, max_wl = 0, max_bm = 0;
    void *mem = nullptr;
    phem::BatchBuffers buf{};
    phem::BatchLaunch launch{};
    float ratio = 0.5f;
    phem::BatchItem *h_items = nullptr;  // pinned staging of the work items
    uint32_t *h_num = nullptr;     // pinned batch size
    uint32_t *h_status = nullptr;  // pinned per-graph status
    cudaEvent_t staged = nullptr;  // the pinned staging has been consumed
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t num_graphs = 0, total_vertices = 0;
};

namespace phem {
phem_status batch_plan_capture(phem_batch_plan *p, const unsigned long long *pairs);
}  // namespace phem
