// batch.h -- device layout and launch plumbing of the batched engine.
#pragma once

#include "internal.h"

namespace phem {

// One graph as the kernel sees it, in queue order (largest first).  Scratch
// offsets are the host's exclusive prefix sums, so graphs whose caller edge
// ranges overlap or leave gaps still get private scratch.
struct BatchItem {
    uint64_t e_off;   // first input record (caller's edge_offset)
    uint64_t wl_off;  // first survivor-list record (prefix sum of m)
    uint32_t m, n;
    uint32_t v_off;   // caller's vertex_offset: outputs and global vertex state
    uint32_t kind;    // PHEM_BATCH_MSF or PHEM_BATCH_CC
    uint32_t bm_off;  // first word of the graph's forest bitmap (prefix sum of ceil(m / 32))
    uint32_t index;   // caller's graph index: per-graph outputs
};
static_assert(sizeof(BatchItem) == 40, "BatchItem layout");

struct BatchArgs {
    const BatchItem *items;
    const uint32_t *num_graphs;  // device word, so one captured launch serves any batch size
    uint32_t *queue;             // next item to take (zeroed before each launch)
    const phem_edge *edges;
    uint4 *wl;                   // sum of m records
    uint32_t *bitmap;            // sum of ceil(m / 32) words
    uint32_t *g_parent;          // vertex state of graphs too large for shared memory
    uint32_t *g_comp;
    unsigned long long *g_best;
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

// Resolves the kernel for (block, items), sets its shared-memory attribute and
// sizes the persistent grid from the occupancy API.
phem_status batch_launch_config(int device, int sm_count, int block, int items, BatchLaunch *out);
phem_status batch_launch(cudaStream_t stream, const BatchLaunch &l, BatchArgs args);

}  // namespace phem
