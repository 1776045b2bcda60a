// hast_compat.cpp -- the reference CC driver's GPU entry points over libphem.
//
// CC/Makefile builds the driver from graph.cu, main.cu, host_spanning_tree.cu,
// ExternalSpanningTree.cu and GPUSpanningTree.cu.  Compiling this file in
// place of the last two (and linking -lphem) keeps main.cu unchanged: the
// functions below have the reference's names, signatures and buffer
// semantics (CC/include/ExternalSpanningTree.cuh:1, GPUSpanningtree.cuh:1-2)
// and run on libphem's C ABI instead of the reference kernels.  Errors are
// reported the way the reference reports CUDA errors: a message on stderr
// and exit(EXIT_FAILURE) (CC/GPUSpanningTree.cu:17).
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "../../include/phem.h"

extern int Batch_Size;  // the driver's globals (CC/main.cu:21-22)
extern float GPU_share;

// The driver's pointer bundle, member for member as CC/include/hbcg_utils.cuh:20-42
// declares it (same name and layout, so main.cu's objects pass straight through).
struct graph_data {
    uint64_t *edges;
    uint64_t *edges2;
    int *temp_label;
    int *label;
    int *V;
    long *E;
    long *size;
    long *size2;
    uint64_t *T1edges;
    uint64_t *T2edges;
    int *first_occ;
    int *last_occ;
    int *parent;
    int *w1;
    int *w2;
    int *w1_copy;
    int *w2_copy;
    uint64_t *SpanningForest;
    int *low;
    int *high;
    bool *fg1;
};
struct graph_data_host;  // the CPU share's bundle; not read here

namespace {

void check(phem_status s, const char *what)
{
    if (s != PHEM_OK) {
        fprintf(stderr, "%s: %s: %s\n", what, phem_status_string(s), phem_last_error());
        exit(EXIT_FAILURE);
    }
}

phem_context *context()
{
    static phem_context *c = [] {
        phem_context *p = nullptr;
        check(phem_context_create(0, &p), "phem_context_create");
        return p;
    }();
    return c;
}

}  // namespace

// SpanningTree (CC/ExternalSpanningTree.cu:133-218): parent = temp_label,
// label = identity, forest slots in T1edges; the host edges h_input->edges
// (pinned, E[0] of them) stream through the GPU in batches of Batch_Size.
// The heterogeneous CPU share is not part of this build: GPU_share must be 1.
float SpanningTree(graph_data *h_input, graph_data *d_input, graph_data_host *)
{
    if (!(GPU_share == 1.0f)) {  // a float: 1.9 and 0.9999 are both a CPU share
        fprintf(stderr, "SpanningTree: GPU_share = %f; this build runs every edge on the GPU (use 1)\n",
                (double)GPU_share);
        exit(EXIT_FAILURE);
    }
    float ms = 0.f;
    check(phem_cc_stream(context(), h_input->edges, (int64_t)h_input->E[0], h_input->V[0], (int64_t)Batch_Size,
                         d_input->temp_label, d_input->label, d_input->T1edges, &ms),
          "SpanningTree");
    return ms;
}

// gpu_spanning_tree (CC/GPUSpanningTree.cu:169-198): unions T1edges and the
// caller's extraedges (n slots each) into a fresh state; final min-id labels
// in label, final forest in T2edges.
float gpu_spanning_tree(graph_data *d_input, uint64_t *extraedges, int vert)
{
    float ms = 0.f;
    check(phem_cc_merge(context(), d_input->T1edges, extraedges, vert, d_input->temp_label, d_input->label,
                        d_input->T2edges, &ms),
          "gpu_spanning_tree");
    return ms;
}

// gpu_spanning_tree_2 (CC/GPUSpanningTree.cu:200-229): the same merge with the
// final forest in SpanningForest.
float gpu_spanning_tree_2(graph_data *d_input, uint64_t *extraedges, int vert)
{
    float ms = 0.f;
    check(phem_cc_merge(context(), d_input->T1edges, extraedges, vert, d_input->temp_label, d_input->label,
                        d_input->SpanningForest, &ms),
          "gpu_spanning_tree_2");
    return ms;
}
