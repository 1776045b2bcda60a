// ref_cc.cpp -- exposes the reference's CC CPU path through a C ABI for the tests.
//
// TEST INFRASTRUCTURE ONLY.  host_spanning_tree() itself is the reference's
// CC/host_spanning_tree.cu, compiled unchanged from the reference tree by
// oracle/Makefile; this file only builds the graph_data_host it expects
// (CC/include/hbcg_utils.cuh:4-18) and times the call.  The number of Parlay
// workers is taken from PARLAY_NUM_THREADS when the library is first used
// (CC/parlay/scheduler.h:203-209); with one worker the edges are united in
// index order.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <thread>

#include "include/hbcg_utils.cuh"

int host_spanning_tree(struct graph_data_host *);  // CC/include/host_spanning_tree.cuh:1

namespace {
struct RefCC {
    graph_data_host h;
    int V = 0;
    long E = 0;
    long edges_size = 0;
    long edge_list_size = 0;
};
}  // namespace

extern "C" {

// Fresh state for n vertices: temp_label[i] = label[i] = i, sptree[i] = INT_MAX
// (CC/main.cu:432-434).
void *ref_cc_create(int32_t n)
{
    RefCC *s = new RefCC();
    s->V = n;
    s->h.V = &s->V;
    s->h.E = &s->E;
    s->h.edges_size = &s->edges_size;
    s->h.edge_list_size = &s->edge_list_size;
    s->h.label = parlay::sequence<int>::from_function(n, [](size_t i) { return (int)i; });
    s->h.temp_label = parlay::sequence<int>::from_function(n, [](size_t i) { return (int)i; });
    s->h.sptree = parlay::sequence<uint64_t>::from_function(n, [](size_t) { return (uint64_t)0x7fffffff; });
    return s;
}

void ref_cc_destroy(void *p) { delete static_cast<RefCC *>(p); }

// Installs the CPU share of the edge list (packed u << 32 | v).
void ref_cc_set_edges(void *p, const uint64_t *edges, int64_t m)
{
    RefCC *s = static_cast<RefCC *>(p);
    s->h.edges = parlay::sequence<uint64_t>::from_function(m, [&](size_t i) { return edges[i]; });
    s->E = m;
    s->edges_size = m;
}

// Runs host_spanning_tree once over the installed edges; state carries over
// between calls exactly as in the reference.  Returns wall seconds of the call.
double ref_cc_run(void *p)
{
    RefCC *s = static_cast<RefCC *>(p);
    auto t0 = std::chrono::steady_clock::now();
    host_spanning_tree(&s->h);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// Resets parents and forest slots to the fresh state without reallocating.
void ref_cc_reset(void *p)
{
    RefCC *s = static_cast<RefCC *>(p);
    for (int i = 0; i < s->V; i++) {
        s->h.temp_label[i] = i;
        s->h.sptree[i] = 0x7fffffff;
    }
}

void ref_cc_get(void *p, int32_t *temp_label, uint64_t *sptree)
{
    RefCC *s = static_cast<RefCC *>(p);
    if (temp_label)
        std::memcpy(temp_label, s->h.temp_label.begin(), sizeof(int32_t) * s->V);
    if (sptree)
        std::memcpy(sptree, s->h.sptree.begin(), sizeof(uint64_t) * s->V);
}

int32_t ref_cc_workers(void) { return (int32_t)parlay::num_workers(); }

}  // extern "C"
