// ref_mst.cu -- exposes the reference's PBBS MST CPU path through a C ABI.
//
// TEST INFRASTRUCTURE ONLY.  mst(), create_wghEdgeArray() and the PBBS/Parlay
// code under them are the reference's MST/src/utils.cu (:794-867), included
// from the reference tree unchanged by oracle/Makefile; this file only converts
// the uint32 {u, v, w} edge array the way new_boruvka.cu:469-475 does, runs
// mst() and reports the MSF edge ids it returns (ascending, from pack_index).
#include <fstream>
#include <sstream>
#include <cstring>
#include <cassert>
#include <chrono>
#include <cstdio>
#include <unistd.h>

#include "utils.cu"

namespace {
// mst() prints one line per phase through parlay's timer; keep the caller's
// stdout clean by pointing fd 1 at /dev/null for the duration of the call.
struct QuietStdout {
    int saved = -1;
    QuietStdout()
    {
        fflush(stdout);
        std::cout.flush();
        saved = dup(1);
        FILE *devnull = fopen("/dev/null", "w");
        if (devnull) {
            dup2(fileno(devnull), 1);
            fclose(devnull);
        }
    }
    ~QuietStdout()
    {
        fflush(stdout);
        std::cout.flush();
        if (saved >= 0) {
            dup2(saved, 1);
            close(saved);
        }
    }
};

struct RefMST {
    wghEdgeArray<vertexId, vertexId> ea;
    parlay::sequence<edgeId> result;
};
}  // namespace

extern "C" {

// Builds the PBBS edge array (n = max vertex id + 1, create_wghEdgeArray).
// uvw holds m records of three uint32 (MST/src/constants.h:15-19).
void *ref_mst_create(const uint32_t *uvw, uint64_t m)
{
    edge_pbbs *e = (edge_pbbs *)malloc((m ? m : 1) * sizeof(edge_pbbs));
    for (uint64_t i = 0; i < m; i++) {
        e[i].u = (int)uvw[3 * i];
        e[i].v = (int)uvw[3 * i + 1];
        e[i].w = (int)uvw[3 * i + 2];
    }
    RefMST *s = new RefMST();
    s->ea = create_wghEdgeArray(e, m);
    free(e);
    return s;
}

void ref_mst_destroy(void *p) { delete static_cast<RefMST *>(p); }

// Runs mst() once.  threads > 0 runs it inside a private Parlay scheduler with
// that many workers; 0 uses the default scheduler.  Returns 0 on success with
// *seconds = wall time of mst(), 2 when PBBS throws (speculative_for gives up
// on phases of 1..14 edges, MST/src/common/speculative_for.h:54-71).
int ref_mst_run(void *p, int32_t threads, double *seconds)
{
    RefMST *s = static_cast<RefMST *>(p);
    int rc = 0;
    auto body = [&]() {
        QuietStdout quiet;
        try {
            auto t0 = std::chrono::steady_clock::now();
            s->result = mst(s->ea);
            auto t1 = std::chrono::steady_clock::now();
            *seconds = std::chrono::duration<double>(t1 - t0).count();
        } catch (const std::exception &) {
            rc = 2;
        }
    };
    if (threads > 0)
        parlay::execute_with_scheduler((unsigned)threads, body);
    else
        body();
    return rc;
}

uint64_t ref_mst_count(void *p) { return static_cast<RefMST *>(p)->result.size(); }

void ref_mst_ids(void *p, uint32_t *out)
{
    RefMST *s = static_cast<RefMST *>(p);
    for (size_t i = 0; i < s->result.size(); i++)
        out[i] = s->result[i];
}

int32_t ref_mst_workers(void) { return (int32_t)parlay::num_workers(); }

}  // extern "C"

extern "C" {

// The MST driver's MatrixMarket reader (getGraphInfo + mmapPopulateEdgeArray,
// MST/src/utils.cu:160-180, 896-1036) on `path`: *n, *m from the size line;
// uvw (3 * capacity uint32, zero-filled here as fresh pinned pages are) gets
// the records.  Returns 0, or 1 when capacity < m.
int ref_mtx_read(const char *path, int generate_weights, uint32_t *uvw, uint64_t capacity, uint32_t *n, uint64_t *m)
{
    std::ifstream file(path);
    vertex num_nodes = 0;
    large_vertex num_edges = 0;
    {
        QuietStdout quiet;
        getGraphInfo(file, num_nodes, num_edges);
    }
    *n = num_nodes;
    *m = num_edges;
    if (!uvw)
        return 0;
    if (capacity < num_edges)
        return 1;
    std::vector<edge> e(num_edges ? num_edges : 1, edge{0, 0, 0});
    {
        QuietStdout quiet;
        mmapPopulateEdgeArray(path, e.data(), (vertex)num_edges, num_nodes, generate_weights != 0);
    }
    memcpy(uvw, e.data(), sizeof(edge) * num_edges);
    return 0;
}

}  // extern "C"

