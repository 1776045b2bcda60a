// ref_serial_mst.cpp -- exposes PBBS's serial Kruskal (MST/src/bench/serialMST.C)
// through a C ABI for the tests.
//
// TEST INFRASTRUCTURE ONLY.  serialMST.C is compiled unchanged from the
// reference tree by oracle/Makefile.  It orders edges by (weight, id) with
// float weights (bench/MST.h:7), exact for the integer weights < 2^24 the
// tests use, and it has no minimum-size limit, so it pins the tiny graphs on
// which the parallel PBBS mst() gives up.
#include <cstdint>
#include <cstdlib>

#include "bench/MST.h"

extern "C" {

// uvw: m records of three uint32.  n = max vertex id + 1, as create_wghEdgeArray
// (MST/src/utils.cu:854-867) sets it.  out_ids needs room for m ids; the ids
// come back in the order Kruskal accepted them.  Returns the count.
uint64_t ref_serial_mst(const uint32_t *uvw, uint64_t m, uint32_t *out_ids)
{
    size_t maxv = 0;
    for (uint64_t i = 0; i < m; i++) {
        size_t a = uvw[3 * i], b = uvw[3 * i + 1];
        maxv = std::max(maxv, std::max(a, b));
    }
    auto E = parlay::sequence<wghEdge<vertexId, edgeWeight>>::from_function(m, [&](size_t i) {
        return wghEdge<vertexId, edgeWeight>((int)uvw[3 * i], (int)uvw[3 * i + 1], (float)uvw[3 * i + 2]);
    });
    wghEdgeArray<vertexId, edgeWeight> G(std::move(E), (int)(m ? maxv + 1 : 0));
    parlay::sequence<edgeId> r = mst(G);
    for (size_t i = 0; i < r.size(); i++)
        out_ids[i] = r[i];
    return r.size();
}

}  // extern "C"
