// mst_stream_compat_driver.cu -- TEST INFRASTRUCTURE: the reference's own
// graph-info and chunk readers (getGraphInfo and populateEdgeChunksLarge from
// MST/src/utils.cu, included from the reference tree unchanged) feeding
// streamline_boruvka from phem_graph_b200/compat/mst_compat.cuh, called the way
// new_boruvka calls it (MST/src/new_boruvka.cu:339-380).
//
//   mst_stream_phem <graph.mtx> <num_chunks> <result file>
// writes the forest to the result file ("u+1 v+1 w" per line) and prints the
// reference's lines, "final weight by streamline approach <total>" among them.
#include <fstream>
#include <sstream>
#include <cstring>
#include <cassert>
#include <unistd.h>

#include "utils.cu"
#include "../phem_graph_b200/compat/mst_compat.cuh"

int main(int argc, char **argv)
{
    if (argc != 4)
        return 2;
    std::ifstream file(argv[1]);
    vertex num_nodes = 0;
    large_vertex num_edges = 0;
    getGraphInfo(file, num_nodes, num_edges);
    // chunk size from the requested chunk count, as new_boruvka.cu:349-353
    const vertex chunk_size = vertex(num_edges / (float)atoi(argv[2]));
    streamline_boruvka(file, num_nodes, num_edges, chunk_size, argv[3], false, false, 2);
    return 0;
}
