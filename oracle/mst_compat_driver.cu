// mst_compat_driver.cu -- TEST INFRASTRUCTURE: a minimal MST driver built
// against the reference's own types (MST/src/constants.h, from the reference
// tree) and phem_graph_b200/compat/mst_compat.cuh, to check that the compat
// functions compile with the reference's declarations and return its results.
//
//   mst_phem <edges.bin> <n>     edges.bin: m records of three uint32 {u, v, w}
// prints "host <count> <total>" (boruvka_for_edge_array) and
//        "device <count> <total> <nodes left>" (device_boruvka).
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <vector>

#include "constants.h"
#include "../phem_graph_b200/compat/mst_compat.cuh"

int main(int argc, char **argv)
{
    if (argc != 3)
        return 2;
    std::ifstream f(argv[1], std::ios::binary | std::ios::ate);
    const size_t bytes = (size_t)f.tellg();
    f.seekg(0);
    std::vector<edge> e(bytes / sizeof(edge));
    f.read(reinterpret_cast<char *>(e.data()), (std::streamsize)bytes);
    vertex n = (vertex)atol(argv[2]), m = (vertex)e.size();
    std::vector<edge> msf(n);
    vertex filled = 0;
    boruvka_for_edge_array(e.data(), n, m, msf.data(), filled);
    unsigned long long total = 0;
    for (vertex i = 0; i < filled; i++)
        total += msf[i].w;
    printf("host %u %llu\n", filled, total);

    edge *d_e = nullptr, *d_out = nullptr;
    cudaMalloc(&d_e, sizeof(edge) * (m ? m : 1));
    cudaMalloc(&d_out, sizeof(edge) * n);
    cudaMemcpy(d_e, e.data(), sizeof(edge) * m, cudaMemcpyHostToDevice);
    vertex nodes = n, edges_left = m, filled_d = 0;
    device_boruvka(d_e, d_out, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nodes, edges_left, filled_d,
                   thrust::device_ptr<vertex>(), thrust::device_ptr<vertex>(), thrust::device_ptr<vertex>(),
                   thrust::device_ptr<edge>(d_out));
    std::vector<edge> out(filled_d);
    cudaMemcpy(out.data(), d_out, sizeof(edge) * filled_d, cudaMemcpyDeviceToHost);
    unsigned long long total_d = 0;
    for (auto &x : out)
        total_d += x.w;
    printf("device %u %llu %u\n", filled_d, total_d, nodes);
    return 0;
}
