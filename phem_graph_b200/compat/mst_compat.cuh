// mst_compat.cuh -- the reference MST entry points over libphem.
//
// The MST driver is one translation unit (MST/main.cu includes
// src/new_boruvka.cu, which includes the kernels and utilities).  To run it
// on libphem, delete the definitions of boruvka_for_edge_array
// (MST/src/new_boruvka.cu:40-179), device_boruvka (MST/src/kernels.cu:507-689)
// and streamline_boruvka (MST/src/kernels.cu:849-1154), include this header
// after MST/src/constants.h, and link -lphem.  The
// functions keep the reference's names, signatures and buffer semantics;
// errors print to stderr and exit(EXIT_FAILURE), as the reference does on
// CUDA errors.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#include <thrust/device_ptr.h>

#include "../../include/phem.h"

static_assert(sizeof(edge) == sizeof(phem_edge), "edge must be three 32-bit fields (MST/src/constants.h:15-19)");

inline void phem_compat_check(phem_status s, const char *what)
{
    if (s != PHEM_OK) {
        fprintf(stderr, "%s: %s: %s\n", what, phem_status_string(s), phem_last_error());
        exit(EXIT_FAILURE);
    }
}

inline phem_context *phem_compat_context()
{
    static phem_context *c = [] {
        phem_context *p = nullptr;
        phem_compat_check(phem_context_create(0, &p), "phem_context_create");
        return p;
    }();
    return c;
}

// boruvka_for_edge_array (MST/src/new_boruvka.cu:40-179): host edges in,
// host final_msf out (the forest ascending by edge index, the PBBS order),
// number_of_filled_edges = forest size; prints the total weight as the
// reference does (its total summed only the written slots here).
inline void boruvka_for_edge_array(edge *edges, vertex num_nodes, vertex num_edges, edge *final_msf,
                                   vertex &number_of_filled_edges, std::string result = "res.txt")
{
    (void)result;
    uint64_t count = 0, total = 0;
    phem_compat_check(phem_msf_solve(phem_compat_context(), reinterpret_cast<const phem_edge *>(edges), num_edges,
                                     num_nodes, reinterpret_cast<phem_edge *>(final_msf), &count, &total, nullptr),
                      "boruvka_for_edge_array");
    number_of_filled_edges = (vertex)count;
    std::cout << "total weight " << total << std::endl;
    std::cout << "number of filled edges " << number_of_filled_edges << std::endl;
}

// device_boruvka (MST/src/kernels.cu:507-689): device edges in; the forest
// is appended to d_final_msf at number_of_filled_edges (which grows by the
// forest size); on return num_edges = 0 and num_nodes = the number of
// components, as after the reference's last round.  The work buffers the
// reference needs are accepted and left untouched.
inline void device_boruvka(edge *d_edges, edge *d_final_msf, edge *d_iter_edges, edge *d_msf,
                           vertex *d_representatives, vertex *d_new_representatives,
                           vertex *d_iter_representatives, outgoing_edge_id *d_outgoing_edges, vertex &num_nodes,
                           vertex &num_edges, vertex &number_of_filled_edges,
                           thrust::device_ptr<vertex> d_new_representatives_ptr,
                           thrust::device_ptr<vertex> d_representatives_ptr,
                           thrust::device_ptr<vertex> d_iter_representatives_ptr,
                           thrust::device_ptr<edge> d_final_msf_ptr, cudaStream_t kernel_stream = 0)
{
    (void)d_iter_edges, (void)d_msf, (void)d_representatives, (void)d_new_representatives;
    (void)d_iter_representatives, (void)d_outgoing_edges, (void)d_new_representatives_ptr;
    (void)d_representatives_ptr, (void)d_iter_representatives_ptr, (void)d_final_msf_ptr;
    phem_context *ctx = phem_compat_context();
    if (kernel_stream)
        phem_compat_check(phem_context_set_stream(ctx, kernel_stream), "device_boruvka");
    phem_msf_stats st{};
    phem_compat_check(phem_msf_solve_device(ctx, reinterpret_cast<const phem_edge *>(d_edges), num_edges, num_nodes,
                                            reinterpret_cast<phem_edge *>(d_final_msf + number_of_filled_edges),
                                            nullptr, &st),
                      "device_boruvka");
    if (kernel_stream)
        phem_compat_check(phem_context_set_stream(ctx, nullptr), "device_boruvka");
    number_of_filled_edges += (vertex)st.msf_edges;
    num_nodes -= (vertex)st.msf_edges;
    num_edges = 0;
}

// The reference's chunk reader (MST/src/utils.cu:300), defined by the driver
// that includes this header; streamline_boruvka fills its chunks with it.
void populateEdgeChunksLarge(std::ifstream &file, edge **chunks_of_edges, large_vertex num_edges, vertex num_nodes,
                             vertex chunk_size, vertex last_chunk_size, int num_chunks, bool generate_random_weights,
                             bool is_weight_float);

// streamline_boruvka (MST/src/kernels.cu:849-1154): the reference's reader
// fills the chunks (views into one pinned block), phem_msf_stream solves them
// in order with the forest carried from chunk to chunk and the next chunk's
// copy overlapped, and each of the execution_time_iterations runs prints its
// time and the forest's total weight as the reference does.  Unless
// result_filename is "res.txt" the forest is written as the reference writes
// it, "u+1 v+1 w" per line; it holds the forest's edges only (the reference
// writes num_nodes - 1 slots whether filled or not), ascending by edge index.
inline void streamline_boruvka(std::ifstream &input_stream, vertex num_nodes, large_vertex num_edges,
                               vertex chunk_size, std::string result_filename = "res.txt",
                               bool generate_random_weights = false, bool is_weight_float = false,
                               int execution_time_iterations = 1)
{
    std::cout << "streamline chunk boruvka " << std::endl;
    if (chunk_size == 0 || num_nodes == 0) {
        fprintf(stderr, "streamline_boruvka: chunk size and node count must be positive\n");
        exit(EXIT_FAILURE);
    }
    const int num_chunks = (int)((num_edges + chunk_size - 1) / chunk_size);
    const vertex last_chunk_size =
        num_chunks ? (vertex)(num_edges - (large_vertex)(num_chunks - 1) * chunk_size) : 0;
    edge *block = nullptr, *final_msf = nullptr;
    if (cudaMallocHost(reinterpret_cast<void **>(&block), (num_edges ? num_edges : 1) * sizeof(edge)) !=
            cudaSuccess ||
        cudaMallocHost(reinterpret_cast<void **>(&final_msf), (size_t)num_nodes * sizeof(edge)) != cudaSuccess) {
        fprintf(stderr, "streamline_boruvka: cannot allocate pinned host memory\n");
        exit(EXIT_FAILURE);
    }
    std::vector<edge *> chunks(num_chunks);
    for (int i = 0; i < num_chunks; i++)
        chunks[i] = block + (size_t)i * chunk_size;
    if (num_chunks)
        populateEdgeChunksLarge(input_stream, chunks.data(), num_edges, num_nodes, chunk_size, last_chunk_size,
                                num_chunks, generate_random_weights, is_weight_float);
    std::vector<long long> times;
    for (int it = 0; it < execution_time_iterations; it++) {
        uint64_t count = 0, total = 0;
        const auto t0 = std::chrono::high_resolution_clock::now();
        phem_compat_check(phem_msf_stream(phem_compat_context(), reinterpret_cast<const phem_edge *>(block),
                                          num_edges, num_nodes, chunk_size, reinterpret_cast<phem_edge *>(final_msf),
                                          &count, &total, nullptr),
                          "streamline_boruvka");
        const long long us = std::chrono::duration_cast<std::chrono::microseconds>(
                                 std::chrono::high_resolution_clock::now() - t0)
                                 .count();
        std::cout << "streamline execution time " << us << " microseconds\n";
        times.push_back(us);
        if (result_filename != "res.txt") {
            std::ofstream result(result_filename);
            for (uint64_t i = 0; i < count; i++)
                result << final_msf[i].u + 1 << " " << final_msf[i].v + 1 << " " << final_msf[i].w << "\n";
        }
        std::cout << "final weight by streamline approach " << total << "\n";
    }
    long long sum = 0;
    for (size_t i = 0; i < times.size(); i++) {
        std::cout << i << "th execution time " << times[i] << std::endl;
        sum += times[i];
    }
    if (!times.empty())
        std::cout << "Average exec time " << sum / (long long)times.size() << std::endl;
    cudaFreeHost(final_msf);
    cudaFreeHost(block);
}
