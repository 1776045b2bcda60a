// mst_compat.cuh -- the reference MST entry points over libphem.
//
// The MST driver is one translation unit (MST/main.cu includes
// src/new_boruvka.cu, which includes the kernels and utilities).  To run it
// on libphem, delete the definitions of boruvka_for_edge_array
// (MST/src/new_boruvka.cu:40-179) and device_boruvka (MST/src/kernels.cu:507-689),
// include this header after MST/src/constants.h, and link -lphem.  The
// functions keep the reference's names, signatures and buffer semantics;
// errors print to stderr and exit(EXIT_FAILURE), as the reference does on
// CUDA errors.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

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
