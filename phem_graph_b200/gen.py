"""Seeded synthetic graphs (host side: the phem_gen_* entry points, loaded from
libphem_gen.so, which holds the generators alone).

The reference benchmarks on graph files that are not shipped; these stand in
with seeded inputs of the same shapes.  Every value is a pure function of
(seed, stream, index), so any thread count gives the same graph.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check_gen as check, gen_lib as lib

# R-MAT quadrant probabilities of the benchmark configurations (a, b, c; d = 1 - a - b - c)
RMAT_ABC = (0.57, 0.19, 0.19)
WEIGHT_BITS = 20  # weights uniform in [1, 2^20]


def er(n: int, draws: int, seed: int) -> np.ndarray:
    """Erdos-Renyi pairs: packed (min << 32 | max), self-loops dropped, duplicates
    kept, in draw order."""
    out = np.empty(max(draws, 1), np.uint64)
    m = C.c_uint64()
    check(lib().phem_gen_er(n, draws, seed, out.ctypes.data, C.byref(m)), "phem_gen_er")
    return out[: m.value]


def rmat(scale: int, draws: int, seed: int, abc=RMAT_ABC) -> np.ndarray:
    """R-MAT pairs packed (min << 32 | max), sorted ascending (upper triangle of
    the symmetrised CSR in row-major order), self-loops dropped, duplicates kept."""
    out = np.empty(max(draws, 1), np.uint64)
    m = C.c_uint64()
    a, b, c = abc
    check(lib().phem_gen_rmat(scale, draws, a, b, c, seed, out.ctypes.data, C.byref(m)), "phem_gen_rmat")
    return out[: m.value]


def rmat_range(scale: int, first: int, count: int, seed: int, abc=RMAT_ABC) -> np.ndarray:
    """Draws [first, first + count) of the rmat() stream, unsorted, in draw order
    (self-loops dropped): a huge graph batch by batch."""
    out = np.empty(max(count, 1), np.uint64)
    m = C.c_uint64()
    a, b, c = abc
    check(lib().phem_gen_rmat_range(scale, first, count, a, b, c, seed, out.ctypes.data, C.byref(m)),
          "phem_gen_rmat_range")
    return out[: m.value]


def rmat_range_device(ctx, scale: int, first: int, count: int, seed: int, out, abc=RMAT_ABC) -> int:
    """rmat_range on the GPU (libphem's phem_gen_rmat_range_device) into the
    device tensor `out` (>= count int64 entries); returns the number written."""
    from ._lib import check as check_phem, lib as phem_lib
    m = C.c_uint64()
    a, b, c = abc
    check_phem(phem_lib().phem_gen_rmat_range_device(ctx.handle, scale, first, count, a, b, c, seed,
                                                     out.data_ptr(), C.byref(m)), "phem_gen_rmat_range_device")
    return m.value


def weights(m: int, seed: int, bits: int = WEIGHT_BITS) -> np.ndarray:
    w = np.empty(max(m, 1), np.uint32)
    check(lib().phem_gen_weights(m, seed, bits, w.ctypes.data), "phem_gen_weights")
    return w[:m]


def msf_edges(pairs: np.ndarray, w: np.ndarray | None) -> np.ndarray:
    """(m, 3) uint32 {u, v, w} records from packed pairs and weights."""
    pairs = np.ascontiguousarray(pairs, np.uint64)
    out = np.empty((max(len(pairs), 1), 3), np.uint32)
    wp = None if w is None else np.ascontiguousarray(w, np.uint32).ctypes.data
    check(lib().phem_pack_msf_edges(pairs.ctypes.data, wp, len(pairs), out.ctypes.data), "phem_pack_msf_edges")
    return out[: len(pairs)]


def csr_from_pairs(pairs: np.ndarray, n: int):
    """Symmetrised CSR (int64 offsets[n + 1], uint32 cols[2m]) from sorted pairs."""
    pairs = np.ascontiguousarray(pairs, np.uint64)
    offsets = np.empty(n + 1, np.int64)
    cols = np.empty(max(2 * len(pairs), 1), np.uint32)
    check(lib().phem_csr_from_sorted_pairs(pairs.ctypes.data, len(pairs), n, offsets.ctypes.data, cols.ctypes.data),
          "phem_csr_from_sorted_pairs")
    return offsets, cols[: 2 * len(pairs)]


@dataclass
class Graph:
    name: str
    n: int
    pairs: np.ndarray            # packed (u << 32 | v), u < v
    w: np.ndarray | None = None  # uint32 weights by edge id

    @property
    def m(self) -> int:
        return len(self.pairs)

    def msf_edges(self) -> np.ndarray:
        return msf_edges(self.pairs, self.w)


def er_graph(n: int, draws: int, seed: int = 1) -> Graph:
    """Connected-components workload: ER over n vertices with `draws` pair draws."""
    return Graph(f"er_n{n}_d{draws}_s{seed}", n, er(n, draws, seed))


def rmat_graph(scale: int, edge_factor: int = 16, seed: int = 22, weight_seed: int | None = None,
               bits: int = WEIGHT_BITS) -> Graph:
    """MSF workload: R-MAT on 2^scale vertices with edge_factor * 2^scale draws
    and weights uniform in [1, 2^bits] by edge id."""
    n = 1 << scale
    pairs = rmat(scale, edge_factor * n, seed)
    ws = seed + 1000 if weight_seed is None else weight_seed
    return Graph(f"rmat{scale}_ef{edge_factor}_s{seed}", n, pairs, weights(len(pairs), ws, bits))


def rgg(n: int, k: int, seed: int):
    """2-D random geometric k-nearest-neighbour graph: (pairs, weights), pairs
    packed (min << 32 | max) and sorted, weights floor(distance * 2^24)."""
    cap = max(n * k, 1)
    out = np.empty(cap, np.uint64)
    w = np.empty(cap, np.uint32)
    m = C.c_uint64()
    check(lib().phem_gen_rgg(n, k, seed, out.ctypes.data, w.ctypes.data, C.byref(m)), "phem_gen_rgg")
    return out[: m.value], w[: m.value]


def rgg_graph(n: int, k: int = 8, seed: int = 1) -> Graph:
    pairs, w = rgg(n, k, seed)
    return Graph(f"rgg_n{n}_k{k}_s{seed}", n, pairs, w)


# ------------------------------------------------------------------ batches

PHEM_BATCH_MSF = 0
PHEM_BATCH_CC = 1

# phem_batch_graph (include/phem.h)
BATCH_GRAPH = np.dtype([("edge_offset", "<u8"), ("num_edges", "<u4"), ("num_vertices", "<u4"),
                        ("vertex_offset", "<u4"), ("kind", "<u4")])
assert BATCH_GRAPH.itemsize == 24


@dataclass
class Batch:
    graphs: np.ndarray   # BATCH_GRAPH records
    edges: np.ndarray    # (E, 3) uint32 {u, v, w}, vertex ids local to each graph
    total_vertices: int
    names: list

    @property
    def num_graphs(self) -> int:
        return len(self.graphs)

    @property
    def total_edges(self) -> int:
        return len(self.edges)

    def graph_edges(self, g: int) -> np.ndarray:
        r = self.graphs[g]
        o = int(r["edge_offset"])
        return self.edges[o: o + int(r["num_edges"])]


def batch_from(parts) -> Batch:
    """Concatenates (name, n, edges (m, 3) uint32, kind) tuples into one batch."""
    parts = list(parts)
    graphs = np.zeros(len(parts), BATCH_GRAPH)
    e_off = v_off = 0
    for g, (_, n, e, kind) in enumerate(parts):
        graphs[g] = (e_off, len(e), n, v_off, kind)
        e_off += len(e)
        v_off += n
    edges = np.concatenate([p[2].reshape(-1, 3) for p in parts]) if parts else np.empty((0, 3), np.uint32)
    return Batch(graphs, np.ascontiguousarray(edges, np.uint32), v_off, [p[0] for p in parts])


_TAG_BATCH = 0x42415443482D47  # "BATCH-G"


def _unit(seed: int, i: int) -> float:
    return (int(lib().phem_gen_mix64(seed, _TAG_BATCH, i)) >> 11) * 2.0 ** -53


def mixed_graph(i: int, seed: int, n_lo: int = 64, n_hi: int = 65536):
    """Graph i of the many-small-graphs workload: n log-uniform in [n_lo, n_hi];
    even i Erdos-Renyi with mean degree uniform in [2, 16] and weights uniform
    in [1, 2^20], odd i a 2-D random geometric 8-nearest-neighbour graph with
    weights floor(distance * 2^24)."""
    n = int(n_lo * (n_hi / n_lo) ** _unit(seed, 4 * i))
    n = max(n_lo, min(n, n_hi))
    gs = seed * 1000003 + i
    if i % 2 == 0:
        deg = 2.0 + 14.0 * _unit(seed, 4 * i + 1)
        pairs = er(n, int(round(n * deg / 2)), gs)
        w = weights(len(pairs), gs + 7)
        name = f"er{i}_n{n}"
    else:
        pairs, w = rgg(n, 8, gs)
        name = f"rgg{i}_n{n}"
    return name, n, msf_edges(pairs, w)


def mixed_batch(num_graphs: int = 4096, seed: int = 4, n_lo: int = 64, n_hi: int = 65536, kind=PHEM_BATCH_MSF,
                threads: int = 16) -> Batch:
    """The many-small-graphs workload (4096 graphs by default); graphs are
    generated on `threads` host threads (the generators release the GIL).
    `kind` is a batch kind or a function of the graph index."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(threads) as ex:
        parts = list(ex.map(lambda i: mixed_graph(i, seed, n_lo, n_hi), range(num_graphs)))
    kinds = kind if callable(kind) else (lambda i: kind)
    return batch_from((name, n, e, kinds(i)) for i, (name, n, e) in enumerate(parts))
