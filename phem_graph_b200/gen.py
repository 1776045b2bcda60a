"""Seeded synthetic graphs (host side, libphem's phem_gen_* entry points).

The reference benchmarks on graph files that are not shipped; these stand in
with seeded inputs of the same shapes.  Every value is a pure function of
(seed, stream, index), so any thread count gives the same graph.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib

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
