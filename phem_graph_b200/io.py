"""Graph files in the reference drivers' formats (readers in csrc/io.cpp).

read_mtx          MatrixMarket coordinate files as the MST driver reads them
read_ecl          ECL binary CSR as the CC driver reads it
read_graph_pairs  the CC driver's input (edge list or ECL) as packed u < v pairs

The writers produce files in the same formats (for tests and for converting
generated graphs into inputs the reference drivers accept).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import lib


class GraphFileError(ValueError):
    pass


def _check(status: int, what: str) -> None:
    if status != 0:
        raise GraphFileError(f"{what}: {lib().phem_io_last_error().decode()}")


def read_mtx(path, generate_weights: bool = False):
    """(edges (m, 3) uint32 {u, v, w} with u <= v, n) of a MatrixMarket file."""
    p = os.fsencode(path)
    n, m = C.c_uint32(), C.c_uint64()
    _check(lib().phem_read_mtx(p, int(generate_weights), None, 0, C.byref(n), C.byref(m)), "read_mtx")
    out = np.empty((max(m.value, 1), 3), np.uint32)
    _check(lib().phem_read_mtx(p, int(generate_weights), out.ctypes.data, m.value, C.byref(n), C.byref(m)),
           "read_mtx")
    return out[: m.value], n.value


def read_ecl(path):
    """(offsets int64[n + 1], cols uint32[nnz], n) of an ECL binary CSR file."""
    p = os.fsencode(path)
    n, nnz = C.c_uint32(), C.c_uint64()
    _check(lib().phem_read_ecl(p, None, None, 0, C.byref(n), C.byref(nnz)), "read_ecl")
    off = np.empty(n.value + 1, np.int64)
    cols = np.empty(max(nnz.value, 1), np.uint32)
    _check(lib().phem_read_ecl(p, off.ctypes.data, cols.ctypes.data, nnz.value, C.byref(n), C.byref(nnz)),
           "read_ecl")
    return off, cols[: nnz.value], n.value


def read_graph_pairs(path):
    """(pairs uint64 packed (u << 32 | v) with u < v, n) as the CC driver reads a file."""
    p = os.fsencode(path)
    n, m = C.c_uint32(), C.c_uint64()
    _check(lib().phem_read_graph_pairs(p, None, 0, C.byref(n), C.byref(m)), "read_graph_pairs")
    out = np.empty(max(m.value, 1), np.uint64)
    _check(lib().phem_read_graph_pairs(p, out.ctypes.data, m.value, C.byref(n), C.byref(m)), "read_graph_pairs")
    return out[: m.value], n.value


def write_mtx(path, edges, n: int, weights: bool = True) -> None:
    """MatrixMarket coordinate file of (m, 3) {u, v, w} records (0-based in, 1-based out)."""
    e = np.asarray(edges, np.uint64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate integer symmetric\n")
        f.write(f"{n} {n} {len(e)}\n")
        cols = [e[:, 0] + 1, e[:, 1] + 1] + ([e[:, 2]] if weights else [])
        np.savetxt(f, np.column_stack(cols), fmt="%d")


def write_ecl(path, offsets, cols) -> None:
    off = np.ascontiguousarray(offsets, np.int64)
    c = np.ascontiguousarray(cols, np.int32)
    with open(path, "wb") as f:
        f.write(np.array([len(off) - 1, len(c)], np.int64).tobytes())
        f.write(off.tobytes())
        f.write(c.tobytes())


def write_edge_list(path, pairs, n: int) -> None:
    """Text edge list with both directions of every packed u < v pair."""
    p = np.asarray(pairs, np.uint64)
    u, v = (p >> np.uint64(32)).astype(np.int64), (p & np.uint64(0xFFFFFFFF)).astype(np.int64)
    with open(path, "w") as f:
        f.write(f"{n} {2 * len(p)}\n")
        np.savetxt(f, np.column_stack([np.concatenate([u, v]), np.concatenate([v, u])]), fmt="%d")
