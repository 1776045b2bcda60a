"""Python view of the serving loop (phem_server_*, include/phem.h).

The loop itself is native (csrc/server.cu): worker threads, continuous
batching, memory-budget admission.  This module builds requests from numpy
arrays, keeps their buffers alive while they are in flight and turns results
into records.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import (PHEM_BATCH_CC, PHEM_BATCH_MSF, Request, RequestResult, ServerConfig, check, lib, ptr)


@dataclass
class ServedGraph:
    """One request: an MSF graph ({u, v, w} records) or a CC graph (packed pairs)."""
    kind: int
    n: int
    edges: np.ndarray | None = None   # (m, 3) uint32, MSF
    pairs: np.ndarray | None = None   # (m,) uint64, CC

    @property
    def m(self) -> int:
        return len(self.edges) if self.kind == PHEM_BATCH_MSF else len(self.pairs)


@dataclass
class Served:
    status: int
    path: int
    forest_edges: int
    total_weight: int
    latency_ns: int
    queue_ns: int
    forest: np.ndarray | None   # MSF: (count, 3) uint32 ascending by edge id
    labels: np.ndarray | None   # CC: min-id labels
    submit_ns: int = 0          # steady-clock times of submission and completion (native)
    done_ns: int = 0


class Server:
    def __init__(self, device: int = 0, memory_budget: int = 8 << 30, slots: int = 2, max_batch_graphs: int = 1024,
                 large_edges: int = 1 << 18, large_workers: int = 2):
        cfg = ServerConfig(memory_budget, slots, max_batch_graphs, large_edges, large_workers, 0)
        self._h = C.c_void_p()
        check(lib().phem_server_create(device, C.byref(cfg), C.byref(self._h)), "phem_server_create")

    def close(self) -> None:
        if self._h:
            lib().phem_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _request(g: ServedGraph):
        """(Request, keep-alive arrays, output arrays)."""
        r = Request()
        r.kind = g.kind
        r.num_vertices = g.n
        if g.kind == PHEM_BATCH_MSF:
            e = np.ascontiguousarray(g.edges, np.uint32).reshape(-1, 3)
            out = np.empty((max(g.n - 1, 1), 3), np.uint32)
            r.num_edges = len(e)
            r.edges = ptr(e)
            r.forest = ptr(out)
            return r, (e, out), out
        p = np.ascontiguousarray(g.pairs, np.uint64)
        out = np.empty(g.n, np.int32)
        r.num_edges = len(p)
        r.pairs = ptr(p)
        r.labels = ptr(out)
        return r, (p, out), out

    @staticmethod
    def _served(g: ServedGraph, res: RequestResult, out) -> Served:
        forest = labels = None
        if res.status == 0:
            if g.kind == PHEM_BATCH_MSF:
                forest = out[: res.forest_edges]
            else:
                labels = out
        return Served(int(res.status), int(res.path), int(res.forest_edges), int(res.total_weight),
                      int(res.done_ns - res.submit_ns), int(res.start_ns - res.submit_ns), forest, labels,
                      int(res.submit_ns), int(res.done_ns))

    def solve(self, g: ServedGraph) -> Served:
        """Submits one request and waits for it."""
        r, keep, out = self._request(g)
        t = C.c_uint64()
        check(lib().phem_server_submit(self._h, C.byref(r), C.byref(t)), "phem_server_submit")
        res = RequestResult()
        check(lib().phem_server_wait(self._h, t.value, 0, C.byref(res)), "phem_server_wait")
        return self._served(g, res, out)

    def replay(self, graphs, arrival_ns) -> list:
        """Open-loop load: graphs[i] is submitted arrival_ns[i] nanoseconds after
        the call starts (by a native thread); returns every result in order."""
        graphs = list(graphs)
        reqs = (Request * max(len(graphs), 1))()
        keep, outs = [], []
        for i, g in enumerate(graphs):
            r, k, o = self._request(g)
            reqs[i] = r
            keep.append(k)
            outs.append(o)
        arr = np.ascontiguousarray(arrival_ns, np.uint64)
        res = (RequestResult * max(len(graphs), 1))()
        lib().phem_server_replay(self._h, reqs, ptr(arr), len(graphs), res)
        return [self._served(g, res[i], outs[i]) for i, g in enumerate(graphs)]


_TAG_SERVE = 0x53455256452D47  # "SERVE-G"


def request_graph(i: int, seed: int = 5, m_lo: int = 1 << 10, m_hi: int = 1 << 24, cc_share: float = 0.7) -> ServedGraph:
    """Request i of the served stream: m log-uniform in [m_lo, m_hi]; 70% CC
    (packed pairs) / 30% MSF ({u, v, w}, weights uniform in [1, 2^20]); half
    Erdos-Renyi (n = m / 4), half R-MAT (edge factor 8)."""
    from . import gen

    def unit(t):
        return (int(lib().phem_gen_mix64(seed, _TAG_SERVE, 4 * i + t)) >> 11) * 2.0 ** -53

    m = int(m_lo * (m_hi / m_lo) ** unit(0))
    kind = PHEM_BATCH_CC if unit(1) < cc_share else PHEM_BATCH_MSF
    gs = seed * 7919 + i
    if unit(2) < 0.5:
        n = max(16, m // 4)
        pairs = gen.er(n, m, gs)
    else:
        scale = max(4, int(round(np.log2(max(m, 16) / 8))))
        n = 1 << scale
        pairs = gen.rmat(scale, m, gs)
    if kind == PHEM_BATCH_CC:
        return ServedGraph(kind, n, pairs=pairs)
    return ServedGraph(kind, n, edges=gen.msf_edges(pairs, gen.weights(len(pairs), gs + 3)))


def request_pool(count: int, seed: int = 5, m_lo: int = 1 << 10, m_hi: int = 1 << 24, threads: int = 16) -> list:
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(threads) as ex:
        return list(ex.map(lambda i: request_graph(i, seed, m_lo, m_hi), range(count)))


def poisson_arrivals(count: int, rate: float, seed: int = 0) -> np.ndarray:
    """Arrival times (ns) of a Poisson process at `rate` requests per second."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1e9 / rate, count)
    return np.cumsum(gaps).astype(np.uint64)


__all__ = ["Server", "ServedGraph", "Served", "poisson_arrivals", "request_graph", "request_pool", "PHEM_BATCH_MSF", "PHEM_BATCH_CC"]
