"""Python view of the C ABI: a Context bound to one GPU and its solves.

Arrays may be numpy (host) or torch CUDA tensors (device); the library stages
host arrays itself.  Results come back as numpy arrays unless device outputs
are passed in.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import (BatchStats, CCStats, KernelProfile, MSFStats, PHEM_CC_CANONICAL, PHEM_FOREST_EMPTY, check, lib,
                   ptr)

# phem_edge as a numpy structured dtype (MST/src/constants.h:15-19)
EDGE_DTYPE = np.dtype([("u", "<u4"), ("v", "<u4"), ("w", "<u4")])


def as_edges(E) -> np.ndarray:
    """{u, v, w} records as an (m, 3) uint32 C array."""
    if isinstance(E, np.ndarray) and E.dtype == EDGE_DTYPE:
        return E.view(np.uint32).reshape(-1, 3)
    if isinstance(E, np.ndarray) and E.dtype.itemsize == 4 and E.dtype.kind in "iu" and E.flags["C_CONTIGUOUS"]:
        return E.view(np.uint32).reshape(-1, 3)  # same bits, no copy (keeps pinned memory pinned)
    E = np.ascontiguousarray(E, np.uint32)
    return E.reshape(-1, 3)


@dataclass
class CCResult:
    labels: np.ndarray
    forest: np.ndarray | None
    components: int
    forest_edges: int
    rounds: int
    device_ms: float


@dataclass
class MSFResult:
    edges: np.ndarray          # (count, 3) uint32, ascending by edge id
    count: int
    total: int
    rounds: int
    m_r: list = field(default_factory=list)
    n_r: list = field(default_factory=list)
    device_ms: float = 0.0
    light_rounds: int = 0
    threshold: int = 0


@dataclass
class BatchResult:
    ids: np.ndarray            # vertex-indexed: graph g's forest ids at [vertex_offset, + count[g])
    count: np.ndarray          # (G,) uint32
    total: np.ndarray          # (G,) uint64
    labels: np.ndarray | None  # vertex-indexed local min-id labels
    stats: dict

    def forest(self, batch, g: int) -> np.ndarray:
        """Forest edge ids of graph g, ascending."""
        o = int(batch.graphs[g]["vertex_offset"])
        return self.ids[o: o + int(self.count[g])]

    def graph_labels(self, batch, g: int) -> np.ndarray:
        r = batch.graphs[g]
        o = int(r["vertex_offset"])
        return self.labels[o: o + int(r["num_vertices"])]


def _stats_dict(st: BatchStats) -> dict:
    return {"max_rounds": int(st.max_rounds), "block_size": int(st.block_size), "items": int(st.items),
            "compact_ratio": float(st.compact_ratio), "grid": int(st.grid), "smem_vertices": int(st.smem_vertices),
            "device_ms": float(st.device_ms)}


def _batch_args(batch):
    graphs = np.ascontiguousarray(batch.graphs)
    edges = batch.edges if hasattr(batch.edges, "data_ptr") else np.ascontiguousarray(batch.edges, np.uint32)
    return graphs, edges


class BatchPlan:
    """A replayable batch (phem_batch_plan): device buffers for up to
    max_graphs / max_edges / max_vertices and one captured CUDA graph."""

    def __init__(self, ctx: "Context", max_graphs: int, max_edges: int, max_vertices: int):
        self._h = C.c_void_p()
        check(lib().phem_batch_plan_create(ctx.handle, max_graphs, max_edges, max_vertices, C.byref(self._h)),
              "phem_batch_plan_create")
        self._batch = None

    def upload(self, batch) -> None:
        self._graphs, self._edges = _batch_args(batch)  # kept alive until the copies are done
        check(lib().phem_batch_plan_upload(self._h, ptr(self._graphs), len(self._graphs), ptr(self._edges),
                                           len(self._edges), batch.total_vertices), "phem_batch_plan_upload")
        self._batch = batch

    def run(self) -> None:
        check(lib().phem_batch_plan_run(self._h), "phem_batch_plan_run")

    def download(self, labels: bool = True) -> BatchResult:
        b = self._batch
        G, V = b.num_graphs, b.total_vertices
        ids = np.empty(max(V, 1), np.uint32)
        cnt = np.empty(max(G, 1), np.uint32)
        tot = np.empty(max(G, 1), np.uint64)
        lab = np.empty(max(V, 1), np.int32) if labels else None
        check(lib().phem_batch_plan_download(self._h, ptr(ids), ptr(cnt), ptr(tot), ptr(lab)),
              "phem_batch_plan_download")
        return BatchResult(ids[:V], cnt[:G], tot[:G], lab[:V] if labels else None, {})

    def device(self) -> dict:
        ps = [C.c_void_p() for _ in range(5)]
        check(lib().phem_batch_plan_device(self._h, *[C.byref(p) for p in ps]), "phem_batch_plan_device")
        return dict(zip(["edges", "msf_ids", "msf_count", "msf_total", "labels"], [p.value for p in ps]))

    def close(self) -> None:
        if self._h:
            lib().phem_batch_plan_destroy(self._h)
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


class Context:
    """A libphem context on CUDA device `device` (its own stream and workspace)."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        check(lib().phem_context_create(device, C.byref(self._h)), "phem_context_create")
        self.device = device

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self) -> None:
        if self._h:
            lib().phem_context_destroy(self._h)
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

    def set_stream(self, stream) -> None:
        """Orders work on a CUDA stream (torch.cuda.Stream, raw handle, or None)."""
        h = getattr(stream, "cuda_stream", stream)
        check(lib().phem_context_set_stream(self._h, h), "phem_context_set_stream")

    def set_timeout_ms(self, ms: int) -> None:
        check(lib().phem_context_set_timeout_ms(self._h, ms), "phem_context_set_timeout_ms")

    def trim(self) -> None:
        check(lib().phem_context_trim(self._h), "phem_context_trim")

    def set_tuning(self, key: str, value: float) -> None:
        """Sets a tuning knob (see phem_context_set_tuning); results never depend on it."""
        check(lib().phem_context_set_tuning(self._h, key.encode(), float(value)), "phem_context_set_tuning")

    def get_tuning(self, key: str) -> float:
        v = C.c_double()
        check(lib().phem_context_get_tuning(self._h, key.encode(), C.byref(v)), "phem_context_get_tuning")
        return v.value

    def set_profiling(self, on: bool) -> None:
        """Brackets every kernel launch with CUDA events (per-kernel durations)."""
        check(lib().phem_context_set_profiling(self._h, 1 if on else 0), "phem_context_set_profiling")

    def profile(self) -> dict:
        """{kernel name: {"launches", "timed_launches", "total_ms"}} since the last reset."""
        buf = (KernelProfile * 64)()
        cnt = C.c_uint32()
        check(lib().phem_context_profile(self._h, buf, 64, C.byref(cnt)), "phem_context_profile")
        return {buf[i].name.decode(): {"launches": int(buf[i].launches), "timed_launches": int(buf[i].timed_launches),
                                       "total_ms": float(buf[i].total_ms)} for i in range(min(cnt.value, 64))}

    def profile_reset(self) -> None:
        check(lib().phem_context_profile_reset(self._h), "phem_context_profile_reset")

    def launches(self) -> int:
        return sum(v["launches"] for v in self.profile().values())

    def launch_log(self) -> list:
        """[(kernel name, ms)] of the event-timed launches since the last reset."""
        from ._lib import LaunchRecord
        cnt = C.c_uint32()
        check(lib().phem_context_launch_log(self._h, None, 0, C.byref(cnt)), "phem_context_launch_log")
        buf = (LaunchRecord * max(cnt.value, 1))()
        check(lib().phem_context_launch_log(self._h, buf, cnt.value, C.byref(cnt)), "phem_context_launch_log")
        return [(buf[i].name.decode(), float(buf[i].ms)) for i in range(cnt.value)]

    # ------------------------------------------------------------ CC
    def cc_solve(self, edges, n: int, canonical: bool = False, labels=None, forest=None,
                 want_forest: bool = True) -> CCResult:
        """Labels (min vertex id per component) and forest slots of packed
        edges (u << 32 | v); see phem_cc_solve."""
        m = int(edges.numel() if hasattr(edges, "numel") else len(edges))
        if isinstance(edges, np.ndarray):
            edges = np.ascontiguousarray(edges, np.uint64)
        out_l = labels if labels is not None else np.empty(n, np.int32)
        out_f = forest if forest is not None else (np.empty(n, np.uint64) if want_forest else None)
        st = CCStats()
        check(lib().phem_cc_solve(self._h, ptr(edges), m, n, ptr(out_l), ptr(out_f),
                                  PHEM_CC_CANONICAL if canonical else 0, C.byref(st)), "phem_cc_solve")
        return CCResult(out_l, out_f, int(st.components), int(st.forest_edges), int(st.rounds),
                        float(st.device_ms))

    def cc_init(self, n, parent, label=None, forest=None):
        check(lib().phem_cc_init(self._h, n, ptr(parent), ptr(label), ptr(forest)), "phem_cc_init")

    def cc_unite(self, edges, m, n, parent, forest=None):
        check(lib().phem_cc_unite(self._h, ptr(edges), m, n, ptr(parent), ptr(forest)), "phem_cc_unite")

    def cc_label(self, n, parent, label):
        check(lib().phem_cc_label(self._h, n, ptr(parent), ptr(label)), "phem_cc_label")

    def cc_stream(self, h_edges, n: int, batch: int, parent, label, forest) -> float:
        """SpanningTree: host-resident batches through overlapped copies."""
        ms = C.c_float()
        m = len(h_edges) if isinstance(h_edges, np.ndarray) else int(h_edges.numel())
        check(lib().phem_cc_stream(self._h, ptr(h_edges), m, n, batch, ptr(parent), ptr(label), ptr(forest),
                                   C.byref(ms)), "phem_cc_stream")
        return ms.value

    def cc_stream_begin(self, n: int, parent, label=None, forest=None):
        """Opens an incremental stream (SpanningTree fed one batch per push)."""
        check(lib().phem_cc_stream_begin(self._h, n, ptr(parent), ptr(label), ptr(forest)),
              "phem_cc_stream_begin")

    def cc_stream_push(self, edges):
        """Unites one batch of packed edges (host or device); returns once a
        host batch has been copied."""
        m = len(edges) if isinstance(edges, np.ndarray) else int(edges.numel())
        if isinstance(edges, np.ndarray):
            edges = np.ascontiguousarray(edges, np.uint64)
        check(lib().phem_cc_stream_push(self._h, ptr(edges), m), "phem_cc_stream_push")

    def cc_stream_end(self) -> float:
        """Waits for the stream's unions; the time from begin to the last one."""
        ms = C.c_float()
        check(lib().phem_cc_stream_end(self._h, C.byref(ms)), "phem_cc_stream_end")
        return ms.value

    def cc_merge(self, forest_a, forest_b, n: int, parent, label, forest_out) -> float:
        """gpu_spanning_tree: merge two forests into final labels + forest."""
        ms = C.c_float()
        check(lib().phem_cc_merge(self._h, ptr(forest_a), ptr(forest_b), n, ptr(parent), ptr(label),
                                  ptr(forest_out), C.byref(ms)), "phem_cc_merge")
        return ms.value

    # ------------------------------------------------------------ MSF
    def msf_solve(self, edges, n: int, want_edges: bool = True, out=None) -> MSFResult:
        """Unique MSF under (w, id) of {u, v, w} records; see phem_msf_solve.
        `out` may supply the (>= n - 1, 3) result buffer (e.g. pinned memory)."""
        if isinstance(edges, np.ndarray):
            edges = as_edges(edges)
            m = len(edges)
        else:  # torch tensor of shape (m, 3) uint32/int32, host or device
            m = int(edges.shape[0])
        if out is not None:
            out = as_edges(out) if isinstance(out, np.ndarray) else out
        elif want_edges:
            out = np.empty((max(n - 1, 1), 3), np.uint32)
        cnt, tot = C.c_uint64(), C.c_uint64()
        st = MSFStats()
        check(lib().phem_msf_solve(self._h, ptr(edges), m, n, ptr(out), C.byref(cnt), C.byref(tot), C.byref(st)),
              "phem_msf_solve")
        k = int(cnt.value)
        return _msf_result(out[:k] if out is not None else None, k, int(tot.value), st)

    def msf_solve_device(self, d_edges, m: int, n: int, d_msf=None, d_count_total=None) -> MSFResult:
        """Device-resident solve (torch tensors); counts stay on the device
        unless d_count_total is given."""
        st = MSFStats()
        check(lib().phem_msf_solve_device(self._h, ptr(d_edges), m, n, ptr(d_msf), ptr(d_count_total),
                                          C.byref(st)), "phem_msf_solve_device")
        return _msf_result(None, int(st.msf_edges), int(st.total_weight), st)

    def msf_stream(self, edges, n: int, chunk: int, want_edges: bool = True, out=None) -> MSFResult:
        """Chunked MSF (streamline_boruvka): the same forest as msf_solve,
        solved chunk by chunk with the forest carried over, so the edge count
        is not limited to 2^32.  `edges` is (m, 3) host (pinned for overlap) or
        device records; device_ms is the time from the first copy to the last
        solve; rounds and per-round counts are not reported."""
        if isinstance(edges, np.ndarray):
            edges = as_edges(edges)
            m = len(edges)
        else:
            m = int(edges.shape[0])
        if out is not None:
            out = as_edges(out) if isinstance(out, np.ndarray) else out
        elif want_edges:
            out = np.empty((max(n - 1, 1), 3), np.uint32)
        cnt, tot, ms = C.c_uint64(), C.c_uint64(), C.c_float()
        check(lib().phem_msf_stream(self._h, ptr(edges), m, n, chunk, ptr(out), C.byref(cnt), C.byref(tot),
                                    C.byref(ms)), "phem_msf_stream")
        k = int(cnt.value)
        return MSFResult(out[:k] if out is not None else None, k, int(tot.value), 0, device_ms=float(ms.value))

    def msf_solve_csr(self, offsets, cols, n: int, weights, m_upper: int) -> MSFResult:
        out = np.empty((max(n - 1, 1), 3), np.uint32)
        cnt, tot = C.c_uint64(), C.c_uint64()
        st = MSFStats()
        check(lib().phem_msf_solve_csr(self._h, ptr(offsets), ptr(cols), n, ptr(weights), m_upper, ptr(out),
                                       C.byref(cnt), C.byref(tot), C.byref(st)), "phem_msf_solve_csr")
        k = int(cnt.value)
        return _msf_result(out[:k], k, int(tot.value), st)

    def csr_to_coo(self, offsets, cols, n: int) -> np.ndarray:
        nnz = int(offsets[n])
        out = np.empty(max(nnz, 1), np.uint64)
        k = C.c_int64()
        check(lib().phem_csr_to_coo(self._h, ptr(offsets), ptr(cols), n, ptr(out), C.byref(k)), "phem_csr_to_coo")
        return out[: k.value]

    # ------------------------------------------------------------ batches

    def batch_solve(self, batch, labels: bool = True, out: dict | None = None) -> BatchResult:
        """Every graph of a gen.Batch in one persistent launch.  `out` may hold
        caller arrays (for instance in pinned memory) for any of "ids" (uint32,
        >= total vertices), "count" (uint32, >= graphs), "total" (uint64,
        >= graphs) and "labels" (int32, >= total vertices)."""
        graphs, edges = _batch_args(batch)
        G, V = len(graphs), batch.total_vertices
        out = out or {}
        ids = out["ids"] if "ids" in out else np.empty(max(V, 1), np.uint32)
        cnt = out["count"] if "count" in out else np.empty(max(G, 1), np.uint32)
        tot = out["total"] if "total" in out else np.empty(max(G, 1), np.uint64)
        lab = None
        if labels:
            lab = out["labels"] if "labels" in out else np.empty(max(V, 1), np.int32)
        for name, a, need, dt in (("ids", ids, V, np.uint32), ("count", cnt, G, np.uint32),
                                  ("total", tot, G, np.uint64), ("labels", lab, V, np.int32)):
            if a is not None and (a.dtype != dt or len(a) < need or not a.flags.c_contiguous):
                raise ValueError(f"batch_solve: out[{name!r}] must be a contiguous {np.dtype(dt).name} array "
                                 f"of at least {need} entries")
        st = BatchStats()
        check(lib().phem_batch_solve(self._h, ptr(graphs), G, ptr(edges), len(edges), V, ptr(ids), ptr(cnt),
                                     ptr(tot), ptr(lab), C.byref(st)), "phem_batch_solve")
        return BatchResult(ids[:V], cnt[:G], tot[:G], lab[:V] if labels else None, _stats_dict(st))

    def batch_autotune(self, batch, reps: int = 3) -> dict:
        """Times every batched-kernel configuration on `batch`, keeps the
        fastest in this context's batch.* tuning and returns it."""
        graphs, edges = _batch_args(batch)
        st = BatchStats()
        check(lib().phem_batch_autotune(self._h, ptr(graphs), len(graphs), ptr(edges), len(edges),
                                        batch.total_vertices, reps, C.byref(st)), "phem_batch_autotune")
        return _stats_dict(st)

    def batch_plan(self, max_graphs: int, max_edges: int, max_vertices: int) -> BatchPlan:
        return BatchPlan(self, max_graphs, max_edges, max_vertices)


def _msf_result(edges, count: int, total: int, st) -> MSFResult:
    r = min(int(st.rounds), len(st.m_r))
    return MSFResult(edges, count, total, int(st.rounds), [int(x) for x in st.m_r[:r]], [int(x) for x in st.n_r[:r]],
                     float(st.device_ms), int(st.light_rounds), int(st.threshold))


def forest_set(forest: np.ndarray) -> np.ndarray:
    f = np.asarray(forest, np.uint64)
    return np.sort(f[f != np.uint64(PHEM_FOREST_EMPTY)])
