#!/usr/bin/env python
"""Benchmark of the MSF hot path on the R-MAT scale-22 workload.

Workload (one "step" = one full minimum-spanning-forest solve):
  R-MAT scale 22 (4,194,304 vertices), edge factor 16 (2^26 draws, a, b, c, d =
  .57, .19, .19, .05, no vertex permutation), self-loops dropped, duplicates
  kept, uint32 weights uniform in [1, 2^20], edge ids in upper-triangle CSR
  order; output = the unique MSF under (weight, edge id), its count and uint64
  total.  Synthetic (seeded) input: the reference's benchmark files are not
  available.

  value   Gedges/s = input edges / device time per solve, edges resident in HBM
          (805 MB, larger than L2, so no flush is needed between steps).
  e2e     the same metric through the C ABI call phem_msf_solve with pinned HOST
          edges in and host MSF records out (copies inside the timed region).
  roofline  the dominant kernel's algorithmic bytes / its event-timed duration
          against the measured HBM copy bandwidth.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl phem|reference]

On one GPU the same JSON line also carries the metric's other workloads:
  csr_input  the same R-MAT solve fed as its symmetrised CSR (int64 offsets,
           uint32 columns) and per-edge weights, converted on the device;
  msf_chunked  the same pinned host edges through phem_msf_stream (the
           reference's chunked streamline mode), 2^24 edges per chunk;
  cc       connected components + forest, Erdos-Renyi n = 2^20, 8 * 2^20 draws;
  batched  4096 small graphs (ER and geometric) in one persistent launch,
           against one solve per graph;
  served   Poisson request streams at 1k-100k req/s through the serving loop
           (p50 / p99 latency, throughput), against serial one-graph solves.

Host only: `python bench.py --ingest-only SCALE` times the MatrixMarket reader
against the reference's own reader and exits.  `python bench.py
--profile-sample` makes one small call of every kernel family (the profilers'
fixed target) and exits.

Multi-GPU (torchrun, one rank per GPU): every rank solves its own shard of a
global multigraph (same vertex set, seed 22 + rank, 2^26 draws each), the local
forests are all-gathered over NCCL and every rank solves their union; value =
all ranks' input edges / max-over-ranks time ("weak" scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gedges/s + % HBM roofline for MST/CC; batched p50/p99 vs one-launch-per-solve"
UNIT = "Gedges/s"


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed work runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [x for x in sm if x > 0.5 * (mx or 1)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def rmat22(rank: int = 0, scale: int = 22, edge_factor: int = 16):
    from phem_graph_b200 import gen
    g = gen.rmat_graph(scale, edge_factor, seed=22 + rank)
    return g, g.msf_edges()


def survey_bytes(m_r: list, n_r: list, count: int) -> int:
    """Algorithmic bytes of one solve in the Boruvka model
    sum_r (32 m_r + 16 m_{r+1}) + 16 sum_r n_r + 12 (n - c), with m_r / n_r the
    live edges / components entering round r of the CPU Boruvka restatement."""
    total = 0
    for r, mr in enumerate(m_r):
        nxt = m_r[r + 1] if r + 1 < len(m_r) else 0
        total += 32 * mr + 16 * nxt
    return total + 16 * sum(n_r) + 12 * count


def kernel_bytes(m: int, stats) -> dict:
    """Algorithmic bytes per solve of each kernel, from the rounds it ran: an
    edge pass reads its input (12-byte caller records in round 0 and in the
    heavy pass, 16-byte survivor records otherwise) and writes 16 bytes per
    survivor; the hook reads best (8), the survivor record (16), the partner's
    best (8) and writes parent (4) per choosing component; the gather reads the
    bitmap and gathers + writes 12 bytes per MSF edge."""
    m_r = stats.m_r
    ep = 0
    for r, mr in enumerate(m_r):
        from_input = r == 0 or r == stats.light_rounds
        ep += (12 * m if from_input else 16 * m_r[r - 1]) + 16 * mr
    return {"msf_edge_pass": ep, "msf_hook": 36 * sum(stats.n_r),
            "msf_gather": (m + 31) // 32 * 4 + 24 * stats.count}


def rounds_fixture(scale: int, edge_factor: int):
    p = ROOT / "tests" / "golden" / f"rmat{scale}_boruvka_rounds.json"
    if scale == 22 and edge_factor == 16 and p.exists():
        return json.loads(p.read_text())
    return None


def cpu_baseline_pbbs(E: np.ndarray, budget_s: float = 20.0, max_runs: int = 5) -> dict:
    """The reference's PBBS mst() (oracle/_ref) on all host cores, call time only,
    median of up to `max_runs` runs after one warm-up, bounded by `budget_s`."""
    import oracle
    if not oracle.ref_available():
        flags, cnt, _ = None, None, None
        t0 = time.perf_counter()
        oracle.msf_kruskal(E, int(E[:, :2].max()) + 1)
        dt = time.perf_counter() - t0
        return {"value": len(E) / dt / 1e9, "unit": UNIT, "cores": 1, "kind": "port",
                "sample": f"oracle Kruskal (w, id) on the full {len(E)}-edge array, 1 run"}
    ref = oracle.RefPBBS(E)
    times = []
    t_start = time.perf_counter()
    ref.run()  # warm-up
    while len(times) < max_runs and time.perf_counter() - t_start < budget_s:
        times.append(ref.run())
    workers = ref.workers()
    ref.close()
    med = statistics.median(times)
    return {"value": len(E) / med / 1e9, "unit": UNIT, "cores": workers, "kind": "reference",
            "sample": f"PBBS mst() (MST/src/utils.cu) on the full {len(E)}-edge R-MAT-22 array, "
                      f"median of {len(times)} runs after 1 warm-up, call time only",
            "seconds_median": med}


def bench_reference_gpu(E: np.ndarray, n: int, expect: tuple, runs: int = 3) -> dict:
    """The reference's own GPU Boruvka (device_boruvka, MST/src/kernels.cu:507-689,
    built unchanged for sm_100a into oracle/_ref) on the same edges, device
    resident: CUDA events around the call, median of `runs` after one warm-up,
    with its forest count and total against ours."""
    import oracle
    if not oracle.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libref_gpu_mst.so was not built (reference tree absent)"}
    ref = oracle.RefGpuMST(E, n)
    try:
        ref.run()
        out = [ref.run() for _ in range(runs)]
    finally:
        ref.close()
    ms = statistics.median(o[0] for o in out)
    cnt, tot = out[-1][1], out[-1][2]
    return {"value": len(E) / (ms / 1e3) / 1e9, "unit": UNIT, "ms": ms, "runs": runs,
            "count": cnt, "total": tot, "equal_to_ours": (cnt, tot) == tuple(expect),
            "what": "device_boruvka (MST/src/kernels.cu) on device-resident records, CUDA events around the call"}


def bench_cc(ctx, torch, peaks: dict, steps: int, warmup: int, cpu: bool) -> dict:
    """Connected components + spanning forest on Erdos-Renyi n = 2^20 with
    8 * 2^20 uniform draws (seed 1; self-loops dropped, duplicates kept):
    device time of phem_cc_solve on resident packed edges (CUDA events around
    init + union + label), the algorithmic bytes 8 m + 16 n against the
    measured HBM bandwidth, end to end from pinned host pairs to host labels,
    and the reference's host_spanning_tree on the host cores."""
    from phem_graph_b200 import gen
    g = gen.er_graph(1 << 20, 8 << 20, 1)
    n, m = g.n, g.m
    dev = torch.device("cuda", ctx.device)
    d_pairs = torch.from_numpy(g.pairs.view(np.int64)).to(dev)
    d_lab = torch.empty(n, dtype=torch.int32, device=dev)
    d_for = torch.empty(n, dtype=torch.int64, device=dev)
    out = {}
    for name, canon in (("default", False), ("canonical", True)):
        for _ in range(warmup):
            ctx.cc_solve(d_pairs, n, canonical=canon, labels=d_lab, forest=d_for)
        ms = [ctx.cc_solve(d_pairs, n, canonical=canon, labels=d_lab, forest=d_for).device_ms for _ in range(steps)]
        t = statistics.median(ms)
        byts = 8 * m + 16 * n
        out[name] = {"value": m / (t / 1e3) / 1e9, "ms": t, "algorithmic_bytes": byts,
                     "achieved_gbs": byts / (t / 1e3) / 1e9, "frac": byts / (t / 1e3) / 1e9 / peaks["hbm_gbs"]}
    h_pairs = torch.from_numpy(g.pairs.view(np.int64)).pin_memory()
    h_lab = torch.empty(n, dtype=torch.int32).pin_memory()
    hp, hl = h_pairs.numpy().view(np.uint64), h_lab.numpy()
    ctx.cc_solve(hp, n, labels=hl, want_forest=False)
    t0 = time.perf_counter()
    reps = max(3, steps // 2)
    for _ in range(reps):
        r = ctx.cc_solve(hp, n, labels=hl, want_forest=False)
    e2e = (time.perf_counter() - t0) / reps
    line = {"workload": "cc_er_n2^20_d8x2^20_s1", "n": n, "m": m, "unit": UNIT, "components": r.components,
            "value": out["default"]["value"], "ms_per_solve": out["default"]["ms"],
            "roofline": {"bound": "hbm", "achieved": out["default"]["achieved_gbs"], "peak": peaks["hbm_gbs"],
                         "unit": "GB/s", "frac": out["default"]["frac"], "bytes_model": "8 m + 16 n"},
            "canonical_forest": out["canonical"],
            "e2e": {"value": m / e2e / 1e9, "unit": UNIT, "ms_per_step": e2e * 1e3, "h2d_bytes_per_step": 8 * m,
                    "d2h_bytes_per_step": 4 * n, "api": "phem_cc_solve (C ABI), pinned host pairs"}}
    if cpu:
        import oracle
        if oracle.ref_available():
            ref = oracle.RefCC(n)
            ref.set_edges(g.pairs)
            ref.run()
            times = []
            for _ in range(3):
                ref.reset()
                times.append(ref.run())
            line["cpu_baseline"] = {"value": m / statistics.median(times) / 1e9, "unit": UNIT,
                                    "cores": ref.workers(), "kind": "reference",
                                    "sample": "host_spanning_tree (CC/host_spanning_tree.cu) on the full edge list, "
                                              "median of 3 after 1 warm-up, call time only"}
            ref.close()
    return line


def bench_csr_input(ctx, torch, g, steps: int, warmup: int, expect: tuple) -> dict:
    """The same R-MAT solve fed as the symmetrised CSR of the workload (int64
    offsets, uint32 columns) with one uint32 weight per edge: phem_msf_solve_csr
    with device-resident CSR and forest, which converts the CSR on the device
    (edge ids in row-walk order) and solves; per-kernel event times give the
    conversion's share."""
    import ctypes as C

    from phem_graph_b200 import _lib, gen
    off, cols = gen.csr_from_pairs(g.pairs, g.n)
    dev = torch.device("cuda", ctx.device)
    d_off = torch.from_numpy(off).to(dev)
    d_cols = torch.from_numpy(cols.view(np.int32)).to(dev)
    d_w = torch.from_numpy(g.w.view(np.int32)).to(dev)
    d_out = torch.empty((g.n, 3), dtype=torch.int32, device=dev)
    cnt, tot = C.c_uint64(), C.c_uint64()

    def solve():
        _lib.check(_lib.lib().phem_msf_solve_csr(ctx.handle, d_off.data_ptr(), d_cols.data_ptr(), g.n,
                                                 d_w.data_ptr(), g.m, d_out.data_ptr(), C.byref(cnt), C.byref(tot),
                                                 None), "phem_msf_solve_csr")

    for _ in range(warmup):
        solve()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        solve()  # returns after the count and total are on the host
    t = (time.perf_counter() - t0) / steps
    ctx.profile_reset()
    ctx.set_profiling(True)
    solve()
    prof = ctx.profile()
    ctx.set_profiling(False)
    conv = prof.get("csr_to_coo", {})
    del d_off, d_cols, d_w, d_out
    torch.cuda.empty_cache()
    nnz = len(cols)
    return {"workload": f"msf_rmat_csr_nnz{nnz}", "n": g.n, "m": g.m, "csr_entries": nnz, "unit": UNIT,
            "value": g.m / t / 1e9, "ms_per_solve": t * 1e3,
            "csr_to_coo_ms": conv.get("total_ms"), "csr_to_coo_launches": conv.get("launches"),
            "csr_to_coo_bytes": 4 * nnz + 8 * (g.n + 1) + 16 * g.m,
            "result_matches_edge_list_solve": (cnt.value, tot.value) == expect,
            "api": "phem_msf_solve_csr (C ABI), device CSR, weights and forest; host count and total"}


def bench_batched(ctx, torch, num_graphs: int = 4096) -> dict:
    """Many small graphs: 4096 graphs, n log-uniform in [64, 65536], half
    Erdos-Renyi (mean degree U[2, 16], weights U[1, 2^20]), half 2-D random
    geometric 8-NN (weights floor(distance * 2^24)), every graph solved for
    MSF + labels.  The autotuner picks the kernel configuration, then the
    captured launch is replayed (CUDA events); the one-solve-per-launch path
    is timed on a 256-graph sample, with the inputs on the host
    (phem_msf_solve per graph) and resident on the device
    (phem_msf_solve_device per graph), each scaled to the batch by the
    sample's share of the edges."""
    from phem_graph_b200 import gen
    b = gen.mixed_batch(num_graphs, 4)
    tuned = ctx.batch_autotune(b, reps=2)
    dev = torch.device("cuda", ctx.device)
    with ctx.batch_plan(b.num_graphs, b.total_edges, b.total_vertices) as p:
        p.upload(b)
        for _ in range(3):
            p.run()
        stream = torch.cuda.ExternalStream(__import__("phem_graph_b200").lib().phem_context_stream(ctx.handle),
                                           device=dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        reps = 10
        e0.record(stream)
        for _ in range(reps):
            p.run()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / reps
        res = p.download(labels=False)
    # end to end: pinned host batch in, host results out, through phem_batch_solve
    pinned = torch.from_numpy(b.edges.view(np.int32)).pin_memory()
    b.edges = pinned.numpy().view(np.uint32)
    V, G = b.total_vertices, b.num_graphs
    outs = {"ids": torch.empty(V, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
            "count": torch.empty(G, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
            "total": torch.empty(G, dtype=torch.int64).pin_memory().numpy().view(np.uint64),
            "labels": torch.empty(V, dtype=torch.int32).pin_memory().numpy()}
    ctx.batch_solve(b, labels=True, out=outs)
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        r = ctx.batch_solve(b, labels=True, out=outs)
        times.append(time.perf_counter() - t0)
    e2e = statistics.median(times)
    assert np.array_equal(r.count, res.count) and np.array_equal(r.total, res.total)
    idx = np.random.default_rng(0).choice(b.num_graphs, 256, replace=False)
    sample = [(np.ascontiguousarray(b.graph_edges(g)), int(b.graphs[g]["num_vertices"])) for g in idx]
    for e, n in sample[:8]:
        ctx.msf_solve(e, n)
    t0 = time.perf_counter()
    for e, n in sample:
        one = ctx.msf_solve(e, n)
    plain_s = time.perf_counter() - t0
    frac = sum(len(e) for e, _ in sample) / b.total_edges
    plain_batch_s = plain_s / frac
    # the like-for-like baseline: the same sample already resident on the
    # device, one phem_msf_solve_device call (one launch sequence) per graph
    d_sample = [(torch.from_numpy(e.view(np.int32)).to(dev), len(e), n) for e, n in sample]
    d_out = torch.empty((max(n for _, _, n in d_sample), 3), dtype=torch.int32, device=dev)
    d_ct = torch.zeros(2, dtype=torch.int64, device=dev)
    for d_e, m_g, n_g in d_sample[:8]:
        ctx.msf_solve_device(d_e, m_g, n_g, d_out, d_ct)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for d_e, m_g, n_g in d_sample:
        ctx.msf_solve_device(d_e, m_g, n_g, d_out, d_ct)
    torch.cuda.synchronize()
    dev_batch_s = (time.perf_counter() - t0) / frac
    del d_sample, d_out
    return {"workload": "batched_4096_mixed_er_rgg", "graphs": b.num_graphs, "edges": b.total_edges,
            "vertices": b.total_vertices, "unit": UNIT, "value": b.total_edges / (ms / 1e3) / 1e9,
            "ms_per_batch": ms, "graphs_per_s": b.num_graphs / (ms / 1e3), "launches_per_batch": 1,
            "config": {k: tuned[k] for k in ("block_size", "items", "compact_ratio", "grid", "smem_vertices")},
            "replay": "captured CUDA graph (queue reset + persistent kernel)",
            "one_launch_per_graph": {"value": b.total_edges / plain_batch_s / 1e9, "s_per_batch": plain_batch_s,
                                     "sample": "256 graphs through phem_msf_solve, scaled by edge share"},
            "speedup_vs_one_launch_per_graph": plain_batch_s / (ms / 1e3),
            "one_launch_per_graph_device": {"value": b.total_edges / dev_batch_s / 1e9, "s_per_batch": dev_batch_s,
                                            "sample": "the same 256 graphs resident on the device, one "
                                                      "phem_msf_solve_device per graph, scaled by edge share; "
                                                      "that path waits on the host between round batches, so "
                                                      "it has no captured form"},
            "speedup_vs_one_launch_per_graph_device": dev_batch_s / (ms / 1e3),
            "e2e": {"value": b.total_edges / e2e / 1e9, "unit": UNIT, "ms_per_step": e2e * 1e3,
                    "h2d_bytes_per_step": 12 * b.total_edges + 24 * b.num_graphs,
                    "d2h_bytes_per_step": 8 * b.total_vertices + 12 * b.num_graphs,
                    "api": "phem_batch_solve (C ABI), pinned host edges and results, median of 3"}}


def _pin_pool(torch, pool, keep):
    """Moves every request buffer of a pool to pinned host memory (a server's
    receive path would hold them that way)."""
    from phem_graph_b200.serve import PHEM_BATCH_MSF
    for g in pool:
        if g.kind == PHEM_BATCH_MSF:
            t = torch.from_numpy(g.edges.view(np.int32)).pin_memory()
            keep.append(t)
            g.edges = t.numpy().view(np.uint32)
        else:
            t = torch.from_numpy(g.pairs.view(np.int64)).pin_memory()
            keep.append(t)
            g.pairs = t.numpy().view(np.uint64)


def _served_stream(torch, srv, pool, rates, requests: int, rng, h2d_gbs: float) -> dict:
    """One request stream through the server at every offered rate: achieved
    vs offered req/s, p50 / p99 latency (submission to result in host memory),
    throughput, the share of requests on the batched path and the host-link
    fraction (request bytes in + result bytes out over the wall time, against
    a plain pinned copy).  A rate is sustained when the server achieved >= 95 %
    of it; latencies at unsustained rates measure queue growth, not service."""
    import phem_graph_b200 as P
    from phem_graph_b200.serve import PHEM_BATCH_MSF, poisson_arrivals
    ctx = P.Context(0)
    solve = (lambda g: ctx.msf_solve(g.edges, g.n) if g.kind == PHEM_BATCH_MSF
             else ctx.cc_solve(g.pairs, g.n, want_forest=False))
    for g in pool:  # warm-up: the context's workspace reaches its largest size once
        solve(g)
    t0 = time.perf_counter()
    for g in pool:
        solve(g)
    serial_s = time.perf_counter() - t0
    ctx.close()
    pool_edges = sum(g.m for g in pool)
    serial = {"value": pool_edges / serial_s / 1e9, "req_s": len(pool) / serial_s,
              "api": "phem_msf_solve / phem_cc_solve one request at a time (one solve per launch sequence), "
                     "pinned host inputs, host results"}
    srv.replay(pool, np.zeros(len(pool), np.uint64))  # warm-up: every worker sizes its workspace
    points = []
    for rate in rates:
        idx = rng.integers(0, len(pool), requests)
        reqs = [pool[i] for i in idx]
        arr = poisson_arrivals(requests, rate, seed=rate)
        res = srv.replay(reqs, arr)
        # the served span on the server's own clock: first submission to last
        # result (building the requests in Python is not serving time)
        wall = (max(r.done_ns for r in res) - min(r.submit_ns for r in res)) / 1e9
        assert all(r.status == 0 for r in res)
        lat = np.array([r.latency_ns for r in res]) / 1e6
        e = sum(g.m for g in reqs)
        io = sum((g.m * 12 + 12 * max(g.n - 1, 1)) if g.kind == PHEM_BATCH_MSF else (g.m * 8 + 4 * g.n)
                 for g in reqs)
        achieved = requests / wall
        points.append({"rate_req_s": rate, "requests": requests, "seconds": wall, "req_s": achieved,
                       "sustained": achieved >= 0.95 * rate, "p50_ms": float(np.percentile(lat, 50)),
                       "p99_ms": float(np.percentile(lat, 99)), "throughput": e / wall / 1e9,
                       "batched_share": float(np.mean([r.path == 0 for r in res])),
                       "host_link_frac": io / wall / 1e9 / h2d_gbs})
    sus = [p for p in points if p["sustained"]]
    best = max(points, key=lambda p: p["throughput"])
    return {"points": points, "value": best["throughput"], "serial_plain": serial,
            "speedup_vs_serial_plain": best["throughput"] / serial["value"],
            "saturation_req_s": max(p["req_s"] for p in points),
            "knee_rate_req_s": max((p["rate_req_s"] for p in sus), default=None),
            "latency_at_knee": ({"p50_ms": sus[-1]["p50_ms"], "p99_ms": sus[-1]["p99_ms"]} if sus else None),
            "pool_graphs": len(pool), "pool_edges": pool_edges}


def bench_served(torch, rates=(1000, 3000, 10000, 30000, 100000), requests: int = 2000, slots: int = 4) -> dict:
    """Served request streams (Poisson arrivals at each offered rate, 2000
    requests per rate, a 64 GB device budget, request buffers in pinned host
    memory):
      mixed  -- the configured stream: m log-uniform in [2^10, 2^24], 70% CC
                packed pairs / 30% MSF records (weights U[1, 2^20]), half
                Erdos-Renyi, half R-MAT (a pool of 64 graphs);
      small  -- the same stream limited to m <= 2^18 (the server's batched
                path; a pool of 256 graphs), the small-graph case whose
                throughput the target compares with one solve per launch.
    Each stream is compared with its own pool solved one request at a time
    through the one-graph entry points."""
    from phem_graph_b200.serve import Server, request_pool
    keep = []
    mixed = request_pool(64, seed=5)
    small = request_pool(256, seed=6, m_hi=1 << 18)
    _pin_pool(torch, mixed, keep)
    _pin_pool(torch, small, keep)
    # host link: one pinned copy of 256 MB
    h = torch.empty(1 << 25, dtype=torch.int64, pin_memory=True)
    d = torch.empty(1 << 25, dtype=torch.int64, device="cuda")
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    d.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    h2d_gbs = 8 * (1 << 25) / (time.perf_counter() - t0) / 1e9
    del h, d
    rng = np.random.default_rng(1)
    cfg = {"memory_budget_gb": 64, "slots": slots, "max_batch_graphs": 1024, "large_edges": 1 << 18,
           "large_workers": 2, "requests_per_rate": requests, "h2d_gbs": h2d_gbs}
    with Server(memory_budget=64 << 30, slots=slots, max_batch_graphs=1024, large_edges=1 << 18,
                large_workers=2) as srv:
        out_mixed = _served_stream(torch, srv, mixed, rates, requests, rng, h2d_gbs)
        out_small = _served_stream(torch, srv, small, rates, requests, rng, h2d_gbs)
    return {"workload": "served_poisson_m_loguniform_2^10_2^24_70cc_30msf", "unit": UNIT,
            "value": out_mixed["value"], "mixed": out_mixed, "small": out_small, "config": cfg}


def bench_streamed(ctx, torch, scale: int, edge_factor: int = 32, batch: int = 1 << 28, cpu: bool = True) -> dict:
    """Streaming spanning forest (the reference's SpanningTree): R-MAT at
    `scale` with edge_factor * 2^scale draws (seed 28, self-loops dropped,
    unsorted, ~69 GB of pairs at scale 28), generated on the GPU batch by batch
    (phem_gen_rmat_range_device, the host generator's exact stream) and copied
    into pinned host memory before timing, then streamed to the GPU in batches
    of `batch` pairs through triple-buffered copies overlapped with the union
    kernels (phem_cc_stream); device memory: parent + labels + forest + 3 batch
    buffers.  Parity: the reference's own host_spanning_tree
    (CC/host_spanning_tree.cu:89, oracle/_ref) consumes the same batches in
    the same order on all host cores, its state carried from batch to batch as
    in the reference; its root of every vertex (the smallest id of the
    component, by its max -> min hook rule) must equal our label bit for bit.
    Also checked: the forest has n - components edges."""
    import oracle
    from phem_graph_b200 import gen
    n = 1 << scale
    draws = edge_factor << scale
    need = 8 * draws + (16 << scale)
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    avail = int(ln.split()[1]) * 1024
    except OSError:
        pass
    workload = f"stream_rmat{scale}_ef{edge_factor}_batch2^{batch.bit_length() - 1}"
    if avail is not None and avail < need + (8 << 30):
        return {"workload": workload, "skipped": f"host memory: {avail / 1e9:.0f} GB available, "
                                                 f"{(need + (8 << 30)) / 1e9:.0f} GB needed"}
    dev = torch.device("cuda", ctx.device)
    t_gen = time.perf_counter()
    h = torch.empty(draws, dtype=torch.int64, pin_memory=True)
    gen_chunk = 1 << 28
    buf = torch.empty(gen_chunk, dtype=torch.int64, device=dev)
    filled = 0
    for first in range(0, draws, gen_chunk):
        k = gen.rmat_range_device(ctx, scale, first, min(gen_chunk, draws - first), 28, buf)
        h[filled:filled + k].copy_(buf[:k])
        filled += k
    del buf
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    m = filled
    parent = torch.empty(n, dtype=torch.int32, device=dev)
    label = torch.empty(n, dtype=torch.int32, device=dev)
    forest = torch.empty(n, dtype=torch.int64, device=dev)
    hv = h[:m].numpy().view(np.uint64)
    # host link bandwidth for the roofline: one pinned copy of a batch
    probe = torch.empty(min(batch, m), dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    probe.copy_(h[: probe.numel()], non_blocking=True)
    torch.cuda.synchronize()
    h2d_gbs = 8 * probe.numel() / (time.perf_counter() - t0) / 1e9
    del probe
    ms = ctx.cc_stream(hv, n, batch, parent, label, forest)
    ctx.cc_label(n, parent, label)
    torch.cuda.synchronize()
    ar = torch.arange(n, dtype=torch.int32, device=dev)
    comps = int((label == ar).sum())
    filled_slots = int((forest != 0x7FFFFFFF).sum())
    del parent, forest, ar
    out = {"workload": workload, "n": n, "m": m, "unit": UNIT, "value": m / (ms / 1e3) / 1e9, "ms": ms,
           "generation_s": t_gen, "generator": "phem_gen_rmat_range_device (the host stream, on the GPU)",
           "roofline": {"bound": "host link", "achieved": 8 * m / (ms / 1e3) / 1e9, "peak": h2d_gbs,
                        "unit": "GB/s", "frac": 8 * m / (ms / 1e3) / 1e9 / h2d_gbs,
                        "peak_source": "one pinned host-to-device copy of a batch, measured here"},
           "device_bytes": 16 * n + 3 * 8 * batch, "components": comps,
           "checks": {"forest_edges_eq_n_minus_c": filled_slots == n - comps}}
    if cpu and oracle.ref_available():
        ref = oracle.RefCC(n)
        t_ref = 0.0
        for off in range(0, m, batch):
            ref.set_edges(hv[off:off + batch])
            t_ref += ref.run()
        rp, _ = ref.state()
        workers = ref.workers()
        ref.close()
        # the reference's root of every vertex, by pointer jumping over its parents on the device
        P = torch.from_numpy(rp).to(dev).long()
        del rp
        for _ in range(64):
            Q = P[P]
            if torch.equal(Q, P):
                break
            P = Q
        del Q
        out["checks"]["labels_equal_reference"] = bool(torch.equal(P.int(), label))
        out["cpu_baseline"] = {"value": m / t_ref / 1e9, "unit": UNIT, "cores": workers, "kind": "reference",
                               "sample": f"host_spanning_tree (CC/host_spanning_tree.cu) fed the same {m} pairs in "
                                         f"the same batches of {batch}, state carried over; call time only"}
        del P
    del label, h
    torch.cuda.empty_cache()
    return out


def bench_msf_chunked(ctx, h_pinned, n: int, one_shot_s: float, expect: tuple, chunk: int = 1 << 24) -> dict:
    """The MSF workload through phem_msf_stream (the reference's
    streamline_boruvka): pinned host records in chunks of `chunk` edges, each
    solved with the forest so far while the next chunk is copied; host forest
    out.  Wall time per call, median of 3, beside the one-shot phem_msf_solve
    of the same pinned input (the headline e2e)."""
    m = int(h_pinned.shape[0])
    out = np.empty((n, 3), np.uint32)
    ctx.msf_stream(h_pinned, n, chunk, out=out)  # warm-up
    times, dev_ms, r = [], [], None
    for _ in range(3):
        t0 = time.perf_counter()
        r = ctx.msf_stream(h_pinned, n, chunk, out=out)
        times.append(time.perf_counter() - t0)
        dev_ms.append(r.device_ms)
    t = float(np.median(times))
    return {"workload": f"msf_rmat_chunked_{m}_chunk2^{chunk.bit_length() - 1}", "n": n, "m": m, "unit": UNIT,
            "chunks": -(-m // chunk), "value": m / t / 1e9, "ms_per_solve": t * 1e3,
            "device_ms": float(np.median(dev_ms)), "one_shot_e2e_ms": one_shot_s * 1e3,
            "result_matches_one_shot": (r.count, r.total) == expect,
            "api": "phem_msf_stream (C ABI), pinned host edges and forest, median of 3"}


def bench_msf_chunked_large(ctx, torch, scale: int, edge_factor: int = 16, chunk: int = 1 << 28) -> dict:
    """Chunked MSF beyond one solve's 2^32-edge limit: R-MAT at `scale` with
    edge_factor * 2^scale draws (seed 28, self-loops dropped, unsorted; at
    scale 28 about 4.29 G edges, 51.5 GB of records), weights uniform in
    [1, 2^20] from a SplitMix64 stream per 2^28 draws, generated into pinned
    host memory before timing and streamed through phem_msf_stream.  Checked
    by size-independent properties: a second run with a ragged chunk size
    returns the identical forest; the forest is acyclic (connected components
    of the forest edges alone number n - count); its weights sum to the total."""
    import ctypes as C

    from phem_graph_b200 import _lib
    n = 1 << scale
    draws = edge_factor << scale
    h = torch.empty((draws, 3), dtype=torch.int32, pin_memory=True)
    gen_chunk = 1 << 28
    pairs = np.empty(gen_chunk, np.uint64)
    w = np.empty(gen_chunk, np.uint32)
    filled = 0
    t_gen = time.perf_counter()
    for k, first in enumerate(range(0, draws, gen_chunk)):
        cnt = C.c_uint64()
        want = min(gen_chunk, draws - first)
        _lib.check(_lib.lib().phem_gen_rmat_range(scale, first, want, 0.57, 0.19, 0.19, 28, pairs.ctypes.data,
                                                  C.byref(cnt)), "phem_gen_rmat_range")
        c = cnt.value
        _lib.check(_lib.lib().phem_gen_weights(c, 1000 + k, 20, w.ctypes.data), "phem_gen_weights")
        _lib.check(_lib.lib().phem_pack_msf_edges(pairs.ctypes.data, w.ctypes.data, c,
                                                  h.data_ptr() + 12 * filled), "phem_pack_msf_edges")
        filled += c
    t_gen = time.perf_counter() - t_gen
    del pairs, w
    m = filled
    hv = h[:m]
    dev = torch.device("cuda", ctx.device)
    # host link bandwidth for the roofline: one pinned copy of a chunk
    probe = torch.empty((min(chunk, m), 3), dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    probe.copy_(hv[: probe.shape[0]], non_blocking=True)
    torch.cuda.synchronize()
    h2d_gbs = 12 * probe.shape[0] / (time.perf_counter() - t0) / 1e9
    del probe
    torch.cuda.empty_cache()
    out_a = torch.empty((n, 3), dtype=torch.int32, pin_memory=True)
    out_b = torch.empty((n, 3), dtype=torch.int32, pin_memory=True)
    t0 = time.perf_counter()
    ra = ctx.msf_stream(hv, n, chunk, out=out_a)
    t_a = time.perf_counter() - t0
    ragged = chunk - (1 << 20) + 7
    rb = ctx.msf_stream(hv, n, ragged, out=out_b)
    same = (ra.count, ra.total) == (rb.count, rb.total) and bool(torch.equal(out_a[:ra.count], out_b[:rb.count]))
    del out_b
    f = out_a[:ra.count].numpy().view(np.uint32)
    total_ok = int(f[:, 2].sum(dtype=np.uint64)) == ra.total
    fd = torch.from_numpy(f.view(np.int32)).to(dev).long() & 0xFFFFFFFF
    lo, hi = torch.minimum(fd[:, 0], fd[:, 1]), torch.maximum(fd[:, 0], fd[:, 1])
    packed = (lo << 32) | hi
    labels = torch.empty(n, dtype=torch.int32, device=dev)
    comps = ctx.cc_solve(packed, n, labels=labels).components
    del fd, lo, hi, packed, labels
    torch.cuda.empty_cache()
    return {"workload": f"msf_rmat{scale}_ef{edge_factor}_chunked_chunk2^{chunk.bit_length() - 1}", "n": n, "m": m,
            "chunks": -(-m // chunk), "unit": UNIT, "value": m / t_a / 1e9, "ms": t_a * 1e3,
            "device_ms": ra.device_ms, "generation_s": t_gen, "msf_edges": ra.count, "total_weight": ra.total,
            "roofline": {"bound": "host link", "achieved": 12 * m / (ra.device_ms / 1e3) / 1e9, "peak": h2d_gbs,
                         "unit": "GB/s", "frac": 12 * m / (ra.device_ms / 1e3) / 1e9 / h2d_gbs,
                         "peak_source": "one pinned host-to-device copy of a chunk, measured here"},
            "host_bytes": 12 * m,
            "device_bytes": "2 x (n - 1 + chunk) records of input slots, n - 1 output records, one solve's workspace",
            "api": "phem_msf_stream (C ABI), pinned host records, pinned host forest",
            "checks": {"ragged_chunks_same_forest": same, "forest_acyclic": comps == n - ra.count,
                       "weights_sum_to_total": total_ok}}


def bench_ingest(scale: int, reps: int = 3) -> dict:
    """Host-side ingest: phem_read_mtx on the MatrixMarket file of an R-MAT
    graph (edge factor 16, weights uniform in [1, 2^20], written to a
    temporary directory first), median of `reps` reads, beside the MST
    driver's own reader (getGraphInfo + mmapPopulateEdgeArray,
    MST/src/utils.cu, compiled into oracle/_ref) on the same file and host
    cores; the two outputs must be identical."""
    import tempfile

    import oracle
    from phem_graph_b200 import gen, io
    g = gen.rmat_graph(scale, 16, seed=3)
    E = g.msf_edges()
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "g.mtx"
        io.write_mtx(path, E, g.n)
        size = path.stat().st_size
        ours, theirs, same = [], [], None
        for _ in range(reps):
            t0 = time.perf_counter()
            a, _ = io.read_mtx(path)
            ours.append(time.perf_counter() - t0)
            if oracle.ref_available():
                t0 = time.perf_counter()
                b, _ = oracle.ref_mtx_read(path)
                theirs.append(time.perf_counter() - t0)
                same = bool(np.array_equal(a, b))
    t = statistics.median(ours)
    line = {"metric": "MatrixMarket read", "unit": "MB/s", "value": size / t / 1e6, "higher_is_better": True,
            "config": {"workload": f"mtx_rmat{scale}_ef16", "bytes": size, "m": len(E), "n": g.n},
            "seconds": t, "cores": os.cpu_count(), "api": "phem_read_mtx (C ABI)"}
    if theirs:
        tr = statistics.median(theirs)
        line["cpu_baseline"] = {"value": size / tr / 1e6, "unit": "MB/s", "seconds": tr, "cores": os.cpu_count(),
                                "kind": "reference", "sample": "the same file, median of %d reads" % reps,
                                "identical_records": same}
    return line


def profile_sample() -> None:
    """--profile-sample: one small call of every kernel family on
    device-resident synthetic inputs, a fixed target for profilers (each launch
    list names the same kernels).  R-MAT scale 20, edge factor 16 for the MSF
    solve and the CSR conversion; Erdos-Renyi n = 2^20 with 8 * 2^20 draws for
    connected components (default, canonical-forest and no-allocation entry
    points); 256 mixed small graphs for the batched kernel.  Every input array
    is larger than L2 except the batch.  Results are not checked here (the GPU
    tests do that)."""
    import ctypes as C

    import torch

    from phem_graph_b200 import Context, _lib, gen

    dev = torch.device("cuda", 0)
    with Context(0) as ctx:
        g = gen.rmat_graph(20, 16, seed=1)
        E = g.msf_edges()
        d_e = torch.from_numpy(E.view(np.int32)).to(dev)
        d_msf = torch.empty((g.n, 3), dtype=torch.int32, device=dev)
        d_ct = torch.zeros(2, dtype=torch.int64, device=dev)
        r = ctx.msf_solve_device(d_e, g.m, g.n, d_msf, d_ct)
        print("msf", g.m, "edges ->", r.count, "forest edges, total", r.total)

        er = gen.er_graph(1 << 20, 8 << 20, 1)
        d_p = torch.from_numpy(er.pairs.view(np.int64)).to(dev)
        d_lab = torch.empty(er.n, dtype=torch.int32, device=dev)
        d_for = torch.empty(er.n, dtype=torch.int64, device=dev)
        c = ctx.cc_solve(d_p, er.n, labels=d_lab, forest=d_for)
        print("cc", er.m, "edges ->", c.components, "components")
        c = ctx.cc_solve(d_p, er.n, canonical=True, labels=d_lab, forest=d_for)
        print("cc canonical", c.components, "components")

        off, cols = gen.csr_from_pairs(g.pairs, g.n)
        d_off = torch.from_numpy(off).to(dev)
        d_cols = torch.from_numpy(cols.view(np.int32)).to(dev)
        d_coo = torch.empty(len(cols), dtype=torch.int64, device=dev)
        k = C.c_int64()
        _lib.check(_lib.lib().phem_csr_to_coo(ctx.handle, d_off.data_ptr(), d_cols.data_ptr(), g.n,
                                              d_coo.data_ptr(), C.byref(k)), "phem_csr_to_coo")
        print("csr_to_coo", len(cols), "entries ->", k.value, "pairs")

        st = _lib.lib().phem_cc_solve_noalloc(C.c_void_p(d_p.data_ptr()), er.m, er.n,
                                               C.c_void_p(d_lab.data_ptr()), C.c_void_p(d_for.data_ptr()), None)
        _lib.check(st, "phem_cc_solve_noalloc")
        print("cc no-alloc ok")

        b = gen.mixed_batch(256, 4)
        with ctx.batch_plan(b.num_graphs, b.total_edges, b.total_vertices) as plan:
            plan.upload(b)  # device-resident edges: one launch, no overlapped copies
            plan.run()
            r = plan.download(labels=False)
        print("batch", b.num_graphs, "graphs ->", int(r.count.sum()), "forest edges")
        torch.cuda.synchronize()


def run_reference(args) -> None:
    """--impl reference: the reference's own CPU path (PBBS mst()) on the same
    workload, all host threads; one step = one full solve."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import tempfile

    import oracle
    # The input is generated in a child process (phem_graph_b200.gen, host
    # code of this build) and handed over as a file, so this process maps the
    # reference's libraries only.
    with tempfile.TemporaryDirectory() as tmp:
        f = os.path.join(tmp, "edges.npy")
        code = ("import sys, numpy as np; sys.path.insert(0, sys.argv[1]); from phem_graph_b200 import gen; "
                "g = gen.rmat_graph(int(sys.argv[2]), int(sys.argv[3]), seed=22); "
                "np.save(sys.argv[4], g.msf_edges()); print(g.n)")
        out = subprocess.run([sys.executable, "-c", code, str(ROOT), str(args.scale), str(args.edge_factor), f],
                             check=True, capture_output=True, text=True).stdout
        E = np.load(f)
    n = int(out.split()[-1])
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference tree absent)"}))
        return
    ref = oracle.RefPBBS(E)
    for _ in range(args.warmup):
        ref.run()
    times = [ref.run() for _ in range(args.steps)]
    workers = ref.workers()
    total = sum(times)
    m = len(E)
    value = args.steps * m / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"msf_rmat{args.scale}_ef{args.edge_factor}", "n": n, "m": m, "seed": 22,
                   "weights": "uniform [1, 2^20]"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "reference",
                         "sample": f"PBBS mst() on the full {m}-edge array, {args.steps} timed runs"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


_UNITS = {"byte": 1, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}


def profile_traffic(kernel: str, csv_name: str, solves: int):
    """DRAM bytes (read + write) per solve of every launch of `kernel`, from the
    ncu CSV that the capture command in profiles/ wrote (--csv --log-file):
    the capture profiles `solves` solves; None when the file is absent."""
    import csv
    p = ROOT / "profiles" / csv_name
    if not p.exists():
        return None
    lines = [ln for ln in p.read_text().splitlines() if ln.startswith('"')]
    total = 0.0
    for row in csv.DictReader(lines):
        if kernel in row.get("Kernel Name", "") and row.get("Metric Name") in ("dram__bytes_read.sum",
                                                                                "dram__bytes_write.sum"):
            total += float(row["Metric Value"].replace(",", "")) * _UNITS.get(row.get("Metric Unit", "byte"), 1)
    return total / solves if total else None


def profile_solves(args) -> None:
    """--profile-solves N: N plain solves of the benchmark workload on device
    memory and nothing else, a fixed target for per-launch profiles."""
    import torch

    import phem_graph_b200 as P
    g, E = rmat22(0, args.scale, args.edge_factor)
    ctx = P.Context(0)
    # the rounds queued on the stream: ncu does not profile the kernel nodes
    # of a graph that has conditional nodes
    ctx.set_tuning("msf.graph", 0)
    d = torch.from_numpy(E.view(np.int32)).to("cuda:0")
    o = torch.empty((g.n, 3), dtype=torch.int32, device="cuda:0")
    ct = torch.zeros(2, dtype=torch.int64, device="cuda:0")
    for _ in range(args.profile_solves):
        r = ctx.msf_solve_device(d, g.m, g.n, o, ct)
    torch.cuda.synchronize()
    print(json.dumps({"solves": args.profile_solves, "m": g.m, "n": g.n, "count": r.count, "total": r.total,
                      "rounds": r.rounds}))
    ctx.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["phem", "reference"], default="phem")
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stream-scale", type=int, default=28,
                    help="also stream an R-MAT graph of this scale (edge factor 32) from pinned host memory and "
                         "check its labels against the reference's host_spanning_tree (0: skip)")
    ap.add_argument("--msf-stream-scale", type=int, default=0,
                    help="also solve an R-MAT graph of this scale (edge factor 16) by chunked MSF from pinned "
                         "host memory (scale 28: 4.29 G edges, beyond one solve's 2^32 limit)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the connected-components, batched and served workloads")
    ap.add_argument("--profile-solves", type=int, default=0, metavar="N",
                    help="N plain solves of the workload on device memory (a fixed profiler target), then exit")
    ap.add_argument("--profile-sample", action="store_true",
                    help="one small call of every kernel family (a fixed target for profilers), then exit")
    ap.add_argument("--ingest-only", type=int, default=0, metavar="SCALE",
                    help="host only: time the MatrixMarket reader on an R-MAT graph of this scale against the "
                         "reference's own reader, then exit (no GPU needed)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.ingest_only:
        print(json.dumps(bench_ingest(args.ingest_only)))
        return
    if args.profile_sample:
        profile_sample()
        return
    if args.profile_solves:
        profile_solves(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    import phem_graph_b200 as P
    from phem_graph_b200 import dist as pdist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    g, E = rmat22(rank, args.scale, args.edge_factor)
    n, m = g.n, g.m
    ctx = P.Context(local)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream)
    d_edges = torch.from_numpy(E.view(np.int32)).to(f"cuda:{local}")
    d_out = torch.empty((n, 3), dtype=torch.int32, device=f"cuda:{local}")
    d_ct = torch.zeros(2, dtype=torch.int64, device=f"cuda:{local}")
    h_pinned = torch.from_numpy(E.view(np.int32)).pin_memory()
    h_out = torch.empty((n, 3), dtype=torch.int32).pin_memory()

    def step():
        if world > 1:
            return pdist.sharded_msf_device(ctx, d_edges, m, n, stream)
        return ctx.msf_solve_device(d_edges, m, n, d_out, d_ct)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            res = step()
    torch.cuda.synchronize()

    peaks = measured_peaks()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.profile_reset()
    with ClockSampler(local) as clocks:
        # the timed steps run as a user runs them, without per-launch events
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                res = step()
        ev1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t_ms = ev0.elapsed_time(ev1)
        launches = ctx.profile()
        # the same steps again with every launch bracketed by CUDA events on
        # the solve's stream: per-kernel durations for the roofline
        ctx.profile_reset()
        ctx.set_profiling(True)
        with torch.cuda.stream(stream):
            for _ in range(args.steps):
                step()
        torch.cuda.synchronize()
        prof = ctx.profile()
        ctx.set_profiling(False)

        # end to end through the C ABI: pinned host edges in, host records out
        e2e_steps = args.e2e_steps or max(3, min(args.steps, 10))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h_edges, h_res = h_pinned.numpy().view(np.uint32), h_out.numpy().view(np.uint32)
        for _ in range(e2e_steps):
            r_host = ctx.msf_solve(h_edges, n, out=h_res)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / e2e_steps
        # the host link alone: one plain pinned copy of the same edges
        d_copy = torch.empty_like(h_pinned, device=f"cuda:{local}")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d_copy.copy_(h_pinned, non_blocking=True)
        torch.cuda.synchronize()
        copy_s = time.perf_counter() - t0
        del d_copy
    if world > 1:
        tt = torch.tensor([t_ms, e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms, e2e_s = float(tt[0]), float(tt[1])

    ms_per_step = t_ms / args.steps
    value = world * m / (ms_per_step / 1e3) / 1e9
    gpu_launches = sum(v["launches"] for v in launches.values())

    # roofline of the dominant kernel, event-timed inside the timed region
    stats = ctx.msf_solve_device(d_edges, m, n, d_out, d_ct) if world > 1 else res
    byts = kernel_bytes(m, stats)
    fx = rounds_fixture(args.scale, args.edge_factor)
    if fx is not None:
        assert (fx["msf_edges"], fx["total_weight"]) == (stats.count, stats.total), "result differs from fixture"
        byts["survey"] = survey_bytes(fx["m_r"], fx["n_r"], fx["msf_edges"])
        survey_src = "tests/golden/rmat22_boruvka_rounds.json (CPU Boruvka restatement)"
    else:
        byts["survey"] = None  # the committed restatement counts cover the R-MAT-22 workload only
        survey_src = None
    timed = {k: v for k, v in prof.items() if v["timed_launches"]}
    dom = max(timed, key=lambda k: timed[k]["total_ms"]) if timed else None
    kernels = {}
    total_kernel_ms = sum(v["total_ms"] for v in timed.values()) or 1.0
    for k, v in timed.items():
        entry = {"launches": v["launches"], "ms_per_step": v["total_ms"] / args.steps,
                 "share": v["total_ms"] / total_kernel_ms}
        if k in byts:
            gbs = byts[k] * args.steps / (v["total_ms"] / 1e3) / 1e9
            entry.update({"bytes_per_step": byts[k], "achieved_gbs": gbs, "frac": gbs / peaks["hbm_gbs"]})
        kernels[k] = entry
    roofline = None
    if dom:
        achieved = kernels[dom].get("achieved_gbs")
        traffic = (profile_traffic("edge_pass", "msf_edge_pass_rmat22_dram.csv", 1)
                   if (dom == "msf_edge_pass" and args.scale == 22 and args.edge_factor == 16) else None)
        roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": (achieved / peaks["hbm_gbs"]) if achieved else None,
                    "traffic": traffic,
                    "traffic_basis": "ncu dram__bytes_read + write of the edge-pass launches of one solve "
                                     "(profiles/msf_edge_pass_rmat22_dram.csv, bench.py --profile-solves 1)",
                    "peak_source": f"{peaks['source']} (MEASURED_PEAKS.json hbm_gbs)",
                    "algorithmic_bytes_per_step": byts.get(dom)}
    solve_gbs = byts["survey"] / (ms_per_step / 1e3) / 1e9 if byts["survey"] else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"msf_rmat{args.scale}_ef{args.edge_factor}", "n": n, "m": m, "seed": 22,
                   "weights": "uniform [1, 2^20]", "l2": "inputs larger than L2 (805 MB edge array), no flush",
                   "parallelism": f"shard{world}" if world > 1 else "single"},
        "roofline": roofline,
        "solve_roofline": {"model": "sum_r(32 m_r + 16 m_r+1) + 16 sum_r n_r + 12 (n - c)",
                           "bytes": byts["survey"], "counts_from": survey_src, "achieved": solve_gbs,
                           "peak": peaks["hbm_gbs"], "frac": solve_gbs / peaks["hbm_gbs"] if solve_gbs else None,
                           "note": "Boruvka byte model; the filtered solve moves fewer bytes than it counts"},
        "device_rounds": {"m_r": stats.m_r, "n_r": stats.n_r, "light_rounds": stats.light_rounds,
                          "threshold_weight": stats.threshold >> 32},
        "kernels": kernels,
        "kernel_timing": "the timed steps repeated with CUDA events around every launch on the solve's stream",
        "result": {"msf_edges": stats.count, "total_weight": stats.total, "rounds": stats.rounds},
        "e2e": {"value": world * m / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": m * 12,
                "d2h_bytes_per_step": r_host.count * 12 + 16, "ms_per_step": e2e_s * 1e3,
                "plain_copy_ms": copy_s * 1e3,
                "api": "phem_msf_solve (C ABI), pinned host edges (four chunks, each solved while the next "
                       "is copied)"},
        "gpu_launches": gpu_launches,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_pbbs(E)
    if rank == 0 and world == 1 and not args.no_extra:
        # the other workloads of the metric, measured after the headline run
        del d_edges, d_out
        torch.cuda.empty_cache()
        try:
            line["reference_gpu"] = bench_reference_gpu(E, n, (stats.count, stats.total))
        except RuntimeError as e:
            line["reference_gpu"] = {"error": str(e)[:300]}
        torch.cuda.empty_cache()
        line["csr_input"] = bench_csr_input(ctx, torch, g, max(3, args.steps // 2), args.warmup,
                                            (stats.count, stats.total))
        line["msf_chunked"] = bench_msf_chunked(ctx, h_pinned, n, e2e_s, (stats.count, stats.total))
        line["cc"] = bench_cc(ctx, torch, peaks, args.steps, args.warmup, not args.no_cpu_baseline)
        line["batched"] = bench_batched(ctx, torch)
        line["served"] = bench_served(torch)
    if rank == 0 and world == 1 and args.stream_scale and not args.no_extra:
        try:
            line["streamed"] = bench_streamed(ctx, torch, args.stream_scale, cpu=not args.no_cpu_baseline)
        except (RuntimeError, MemoryError) as e:  # e.g. pinned host memory refused: report, keep the line
            line["streamed"] = {"workload": f"stream_rmat{args.stream_scale}_ef32", "error": str(e)[:300]}
    if rank == 0 and world == 1 and args.msf_stream_scale:
        del h_pinned, h_out
        line["msf_chunked_large"] = bench_msf_chunked_large(ctx, torch, args.msf_stream_scale)
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
