"""Edge-sharded MSF / CC across ranks (one process per GPU).

Each rank holds a contiguous share of the global edge list (global edge id =
(rank, local id) in lexicographic order).  A solve is

  1. local MSF (or spanning forest) of the rank's share on its GPU;
  2. all-gather of the local forests (at most n - 1 records each, padded with
     self-loops, which every solver ignores) over NCCL;
  3. MSF of the union of the gathered forests, on every rank.

This is exact because an edge that is not in the MSF of its own share is the
heaviest edge of a cycle there, hence of a cycle in the whole graph, and the
gathered records stay in global-id order (rank blocks, each ascending), so the
(weight, id) tie-break is the global one.  The reference merges a GPU forest
with a CPU forest the same way (CC/GPUSpanningTree.cu:74-96) and merges chunk
forests in its streaming MSF (MST/src/kernels.cu:950-953).

The gather crosses NVLink once per rank: (n - 1) * 12 bytes; there is no other
data-path collective.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def pad_forest(records, n: int):
    """(k, 3) records -> (n - 1, 3) with self-loop padding (0, 0, 0)."""
    import torch
    rows = max(n - 1, 1)
    if isinstance(records, np.ndarray):
        out = np.zeros((rows, 3), records.dtype)
        out[: len(records)] = records
        return out
    out = torch.zeros((rows, 3), dtype=records.dtype, device=records.device)
    out[: records.shape[0]] = records
    return out


def sharded_msf(local_solve: Callable, merge_solve: Callable, edges_local, n: int, group=None):
    """Generic three-step sharded solve.

    local_solve(edges) -> (k, 3) forest records ascending by local id;
    merge_solve(records) -> result of the union solve.  Works with any
    torch.distributed backend (NCCL on GPUs, gloo in the CPU tests)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    forest = local_solve(edges_local)
    padded = pad_forest(forest, n)
    t = (padded if isinstance(padded, torch.Tensor) else torch.from_numpy(padded.view(np.int32))).contiguous()
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    return merge_solve(torch.cat(parts, 0))


def sharded_msf_device(ctx, d_edges, m_local: int, n: int, stream=None, group=None):
    """The GPU form: local solve and merge through libphem on device tensors;
    returns the merged MSFResult (count, total and per-round stats of the merge)."""
    import torch
    dev = d_edges.device
    d_out = torch.empty((max(n - 1, 1), 3), dtype=torch.int32, device=dev)
    d_ct = torch.zeros(2, dtype=torch.int64, device=dev)

    def local_solve(e):
        ctx.msf_solve_device(e, m_local, n, d_out, d_ct)
        # zero the unused tail on the device: those rows become self-loops
        idx = torch.arange(d_out.shape[0], device=dev)
        d_out.masked_fill_((idx >= d_ct[0]).unsqueeze(1), 0)
        return d_out

    d_final = torch.empty((max(n - 1, 1), 3), dtype=torch.int32, device=dev)
    d_ct2 = torch.zeros(2, dtype=torch.int64, device=dev)

    def merge_solve(records):
        return ctx.msf_solve_device(records, records.shape[0], n, d_final, d_ct2)

    return sharded_msf(local_solve, merge_solve, d_edges, n, group)
