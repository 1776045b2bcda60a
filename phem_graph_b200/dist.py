"""Edge-sharded MSF / CC across ranks (one process per GPU).

Each rank holds a contiguous share of the global edge list (global edge id =
(rank, local id) in lexicographic order).  A solve is

  1. the local MSF (or spanning forest) of the rank's share on its GPU;
  2. an all-gather of the local forests over NCCL;
  3. the MSF (or the spanning forest and labels) of the union of the gathered
     forests, on every rank.

MSF: exact because an edge that is not in the MSF of its own share is the
heaviest edge of a cycle there, hence of a cycle in the whole graph, and the
gathered records stay in global-id order (rank blocks, each ascending), so the
(weight, id) tie-break is the global one.  A local forest has at most n - 1
records and is padded with self-loops, which every solver ignores.

CC: a spanning forest of each share connects exactly what the share connects,
so the union of the local forests has the components of the whole graph; the
local forests are the reference's slot arrays (forest[hooked root] = edge, the
rest PHEM_FOREST_EMPTY, n slots each) and are merged pairwise by
phem_cc_merge, which is the reference's own merge of two forests
(gpu_spanning_tree, CC/GPUSpanningTree.cu:74-96,169-198).  Labels are the
min-id labels of the whole graph; the forest is a spanning forest of it.

The reference merges a GPU forest with a CPU forest the same way and merges
chunk forests in its streaming MSF (MST/src/kernels.cu:950-953).  The gather
crosses NVLink once per rank: (n - 1) * 12 bytes (MSF) or n * 8 bytes (CC);
there is no other data-path collective.

`gather` (every function): a callable taking this rank's tensor and returning
every rank's, in rank order; the default is torch.distributed.all_gather over
`group`.  The one-GPU tests pass a local stand-in for it.
"""
from __future__ import annotations

from typing import Callable

import numpy as np

FOREST_EMPTY = 0x7FFFFFFF


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


def all_gather(group=None) -> Callable:
    """The default gather: torch.distributed.all_gather over `group`."""
    import torch
    import torch.distributed as dist

    def gather(t):
        parts = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
        dist.all_gather(parts, t, group=group)
        return parts
    return gather


def sharded_msf(local_solve: Callable, merge_solve: Callable, edges_local, n: int, group=None,
                gather: Callable | None = None):
    """Generic three-step sharded MSF.

    local_solve(edges) -> (k, 3) forest records ascending by local id;
    merge_solve(records) -> result of the union solve.  Works with any
    torch.distributed backend (NCCL on GPUs, gloo in the CPU tests)."""
    import torch
    forest = local_solve(edges_local)
    padded = pad_forest(forest, n)
    t = (padded if isinstance(padded, torch.Tensor) else torch.from_numpy(padded.view(np.int32))).contiguous()
    parts = (gather or all_gather(group))(t)
    return merge_solve(torch.cat(list(parts), 0))


def sharded_cc(local_solve: Callable, merge: Callable, pairs_local, n: int, group=None,
               gather: Callable | None = None):
    """Generic three-step sharded CC.

    local_solve(pairs) -> the n forest slots of the share (uint64 numpy array
    or int64 tensor, PHEM_FOREST_EMPTY where no edge hooked);
    merge(slots_a, slots_b) -> (labels, slots) of the union of two slot arrays.
    The gathered slot arrays are merged left to right in rank order; returns
    the last merge's (labels, slots)."""
    import torch
    slots = local_solve(pairs_local)
    t = (slots if isinstance(slots, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(slots).view(np.int64)))
    parts = list((gather or all_gather(group))(t.contiguous()))
    labels, acc = merge(parts[0], parts[1] if len(parts) > 1 else None)
    for p in parts[2:]:
        labels, acc = merge(acc, p)
    return labels, acc


def local_msf_forest_device(ctx, d_edges, m_local: int, n: int):
    """Local step on the GPU: the share's MSF records, padded to n - 1 rows of
    self-loops on the device."""
    import torch
    dev = d_edges.device
    d_out = torch.empty((max(n - 1, 1), 3), dtype=torch.int32, device=dev)
    d_ct = torch.zeros(2, dtype=torch.int64, device=dev)
    ctx.msf_solve_device(d_edges, m_local, n, d_out, d_ct)
    # zero the unused tail on the device: those rows become self-loops
    idx = torch.arange(d_out.shape[0], device=dev)
    d_out.masked_fill_((idx >= d_ct[0]).unsqueeze(1), 0)
    return d_out


def sharded_msf_device(ctx, d_edges, m_local: int, n: int, stream=None, group=None,
                       gather: Callable | None = None):
    """The GPU form: local solve and merge through libphem on device tensors;
    returns the merged MSFResult (count, total and per-round stats of the
    merge; edges = the forest records as a device tensor)."""
    import torch
    dev = d_edges.device
    d_final = torch.empty((max(n - 1, 1), 3), dtype=torch.int32, device=dev)
    d_ct2 = torch.zeros(2, dtype=torch.int64, device=dev)

    def merge_solve(records):
        res = ctx.msf_solve_device(records, records.shape[0], n, d_final, d_ct2)
        res.edges = d_final[: res.count]  # the forest records (device), ascending by global id
        return res

    return sharded_msf(lambda e: local_msf_forest_device(ctx, e, m_local, n), merge_solve, d_edges, n, group, gather)


def local_cc_forest_device(ctx, d_pairs, n: int):
    """Local step on the GPU: union-find over the share's packed pairs; returns
    its n forest slots (int64 device tensor)."""
    import torch
    dev = d_pairs.device
    labels = torch.empty(n, dtype=torch.int32, device=dev)
    slots = torch.empty(n, dtype=torch.int64, device=dev)
    ctx.cc_solve(d_pairs, n, labels=labels, forest=slots)
    return slots


def sharded_cc_device(ctx, d_pairs, n: int, group=None, gather: Callable | None = None):
    """The GPU form of sharded_cc: local phem_cc_solve, all-gather of the slot
    arrays, pairwise phem_cc_merge.  Returns (labels, forest slots) as device
    tensors."""
    import torch
    dev = d_pairs.device

    def merge(a, b):
        parent = torch.empty(n, dtype=torch.int32, device=dev)
        labels = torch.empty(n, dtype=torch.int32, device=dev)
        out = torch.empty(n, dtype=torch.int64, device=dev)
        ctx.cc_merge(a, b, n, parent, labels, out)
        return labels, out

    return sharded_cc(lambda p: local_cc_forest_device(ctx, p, n), merge, d_pairs, n, group, gather)
