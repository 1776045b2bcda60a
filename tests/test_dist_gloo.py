"""The sharded (multi-rank) solve on CPU: two gloo ranks, each with its own edge
share; local forests are all-gathered and merged.  The solver calls are
injected, so the oracle plays the GPU solver here -- what is tested is the
sharding, padding, gather order and merge logic of phem_graph_b200.dist."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

WORLD = 2


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def shard(rank: int, bits: int):
    from phem_graph_b200 import gen
    g = gen.rmat_graph(11, 8, seed=40 + rank, bits=bits)
    return g.msf_edges(), g.n


def _worker(rank: int, port: int, bits: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        import oracle
        from phem_graph_b200.dist import sharded_msf
        E, n = shard(rank, bits)

        def local_solve(e):
            flags, _, _ = oracle.msf_kruskal(e, n)
            return e[np.nonzero(flags)[0]]

        def merge_solve(rec):
            rec = rec.numpy().view(np.uint32).reshape(-1, 3)
            flags, cnt, tot = oracle.msf_kruskal(rec, n)
            return rec[np.nonzero(flags)[0]], cnt, tot

        recs, cnt, tot = sharded_msf(local_solve, merge_solve, E, n)
        q.put((rank, recs, cnt, tot))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("bits", [20, 2])
def test_two_rank_sharded_msf_equals_global(bits):
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, bits, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(WORLD):
        rank, recs, cnt, tot = q.get(timeout=240)
        out[rank] = (recs, cnt, tot)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # global reference: both shards concatenated in rank order (global ids)
    E0, n = shard(0, bits)
    E1, _ = shard(1, bits)
    E = np.concatenate([E0, E1])
    flags, cnt, tot = oracle.msf_kruskal(E, n)
    for rank in range(WORLD):
        recs, c, t = out[rank]
        assert (c, t) == (cnt, tot)
        np.testing.assert_array_equal(recs, E[np.nonzero(flags)[0]])


EMPTY = np.uint64(0x7FFFFFFF)


def cc_shard(rank: int):
    from phem_graph_b200 import gen
    g = gen.rmat_graph(12, 4, seed=60 + rank)
    return g.pairs, g.n


def _oracle_merge(a, b):
    """Union of two slot arrays on the CPU (the role phem_cc_merge plays on the GPU)."""
    import oracle
    a = a.numpy().view(np.uint64)
    b = b.numpy().view(np.uint64) if b is not None else np.full_like(a, EMPTY)
    both = np.concatenate([a, b])
    both = np.where(both == EMPTY, np.uint64(0), both)  # empty slot -> self-loop (skipped)
    labels, slots = oracle.cc_solve(both, len(a))
    return labels, slots


def _cc_worker(rank: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    try:
        import oracle
        from phem_graph_b200.dist import sharded_cc
        pairs, n = cc_shard(rank)

        def merge(a, b):
            labels, slots = _oracle_merge(a, b)
            return labels, torch.from_numpy(slots.view(np.int64))

        labels, slots = sharded_cc(lambda p: oracle.cc_solve(p, n)[1], merge, pairs, n)
        q.put((rank, labels, slots.numpy().view(np.uint64)))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_cc_equals_global():
    """Local union-find per share, all-gather of the slot arrays, merge: the
    labels are the whole graph's and the merged slots are a spanning forest of
    it made of input edges."""
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cc_worker, args=(r, port, q)) for r in range(WORLD)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(WORLD):
        rank, labels, slots = q.get(timeout=240)
        out[rank] = (labels, slots)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    P0, n = cc_shard(0)
    P1, _ = cc_shard(1)
    P = np.concatenate([P0, P1])
    ref_labels, _ = oracle.cc_solve(P, n)
    comps = len(np.unique(ref_labels))
    for rank in range(WORLD):
        labels, slots = out[rank]
        np.testing.assert_array_equal(labels, ref_labels)
        f = oracle.forest_set(slots)
        assert len(f) == n - comps
        assert np.all(np.isin(f, P))
        np.testing.assert_array_equal(oracle.cc_solve(f, n)[0], ref_labels)
