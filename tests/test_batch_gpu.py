"""GPU parity of the batched engine (many graphs, one persistent launch)
against the oracle: per graph, the forest edge ids (ascending), count and
uint64 total equal the (w, id) Kruskal restatement for MSF graphs and the
index-order Kruskal (the canonical forest) for CC graphs; labels equal the
oracle's min-id labels.  Every kernel configuration the autotuner can pick
gives the same results."""
import numpy as np
import pytest

import oracle
from phem_graph_b200 import _lib, gen
from phem_graph_b200._lib import PhemError

pytestmark = pytest.mark.gpu
TUNING = ("batch.block_size", "batch.items", "batch.compact_ratio")


def _pack(e):
    u = e[:, 0].astype(np.uint64)
    v = e[:, 1].astype(np.uint64)
    lo, hi = np.minimum(u, v), np.maximum(u, v)
    return (lo << np.uint64(32)) | hi


def expected(batch, g):
    """(ids, total, labels) of graph g from the oracle."""
    r = batch.graphs[g]
    n, kind = int(r["num_vertices"]), int(r["kind"])
    e = batch.graph_edges(g)
    if n == 0:
        return np.empty(0, np.uint32), 0, np.empty(0, np.int32)
    if kind == gen.PHEM_BATCH_MSF:
        flags, _, total = oracle.msf_kruskal(e, n)
    else:
        z = e.copy()
        z[:, 2] = 0  # Kruskal under edge index order
        flags, _, _ = oracle.msf_kruskal(z, n)
        total = 0
    keep = e[:, 0] != e[:, 1]
    labels, _ = oracle.cc_solve(_pack(e[keep]), n)
    return np.nonzero(flags)[0].astype(np.uint32), total, labels


def check_batch(batch, res, graphs=None):
    for g in (range(batch.num_graphs) if graphs is None else graphs):
        ids, total, labels = expected(batch, g)
        np.testing.assert_array_equal(res.forest(batch, g), ids, err_msg=f"graph {g} {batch.names[g]}")
        assert int(res.count[g]) == len(ids)
        assert int(res.total[g]) == total, f"graph {g}"
        if res.labels is not None:
            np.testing.assert_array_equal(res.graph_labels(batch, g), labels, err_msg=f"graph {g}")


def small_mixed(num=64, seed=9, n_lo=16, n_hi=12000, kind=gen.PHEM_BATCH_MSF):
    return gen.mixed_batch(num, seed, n_lo=n_lo, n_hi=n_hi, kind=kind, threads=8)


def edge_case_batch():
    """Empty, single-vertex, self-loop-only, duplicate/tie, reversed (u > v)
    and disconnected graphs, MSF and CC kinds."""
    rng = np.random.default_rng(5)
    parts = [("empty_n0", 0, np.empty((0, 3), np.uint32), gen.PHEM_BATCH_MSF),
             ("single", 1, np.empty((0, 3), np.uint32), gen.PHEM_BATCH_MSF),
             ("loops", 4, np.array([[0, 0, 5], [3, 3, 1]], np.uint32), gen.PHEM_BATCH_MSF),
             ("isolated", 50, np.array([[1, 2, 7]], np.uint32), gen.PHEM_BATCH_CC)]
    ties = rng.integers(0, 40, (400, 2)).astype(np.uint32)
    parts.append(("ties", 40, np.column_stack([ties, np.full(400, 3, np.uint32)]), gen.PHEM_BATCH_MSF))
    rev = rng.integers(0, 300, (900, 2)).astype(np.uint32)
    parts.append(("reversed", 300, np.column_stack([rev, rng.integers(1, 4, 900).astype(np.uint32)]),
                  gen.PHEM_BATCH_MSF))
    parts.append(("reversed_cc", 300, np.column_stack([rev, np.zeros(900, np.uint32)]), gen.PHEM_BATCH_CC))
    blocks = np.concatenate([rng.integers(0, 100, (300, 2)), rng.integers(100, 200, (300, 2))]).astype(np.uint32)
    parts.append(("two_blocks", 200, np.column_stack([blocks, rng.integers(1, 1 << 20, 600).astype(np.uint32)]),
                  gen.PHEM_BATCH_MSF))
    return gen.batch_from(parts)


def test_mixed_batch_matches_oracle(ctx):
    b = small_mixed()
    res = ctx.batch_solve(b)
    assert res.stats["max_rounds"] >= 1
    check_batch(b, res)


def test_caller_output_arrays(ctx):
    """Results written into caller arrays (pinned, and larger than needed)
    equal the ones the call allocates; a wrong dtype is refused."""
    import torch
    b = small_mixed(24, seed=7)
    want = ctx.batch_solve(b)
    V, G = b.total_vertices, b.num_graphs
    out = {"ids": torch.empty(V + 5, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
           "count": torch.empty(G, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
           "total": torch.empty(G + 1, dtype=torch.int64).pin_memory().numpy().view(np.uint64),
           "labels": torch.empty(V, dtype=torch.int32).pin_memory().numpy()}
    for _ in range(2):
        got = ctx.batch_solve(b, out=out)
        np.testing.assert_array_equal(got.count, want.count)
        np.testing.assert_array_equal(got.total, want.total)
        np.testing.assert_array_equal(got.labels, want.labels)
        for g in range(G):
            np.testing.assert_array_equal(got.forest(b, g), want.forest(b, g))
    with pytest.raises(ValueError):
        ctx.batch_solve(b, out={"count": np.empty(G, np.int64)})


def test_cc_kind_canonical_forest(ctx):
    b = small_mixed(32, seed=3, kind=gen.PHEM_BATCH_CC)
    res = ctx.batch_solve(b)
    check_batch(b, res)
    assert np.all(res.total == 0)


def test_edge_cases(ctx):
    b = edge_case_batch()
    check_batch(b, ctx.batch_solve(b))


def test_empty_batch(ctx):
    res = ctx.batch_solve(gen.batch_from([]))
    assert len(res.count) == 0


@pytest.mark.parametrize("block", [256, 512, 1024])
@pytest.mark.parametrize("items", [1, 2, 4])
def test_every_configuration(ctx, block, items):
    b = small_mixed(24, seed=11, n_lo=16, n_hi=20000)
    saved = [ctx.get_tuning(k) for k in TUNING]
    try:
        for ratio in (0.0, 0.5, 1.0):
            ctx.set_tuning("batch.block_size", block)
            ctx.set_tuning("batch.items", items)
            ctx.set_tuning("batch.compact_ratio", ratio)
            res = ctx.batch_solve(b)
            assert res.stats["block_size"] == block and res.stats["items"] == items
            check_batch(b, res)
    finally:
        for k, v in zip(TUNING, saved):
            ctx.set_tuning(k, v)


def test_large_graphs_use_global_state(ctx):
    """Graphs above the shared-memory capacity keep their state in HBM."""
    b = small_mixed(6, seed=21, n_lo=30000, n_hi=65536)
    res = ctx.batch_solve(b)
    assert int(b.graphs["num_vertices"].min()) > res.stats["smem_vertices"]
    check_batch(b, res)


def test_plan_replay_two_batches(ctx):
    a = small_mixed(40, seed=1)
    c = small_mixed(70, seed=2, n_hi=5000)
    with ctx.batch_plan(128, max(a.total_edges, c.total_edges), max(a.total_vertices, c.total_vertices)) as p:
        for b in (a, c, a):
            p.upload(b)
            p.run()
            check_batch(b, p.download())
        assert all(v for v in p.device().values())


def test_large_host_batch_overlapped_launches(ctx):
    """A batch of host edges past the overlap size is copied in chunks and
    solved by one launch per chunk group (graphs straddling chunk ends go
    to the later group); every graph's forest, count, total and labels equal
    the single-launch result of a plan, twice in a row."""
    b = gen.mixed_batch(160, 21, n_lo=64, n_hi=65536, threads=8)
    assert b.total_edges >= 1 << 22
    with ctx.batch_plan(b.num_graphs, b.total_edges, b.total_vertices) as p:
        p.upload(b)
        p.run()
        want = p.download(labels=True)
    for _ in range(2):
        got = ctx.batch_solve(b)
        np.testing.assert_array_equal(got.count, want.count)
        np.testing.assert_array_equal(got.total, want.total)
        np.testing.assert_array_equal(got.labels, want.labels)
        for g in range(b.num_graphs):
            np.testing.assert_array_equal(got.forest(b, g), want.forest(b, g))


def test_plan_rejects_oversized_batch(ctx):
    a = small_mixed(8, seed=4)
    with ctx.batch_plan(4, a.total_edges, a.total_vertices) as p:
        with pytest.raises(PhemError) as e:
            p.upload(a)
        assert e.value.status == _lib.PHEM_ERR_INVALID


def test_invalid_inputs_are_rejected(ctx):
    bad = gen.batch_from([("oob", 5, np.array([[0, 9, 1]], np.uint32), gen.PHEM_BATCH_MSF)])
    with pytest.raises(PhemError) as e:
        ctx.batch_solve(bad)
    assert e.value.status == _lib.PHEM_ERR_INVALID
    one = np.array([[0, 1, 1]], np.uint32)
    ov = gen.batch_from([("a", 10, one, 0), ("b", 10, one, 0)])
    ov.graphs["vertex_offset"][1] = 5  # overlaps graph 0
    with pytest.raises(PhemError) as e:
        ctx.batch_solve(ov)
    assert e.value.status == _lib.PHEM_ERR_INVALID
    b = edge_case_batch()  # the context stays usable
    check_batch(b, ctx.batch_solve(b))


def test_autotune_picks_a_grid_point(ctx):
    b = small_mixed(48, seed=13)
    saved = [ctx.get_tuning(k) for k in TUNING]
    try:
        best = ctx.batch_autotune(b, reps=1)
        assert best["block_size"] in (256, 512, 1024) and best["items"] in (1, 2, 4)
        assert best["compact_ratio"] in (0.25, 0.5, 1.0) and best["device_ms"] > 0
        assert ctx.get_tuning("batch.block_size") == best["block_size"]
        check_batch(b, ctx.batch_solve(b))
    finally:
        for k, v in zip(TUNING, saved):
            ctx.set_tuning(k, v)


def test_batch_equals_one_graph_path(ctx):
    """A graph's batched forest equals phem_msf_solve's on that graph alone."""
    b = small_mixed(12, seed=17, n_lo=1000, n_hi=40000)
    res = ctx.batch_solve(b)
    for g in range(b.num_graphs):
        n = int(b.graphs[g]["num_vertices"])
        one = ctx.msf_solve(b.graph_edges(g), n)
        np.testing.assert_array_equal(b.graph_edges(g)[res.forest(b, g)], one.edges)
        assert one.total == int(res.total[g])


@pytest.mark.slow
def test_full_workload_sampled(ctx):
    """The 4096-graph workload: every graph's forest size agrees with its
    labels, and a sample of graphs matches the oracle exactly."""
    b = gen.mixed_batch(4096, 4)
    res = ctx.batch_solve(b)
    for g in range(b.num_graphs):
        n = int(b.graphs[g]["num_vertices"])
        assert int(res.count[g]) == n - len(np.unique(res.graph_labels(b, g)))
    rng = np.random.default_rng(0)
    check_batch(b, res, graphs=sorted(rng.choice(b.num_graphs, 96, replace=False).tolist()))
