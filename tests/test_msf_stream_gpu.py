"""GPU parity: chunked MSF (phem_msf_stream, the reference's
streamline_boruvka, MST/src/kernels.cu:849-1154) against the oracle.
Bit-exact: the forest records ascending by global edge id, their count and
uint64 total weight are phem_msf_solve's for every chunk size."""
import numpy as np
import pytest

import oracle
import phem_graph_b200 as P
from phem_graph_b200 import _lib, gen
from tests.golden import load, names

pytestmark = pytest.mark.gpu
MSF_CASES = names("msf_")


def expect(E, n):
    flags, cnt, tot = oracle.msf_kruskal(E, n)
    return np.nonzero(flags)[0], cnt, tot


def assert_msf(r, E, ids, cnt, tot):
    assert r.count == cnt and r.total == tot
    np.testing.assert_array_equal(r.edges, np.asarray(E, np.uint32).reshape(-1, 3)[ids])


@pytest.mark.parametrize("name", MSF_CASES)
def test_golden_in_chunks(ctx, name):
    """Every golden MSF vector (PBBS mst() / serial Kruskal outputs of the
    reference's own code) in one-edge (small cases), small ragged and
    three-way chunks."""
    g = load(name)
    E, n = np.asarray(g["edges"], np.uint32).reshape(-1, 3), int(g["n"])
    for chunk in sorted({1 if len(E) <= 6000 else 61, 7, max(1, len(E) // 3 + 1)}):
        assert_msf(ctx.msf_stream(E, n, chunk), E, g["msf_ids"], int(g["count"]), int(g["total"]))


@pytest.mark.parametrize("chunk", [1 << 18, 100_003, 4096, 1 << 30])
def test_stream_equals_whole_graph(ctx, chunk):
    """R-MAT scale 16 (about 1M edges): aligned, ragged and tiny chunks and a
    single chunk give the oracle's forest record for record."""
    g = gen.rmat_graph(16, 16, seed=5)
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    r = ctx.msf_stream(E, g.n, chunk)
    assert_msf(r, E, ids, cnt, tot)
    assert r.device_ms > 0


@pytest.mark.parametrize("bits", [1, 2])
@pytest.mark.parametrize("chunk", [1, 3, 37, 250])
def test_stream_ties_duplicates_self_loops(ctx, bits, chunk):
    """Heavy weight ties resolved by global edge id across chunk boundaries,
    duplicate edges and self-loops, one-edge chunks."""
    rng = np.random.default_rng(bits * 100 + chunk)
    n, m = 97, 600
    E = np.stack([rng.integers(0, n, m), rng.integers(0, n, m), rng.integers(1, 1 + (1 << bits), m)], 1)
    E = E.astype(np.uint32)
    E[::40, 1] = E[::40, 0]
    E[1::7] = E[0:-1:7][: len(E[1::7])]  # duplicates of the previous record
    ids, cnt, tot = expect(E, n)
    assert_msf(ctx.msf_stream(E, n, chunk), E, ids, cnt, tot)


@pytest.mark.parametrize("chunk", [1000, 65_536])
def test_stream_disconnected(ctx, chunk):
    """A sparse Erdos-Renyi graph with many components (about 29.6K of 65.5K
    vertices stay apart): the carried forest is far below n - 1 edges, so
    much of the forest area is unused; a few dozen edges close cycles."""
    n = 1 << 16
    p = gen.er(n, 36_000, 9)
    E = gen.msf_edges(p, gen.weights(len(p), 9, bits=12))
    ids, cnt, tot = expect(E, n)
    assert n - cnt > n // 3 and cnt < len(E)
    assert_msf(ctx.msf_stream(E, n, chunk), E, ids, cnt, tot)


def test_stream_carried_forest_sizes_mod_4(ctx):
    """Carried forests of every size modulo 4 (the solve input starts on a
    rounded-down record with zero padding before the forest)."""
    for n in (2, 3, 4, 5, 6, 9):
        for m in (1, 2, 5, 13):
            rng = np.random.default_rng(n * 31 + m)
            E = np.stack([rng.integers(0, n, m), rng.integers(0, n, m), rng.integers(1, 9, m)], 1).astype(np.uint32)
            ids, cnt, tot = expect(E, n)
            for chunk in (1, 2, 3):
                assert_msf(ctx.msf_stream(E, n, chunk), E, ids, cnt, tot)


def test_stream_edge_cases(ctx):
    r = ctx.msf_stream(np.zeros((0, 3), np.uint32), 4, 16)
    assert (r.count, r.total) == (0, 0)
    r = ctx.msf_stream(np.array([[0, 0, 3]], np.uint32), 1, 1)
    assert (r.count, r.total) == (0, 0)
    E = np.array([[1, 0, 2**31 - 1], [2, 1, 3], [0, 2, 7]], np.uint32)
    r = ctx.msf_stream(E, 3, 2)
    assert r.count == 2 and r.total == 10
    with pytest.raises(P.PhemError) as ei:
        ctx.msf_stream(E, 3, 0)
    assert ei.value.status == _lib.PHEM_ERR_INVALID
    with pytest.raises(P.PhemError) as ei:
        ctx.msf_stream(E, 2**32 - 1, 4, want_edges=False)
    assert ei.value.status == _lib.PHEM_ERR_INVALID


def test_stream_out_of_range_endpoint_in_a_later_chunk(ctx):
    g = gen.rmat_graph(12, 8, seed=3)
    E = g.msf_edges().copy()
    E[-3] = (1, g.n + 2, 5)
    with pytest.raises(P.PhemError) as ei:
        ctx.msf_stream(E, g.n, 4000)
    assert ei.value.status == _lib.PHEM_ERR_INVALID
    # the context stays usable
    ids, cnt, tot = expect(g.msf_edges(), g.n)
    assert_msf(ctx.msf_stream(g.msf_edges(), g.n, 4000), g.msf_edges(), ids, cnt, tot)


def test_stream_pinned_device_and_caller_outputs(ctx):
    import torch
    g = gen.rmat_graph(15, 16, seed=12)
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    pinned = torch.from_numpy(E.view(np.int32)).pin_memory()
    out = torch.empty((g.n, 3), dtype=torch.int32).pin_memory()
    r = ctx.msf_stream(pinned, g.n, 50_000, out=out)
    assert (r.count, r.total) == (cnt, tot)
    np.testing.assert_array_equal(out[:cnt].numpy().view(np.uint32), E[ids])
    dev = pinned.cuda()
    d_out = torch.empty((g.n, 3), dtype=torch.int32, device="cuda")
    r = ctx.msf_stream(dev, g.n, 77_777, out=d_out)
    assert (r.count, r.total) == (cnt, tot)
    np.testing.assert_array_equal(d_out[:cnt].cpu().numpy().view(np.uint32), E[ids])
    # a later one-shot solve on the same context is unaffected
    assert_msf(ctx.msf_solve(E, g.n), E, ids, cnt, tot)


@pytest.mark.slow
def test_stream_full_size_rmat22(ctx):
    """The MSF workload at full size (R-MAT scale 22, edge factor 16) in
    chunks of 2^24 edges: the oracle's forest, record for record."""
    g = gen.rmat_graph(22, 16, seed=22)
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    assert_msf(ctx.msf_stream(E, g.n, 1 << 24), E, ids, cnt, tot)
