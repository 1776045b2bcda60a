"""GPU parity: minimum spanning forest against the reference's golden vectors
and the oracle.  Bit-exact: the MSF edge records (ascending by edge id, as the
PBBS result), their count and the uint64 total weight."""
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
def test_golden(ctx, name):
    g = load(name)
    E, n = g["edges"], int(g["n"])
    r = ctx.msf_solve(E, n)
    assert_msf(r, E, g["msf_ids"], int(g["count"]), int(g["total"]))


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("scale,ef,bits", [(10, 4, 20), (12, 16, 20), (14, 8, 4), (16, 16, 20), (13, 2, 1)])
def test_rmat_random(ctx, seed, scale, ef, bits):
    g = gen.rmat_graph(scale, ef, seed=seed, bits=bits)
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    r = ctx.msf_solve(E, g.n)
    assert_msf(r, E, ids, cnt, tot)
    assert sum(r.n_r) >= cnt  # every MSF edge is hooked by one chooser


@pytest.mark.parametrize("lpv", [0.0, 0.25, 1.0, 2.0, 6.0])
@pytest.mark.parametrize("scale,ef,bits", [(12, 16, 20), (13, 8, 3)])
def test_filter_settings_do_not_change_the_forest(ctx, lpv, scale, ef, bits):
    g = gen.rmat_graph(scale, ef, seed=11, bits=bits)
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    old = ctx.get_tuning("msf.light_per_vertex")
    ctx.set_tuning("msf.light_per_vertex", lpv)
    try:
        r = ctx.msf_solve(E, g.n)
    finally:
        ctx.set_tuning("msf.light_per_vertex", old)
    assert_msf(r, E, ids, cnt, tot)
    if lpv == 0.0:
        assert r.threshold == 2**64 - 1 and r.light_rounds == r.rounds


@pytest.mark.parametrize("scale,ef", [(12, 16), (15, 8)])
def test_unfiltered_rounds_equal_boruvka_restatement(ctx, scale, ef):
    """With the filter off the device runs plain Boruvka: every round the same
    components choose (n_r is the restatement's) and the same forest results.
    The device drops parallel records between two components that cannot win
    (all but the lightest of a group met in one row), so its live edge counts
    are at most the restatement's, which keeps every parallel edge."""
    g = gen.rmat_graph(scale, ef, seed=scale)
    E = g.msf_edges()
    _, _, _, m_r, n_r = oracle.msf_boruvka(E, g.n)
    saved = ctx.get_tuning("msf.light_per_vertex")
    ctx.set_tuning("msf.light_per_vertex", 0)
    try:
        r = ctx.msf_solve(E, g.n)
    finally:
        ctx.set_tuning("msf.light_per_vertex", saved)
    ids, cnt, tot = expect(E, g.n)
    assert_msf(r, E, ids, cnt, tot)
    assert r.n_r == [int(x) for x in n_r] + [0]
    assert len(r.m_r) == len(m_r) + 1 and r.m_r[-1] == 0
    assert all(a <= int(b) for a, b in zip(r.m_r, m_r))


@pytest.mark.parametrize("seed", [5, 6])
def test_er_with_ties_and_duplicates(ctx, seed):
    p = gen.er(5000, 60000, seed)
    p = np.concatenate([p, p[::3]])  # explicit parallel duplicates
    E = gen.msf_edges(p, gen.weights(len(p), seed, bits=2))
    ids, cnt, tot = expect(E, 5000)
    assert_msf(ctx.msf_solve(E, 5000), E, ids, cnt, tot)


@pytest.mark.slow
def test_full_size_rmat22(ctx):
    """The MSF workload at full size (R-MAT scale 22, edge factor 16): count,
    total and every record against
    the oracle; the light/heavy filter is active at this size."""
    g = gen.rmat_graph(22, 16, seed=22)
    E = g.msf_edges()
    flags, cnt, tot, m_r, n_r = oracle.msf_boruvka(E, g.n)
    r = ctx.msf_solve(E, g.n)
    assert_msf(r, E, np.nonzero(flags)[0], cnt, tot)
    assert r.threshold != 2**64 - 1 and r.light_rounds < r.rounds  # the filter ran
    # idempotence: the MSF of the MSF is itself
    r2 = ctx.msf_solve(r.edges, g.n)
    assert (r2.count, r2.total) == (r.count, r.total)


def test_edge_cases(ctx):
    # no edges: empty forest
    r = ctx.msf_solve(np.zeros((0, 3), np.uint32), 4)
    assert (r.count, r.total) == (0, 0)
    # only self-loops
    r = ctx.msf_solve(np.array([[1, 1, 5], [2, 2, 1]], np.uint32), 3)
    assert (r.count, r.total) == (0, 0)
    # u > v and a weight of 2^31 - 1 (largest the reference's int weights hold)
    E = np.array([[1, 0, 2**31 - 1], [2, 1, 3], [0, 2, 7]], np.uint32)
    r = ctx.msf_solve(E, 3)
    assert r.count == 2 and r.total == 10
    # one vertex
    assert ctx.msf_solve(np.zeros((0, 3), np.uint32), 1).count == 0
    # sizes not a multiple of the 4-record vector groups
    for m in (1, 2, 3, 5, 1023, 1025):
        p = gen.er(64, m + 8, m)[:m]
        E = gen.msf_edges(p, gen.weights(len(p), m, bits=3))
        ids, cnt, tot = expect(E, 64)
        assert_msf(ctx.msf_solve(E, 64), E, ids, cnt, tot)


def test_out_of_range_endpoint_rejected(ctx):
    with pytest.raises(P.PhemError) as ei:
        ctx.msf_solve(np.array([[0, 9, 1]], np.uint32), 4)
    assert ei.value.status == _lib.PHEM_ERR_INVALID
    assert ctx.msf_solve(np.array([[0, 1, 1]], np.uint32), 2).count == 1


@pytest.mark.parametrize("weight", [1, (1 << 20) + 7])
def test_out_of_range_endpoint_rejected_filtered(ctx, weight):
    """With the light/heavy filter on, an out-of-range endpoint is reported
    whether its edge is light (checked by the light pass) or heavy (checked
    by the heavy pass), and the context stays usable."""
    g = gen.rmat_graph(14, 16, seed=4)
    E = g.msf_edges().copy()
    E[len(E) // 2] = (3, g.n + 5, weight)
    with pytest.raises(P.PhemError) as ei:
        ctx.msf_solve(E, g.n)
    assert ei.value.status == _lib.PHEM_ERR_INVALID
    r = ctx.msf_solve(g.msf_edges(), g.n)
    ids, cnt, tot = expect(g.msf_edges(), g.n)
    assert_msf(r, g.msf_edges(), ids, cnt, tot)
    assert r.threshold != 2**64 - 1  # the filter was on


def test_device_resident(ctx):
    import torch
    g = gen.rmat_graph(14, 16, seed=7)
    E = g.msf_edges()
    d = torch.from_numpy(E.view(np.int32)).cuda()
    d_out = torch.empty((g.n, 3), dtype=torch.int32, device="cuda")
    d_ct = torch.zeros(2, dtype=torch.int64, device="cuda")
    r = ctx.msf_solve_device(d, len(E), g.n, d_out, d_ct)
    ids, cnt, tot = expect(E, g.n)
    ct = d_ct.cpu().numpy()
    assert (int(ct[0]), int(ct[1])) == (cnt, tot) == (r.count, r.total)
    np.testing.assert_array_equal(d_out[:cnt].cpu().numpy().view(np.uint32), E[ids])


def test_csr_input(ctx):
    """Symmetrised CSR in, edge ids numbered as csr_to_coo numbers them."""
    g = gen.rmat_graph(13, 16, seed=3)
    off, cols = gen.csr_from_pairs(g.pairs, g.n)
    np.testing.assert_array_equal(ctx.csr_to_coo(off, cols, g.n), g.pairs)
    np.testing.assert_array_equal(ctx.csr_to_coo(off, cols, g.n), oracle.csr_to_coo(off, cols, g.n))
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    r = ctx.msf_solve_csr(off, cols, g.n, g.w, g.m)
    assert_msf(r, E, ids, cnt, tot)


def _csr_from_entries(rows, cols, n):
    """CSR of directed entries (rows need not be sorted; a row keeps its
    entries in the given order)."""
    order = np.argsort(rows, kind="stable")
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum(np.bincount(rows, minlength=n))
    return off, np.ascontiguousarray(np.asarray(cols)[order], np.uint32)


def _csr_case(kind):
    rng = np.random.default_rng(17)
    if kind == "sparse_rows":  # long runs of empty rows between and after the entries
        n = 1 << 20
        u = rng.integers(0, n // 2, 3000)
        v = rng.integers(0, n // 2, 3000)
        return _csr_from_entries(np.r_[u, v], np.r_[v, u], n) + (n,)
    if kind == "hub":  # one row spans many tiles
        n = 40000
        u = np.r_[np.full(20000, 5), rng.integers(0, n, 60000)]
        v = np.r_[rng.permutation(np.arange(1, 20001)), rng.integers(0, n, 60000)]
        return _csr_from_entries(np.r_[u, v], np.r_[v, u], n) + (n,)
    if kind == "tile_edges":  # row lengths at and around the 1024-entry tile
        lens = np.array([1024, 1023, 1025, 1, 2048, 0, 0, 1024, 3, 4096, 1022], np.int64)
        n = 8192
        rows = np.repeat(np.arange(len(lens)), lens)
        cols = rng.integers(0, n, len(rows))
        return _csr_from_entries(rows, cols, n) + (n,)
    if kind == "asymmetric":  # directed entries, duplicates, self-loops, unsorted rows
        n = 5000
        u = rng.integers(0, n, 70000)
        v = np.where(rng.random(70000) < 0.05, u, rng.integers(0, n, 70000))
        return _csr_from_entries(u, v, n) + (n,)
    if kind == "tiny":
        return np.array([0, 1, 2, 2], np.int64), np.array([1, 0], np.uint32), 3
    if kind == "empty":
        return np.zeros(9, np.int64), np.zeros(0, np.uint32), 8
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["sparse_rows", "hub", "tile_edges", "asymmetric", "tiny", "empty"])
def test_csr_shapes(ctx, kind):
    """csr_to_coo order and content equal the reference's row walk for empty
    rows, rows spanning many tiles, tile-boundary rows and non-symmetric
    input; the fused CSR MSF input numbers edges the same way."""
    off, cols, n = _csr_case(kind)
    want = oracle.csr_to_coo(off, cols, n)
    np.testing.assert_array_equal(ctx.csr_to_coo(off, cols, n), want)
    m = len(want)
    w = np.random.default_rng(3).integers(1, 1 << 20, max(m, 1)).astype(np.uint32)[:m]
    E = np.zeros((m, 3), np.uint32)
    E[:, 0], E[:, 1], E[:, 2] = want >> np.uint64(32), want & np.uint64(0xFFFFFFFF), w
    ids, cnt, tot = expect(E, n)
    r = ctx.msf_solve_csr(off, cols, n, np.ascontiguousarray(w) if m else np.zeros(1, np.uint32), m)
    assert_msf(r, E, ids, cnt, tot)


def test_csr_many_scan_groups_and_wrong_edge_count(ctx):
    """A CSR of 16.8 M entries (8,192 tiles: two groups of the tile-offset
    scan) converts in the reference's order and solves exactly; an edge count
    that disagrees with the CSR is reported after the solve (too low or too
    high), and the context solves correctly afterwards."""
    g = gen.rmat_graph(19, 16, seed=19)
    off, cols = gen.csr_from_pairs(g.pairs, g.n)
    assert (len(cols) + 2047) // 2048 > 4096
    np.testing.assert_array_equal(ctx.csr_to_coo(off, cols, g.n), oracle.csr_to_coo(off, cols, g.n))
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    for bad in (g.m - 1, g.m + 5):
        w = np.zeros(bad, np.uint32)
        w[: min(bad, g.m)] = g.w[: min(bad, g.m)]
        with pytest.raises(P.PhemError) as ei:
            ctx.msf_solve_csr(off, cols, g.n, w, bad)
        assert ei.value.status == _lib.PHEM_ERR_INVALID
    assert_msf(ctx.msf_solve_csr(off, cols, g.n, g.w, g.m), E, ids, cnt, tot)


def test_csr_device_buffers(ctx):
    """Device offsets/cols/output take the no-staging path."""
    import torch
    g = gen.rmat_graph(15, 16, seed=8)
    off, cols = gen.csr_from_pairs(g.pairs, g.n)
    d_off = torch.from_numpy(off).cuda()
    d_cols = torch.from_numpy(cols.view(np.int32)).cuda()
    d_out = torch.empty(len(cols), dtype=torch.int64, device="cuda")
    k = _lib.C.c_int64()
    _lib.check(_lib.lib().phem_csr_to_coo(ctx._h, d_off.data_ptr(), d_cols.data_ptr(), g.n, d_out.data_ptr(),
                                          _lib.C.byref(k)), "phem_csr_to_coo")
    got = d_out[: k.value].cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(got, g.pairs)


def test_repeated_solves_share_context(ctx):
    """Workspace reuse across sizes, both directions."""
    for scale in (14, 10, 15, 9):
        g = gen.rmat_graph(scale, 8, seed=scale)
        E = g.msf_edges()
        ids, cnt, tot = expect(E, g.n)
        assert_msf(ctx.msf_solve(E, g.n), E, ids, cnt, tot)


@pytest.mark.parametrize("ctas", [1, 2, 4])
def test_edge_pass_grid_sizes(ctx, ctas):
    """Every edge-pass grid size (warps own different tiles, flush in
    different orders) gives the same forest, for weighted edges on a hub-heavy
    R-MAT graph and for packed (canonical CC) edges."""
    g = gen.rmat_graph(15, 16, seed=5)
    E = g.msf_edges()
    ids, cnt, tot = expect(E, g.n)
    c = gen.er_graph(1 << 15, 1 << 17, seed=6)
    labels, forest = oracle.cc_solve(c.pairs, c.n)
    old = ctx.get_tuning("msf.edge_ctas_per_sm")
    ctx.set_tuning("msf.edge_ctas_per_sm", ctas)
    try:
        r = ctx.msf_solve(E, g.n)
        rc = ctx.cc_solve(c.pairs, c.n, canonical=True)
    finally:
        ctx.set_tuning("msf.edge_ctas_per_sm", old)
    assert_msf(r, E, ids, cnt, tot)
    np.testing.assert_array_equal(rc.labels, labels)
    np.testing.assert_array_equal(P.api.forest_set(rc.forest), oracle.forest_set(forest))


@pytest.mark.parametrize("graph", [0, 1])
def test_graph_and_stream_round_loops(ctx, graph):
    """The rounds as a CUDA graph with a device-driven while-node and as
    batches queued on the stream give the same forest and round counts, for
    weighted and packed (canonical CC) edges, across calls whose sizes differ
    (the cached graph is updated or rebuilt)."""
    old = ctx.get_tuning("msf.graph")
    ctx.set_tuning("msf.graph", graph)
    try:
        for scale, seed in ((12, 31), (14, 32), (12, 31)):
            g = gen.rmat_graph(scale, 8, seed=seed)
            E = g.msf_edges()
            ids, cnt, tot = expect(E, g.n)
            r = ctx.msf_solve(E, g.n)
            assert_msf(r, E, ids, cnt, tot)
            _, _, _, m_r, n_r = oracle.msf_boruvka(E, g.n)
            assert r.rounds >= 1
        c = gen.er_graph(1 << 14, 1 << 16, seed=33)
        labels, forest = oracle.cc_solve(c.pairs, c.n)
        rc = ctx.cc_solve(c.pairs, c.n, canonical=True)
        np.testing.assert_array_equal(rc.labels, labels)
        np.testing.assert_array_equal(P.api.forest_set(rc.forest), oracle.forest_set(forest))
    finally:
        ctx.set_tuning("msf.graph", old)
