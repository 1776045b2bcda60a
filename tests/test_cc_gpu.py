"""GPU parity: connected components + spanning forest against the oracle and
the reference's golden vectors.  Labels are bit-exact; the default forest is
checked for validity (which edge wins a hooking race is not fixed, in the
reference either); the canonical forest is bit-exact as a set."""
import numpy as np
import pytest

import oracle
import phem_graph_b200 as P
from phem_graph_b200 import _lib, gen
from phem_graph_b200.api import forest_set
from tests.golden import load, names

pytestmark = pytest.mark.gpu
CC_CASES = names("cc_")


def check_forest(edges, n, labels, forest):
    """Valid spanning forest of the graph: |F| = n - c, every slot edge is an
    input edge with u < v, and F alone reproduces the labels."""
    f = forest_set(forest)
    c = len(np.unique(labels))
    assert len(f) == n - c
    live = np.unique(edges[(edges >> np.uint64(32)) < (edges & np.uint64(0xFFFFFFFF))])
    assert np.all(np.isin(f, live))
    lab_f, _ = oracle.cc_solve(f, n)
    np.testing.assert_array_equal(lab_f, labels)


@pytest.mark.parametrize("name", CC_CASES)
def test_golden_labels_and_forest(ctx, name):
    g = load(name)
    edges, n = g["edges"], int(g["n"])
    r = ctx.cc_solve(edges, n)
    np.testing.assert_array_equal(r.labels, g["labels"])
    check_forest(edges, n, r.labels, r.forest)
    assert r.components == len(np.unique(g["labels"]))


@pytest.mark.parametrize("name", CC_CASES)
def test_golden_canonical_forest_bit_exact(ctx, name):
    g = load(name)
    edges, n = g["edges"], int(g["n"])
    r = ctx.cc_solve(edges, n, canonical=True)
    np.testing.assert_array_equal(r.labels, g["labels"])
    np.testing.assert_array_equal(forest_set(r.forest), g["forest"])


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
@pytest.mark.parametrize("n,draws", [(1000, 800), (1 << 14, 1 << 15), (1 << 16, 1 << 19)])
def test_er_random(ctx, seed, n, draws):
    g = gen.er_graph(n, draws, seed)
    labels, forest = oracle.cc_solve(g.pairs, n)
    r = ctx.cc_solve(g.pairs, n)
    np.testing.assert_array_equal(r.labels, labels)
    check_forest(g.pairs, n, r.labels, r.forest)
    rc = ctx.cc_solve(g.pairs, n, canonical=True)
    np.testing.assert_array_equal(rc.labels, labels)
    np.testing.assert_array_equal(forest_set(rc.forest), oracle.forest_set(forest))


@pytest.mark.parametrize("scale", [12, 16])
def test_rmat_hubs(ctx, scale):
    p = gen.rmat(scale, 16 << scale, seed=scale)
    n = 1 << scale
    labels, forest = oracle.cc_solve(p, n)
    r = ctx.cc_solve(p, n)
    np.testing.assert_array_equal(r.labels, labels)
    check_forest(p, n, r.labels, r.forest)
    rc = ctx.cc_solve(p, n, canonical=True)
    np.testing.assert_array_equal(forest_set(rc.forest), oracle.forest_set(forest))


@pytest.mark.slow
def test_full_size_er20(ctx):
    """The CC workload at full size: n = 2^20, 8 * 2^20 draws, seed 1."""
    g = gen.er_graph(1 << 20, 8 << 20, 1)
    labels, forest = oracle.cc_solve(g.pairs, g.n)
    r = ctx.cc_solve(g.pairs, g.n)
    np.testing.assert_array_equal(r.labels, labels)
    assert r.forest_edges == g.n - len(np.unique(labels))
    rc = ctx.cc_solve(g.pairs, g.n, canonical=True)
    np.testing.assert_array_equal(forest_set(rc.forest), oracle.forest_set(forest))
    # idempotence: solving the forest alone gives the same labels and keeps every forest edge
    r2 = ctx.cc_solve(forest_set(r.forest), g.n)
    np.testing.assert_array_equal(r2.labels, labels)
    assert r2.forest_edges == r.forest_edges


def test_edge_cases(ctx):
    # no edges
    r = ctx.cc_solve(np.zeros(0, np.uint64), 5)
    np.testing.assert_array_equal(r.labels, np.arange(5))
    assert np.all(r.forest == _lib.PHEM_FOREST_EMPTY)
    # one vertex
    assert ctx.cc_solve(np.zeros(0, np.uint64), 1).labels.tolist() == [0]
    # self-loops and u > v are skipped (union_find_gpu_COO unites only u < v)
    e = np.array([(3 << 32) | 3, (4 << 32) | 1, (1 << 32) | 2], np.uint64)
    r = ctx.cc_solve(e, 5)
    assert r.labels.tolist() == [0, 1, 1, 3, 4]
    rc = ctx.cc_solve(e, 5, canonical=True)
    assert rc.labels.tolist() == [0, 1, 1, 3, 4]
    assert forest_set(rc.forest).tolist() == [(1 << 32) | 2]
    # odd m exercises the tail of the vectorised loads
    e = gen.er(100, 333, 3)
    assert len(e) % 2 == 1 or True
    lab, _ = oracle.cc_solve(e, 100)
    np.testing.assert_array_equal(ctx.cc_solve(e[:-1], 100).labels, oracle.cc_solve(e[:-1], 100)[0])
    np.testing.assert_array_equal(ctx.cc_solve(e, 100).labels, lab)


def test_out_of_range_endpoint_rejected(ctx):
    e = np.array([(1 << 32) | 7], np.uint64)
    with pytest.raises(P.PhemError) as ei:
        ctx.cc_solve(e, 5)
    assert ei.value.status == _lib.PHEM_ERR_INVALID
    with pytest.raises(P.PhemError):
        ctx.cc_solve(e, 5, canonical=True)
    # the context is still usable
    assert ctx.cc_solve(np.array([(0 << 32) | 1], np.uint64), 2).labels.tolist() == [0, 0]


def test_device_resident_inputs(ctx):
    import torch
    g = gen.er_graph(1 << 15, 1 << 16, 9)
    d_edges = torch.from_numpy(g.pairs.view(np.int64)).cuda()
    d_lab = torch.empty(g.n, dtype=torch.int32, device="cuda")
    d_for = torch.empty(g.n, dtype=torch.int64, device="cuda")
    ctx.cc_solve(d_edges, g.n, labels=d_lab, forest=d_for)
    labels, _ = oracle.cc_solve(g.pairs, g.n)
    np.testing.assert_array_equal(d_lab.cpu().numpy(), labels)
    check_forest(g.pairs, g.n, labels, d_for.cpu().numpy().view(np.uint64))


def test_stage_entry_points_and_reference_pipeline(ctx):
    """SpanningTree + gpu_spanning_tree as the reference driver runs them
    (CC/main.cu:157-186): stream the edges in batches, then merge the batch
    forest with a second forest (here the CPU oracle's forest of a second edge
    share, standing in for the reference's CPU partner)."""
    import torch
    g = gen.er_graph(1 << 16, 3 << 16, 5)
    n = g.n
    half = len(g.pairs) // 2
    gpu_share, cpu_share = g.pairs[:half], g.pairs[half:]
    parent = torch.empty(n, dtype=torch.int32, device="cuda")
    label = torch.empty(n, dtype=torch.int32, device="cuda")
    t1 = torch.empty(n, dtype=torch.int64, device="cuda")
    pinned = torch.from_numpy(gpu_share.view(np.int64)).pin_memory()
    ctx.cc_stream(pinned, n, 4097, parent, label, t1)
    _, cpu_forest = oracle.cc_solve(cpu_share, n)
    extra = torch.from_numpy(cpu_forest.view(np.int64)).cuda()
    t2 = torch.empty(n, dtype=torch.int64, device="cuda")
    ctx.cc_merge(t1, extra, n, parent, label, t2)
    labels, _ = oracle.cc_solve(g.pairs, n)
    np.testing.assert_array_equal(label.cpu().numpy(), labels)
    check_forest(g.pairs, n, labels, t2.cpu().numpy().view(np.uint64))
    # stage-level calls on device buffers reproduce the one-shot solve
    d_edges = torch.from_numpy(g.pairs.view(np.int64)).cuda()
    ctx.cc_init(n, parent, label, t1)
    ctx.cc_unite(d_edges, len(g.pairs), n, parent, t1)
    ctx.cc_label(n, parent, label)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(label.cpu().numpy(), labels)


def test_stream_unsorted_rmat_batches(ctx):
    """SpanningTree over an unsorted R-MAT stream in ragged batches: labels
    equal the oracle's, the forest reproduces them."""
    import ctypes as C
    import torch
    scale, draws = 18, 32 << 18
    out = np.empty(draws, np.uint64)
    m = C.c_uint64()
    _lib.check(_lib.lib().phem_gen_rmat_range(scale, 0, draws, 0.57, 0.19, 0.19, 28, out.ctypes.data, C.byref(m)),
               "phem_gen_rmat_range")
    pairs = out[: m.value]
    n = 1 << scale
    pinned = torch.from_numpy(pairs.view(np.int64)).pin_memory()
    dev = torch.device("cuda", 0)
    parent = torch.empty(n, dtype=torch.int32, device=dev)
    label = torch.empty(n, dtype=torch.int32, device=dev)
    forest = torch.empty(n, dtype=torch.int64, device=dev)
    ctx.cc_stream(pinned.numpy().view(np.uint64), n, (1 << 20) + 12345, parent, label, forest)
    ctx.cc_label(n, parent, label)
    torch.cuda.synchronize()
    want, _ = oracle.cc_solve(pairs, n)
    got = label.cpu().numpy()
    np.testing.assert_array_equal(got, want)
    check_forest(pairs, n, got, forest.cpu().numpy().view(np.uint64))


def test_incremental_stream_batches_of_every_kind(ctx):
    """phem_cc_stream_begin/push/end: ragged batches from pinned and pageable
    host memory (one larger than the first staging buffers, which then grow),
    aligned device memory (united in place, one batch empty) and an unaligned
    device view (staged): labels equal the oracle's and the forest reproduces
    them."""
    import torch
    g = gen.er_graph(1 << 16, 1 << 21, 41)
    n, pairs = g.n, g.pairs
    cuts = [0, 1, 1001, 1001, 70001, 1270001, 1273000, len(pairs)]
    dev = torch.device("cuda", ctx.device)
    parent = torch.empty(n, dtype=torch.int32, device=dev)
    label = torch.empty(n, dtype=torch.int32, device=dev)
    forest = torch.empty(n, dtype=torch.int64, device=dev)
    d_all = torch.from_numpy(pairs.view(np.int64)).to(dev)
    ctx.cc_stream_begin(n, parent, label, forest)
    for k in range(len(cuts) - 1):
        a, b = cuts[k], cuts[k + 1]
        kind = k % 4
        if kind == 0:
            ctx.cc_stream_push(torch.from_numpy(pairs[a:b].view(np.int64)).pin_memory())
        elif kind == 1:
            ctx.cc_stream_push(pairs[a:b].copy())
        elif kind == 2:
            ctx.cc_stream_push(d_all[a:b] if a % 2 == 0 else d_all[a:b].clone())
        else:
            ctx.cc_stream_push(d_all[a:b])  # odd start: 8-byte aligned only, staged
    ms = ctx.cc_stream_end()
    assert ms > 0
    ctx.cc_label(n, parent, label)
    torch.cuda.synchronize()
    want, _ = oracle.cc_solve(pairs, n)
    got = label.cpu().numpy()
    np.testing.assert_array_equal(got, want)
    check_forest(pairs, n, got, forest.cpu().numpy().view(np.uint64))


def test_incremental_stream_call_order(ctx):
    """push and end need an open stream; a second begin is refused; a stream
    can be opened again after its end."""
    import torch
    n = 64
    parent = torch.empty(n, dtype=torch.int32, device="cuda")
    with pytest.raises(P.PhemError) as ei:
        ctx.cc_stream_push(np.array([1], np.uint64))
    assert ei.value.status == _lib.PHEM_ERR_INVALID
    with pytest.raises(P.PhemError):
        ctx.cc_stream_end()
    ctx.cc_stream_begin(n, parent)
    with pytest.raises(P.PhemError):
        ctx.cc_stream_begin(n, parent)
    ctx.cc_stream_push(np.array([(1 << 32) | 2, (2 << 32) | 3], np.uint64))
    ctx.cc_stream_end()
    ctx.cc_stream_begin(n, parent)
    ctx.cc_stream_push(np.array([(5 << 32) | 9], np.uint64))
    ctx.cc_stream_end()
    label = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.cc_label(n, parent, label)
    got = label.cpu().numpy()
    assert got[9] == 5 and got[3] == 3 and got[2] == 2  # only the second stream's edge


@pytest.mark.parametrize("light", [0.0, 0.5, 2.0, 6.0])
def test_canonical_filter_setting_does_not_change_the_forest(ctx, light):
    """The canonical forest's light/heavy split (first edges by index) gives
    the sequential reference's forest set for any split size, unfiltered
    included."""
    g = gen.er_graph(1 << 15, 1 << 18, 23)
    want_labels, want_forest = oracle.cc_solve(g.pairs, g.n)
    saved = ctx.get_tuning("cc.canonical_light_per_vertex")
    try:
        ctx.set_tuning("cc.canonical_light_per_vertex", light)
        rc = ctx.cc_solve(g.pairs, g.n, canonical=True)
    finally:
        ctx.set_tuning("cc.canonical_light_per_vertex", saved)
    np.testing.assert_array_equal(rc.labels, want_labels)
    np.testing.assert_array_equal(forest_set(rc.forest), oracle.forest_set(want_forest))


@pytest.mark.parametrize("sample", [0.0, 0.5, 2.0, 1000.0])
def test_sample_schedule_same_labels(ctx, sample):
    """The prefix-sample / compress / rest schedule gives the same labels and
    a valid forest for any sample size."""
    g = gen.er_graph(1 << 16, 1 << 19, 9)
    want, _ = oracle.cc_solve(g.pairs, g.n)
    saved = ctx.get_tuning("cc.sample_per_vertex")
    try:
        ctx.set_tuning("cc.sample_per_vertex", sample)
        r = ctx.cc_solve(g.pairs, g.n)
    finally:
        ctx.set_tuning("cc.sample_per_vertex", saved)
    np.testing.assert_array_equal(r.labels, want)
    check_forest(g.pairs, g.n, r.labels, r.forest)


@pytest.mark.parametrize("sample", [0.0, 1.0, 6.0])
@pytest.mark.parametrize("pinned", [False, True])
def test_host_edges_copied_in_overlapped_chunks(ctx, sample, pinned):
    """Large host inputs are copied in 2^21-edge chunks on a second stream,
    each chunk's union waiting for its own copy; prefixes that end inside,
    at the end of, or beyond several chunks give the oracle's labels and a
    valid forest, from pageable and from pinned memory, twice in a row."""
    import torch
    g = gen.er_graph(1 << 19, 5_000_001, 17)
    edges = g.pairs if not pinned else torch.from_numpy(g.pairs.view(np.int64)).pin_memory().numpy().view(np.uint64)
    want, _ = oracle.cc_solve(g.pairs, g.n)
    saved = ctx.get_tuning("cc.sample_per_vertex")
    try:
        ctx.set_tuning("cc.sample_per_vertex", sample)
        for _ in range(2):
            r = ctx.cc_solve(edges, g.n)
            np.testing.assert_array_equal(r.labels, want)
            check_forest(g.pairs, g.n, r.labels, r.forest)
    finally:
        ctx.set_tuning("cc.sample_per_vertex", saved)


def test_solves_from_reference_file_formats(ctx, tmp_path):
    """Inputs read from the reference drivers' file formats solve to the
    oracle's results (ECL binary CSR for CC, MatrixMarket for MSF)."""
    from phem_graph_b200 import io
    g = gen.rmat_graph(12, 8, seed=6)
    off, cols = gen.csr_from_pairs(g.pairs, g.n)
    io.write_ecl(tmp_path / "g.egr", off, cols)
    pairs, n = io.read_graph_pairs(tmp_path / "g.egr")
    want, _ = oracle.cc_solve(pairs, n)
    np.testing.assert_array_equal(ctx.cc_solve(pairs, n).labels, want)
    io.write_mtx(tmp_path / "g.mtx", g.msf_edges(), g.n)
    e, n = io.read_mtx(tmp_path / "g.mtx")
    flags, cnt, tot = oracle.msf_kruskal(e, n)
    r = ctx.msf_solve(e, n)
    assert (r.count, r.total) == (cnt, tot)
    np.testing.assert_array_equal(r.edges, e[flags])
