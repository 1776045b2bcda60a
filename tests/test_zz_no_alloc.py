"""phem_cc_solve_noalloc (fixed static scratch, no device allocation) against
phem_cc_solve on the same inputs, called through the C ABI.

Kept in its own file, collected last, so that it runs both alone and after
every other GPU test of the session."""
import ctypes as C

import numpy as np
import pytest

import oracle
from phem_graph_b200 import _lib, gen
from phem_graph_b200.api import forest_set

pytestmark = pytest.mark.gpu
MAX_N = _lib.PHEM_CC_NOALLOC_MAX_VERTICES


def _noalloc(torch, d_edges, m, n, d_labels, d_forest, stream):
    return _lib.lib().phem_cc_solve_noalloc(
        C.c_void_p(d_edges.data_ptr() if d_edges is not None else None), m, n, C.c_void_p(d_labels.data_ptr()),
        C.c_void_p(d_forest.data_ptr() if d_forest is not None else None), C.c_void_p(stream))


def _solve(torch, pairs, n, stream, with_forest=True):
    dev = torch.device("cuda", 0)
    d_edges = torch.from_numpy(pairs.view(np.int64)).to(dev)
    d_labels = torch.full((n,), -1, dtype=torch.int32, device=dev)
    d_forest = torch.zeros(n, dtype=torch.int64, device=dev) if with_forest else None
    torch.cuda.synchronize()
    st = _noalloc(torch, d_edges, len(pairs), n, d_labels, d_forest, stream)
    _lib.check(st, "phem_cc_solve_noalloc")
    labels = d_labels.cpu().numpy()
    forest = d_forest.cpu().numpy().view(np.uint64) if with_forest else None
    return labels, forest


def _check_against_solve(ctx, pairs, n, labels, forest):
    ref = ctx.cc_solve(pairs, n)
    np.testing.assert_array_equal(labels, ref.labels)
    np.testing.assert_array_equal(labels, oracle.cc_solve(pairs, n)[0])  # and the oracle's, directly
    if forest is not None:
        # which edge wins a hooking race is not fixed: compare forests by
        # validity -- n - c edges, all taken from the input with u < v, and
        # they alone give the same components
        f = forest_set(forest)
        assert len(f) == len(forest_set(ref.forest)) == n - ref.components
        live = pairs[(pairs >> np.uint64(32)) < (pairs & np.uint64(0xFFFFFFFF))]
        assert np.all(np.isin(f, live))
        np.testing.assert_array_equal(ctx.cc_solve(f, n).labels, labels)


def test_two_calls_in_a_row_match_cc_solve(ctx):
    import torch
    stream = torch.cuda.current_stream(0).cuda_stream
    # first call at the scratch limit (the ER config's n = 2^20), then a
    # smaller, differently shaped graph reusing the same scratch
    a = gen.er_graph(MAX_N, 8 << 20, 7)
    la, fa = _solve(torch, a.pairs, MAX_N, stream)
    b = gen.rmat_graph(16, 8, seed=5)
    lb, fb = _solve(torch, b.pairs, b.n, stream)
    _check_against_solve(ctx, a.pairs, MAX_N, la, fa)
    _check_against_solve(ctx, b.pairs, b.n, lb, fb)


def test_side_stream_without_forest(ctx):
    import torch
    s = torch.cuda.Stream(0)
    g = gen.er_graph(50_000, 60_000, 3)
    for _ in range(2):
        labels, _ = _solve(torch, g.pairs, g.n, s.cuda_stream, with_forest=False)
        np.testing.assert_array_equal(labels, ctx.cc_solve(g.pairs, g.n).labels)


def test_rejects_sizes_beyond_scratch_and_bad_pointers():
    import torch
    dev = torch.device("cuda", 0)
    d_edges = torch.zeros(4, dtype=torch.int64, device=dev)
    d_labels = torch.zeros(MAX_N + 1, dtype=torch.int32, device=dev)
    st = _noalloc(torch, d_edges, 4, MAX_N + 1, d_labels, None, 0)
    assert st == _lib.PHEM_ERR_INVALID
    assert str(MAX_N) in _lib.lib().phem_last_error().decode()
    # host labels are not device memory
    h = np.zeros(8, dtype=np.int32)
    st = _lib.lib().phem_cc_solve_noalloc(C.c_void_p(d_edges.data_ptr()), 4, 8, C.c_void_p(h.ctypes.data),
                                          None, None)
    assert st == _lib.PHEM_ERR_INVALID
    # edges not 16-byte aligned
    st = _lib.lib().phem_cc_solve_noalloc(C.c_void_p(d_edges.data_ptr() + 8), 2, 8,
                                          C.c_void_p(d_labels.data_ptr()), None, None)
    assert st == _lib.PHEM_ERR_INVALID


def test_endpoint_out_of_range_then_clean_call(ctx):
    """An endpoint >= n is reported through the device status word; the next
    call clears the word and succeeds."""
    import torch
    stream = torch.cuda.current_stream(0).cuda_stream
    bad = np.array([(1 << 32) | 2, (3 << 32) | 99], dtype=np.uint64)  # 99 >= n = 10
    dev = torch.device("cuda", 0)
    d_edges = torch.from_numpy(bad.view(np.int64)).to(dev)
    d_labels = torch.zeros(10, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    assert _noalloc(torch, d_edges, 2, 10, d_labels, None, stream) == _lib.PHEM_ERR_INVALID
    good = gen.er_graph(1000, 900, 11)
    labels, forest = _solve(torch, good.pairs, good.n, stream)
    _check_against_solve(ctx, good.pairs, good.n, labels, forest)
