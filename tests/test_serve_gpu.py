"""GPU tests of the serving loop: every request's result is the same alone
(one-graph entry points on an idle context) and in a mix of concurrent
requests served by batched launches and device-wide solves; admission by
the memory budget refuses what can never fit."""
import threading

import numpy as np
import pytest

from phem_graph_b200 import _lib
from phem_graph_b200._lib import PhemError
from phem_graph_b200.serve import (PHEM_BATCH_CC, PHEM_BATCH_MSF, Server, ServedGraph, poisson_arrivals,
                                   request_pool)

pytestmark = pytest.mark.gpu


def alone(ctx, g):
    if g.kind == PHEM_BATCH_MSF:
        r = ctx.msf_solve(g.edges, g.n)
        return r.edges, r.count, r.total
    r = ctx.cc_solve(g.pairs, g.n)
    return r.labels, int(g.n - r.components), 0


def check_same(ctx, g, s):
    assert s.status == 0
    want, count, total = alone(ctx, g)
    assert s.forest_edges == count
    if g.kind == PHEM_BATCH_MSF:
        np.testing.assert_array_equal(s.forest, want)
        assert s.total_weight == total
    else:
        np.testing.assert_array_equal(s.labels, want)


@pytest.fixture(scope="module")
def pool():
    # sizes span both paths: large_edges = 2^13 below
    return request_pool(48, seed=3, m_lo=1 << 6, m_hi=1 << 17, threads=8)


def test_alone_equals_in_the_mix(ctx, pool):
    with Server(memory_budget=2 << 30, slots=2, max_batch_graphs=64, large_edges=1 << 13, large_workers=2) as srv:
        # all requests arrive within ~1 ms: they overlap on the device
        res = srv.replay(pool, poisson_arrivals(len(pool), 50000.0, seed=1))
        paths = {s.path for s in res}
        assert paths == {_lib.PHEM_PATH_BATCHED, _lib.PHEM_PATH_DEVICE}
        for g, s in zip(pool, res):
            check_same(ctx, g, s)
            assert s.latency_ns > 0 and s.queue_ns >= 0
        # and again one at a time through the same server
        for g in pool[:8]:
            check_same(ctx, g, srv.solve(g))


def test_concurrent_submitters(ctx, pool):
    with Server(memory_budget=1 << 30, slots=3, max_batch_graphs=16, large_edges=1 << 12, large_workers=1) as srv:
        out = [None] * len(pool)

        def worker(k):
            for i in range(k, len(pool), 4):
                out[i] = srv.solve(pool[i])

        ts = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        for g, s in zip(pool, out):
            check_same(ctx, g, s)


def test_budget_refuses_what_never_fits():
    with Server(memory_budget=64 << 20, slots=1, max_batch_graphs=8, large_edges=1 << 10, large_workers=1) as srv:
        n = 1 << 20
        big = ServedGraph(PHEM_BATCH_CC, n, pairs=np.arange(1, 1 << 22, dtype=np.uint64))
        with pytest.raises(PhemError) as e:
            srv.solve(big)
        assert e.value.status == _lib.PHEM_ERR_NOMEM
        small = ServedGraph(PHEM_BATCH_CC, 4, pairs=np.array([1, (2 << 32) | 3], np.uint64))
        s = srv.solve(small)
        np.testing.assert_array_equal(s.labels, [0, 0, 2, 2])


def test_bad_requests_fail_alone():
    with Server(memory_budget=256 << 20, slots=1, max_batch_graphs=8, large_edges=1 << 10, large_workers=1) as srv:
        bad = ServedGraph(PHEM_BATCH_MSF, 4, edges=np.array([[0, 7, 1]], np.uint32))  # endpoint >= n
        good = ServedGraph(PHEM_BATCH_MSF, 4, edges=np.array([[0, 1, 5], [1, 2, 3], [0, 2, 1]], np.uint32))
        res = srv.replay([bad, good], np.array([0, 0], np.uint64))
        assert res[0].status == _lib.PHEM_ERR_INVALID
        assert res[1].status == 0 and res[1].total_weight == 4
        with pytest.raises(PhemError):
            srv.solve(ServedGraph(PHEM_BATCH_MSF, 0, edges=np.empty((0, 3), np.uint32)))
