"""The sharded solves' GPU forms (phem_graph_b200.dist) on one GPU.

Only one GPU is available to these tests, so two shards are solved on it in
turn and the all-gather is replaced by a local stand-in that returns both
shards' device forests in rank order; everything else -- the device-side
padding of the local forest, the concatenation, the merge solve on
(n - 1) * world records, the pairwise phem_cc_merge -- is the code a multi-GPU
run executes.  Results are compared with the oracle on the whole graph."""
import numpy as np
import pytest

import oracle
from phem_graph_b200 import dist as pdist, gen

pytestmark = pytest.mark.gpu
WORLD = 2


def _msf_shards(bits):
    gs = [gen.rmat_graph(14, 8, seed=40 + r, bits=bits) for r in range(WORLD)]
    return [g.msf_edges() for g in gs], gs[0].n


@pytest.mark.parametrize("bits", [20, 2])
def test_sharded_msf_device_equals_whole_graph(ctx, bits):
    import torch
    Es, n = _msf_shards(bits)
    d = [torch.from_numpy(E.view(np.int32)).cuda() for E in Es]
    local = [pdist.local_msf_forest_device(ctx, d[r], len(Es[r]), n).clone() for r in range(WORLD)]
    E = np.concatenate(Es)
    flags, cnt, tot = oracle.msf_kruskal(E, n)
    want = E[np.nonzero(flags)[0]]
    for rank in range(WORLD):
        def gather(t, rank=rank):
            assert t.shape == local[rank].shape
            return [t if r == rank else local[r] for r in range(WORLD)]
        res = pdist.sharded_msf_device(ctx, d[rank], len(Es[rank]), n, gather=gather)
        assert (res.count, res.total) == (cnt, tot)
        np.testing.assert_array_equal(res.edges.cpu().numpy().view(np.uint32), want)


def test_sharded_msf_device_sparse_shards(ctx):
    """Shards far smaller than n - 1: most of each gathered block is padding."""
    import torch
    gs = [gen.er_graph(20_000, 3_000, 70 + r) for r in range(WORLD)]
    n = 20_000
    Es = [gen.msf_edges(g.pairs, gen.weights(g.m, 80 + r, 12)) for r, g in enumerate(gs)]
    d = [torch.from_numpy(E.view(np.int32)).cuda() for E in Es]
    local = [pdist.local_msf_forest_device(ctx, d[r], len(Es[r]), n).clone() for r in range(WORLD)]
    E = np.concatenate(Es)
    flags, cnt, tot = oracle.msf_kruskal(E, n)
    res = pdist.sharded_msf_device(ctx, d[0], len(Es[0]), n, gather=lambda t: [t, local[1]])
    assert (res.count, res.total) == (cnt, tot)
    np.testing.assert_array_equal(res.edges.cpu().numpy().view(np.uint32), E[np.nonzero(flags)[0]])


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_cc_device_equals_whole_graph(ctx, world):
    import torch
    gs = [gen.rmat_graph(15, 4, seed=60 + r) for r in range(world)]
    n = gs[0].n
    d = [torch.from_numpy(g.pairs.view(np.int64)).cuda() for g in gs]
    local = [pdist.local_cc_forest_device(ctx, d[r], n).clone() for r in range(world)]
    P = np.concatenate([g.pairs for g in gs])
    ref, _ = oracle.cc_solve(P, n)
    comps = len(np.unique(ref))
    for rank in range(world):
        def gather(t, rank=rank):
            return [t if r == rank else local[r] for r in range(world)]
        labels, slots = pdist.sharded_cc_device(ctx, d[rank], n, gather=gather)
        np.testing.assert_array_equal(labels.cpu().numpy(), ref)
        f = oracle.forest_set(slots.cpu().numpy().view(np.uint64))
        assert len(f) == n - comps
        assert np.all(np.isin(f, P))
        np.testing.assert_array_equal(oracle.cc_solve(f, n)[0], ref)
