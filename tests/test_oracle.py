"""The CPU oracle is pinned against the reference's own code: the golden
vectors in tests/golden (made by that code) always, and the compiled reference
in oracle/_ref directly when it is present."""
import os
import subprocess
import sys

import numpy as np
import pytest

import oracle
from tests.golden import load, names

CC_CASES = names("cc_")
MSF_CASES = names("msf_")


@pytest.mark.parametrize("name", CC_CASES)
def test_cc_restatement_equals_reference_golden(name):
    g = load(name)
    n = int(g["n"])
    parent, forest = oracle.cc_state(n)
    oracle.cc_unite(g["edges"], n, parent, forest)
    # same sequential order and hook rule => the very same parent array and slots
    np.testing.assert_array_equal(parent, g["ref_parent"])
    np.testing.assert_array_equal(forest, g["ref_sptree"])
    np.testing.assert_array_equal(oracle.cc_labels(parent), g["labels"])
    np.testing.assert_array_equal(oracle.forest_set(forest), g["forest"])


@pytest.mark.parametrize("name", MSF_CASES)
def test_msf_restatements_equal_reference_golden(name):
    g = load(name)
    E, n = g["edges"], int(g["n"])
    flags, cnt, tot = oracle.msf_kruskal(E, n)
    np.testing.assert_array_equal(np.nonzero(flags)[0], g["msf_ids"])
    assert cnt == int(g["count"]) and tot == int(g["total"])
    bflags, bcnt, btot, m_r, n_r = oracle.msf_boruvka(E, n)
    np.testing.assert_array_equal(bflags, flags)
    assert (bcnt, btot) == (cnt, tot)
    # each round at least halves the components with live edges
    assert all(int(n_r[i + 1]) * 2 <= int(n_r[i]) for i in range(len(n_r) - 1))
    assert all(int(m_r[i + 1]) <= int(m_r[i]) for i in range(len(m_r) - 1))


def test_golden_manifest_covers_edge_cases():
    man = load  # noqa: F841  (manifest is json; the cases below must exist)
    for needed in ("cc_isolated_only", "cc_path300_reversed", "cc_star200_dups", "msf_tiny_ties",
                   "msf_rmat12_ties", "msf_two_blocks"):
        assert needed in CC_CASES + MSF_CASES


def test_kruskal_small_handmade():
    # triangle with a tie: (w, id) order keeps ids 1 and 2
    E = np.array([[0, 1, 5], [1, 2, 3], [0, 2, 3], [2, 3, 1], [3, 3, 0]], np.uint32)
    flags, cnt, tot = oracle.msf_kruskal(E, 4)
    assert list(np.nonzero(flags)[0]) == [1, 2, 3] and (cnt, tot) == (3, 7)


def test_boruvka_round_counts_define_bytes():
    from phem_graph_b200 import gen
    g = gen.rmat_graph(12, 16, seed=3)
    _, cnt, _, m_r, n_r = oracle.msf_boruvka(g.msf_edges(), g.n)
    b = oracle.msf_bytes(m_r, n_r, g.n, g.n - cnt)
    expect = sum(32 * int(m_r[r]) + 16 * (int(m_r[r + 1]) if r + 1 < len(m_r) else 0) for r in range(len(m_r)))
    expect += 16 * int(sum(int(x) for x in n_r)) + 12 * cnt
    assert b == expect


def test_csr_restatement_recovers_generator_order():
    from phem_graph_b200 import gen
    pairs = gen.rmat(11, 8 << 11, seed=2)
    off, cols = gen.csr_from_pairs(pairs, 1 << 11)
    np.testing.assert_array_equal(oracle.csr_to_coo(off, cols, 1 << 11), pairs)


# ---------------------------------------------------------------- live reference (oracle/_ref)

need_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@need_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_cc_labels_equal_parallel_reference(seed):
    """With all Parlay workers the reference's forest depends on the race, but
    its labels (roots) are fixed: they must equal the restatement's."""
    from phem_graph_b200 import gen
    g = gen.er_graph(1 << 15, 3 << 15, seed=seed)
    ref = oracle.RefCC(g.n)
    ref.set_edges(g.pairs)
    ref.run()
    parent, sptree = ref.state()
    labels, _ = oracle.cc_solve(g.pairs, g.n)
    np.testing.assert_array_equal(oracle.cc_labels(parent), labels)
    assert len(oracle.forest_set(sptree)) == g.n - len(np.unique(labels))


@need_ref
def test_cc_single_worker_reference_is_index_order():
    """PARLAY_NUM_THREADS=1: the reference unites in index order, so parent
    array and forest slots equal the sequential restatement bit for bit."""
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r)\n"
        "import oracle\nfrom phem_graph_b200 import gen\n"
        "g = gen.rmat(12, 8 << 12, seed=8)\n"
        "r = oracle.RefCC(1 << 12); assert r.workers() == 1; r.set_edges(g); r.run()\n"
        "p, s = r.state(); p2, s2 = oracle.cc_state(1 << 12); oracle.cc_unite(g, 1 << 12, p2, s2)\n"
        "assert np.array_equal(p, p2) and np.array_equal(s, s2)\n"
    ) % str(oracle.HERE.parent)
    env = dict(os.environ, PARLAY_NUM_THREADS="1")
    subprocess.run([sys.executable, "-c", code], check=True, env=env)


@need_ref
@pytest.mark.parametrize("scale,ef,bits,seed", [(10, 16, 20, 1), (13, 8, 20, 2), (12, 16, 2, 3), (11, 4, 6, 4)])
def test_msf_restatement_equals_pbbs(scale, ef, bits, seed):
    from phem_graph_b200 import gen
    g = gen.rmat_graph(scale, ef, seed=seed, bits=bits)
    E = g.msf_edges()
    flags, cnt, tot = oracle.msf_kruskal(E, g.n)
    ids = oracle.ref_pbbs_mst(E)
    np.testing.assert_array_equal(np.sort(ids), np.nonzero(flags)[0])


@need_ref
@pytest.mark.parametrize("seed", range(6))
def test_msf_restatement_equals_serial_kruskal_tiny(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 9))
    m = int(rng.integers(0, 20))
    E = np.stack([rng.integers(0, n, m), rng.integers(0, n, m), rng.integers(1, 4, m)], 1).astype(np.uint32)
    flags, _, _ = oracle.msf_kruskal(E, n)
    np.testing.assert_array_equal(oracle.ref_serial_mst(E), np.nonzero(flags)[0])


@pytest.mark.parametrize("scale,ef,bits,chunk", [(10, 16, 20, 1000), (11, 8, 2, 777), (9, 4, 1, 1), (12, 16, 20, 1 << 20)])
def test_chunked_msf_restatement_equals_whole_graph(scale, ef, bits, chunk):
    """streamline_boruvka's merge (MSF of each chunk plus the forest so far)
    gives the whole graph's MSF: same edge set under (w, id), same weight --
    heavy ties (1- and 2-bit weights), one-edge chunks and a single chunk."""
    from phem_graph_b200 import gen
    g = gen.rmat_graph(scale, ef, seed=scale + chunk, bits=bits)
    E = g.msf_edges()
    want, cnt, tot = oracle.msf_kruskal(E, g.n)
    got, c2, t2 = oracle.msf_chunked(E, g.n, chunk)
    np.testing.assert_array_equal(got, want)
    assert (c2, t2) == (cnt, tot)


@need_ref
def test_chunked_msf_restatement_equals_pbbs_with_self_loops():
    rng = np.random.default_rng(11)
    n, m = 300, 5000
    E = np.stack([rng.integers(0, n, m), rng.integers(0, n, m), rng.integers(1, 5, m)], 1).astype(np.uint32)
    E[::50, 1] = E[::50, 0]  # self-loops
    got, _, _ = oracle.msf_chunked(E, n, 613)
    np.testing.assert_array_equal(np.sort(oracle.ref_pbbs_mst(E)), np.nonzero(got)[0])
