"""Graph-file readers (csrc/io.cpp) against the reference's own MatrixMarket
reader (compiled from MST/src/utils.cu into oracle/_ref) and against the
restated ECL / edge-list conversions of the CC driver (CC/graph.cu)."""
import numpy as np
import pytest

import oracle
from phem_graph_b200 import gen, io


def _ref_mtx(path, generate_weights):
    return oracle.ref_mtx_read(path, bool(generate_weights))


def _mtx_graph():
    g = gen.rmat_graph(10, 8, seed=3)
    e = g.msf_edges().copy()
    flip = np.arange(len(e)) % 3 == 0  # some lines with u > v
    e[flip, 0], e[flip, 1] = e[flip, 1].copy(), e[flip, 0].copy()
    return e, g.n


@pytest.mark.parametrize("weights", [True, False])
def test_mtx_matches_reference_reader(tmp_path, weights):
    e, n = _mtx_graph()
    p = tmp_path / "g.mtx"
    io.write_mtx(p, e, n, weights=weights)
    got, gn = io.read_mtx(p, generate_weights=not weights)
    assert gn == n and len(got) == len(e)
    lo, hi = np.minimum(e[:, 0], e[:, 1]), np.maximum(e[:, 0], e[:, 1])
    np.testing.assert_array_equal(got[:, 0], lo)
    np.testing.assert_array_equal(got[:, 1], hi)
    if weights:
        np.testing.assert_array_equal(got[:, 2], e[:, 2])
    else:
        u1, v1 = e[:, 0].astype(np.uint64) + 1, e[:, 1].astype(np.uint64) + 1
        w = (((u1 - 1) * (v1 - 1)) & 0xFFFFFFFF) % np.uint64(n) + 1
        np.testing.assert_array_equal(got[:, 2], w.astype(np.uint32))
    if oracle.ref_available():
        ref, rn = _ref_mtx(p, int(not weights))
        assert rn == gn
        np.testing.assert_array_equal(got, ref)


def test_mtx_comments_blank_and_short_files(tmp_path):
    p = tmp_path / "c.mtx"
    p.write_text("%%MatrixMarket matrix coordinate integer general\n% a comment\n5 5 4\n1 2 7\n\n3 1 2\n")
    got, n = io.read_mtx(p)
    assert n == 5
    np.testing.assert_array_equal(got, [[0, 1, 7], [0, 0, 0], [0, 2, 2], [0, 0, 0]])
    if oracle.ref_available():
        ref, _ = _ref_mtx(p, 0)
        np.testing.assert_array_equal(got, ref)


def test_ecl_and_edge_list_pairs(tmp_path):
    g = gen.rmat_graph(9, 8, seed=5)
    off, cols = gen.csr_from_pairs(g.pairs, g.n)
    pe = tmp_path / "g.egr"
    io.write_ecl(pe, off, cols)
    o2, c2, n2 = io.read_ecl(pe)
    np.testing.assert_array_equal(o2, off)
    np.testing.assert_array_equal(c2, cols)
    assert n2 == g.n
    pairs, n = io.read_graph_pairs(pe)
    np.testing.assert_array_equal(pairs, oracle.csr_to_coo(off, cols, g.n))
    # any unknown extension is read as ECL binary, as the reference does
    pb = tmp_path / "g.whatever"
    io.write_ecl(pb, off, cols)
    np.testing.assert_array_equal(io.read_graph_pairs(pb)[0], pairs)
    pt = tmp_path / "g.txt"
    io.write_edge_list(pt, g.pairs, g.n)
    tp, tn = io.read_graph_pairs(pt)
    assert tn == g.n
    np.testing.assert_array_equal(tp, g.pairs)


def test_bad_files_raise(tmp_path):
    with pytest.raises(io.GraphFileError):
        io.read_mtx(tmp_path / "missing.mtx")
    p = tmp_path / "trunc.egr"
    p.write_bytes(np.array([100, 1000], np.int64).tobytes())
    with pytest.raises(io.GraphFileError):
        io.read_ecl(p)
