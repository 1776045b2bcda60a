"""The reference drivers on libphem through the compat layer: the reference's
own CC driver (CC/main.cu, graph.cu, host_spanning_tree.cu, compiled from the
reference tree) linked with phem_graph_b200/compat/hast_compat.cpp in place of
its GPU files, and a driver on the reference's MST types using
compat/mst_compat.cuh.  Their printed results equal the oracle's."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle
from phem_graph_b200 import gen, io

pytestmark = pytest.mark.gpu
REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def _run(args):
    r = subprocess.run([str(a) for a in args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


@pytest.mark.skipif(not (REF / "hast_phem").exists(), reason="compat drivers not built (reference tree absent)")
@pytest.mark.parametrize("fmt,batch", [("txt", 1 << 20), ("txt", 4097), ("egr", 100003)])
def test_reference_cc_driver_on_libphem(tmp_path, fmt, batch):
    g = gen.rmat_graph(14, 8, seed=12)
    labels, _ = oracle.cc_solve(g.pairs, g.n)
    want = len(np.unique(labels))
    if fmt == "txt":
        path = tmp_path / "g.txt"
        io.write_edge_list(path, g.pairs, g.n)
    else:
        path = tmp_path / "g.egr"
        off, cols = gen.csr_from_pairs(g.pairs, g.n)
        io.write_ecl(path, off, cols)
    out = _run([REF / "hast_phem", path, 1, batch])
    m = re.search(r"CC = (\d+)", out)
    assert m, out[-1000:]
    assert int(m.group(1)) == want


@pytest.mark.skipif(not (REF / "mst_phem").exists(), reason="compat drivers not built (reference tree absent)")
def test_reference_mst_entry_points_on_libphem(tmp_path):
    g = gen.rmat_graph(13, 16, seed=4)
    E = g.msf_edges()
    flags, cnt, tot = oracle.msf_kruskal(E, g.n)
    p = tmp_path / "e.bin"
    p.write_bytes(np.ascontiguousarray(E, np.uint32).tobytes())
    out = _run([REF / "mst_phem", p, g.n])
    host = re.search(r"^host (\d+) (\d+)$", out, re.M)
    dev = re.search(r"^device (\d+) (\d+) (\d+)$", out, re.M)
    assert host and dev, out
    assert (int(host.group(1)), int(host.group(2))) == (cnt, tot)
    assert (int(dev.group(1)), int(dev.group(2))) == (cnt, tot)
    assert int(dev.group(3)) == g.n - cnt


@pytest.mark.skipif(not (REF / "mst_stream_phem").exists(), reason="compat drivers not built (reference tree absent)")
@pytest.mark.parametrize("chunks", [1, 3, 7])
def test_reference_streamline_mode_on_libphem(tmp_path, chunks):
    """streamline_boruvka through the compat layer, fed by the reference's own
    MatrixMarket chunk reader: the forest file holds the oracle's MSF (ascending
    by edge id, 1-based endpoints) and the printed total weight is its total,
    on both timed iterations."""
    g = gen.rmat_graph(12, 8, seed=21, bits=6)
    E = g.msf_edges()
    flags, cnt, tot = oracle.msf_kruskal(E, g.n)
    path, res = tmp_path / "g.mtx", tmp_path / "forest.txt"
    io.write_mtx(path, E, g.n)
    out = subprocess.run([str(REF / "mst_stream_phem"), str(path), str(chunks), str(res)], capture_output=True,
                         text=True, timeout=300, cwd=tmp_path)  # the reader writes a temporary copy in its cwd
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    totals = [int(x) for x in re.findall(r"final weight by streamline approach (\d+)", out.stdout)]
    assert totals == [tot, tot]
    got = np.loadtxt(res, dtype=np.int64, ndmin=2)
    want = E[flags].astype(np.int64)
    want[:, :2] += 1
    np.testing.assert_array_equal(got, want)
