"""Regenerates the golden vectors in tests/golden/ from the reference's own CPU
code, compiled from the reference tree into oracle/_ref (oracle/Makefile):

  * CC cases: CC/host_spanning_tree.cu run with ONE Parlay worker (edges are
    united in index order), in a child process so PARLAY_NUM_THREADS takes
    effect.  Stored: the parent array and forest slots it leaves, the min-id
    labels derived from that parent array (root of each vertex), and the
    sorted forest edge set.
  * MSF cases: PBBS mst() (MST/src/utils.cu:794-841), or PBBS serial Kruskal
    (MST/src/bench/serialMST.C) for graphs too small for mst().  Stored: the
    ascending MSF edge ids, their count and uint64 total weight.

Inputs come from the package's seeded generators and are stored next to the
outputs, so each .npz is self-contained.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def cc_cases():
    from phem_graph_b200 import gen
    cases = {}
    g = gen.er_graph(2000, 6000, seed=7)
    cases["cc_er_n2000"] = (g.pairs, g.n)
    g = gen.er_graph(1 << 14, 1 << 15, seed=3)
    cases["cc_er_n16384_sparse"] = (g.pairs, g.n)
    p = gen.rmat(10, 8 << 10, seed=5)
    cases["cc_rmat10"] = (p, 1 << 10)
    n = 300
    path = np.array([(i << 32) | (i + 1) for i in range(n - 1)], np.uint64)
    cases["cc_path300_reversed"] = (path[::-1].copy(), n)
    star = np.array([(0 << 32) | i for i in range(1, 200)], np.uint64)
    cases["cc_star200_dups"] = (np.concatenate([star, star[::7]]), 200)
    cases["cc_isolated_only"] = (np.zeros(0, np.uint64), 50)
    # two ER blocks plus isolated vertices
    a = gen.er(500, 1500, 11)
    b = gen.er(500, 1500, 12) + np.uint64((600 << 32) | 600)
    cases["cc_two_blocks"] = (np.concatenate([a, b]), 1200)
    return cases


def msf_cases():
    from phem_graph_b200 import gen
    cases = {}
    g = gen.rmat_graph(10, 16, seed=9)
    cases["msf_rmat10"] = (g.msf_edges(), g.n, "pbbs")
    g = gen.rmat_graph(12, 8, seed=4, bits=3)
    cases["msf_rmat12_ties"] = (g.msf_edges(), g.n, "pbbs")
    p = gen.er(800, 6000, 21)
    cases["msf_er800_w2"] = (gen.msf_edges(p, gen.weights(len(p), 5, bits=1)), 800, "pbbs")
    a = gen.er(400, 3000, 31)
    b = gen.er(400, 3000, 32) + np.uint64((500 << 32) | 500)
    p = np.concatenate([a, b])
    cases["msf_two_blocks"] = (gen.msf_edges(p, gen.weights(len(p), 6, bits=10)), 1000, "pbbs")
    E = np.array([[0, 1, 4], [1, 2, 4], [0, 2, 4], [2, 3, 1], [3, 4, 7], [1, 4, 2], [0, 4, 2]], np.uint32)
    cases["msf_tiny_ties"] = (E, 5, "serial")
    E = np.array([[0, 1, 9], [2, 3, 9], [1, 0, 3], [3, 2, 1], [4, 5, 2]], np.uint32)
    cases["msf_tiny_forest"] = (E, 6, "serial")
    return cases


def _cc_child(name: str) -> None:
    """Runs in a child with PARLAY_NUM_THREADS=1: reference CC on one case."""
    import oracle
    edges, n = cc_cases()[name]
    ref = oracle.RefCC(n)
    assert ref.workers() == 1, ref.workers()
    ref.set_edges(edges)
    ref.run()
    parent, sptree = ref.state()
    np.savez(HERE / f"_tmp_{name}.npz", parent=parent, sptree=sptree)


def rmat22_rounds() -> None:
    """Per-round live counts of the MSF benchmark workload (R-MAT scale 22, edge
    factor 16, seed 22) from the CPU Boruvka restatement, with the MSF size and
    total pinned by the reference's PBBS mst().  bench.py reads this file for
    the algorithmic byte model of a solve."""
    import oracle
    from phem_graph_b200 import gen
    g = gen.rmat_graph(22, 16, seed=22)
    E = g.msf_edges()
    flags, cnt, tot, m_r, n_r = oracle.msf_boruvka(E, g.n)
    ids = oracle.ref_pbbs_mst(E)
    assert len(ids) == cnt and int(E[ids, 2].astype(np.uint64).sum()) == tot
    out = {"workload": "msf_rmat22_ef16", "n": g.n, "m": g.m, "seed": 22, "weight_seed": 1022,
           "m_r": [int(x) for x in m_r], "n_r": [int(x) for x in n_r], "msf_edges": cnt, "total_weight": tot,
           "source": "oracle/phem_oracle.c oracle_msf_boruvka; count and total equal PBBS mst()"}
    (HERE / "rmat22_boruvka_rounds.json").write_text(json.dumps(out, indent=1) + "\n")
    print(json.dumps(out))


def main() -> None:
    if len(sys.argv) == 3 and sys.argv[1] == "--cc-child":
        _cc_child(sys.argv[2])
        return
    if len(sys.argv) == 2 and sys.argv[1] == "--rmat22":
        rmat22_rounds()
        return
    import oracle
    if not oracle.ref_available():
        oracle.build()
    env = dict(os.environ, PARLAY_NUM_THREADS="1")
    manifest = {}
    for name, (edges, n) in cc_cases().items():
        subprocess.run([sys.executable, __file__, "--cc-child", name], check=True, env=env)
        tmp = HERE / f"_tmp_{name}.npz"
        with np.load(tmp) as z:
            parent, sptree = z["parent"], z["sptree"]
        tmp.unlink()
        # labels = root of each vertex in the reference's parent array
        labels = np.empty(n, np.int32)
        for i in range(n):
            r = i
            while parent[r] != r:
                r = parent[r]
            labels[i] = r
        forest = np.sort(sptree[sptree != np.uint64(0x7FFFFFFF)])
        np.savez_compressed(HERE / f"{name}.npz", edges=edges, n=np.int64(n), ref_parent=parent,
                            ref_sptree=sptree, labels=labels, forest=forest)
        manifest[name] = {"n": n, "m": int(len(edges)), "components": int(len(np.unique(labels))),
                          "forest_edges": int(len(forest)), "source": "CC/host_spanning_tree.cu, 1 worker"}
    for name, (E, n, how) in msf_cases().items():
        ids = oracle.ref_pbbs_mst(E) if how == "pbbs" else oracle.ref_serial_mst(E)
        ids = np.sort(ids).astype(np.uint32)
        total = int(E[ids, 2].astype(np.uint64).sum())
        np.savez_compressed(HERE / f"{name}.npz", edges=E, n=np.int64(n), msf_ids=ids, count=np.int64(len(ids)),
                            total=np.uint64(total))
        manifest[name] = {"n": n, "m": int(len(E)), "count": int(len(ids)), "total": total,
                          "source": "MST/src/utils.cu mst()" if how == "pbbs" else "MST/src/bench/serialMST.C"}
    (HERE / "manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True) + "\n")
    print(json.dumps(manifest, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
