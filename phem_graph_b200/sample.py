"""One small call of every kernel family, on device-resident synthetic inputs:
a fixed target for profilers (each launch list names the same kernels).

    python -m phem_graph_b200.sample

Inputs (seeded): R-MAT scale 20, edge factor 16, for the MSF solve and the CSR
conversion; Erdos-Renyi n = 2^20 with 8 * 2^20 draws for connected components
(default, canonical-forest and no-allocation entry points); 256 mixed small
graphs for the batched kernel.  Every input array is larger than L2 except the
batch.  Prints one line per call; the results are not checked here (the GPU
tests do that).
"""
from __future__ import annotations

import ctypes as C

import numpy as np


def main() -> None:
    import torch

    from . import Context, _lib, gen

    dev = torch.device("cuda", 0)
    with Context(0) as ctx:
        g = gen.rmat_graph(20, 16, seed=1)
        E = g.msf_edges()
        d_e = torch.from_numpy(E.view(np.int32)).to(dev)
        d_msf = torch.empty((g.n, 3), dtype=torch.int32, device=dev)
        d_ct = torch.zeros(2, dtype=torch.int64, device=dev)
        r = ctx.msf_solve_device(d_e, g.m, g.n, d_msf, d_ct)
        print("msf", g.m, "edges ->", r.count, "forest edges, total", r.total)

        er = gen.er_graph(1 << 20, 8 << 20, 1)
        d_p = torch.from_numpy(er.pairs.view(np.int64)).to(dev)
        d_lab = torch.empty(er.n, dtype=torch.int32, device=dev)
        d_for = torch.empty(er.n, dtype=torch.int64, device=dev)
        c = ctx.cc_solve(d_p, er.n, labels=d_lab, forest=d_for)
        print("cc", er.m, "edges ->", c.components, "components")
        c = ctx.cc_solve(d_p, er.n, canonical=True, labels=d_lab, forest=d_for)
        print("cc canonical", c.components, "components")

        off, cols = gen.csr_from_pairs(g.pairs, g.n)
        d_off = torch.from_numpy(off).to(dev)
        d_cols = torch.from_numpy(cols.view(np.int32)).to(dev)
        d_coo = torch.empty(len(cols), dtype=torch.int64, device=dev)
        k = C.c_int64()
        _lib.check(_lib.lib().phem_csr_to_coo(ctx.handle, d_off.data_ptr(), d_cols.data_ptr(), g.n,
                                              d_coo.data_ptr(), C.byref(k)), "phem_csr_to_coo")
        print("csr_to_coo", len(cols), "entries ->", k.value, "pairs")

        st = _lib.lib().phem_cc_solve_noalloc(C.c_void_p(d_p.data_ptr()), er.m, er.n,
                                               C.c_void_p(d_lab.data_ptr()), C.c_void_p(d_for.data_ptr()), None)
        _lib.check(st, "phem_cc_solve_noalloc")
        print("cc no-alloc ok")

        b = gen.mixed_batch(256, 4)
        with ctx.batch_plan(b.num_graphs, b.total_edges, b.total_vertices) as plan:
            plan.upload(b)  # device-resident edges: one launch, no overlapped copies
            plan.run()
            r = plan.download(labels=False)
        print("batch", b.num_graphs, "graphs ->", int(r.count.sum()), "forest edges")
        torch.cuda.synchronize()


if __name__ == "__main__":
    main()
