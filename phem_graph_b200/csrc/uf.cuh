// uf.cuh -- the union-find steps shared by phem_cc_solve (cc.cu) and the
// no-allocation entry point (noalloc.cu): root walks with path halving, the
// lockstep walk of an edge's two endpoints, and the union with the
// reference's hook rule (larger root under the smaller, forest[hooked root] =
// edge; CC/ExternalSpanningTree.cu:27-116, CC/GPUSpanningTree.cu:24-140).
#pragma once

#include "internal.h"

namespace phem {

// parent[i] through L1 (ld.global.ca).  Another SM's hook may not be seen
// yet, but every value read is still an ancestor of i (a vertex's ancestors
// only grow), so a walk on such values ends at an ancestor that may have
// stopped being a root; the CAS that would hook it then fails, and the
// retry reads through L2.  The gain: the few roots that most walks end at
// (a giant component's) are served by each SM's L1 instead of one L2 slice.
__device__ __forceinline__ int32_t ld_ca(const int32_t *p)
{
    int32_t v;
    asm volatile("ld.global.ca.s32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}

// Root of x with path halving.  Writes only touch non-roots (a vertex that is
// not a root never becomes one again), so they cannot race with the CAS that
// hooks a root; each write points a vertex at one of its ancestors, as a
// fire-and-forget atomic min.  A path
// has fewer than n + 1 vertices, so n + 1 steps bound the walk.  CACHED walks
// read through L1 (see ld_ca); the others read L2-coherently.
// Vertex 0 is always a root (nothing is smaller to hook it under), so a walk
// that reaches it stops without reading the word every walk would read.
template <bool CACHED>
__device__ __forceinline__ int32_t uf_find(int32_t *parent, int32_t x, int32_t n, uint32_t *err)
{
    const uint32_t cap = (uint32_t)n + 1;
    for (uint32_t steps = 0; steps < cap; steps++) {
        const int32_t p = CACHED ? ld_ca(parent + x) : __ldcg(parent + x);
        if (p == x || p == 0)
            return p;
        const int32_t gp = CACHED ? ld_ca(parent + p) : __ldcg(parent + p);
        if (gp == p)
            return p;
        // ids fall towards the root (hooks point at smaller ids), so a min
        // never moves x's pointer back below a shortcut another walk made
        // after this one read a (possibly stale) parent
        atomicMin(parent + x, gp);
        x = gp;
    }
    set_err(err, kErrChase);
    return x;
}

// The roots of a and b, walked in lockstep (both walks' loads are in flight
// together) with the same halving as uf_find.  Returns true as soon as the
// walks meet (one component; *ra, *rb are then not set), else false with
// the two roots.
template <bool CACHED>
__device__ __forceinline__ bool uf_find2(int32_t *parent, int32_t a, int32_t b, int32_t n, uint32_t *err,
                                         int32_t *ra, int32_t *rb)
{
    const uint32_t cap = (uint32_t)n + 1;
    bool da = false, db = false;  // walk finished at a root
    for (uint32_t steps = 0; steps < cap; steps++) {
        if (a == b)
            return true;
        if (da && db) {
            *ra = a;
            *rb = b;
            return false;
        }
        const int32_t pa = da ? a : (CACHED ? ld_ca(parent + a) : __ldcg(parent + a));
        const int32_t pb = db ? b : (CACHED ? ld_ca(parent + b) : __ldcg(parent + b));
        const bool ra_now = !da && (pa == a || pa == 0), rb_now = !db && (pb == b || pb == 0);
        const bool step_a = !da && !ra_now, step_b = !db && !rb_now;
        const int32_t ga = step_a ? (CACHED ? ld_ca(parent + pa) : __ldcg(parent + pa)) : pa;
        const int32_t gb = step_b ? (CACHED ? ld_ca(parent + pb) : __ldcg(parent + pb)) : pb;
        if (ra_now) {
            a = pa;
            da = true;
        } else if (step_a) {
            if (ga == pa) {
                da = true;
            } else {
                atomicMin(parent + a, ga);
            }
            a = ga;
        }
        if (rb_now) {
            b = pb;
            db = true;
        } else if (step_b) {
            if (gb == pb) {
                db = true;
            } else {
                atomicMin(parent + b, gb);
            }
            b = gb;
        }
    }
    set_err(err, kErrChase);
    *ra = a;
    *rb = b;
    return a == b;
}

// One union with the reference's hook rule (larger root under smaller root,
// forest[hooked root] = edge).  Returns true when it hooked.
__device__ __forceinline__ bool uf_unite(int32_t *parent, unsigned long long *forest, unsigned long long e,
                                         int32_t u, int32_t v, int32_t n, uint32_t *err)
{
    {
        // two independent loads settle most edges once parents point at roots
        // (after a compress): equal parents mean one component
        const int32_t pu = ld_ca(parent + u), pv = ld_ca(parent + v);
        if (pu == pv)
            return false;
        u = pu;  // ancestors of the endpoints
        v = pv;
    }
    for (uint32_t retry = 0; retry < kUnionRetryCap; retry++) {
        // first attempt through L1; after a failed CAS, coherent walks
        int32_t ru, rv;
        if (retry == 0 ? uf_find2<true>(parent, u, v, n, err, &ru, &rv) : uf_find2<false>(parent, u, v, n, err, &ru, &rv))
            return false;
        if (ru == rv)
            return false;
        if ((retry & 63) == 63 && (*(volatile uint32_t *)err & (kErrChase | kErrRetry)))
            return false;  // another thread already reported a broken state
        const int32_t hi = ru > rv ? ru : rv, lo = ru > rv ? rv : ru;
        const int32_t old = atomicCAS(parent + hi, hi, lo);
        if (old == hi) {
            if (forest)
                forest[hi] = e;
            return true;
        }
        // hi was hooked under `old` meanwhile: walk on from there (both are
        // ancestors of the original endpoints)
        u = old;
        v = lo;
    }
    set_err(err, kErrRetry);
    return false;
}

__device__ __forceinline__ void unite_packed(int32_t *parent, unsigned long long *forest, unsigned long long e,
                                             int32_t n, uint32_t *err)
{
    const int32_t u = (int32_t)(e >> 32), v = (int32_t)(uint32_t)e;
    if (!(u < v))
        return;  // union_find_gpu_COO only unites u < v (CC/ExternalSpanningTree.cu:82)
    if (u < 0 || v >= n) {
        set_err(err, kErrRange);
        return;
    }
    uf_unite(parent, forest, e, u, v, n, err);
}

}  // namespace phem
