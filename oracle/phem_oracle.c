/*
 * phem_oracle.c -- CPU restatement of PHEM's two graph hot paths.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py load it.  No product code
 * links, imports or calls it, and the CUDA library never falls back to it.
 *
 * What it restates (paths relative to the PHEM reference tree):
 *   - CC/SF union-find: find_compress + unite_impl of CC/host_spanning_tree.cu:10-42,
 *     run sequentially in edge-index order (what SimpleUnionAsync at :67-86 does
 *     with one Parlay worker), plus the label step label[i] = find(i) that
 *     CC/GPUSpanningTree.cu:122-128 performs (min vertex id of the component,
 *     because hooks always go from the larger root to the smaller).
 *   - MSF by Kruskal under the strict (weight, edge id) order used by the PBBS
 *     mst() of MST/src/utils.cu:801-802 and by MST/src/bench/serialMST.C:62-101.
 *     Under that order the minimum spanning forest is unique.
 *   - Boruvka rounds as MST/src/kernels.cu:507-689 runs them (min (w,id) edge per
 *     component, mutual pair keeps the lower id as root, contract, drop edges that
 *     became internal), used to count the live edges m_r and live components n_r
 *     entering each round; those counts define the algorithmic byte model.
 *   - CSR -> packed COO in CSR row order keeping i < col (CC/graph.cu:149-196).
 *
 * Parity of this restatement is pinned against the reference's own CPU code
 * compiled from source (oracle/Makefile -> oracle/_ref) and against golden
 * vectors that code produced (tests/golden/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Empty forest slot: INT_MAX stored in a uint64 (CC/main.cu:434,
 * CC/GPUSpanningTree.cu:139). */
#define ORC_FOREST_EMPTY 0x7fffffffULL
#define ORC_KEY_NONE UINT64_MAX

/* MST/src/constants.h:15-19 `edge`: three uint32, 12 bytes. */
typedef struct {
    uint32_t u, v, w;
} orc_edge;

/* ------------------------------------------------------------------------- */
/* CC: union-find with max->min hooking                                       */
/* ------------------------------------------------------------------------- */

/* Root of x; afterwards every node on the path whose parent is still above the
 * root points straight at it.  Same walk and same write rule as find_compress
 * (CC/host_spanning_tree.cu:10-22): ids strictly decrease towards the root. */
static int32_t cc_root(int32_t *parent, int32_t x)
{
    int32_t r = x;
    while (parent[r] != r)
        r = parent[r];
    while (parent[x] > r) {
        int32_t up = parent[x];
        parent[x] = r;
        x = up;
    }
    return r;
}

void oracle_cc_init(int32_t n, int32_t *parent, uint64_t *forest)
{
    for (int32_t i = 0; i < n; i++) {
        parent[i] = i;
        if (forest)
            forest[i] = ORC_FOREST_EMPTY;
    }
}

/* Processes edges[0..m) in index order, as unite_impl does for each edge
 * (CC/host_spanning_tree.cu:25-42): the larger of the two roots is hooked under
 * the smaller and the forest slot of the hooked root records the packed
 * original edge (u << 32 | v).  State in parent/forest carries over between
 * calls, so batches can be fed one after another.  Every edge is processed
 * whatever the order of its endpoints (the CPU reference does not skip u > v).
 * Returns the number of hooks, or -1 when an endpoint is outside [0, n). */
int64_t oracle_cc_unite(const uint64_t *edges, int64_t m, int32_t n,
                        int32_t *parent, uint64_t *forest)
{
    int64_t hooks = 0;
    for (int64_t i = 0; i < m; i++) {
        int32_t u = (int32_t)(edges[i] >> 32);
        int32_t v = (int32_t)(edges[i] & 0xffffffffu);
        if (u < 0 || v < 0 || u >= n || v >= n)
            return -1;
        int32_t a = cc_root(parent, u);
        int32_t b = cc_root(parent, v);
        if (a == b)
            continue;
        int32_t hi = a > b ? a : b, lo = a > b ? b : a;
        parent[hi] = lo;
        if (forest)
            forest[hi] = edges[i];
        hooks++;
    }
    return hooks;
}

/* label[i] = root of i = smallest vertex id of its component. */
void oracle_cc_labels(int32_t n, int32_t *parent, int32_t *label)
{
    for (int32_t i = 0; i < n; i++)
        label[i] = cc_root(parent, i);
}

/* ------------------------------------------------------------------------- */
/* Sorting helper: LSD radix sort of 64-bit keys, 16-bit digits.              */
/* ------------------------------------------------------------------------- */

static int radix_sort_u64(uint64_t *keys, uint64_t count)
{
    if (count < 2)
        return 0;
    uint64_t *tmp = (uint64_t *)malloc(count * sizeof(uint64_t));
    uint64_t *hist = (uint64_t *)malloc(65536 * sizeof(uint64_t));
    if (!tmp || !hist) {
        free(tmp);
        free(hist);
        return -1;
    }
    uint64_t *src = keys, *dst = tmp;
    for (int shift = 0; shift < 64; shift += 16) {
        memset(hist, 0, 65536 * sizeof(uint64_t));
        for (uint64_t i = 0; i < count; i++)
            hist[(src[i] >> shift) & 0xffff]++;
        /* a digit shared by every key leaves the order unchanged */
        if (hist[(src[0] >> shift) & 0xffff] == count)
            continue;
        uint64_t sum = 0;
        for (int d = 0; d < 65536; d++) {
            uint64_t c = hist[d];
            hist[d] = sum;
            sum += c;
        }
        for (uint64_t i = 0; i < count; i++)
            dst[hist[(src[i] >> shift) & 0xffff]++] = src[i];
        uint64_t *t = src;
        src = dst;
        dst = t;
    }
    if (src != keys)
        memcpy(keys, src, count * sizeof(uint64_t));
    free(tmp);
    free(hist);
    return 0;
}

/* Plain union-find (union by size, path halving) for the MSF restatements. */
static uint32_t dsu_find(uint32_t *p, uint32_t x)
{
    while (p[x] != x) {
        p[x] = p[p[x]];
        x = p[x];
    }
    return x;
}

/* ------------------------------------------------------------------------- */
/* MSF: Kruskal under (w, id)                                                 */
/* ------------------------------------------------------------------------- */

/* in_msf[id] = 1 for every edge of the unique minimum spanning forest under the
 * order (w, id); *count and *total receive its size and uint64 weight.
 * Endpoints must be < n; requires m < 2^32 (ids are 32-bit, as edgeId in
 * MST/src/MST.h:6).  Returns 0, or -1 on bad input / allocation failure. */
int oracle_msf_kruskal(const orc_edge *E, uint64_t m, uint32_t n,
                       uint8_t *in_msf, uint64_t *count, uint64_t *total)
{
    if (m >= (1ull << 32))
        return -1;
    memset(in_msf, 0, m);
    uint64_t *keys = (uint64_t *)malloc((m ? m : 1) * sizeof(uint64_t));
    uint32_t *p = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t *sz = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    if (!keys || !p || !sz) {
        free(keys);
        free(p);
        free(sz);
        return -1;
    }
    for (uint64_t i = 0; i < m; i++) {
        if (E[i].u >= n || E[i].v >= n) {
            free(keys);
            free(p);
            free(sz);
            return -1;
        }
        keys[i] = ((uint64_t)E[i].w << 32) | i;
    }
    if (radix_sort_u64(keys, m) != 0) {
        free(keys);
        free(p);
        free(sz);
        return -1;
    }
    for (uint32_t i = 0; i < n; i++) {
        p[i] = i;
        sz[i] = 1;
    }
    uint64_t c = 0, t = 0;
    for (uint64_t k = 0; k < m; k++) {
        uint32_t id = (uint32_t)(keys[k] & 0xffffffffu);
        uint32_t a = dsu_find(p, E[id].u), b = dsu_find(p, E[id].v);
        if (a == b)
            continue;
        if (sz[a] < sz[b]) {
            uint32_t s = a;
            a = b;
            b = s;
        }
        p[b] = a;
        sz[a] += sz[b];
        in_msf[id] = 1;
        c++;
        t += E[id].w;
    }
    *count = c;
    *total = t;
    free(keys);
    free(p);
    free(sz);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* MSF: Boruvka rounds with per-round live counts                             */
/* ------------------------------------------------------------------------- */

/* Round-synchronous Boruvka as MST/src/kernels.cu:507-689 runs it:
 *   - every component with a live edge takes its minimum (w, id) edge
 *     (populate_min_weight / populate_eid, :24-70);
 *   - a mutual pair keeps the lower component id as root, every other chooser
 *     hooks onto the far component and contributes its edge (new_grafting_edges,
 *     :73-134);
 *   - hook chains are jumped to their roots (new_shortcutting_step, :254-271);
 *   - edges whose endpoints now share a component are dropped (relabelling_step,
 *     filtering_step and the two remove_if calls, :273-321, :641-649).
 * m_r[r] = live edges entering round r, n_r[r] = components with a live edge
 * entering round r; *rounds = number of rounds that chose at least one edge.
 * in_msf/count/total as in oracle_msf_kruskal (the sets are equal).
 * Returns 0, -1 on bad input, -2 when max_rounds is exceeded. */
int oracle_msf_boruvka(const orc_edge *E, uint64_t m, uint32_t n,
                       uint8_t *in_msf, uint64_t *count, uint64_t *total,
                       uint64_t *m_r, uint64_t *n_r, int32_t max_rounds,
                       int32_t *rounds)
{
    if (m >= (1ull << 32))
        return -1;
    memset(in_msf, 0, m);
    uint32_t *comp = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t *hook = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint64_t *best = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *live = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    if (!comp || !hook || !best || !live) {
        free(comp);
        free(hook);
        free(best);
        free(live);
        return -1;
    }
    uint64_t nlive = 0;
    for (uint64_t i = 0; i < m; i++) {
        if (E[i].u >= n || E[i].v >= n) {
            free(comp);
            free(hook);
            free(best);
            free(live);
            return -1;
        }
        if (E[i].u != E[i].v)
            live[nlive++] = (uint32_t)i;
    }
    for (uint32_t x = 0; x < n; x++) {
        comp[x] = x;
        best[x] = ORC_KEY_NONE;
    }
    uint64_t c = 0, t = 0;
    int32_t r = 0;
    int rc = 0;
    while (nlive > 0) {
        if (r >= max_rounds) {
            rc = -2;
            break;
        }
        m_r[r] = nlive;
        for (uint64_t k = 0; k < nlive; k++) {
            uint32_t id = live[k];
            uint64_t key = ((uint64_t)E[id].w << 32) | id;
            uint32_t a = comp[E[id].u], b = comp[E[id].v];
            if (key < best[a])
                best[a] = key;
            if (key < best[b])
                best[b] = key;
        }
        uint64_t active = 0;
        for (uint32_t x = 0; x < n; x++) {
            hook[x] = x;
            if (best[x] == ORC_KEY_NONE)
                continue;
            active++;
            uint32_t id = (uint32_t)(best[x] & 0xffffffffu);
            uint32_t a = comp[E[id].u], b = comp[E[id].v];
            uint32_t other = (a == x) ? b : a;
            int mutual = best[other] == best[x];
            if (mutual && x < other)
                continue;
            hook[x] = other;
            in_msf[id] = 1;
            c++;
            t += E[id].w;
        }
        n_r[r] = active;
        for (uint32_t x = 0; x < n; x++) {
            if (best[x] == ORC_KEY_NONE)
                continue;
            uint32_t y = x;
            while (hook[y] != y)
                y = hook[y];
            hook[x] = y; /* shortcut to the root */
        }
        for (uint32_t x = 0; x < n; x++)
            comp[x] = hook[comp[x]];
        for (uint32_t x = 0; x < n; x++)
            best[x] = ORC_KEY_NONE;
        uint64_t kept = 0;
        for (uint64_t k = 0; k < nlive; k++) {
            uint32_t id = live[k];
            if (comp[E[id].u] != comp[E[id].v])
                live[kept++] = id;
        }
        nlive = kept;
        r++;
    }
    *rounds = r;
    *count = c;
    *total = t;
    free(comp);
    free(hook);
    free(best);
    free(live);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* CSR -> packed COO                                                          */
/* ------------------------------------------------------------------------- */

/* Walks rows in order and emits (i << 32 | col) for every entry with i < col,
 * the order csr_to_coo uses (CC/graph.cu:169-187).  out may be NULL to count.
 * Returns the number of edges emitted. */
int64_t oracle_csr_to_coo(const int64_t *offsets, const uint32_t *cols, int32_t n,
                          uint64_t *out)
{
    int64_t k = 0;
    for (int32_t i = 0; i < n; i++)
        for (int64_t j = offsets[i]; j < offsets[i + 1]; j++)
            if ((int64_t)i < (int64_t)cols[j]) {
                if (out)
                    out[k] = ((uint64_t)(uint32_t)i << 32) | cols[j];
                k++;
            }
    return k;
}
