// msf.cu -- minimum spanning forest on sm_100a: Boruvka rounds behind a
// light/heavy edge filter.
//
// Arithmetic is the reference's device_boruvka (MST/src/kernels.cu:507-689):
// per round every component takes its minimum (weight, edge id) edge, a
// mutual pair keeps the lower id as root and every other chooser hooks onto
// the far component (new_grafting_edges, :73-134), hooks are jumped to roots
// (new_shortcutting_step, :254-271) and edges inside a component are dropped
// (relabelling_step / filtering_step / remove_if, :273-321, :641-649).  The
// order (weight, edge id) is strict, so the forest is the unique MSF that the
// reference's PBBS mst() (MST/src/utils.cu:794-841) returns.
//
// Order of work (B200 design, not a translation):
//   1. A one-CTA kernel picks a weight threshold from a stratified sample of
//      the input so that about `light_per_vertex * n` edges are light: the
//      filtering step of PBBS mst() (approximate k-th smallest, :805-813), done
//      on the device.
//   2. Light phase.  Round 0 streams the input once and keeps only light
//      edges; later rounds stream the (small) survivor list.  Each round is ONE
//      pass: relabel both endpoints to their roots, drop internal edges, append
//      survivors as 16-byte {root_u, root_v, w, id} records, and offer each
//      survivor to both roots.
//   3. When no light edge is left the parents of all vertices are compressed
//      and the input is streamed a second time keeping heavy edges whose
//      endpoints lie in different components (PBBS's second filter, :819-823);
//      Boruvka continues on those survivors.  An edge that is heavy and
//      internal after the light phase closes a cycle of lighter edges, so it
//      is in no MSF: the filter changes the work, not the result.
//
// A component's choice is the minimum key (w << 32 | id) offered to it, kept
// with fire-and-forget 64-bit atomicMin.  The hook then runs over the survivor
// records: a record whose key won at an endpoint is that endpoint's choice, so
// no record has to be looked up and the survivor list may be in any order.
// That removes every dependency between CTAs from the edge pass: tiles are
// statically strided over a persistent grid, arrive in shared memory by 1-D
// bulk copies (cp.async.bulk) one tile ahead of use, survivors are staged
// densely in shared memory before their coalesced write, and output space is
// reserved in chunks with one atomicAdd each.  MSF membership is a bitmap over
// edge ids; one ordered gather (decoupled look-back) writes the MSF records
// ascending by id
// with the uint64 total.  Every round kernel reads the round, phase and
// continue flag from the device control block, so rounds are queued ahead
// without host round trips; a round queued after convergence exits at once.
#include <algorithm>
#include <cstring>

#include "internal.h"

namespace phem {
namespace {

struct RoundArgs {
    const void *e0;
    uint64_t m;
    uint32_t n;
    uint32_t *parent;
    unsigned long long *best;  // per component: minimum key (w << 32 | id) offered this round
    uint32_t *cand0;  // the round's choosers
    uint32_t *bitmap;
    uint32_t *chunk_cnt;  // MSF edges per 1024 edge ids, then per-4096-chunk totals and offsets
    uint4 *wl0, *wl1;
    uint64_t *status;
    unsigned long long *forest;
    Ctl *ctl;
    uint64_t light_k;  // light edges the threshold aims at (sizes the edge pass's list chunks)
};

// Count words for the chunks of 1024 edge ids (32 bitmap words) of an m-edge
// solve: one more so a zero-edge solve still has one, padded to a multiple of
// 4096 for the scan's vector loads.
__host__ __device__ inline uint64_t gather_chunks(uint64_t m) { return ((m + 1023) / 1024 + 1 + 4095) / 4096 * 4096; }
// Scan tiles of 4096 counts, and the count array's storage: the counts, then
// the tiles' totals and their exclusive prefixes.
__host__ __device__ inline uint64_t gather_tiles(uint64_t m) { return gather_chunks(m) / 4096; }
__host__ __device__ inline uint64_t gather_words(uint64_t m) { return gather_chunks(m) + 2 * gather_tiles(m) + 4; }

// Survivor records mark in the top bit of each root whether the record's
// offer may have won there; vertex ids leave that bit free up to this n.
constexpr uint32_t kMarkMaxN = 0x80000000u;
constexpr uint32_t kRootMask = 0x7fffffffu;

// An input record takes part in the forest: self-loops never do; packed CC
// edges follow union_find_gpu_COO and only count when u < v
// (CC/ExternalSpanningTree.cu:82).
template <int KIND>
__device__ __forceinline__ bool e0_live(uint32_t u, uint32_t v)
{
    return KIND == kKindMsf ? (u != v) : (u < v);
}

// Key of an edge: (w, id) for weighted edges, id alone for packed CC edges
// (the canonical forest orders edges by index).
template <int KIND>
__device__ __forceinline__ unsigned long long e0_key(uint32_t w, uint64_t id)
{
    return KIND == kKindMsf ? (((unsigned long long)w << 32) | id) : (unsigned long long)id;
}

// Offers.  A survivor offers its key to both of its roots' best[] words.
// Most survivors of hub-heavy rounds (and of the heavy pass, whose records
// mostly touch the light phase's giant component) offer to a handful of
// roots, and atomics on one best[] word serialise on its L2 slice; so a root
// first tries the slot hash(t) of a 512-entry table in the CTA's shared
// memory, claiming it when it is free: offers to a claimed slot are
// shared-memory atomicMins behind a shared read, and the table goes to best[]
// (one atomic per slot) when the CTA's pass ends.  An offer whose slot another
// root holds reads best[t] from L2 first and issues the 64-bit atomicMin only
// when it can still win: the read may be stale but never below the true
// value.  Both roots' reads are issued before either atomic.  (Grouping a
// warp's equal targets with __match_any_sync and reduce first cost more than
// the atomics it saved.)  Shared: tags 2 KB, keys 4 KB.
constexpr int kOfferSlots = 512;
constexpr uint32_t kNoTag = 0xffffffffu;

struct OfferCache {
    unsigned long long key[kOfferSlots];
    uint32_t tag[kOfferSlots];
};

// True when the offer went to (or lost against) t's shared slot; *may is set
// when it went there below the slot's value.
__device__ __forceinline__ bool table_offer(OfferCache &oc, uint32_t t, unsigned long long k, int *may)
{
    const int slot = (int)((t * 0x9E3779B1u) >> 23);  // 9 bits
    uint32_t tag = *(volatile uint32_t *)&oc.tag[slot];
    if (tag == kNoTag)
        tag = atomicCAS(&oc.tag[slot], kNoTag, t);
    if (tag != kNoTag && tag != t)
        return false;
    // most offers to a hub's slot cannot win: a shared read first avoids the
    // 64-bit shared atomic (a compare-and-swap loop under contention)
    if (k < *(volatile unsigned long long *)&oc.key[slot]) {
        atomicMin(&oc.key[slot], k);
        *may = 1;
    }
    return true;
}

// Returns bit 0 / bit 1 set when the offer at ta / tb may still win.  A
// cleared bit means the key lost there for good: it met a lower value (the
// shared slot's, or best[t]'s in L2), and the final minimum is lower still
// (keys are unique).
__device__ __forceinline__ uint32_t offer_pair(unsigned long long *best, OfferCache &oc, uint32_t ta, uint32_t tb,
                                               unsigned long long key, bool on)
{
    if (!on)
        return 0u;
    int wa = 0, wb = 0;
    const bool da = table_offer(oc, ta, key, &wa), db = table_offer(oc, tb, key, &wb);
    const unsigned long long ga = da ? 0ull : __ldcg(best + ta), gb = db ? 0ull : __ldcg(best + tb);
    if (!da && key < ga) {
        atomicMin(best + ta, key);
        wa = 1;
    }
    if (!db && key < gb) {
        atomicMin(best + tb, key);
        wb = 1;
    }
    return (uint32_t)wa | ((uint32_t)wb << 1);
}

__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long x, unsigned long long *s)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, d);
    const int warp = threadIdx.x >> 5;
    if (lane_id() == 0)
        s[warp] = x;
    __syncthreads();
    unsigned long long t = 0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kWarps; i++)
            t += s[i];
    return t;  // valid in thread 0
}

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// ---- kernels -----------------------------------------------------------------

// set_threshold: 0 when the threshold select runs beside this kernel (it
// writes ctl->threshold itself; both follow the control block's reset).
__global__ void __launch_bounds__(kBlock) init_kernel(RoundArgs a, unsigned long long threshold, int set_threshold)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < a.n; x += stride) {
        a.parent[x] = x;
        a.best[x] = kKeyNone;
        if (a.forest)
            a.forest[x] = kForestEmpty;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Ctl *c = a.ctl;
        c->go = 1;
        c->round = 0;
        c->phase = 0;
        c->src = kSrcLight;
        c->cand_all = 1;
        if (set_threshold)
            c->threshold = threshold;
    }
}

// Weight threshold from a stratified sample of kSample input weights: the
// sample's `rank`-th smallest weight, found by a three-digit radix select in
// shared memory (by the last of the sampling CTAs).  Light edges are those
// with w below it.
constexpr int kSample = 8192;
constexpr int kSelectThreads = 1024;
constexpr int kSelectBlocks = kSample / kSelectThreads;

__global__ void __launch_bounds__(kSelectThreads) select_threshold_kernel(const uint32_t *e0, uint64_t m,
                                                                          uint64_t k, uint32_t *g_samp, Ctl *ctl)
{
    __shared__ uint32_t samp[kSample];
    __shared__ uint32_t hist[2048];
    __shared__ uint32_t s_prefix, s_rank, s_or;
    __shared__ bool s_last;
    const int tid = threadIdx.x;
    // One sample per thread over kSelectBlocks blocks (a single block's 8192
    // random reads queue behind one SM's outstanding-miss limit); the last
    // block to finish selects.
    {
        const int i = blockIdx.x * kSelectThreads + tid;
        const uint64_t lo = (uint64_t)i * m / kSample, hi = (uint64_t)(i + 1) * m / kSample;
        const uint64_t pos = hi > lo ? lo + mix64(0x5EED0000ull + i) % (hi - lo) : lo;
        g_samp[i] = __ldg(e0 + pos * 3 + 2);
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        s_last = atomicAdd(&ctl->misc[7], 1ull) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    if (tid == 0)
        ctl->misc[7] = 0;
    constexpr int kPerThread = kSample / kSelectThreads;
    uint32_t v[kPerThread];
#pragma unroll
    for (int q = 0; q < kPerThread; q++)
        v[q] = __ldcg(g_samp + tid + q * kSelectThreads);
    uint32_t orv = 0;
#pragma unroll
    for (int q = 0; q < kPerThread; q++) {
        samp[tid + q * kSelectThreads] = v[q];
        orv |= v[q];
    }
    if (tid == 0) {
        s_prefix = 0;
        s_rank = (uint32_t)(k * kSample / m);
        s_or = 0;
    }
    __syncthreads();
    orv = __reduce_or_sync(0xffffffffu, orv);
    if ((tid & 31) == 0)
        atomicOr(&s_or, orv);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const int sh = d == 0 ? 21 : (d == 1 ? 10 : 0), nb = d == 2 ? 10 : 11, hsh = sh + nb;
        __syncthreads();
        // a digit that is zero in every sample (weights below 2^21 leave the
        // top one empty) puts them all in bin 0: the prefix and rank stand
        if ((s_or >> sh) == 0)
            continue;
        for (int i = tid; i < 2048; i += kSelectThreads)
            hist[i] = 0;
        __syncthreads();
        const uint64_t want_hi = (uint64_t)s_prefix >> hsh;
        for (int i = tid; i < kSample; i += kSelectThreads) {
            const uint32_t x = samp[i];
            if (((uint64_t)x >> hsh) == want_hi)
                atomicAdd(&hist[(x >> sh) & ((1u << nb) - 1)], 1u);
        }
        __syncthreads();
        if (tid < 32) {
            // lane l owns bins [64 l, 64 l + 64)
            uint32_t sum = 0;
            for (int b = 0; b < 64; b++)
                sum += hist[tid * 64 + b];
            uint32_t incl = sum;
#pragma unroll
            for (int s = 1; s < 32; s <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, incl, s);
                if (tid >= s)
                    incl += y;
            }
            const uint32_t excl = incl - sum, rank = s_rank;
            if (rank >= excl && rank < incl) {
                uint32_t c = excl;
                for (int b = 0; b < 64; b++) {
                    const uint32_t h = hist[tid * 64 + b];
                    if (rank < c + h) {
                        s_prefix |= (uint32_t)(tid * 64 + b) << sh;
                        s_rank = rank - c;
                        break;
                    }
                    c += h;
                }
            }
        }
        __syncthreads();
    }
    if (tid == 0)
        ctl->threshold = (unsigned long long)s_prefix << 32;
}

// One Boruvka round's edge pass: relabel + filter + compaction + per-root
// minimum, in one streaming pass over the round's input (the caller's records
// in round 0 and the heavy pass, the previous round's survivor list
// otherwise).
//
// Every warp works alone: no CTA barrier anywhere.  A warp owns the warp
// tiles gw, gw + GW, gw + 2 GW, ... (gw its global index, GW the grid's warp
// count; kEpStageBytes of input each: 128 records of 12 bytes, 192 packed
// pairs or 96 survivor records) and streams them through a two-stage
// pipeline of its own: lane 0 issues a 1-D bulk copy (cp.async.bulk, no
// multicast) of tile k + 1 into one stage while the warp reads tile k from
// the other, completion tracked by a per-stage mbarrier.  Lanes read records
// lane-striped from shared memory (12- and 16-byte strides are conflict-free),
// relabel endpoints to roots (read-only L1/L2 gathers of parent[]), drop
// internal and out-of-pass records, and append survivors by ballot rank to a
// 64-entry ring in the warp's shared memory.  Whenever 32 survivors are
// pending the warp flushes them: one atomicAdd reserves exactly 32 list slots
// (the list has no padding), one coalesced 512-byte store writes them, and
// their keys are offered to both roots (offer_pair).  A warp's last partial
// ring is flushed the same way with its exact count.
constexpr int kEpThreads = 256;
constexpr int kEpWarps = kEpThreads / 32;
constexpr int kEpMaxCtasPerSm = 4;   // 32 warps per SM; registers capped at 64 per thread
constexpr int kEpStages = 2;
constexpr uint32_t kEpStageBytes = 1536;
constexpr uint32_t kRing = 64;       // survivors staged per warp

struct __align__(16) EpWarp {
    unsigned char stage[kEpStages][kEpStageBytes];
    uint4 ring[kRing];
    unsigned long long bar[kEpStages];
};

// Records per warp tile for a record size.
template <uint32_t REC>
__host__ __device__ constexpr uint32_t ep_tile_recs()
{
    return kEpStageBytes / REC;
}
static_assert(kEpStageBytes % 12 == 0 && kEpStageBytes % 16 == 0 && (kEpStageBytes / 12) % 32 == 0 &&
                  (kEpStageBytes / 8) % 32 == 0 && (kEpStageBytes / 16) % 32 == 0,
              "warp tiles hold whole rows of every record size, in 16-byte multiples");

// Appends the lanes' survivors (keep) to the ring in lane order.
__device__ __forceinline__ void ring_append(EpWarp &w, uint32_t &filled, bool keep, uint4 rec, uint32_t lane)
{
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (keep)
        w.ring[(filled + __popc(mask & ((1u << lane) - 1u))) & (kRing - 1)] = rec;
    filled += __popc(mask);
}

// List space of one CTA.  Warps take exact slot ranges from the CTA's current
// chunk (a shared-memory atomic); the warp whose request crosses the chunk's
// end takes the chunk's last slots plus the start of the next chunk, which it
// reserves with one global atomicAdd and publishes; warps that arrive
// meanwhile wait for the new chunk.  One global atomic per chunk, not per
// flush: a single list counter takes about one returning atomic per few
// clocks, which per-flush reservations (10 M survivors / 32) saturated.
// Chunks are taken lazily, so a CTA without survivors reserves nothing; the
// CTA's last chunk is padded with dead records {0, 0, 0, 0} (equal roots:
// the next pass drops them) when the pass ends.
struct EpChunks {
    uint32_t state;              // (chunk number mod 256) << 24 | slots handed out in it
    uint32_t size;               // records per chunk
    unsigned long long base[8];  // list index of chunk c at [c & 7]
};

// Slots of one request: [b1, b1 + split) then [b2, b2 + k - split).
struct EpSlots {
    unsigned long long b1, b2;
    uint32_t split;
};

// The rare part of a reservation: `old` is what the first atomicAdd
// returned and did not fit (close the chunk, or wait for the warp closing it).
__device__ __noinline__ EpSlots chunk_reserve_slow(EpChunks &c, unsigned long long *len, uint32_t k, uint32_t *err,
                                                   uint32_t old)
{
    const uint32_t C = c.size;
    for (uint32_t spins = 0; spins < kMbarSpinCap; spins++) {
        const uint32_t cid = old >> 24, used = old & 0xffffffu;
        if (used + k <= C) {
            const unsigned long long b = *(volatile unsigned long long *)&c.base[cid & 7] + used;
            return EpSlots{b, b, k};
        }
        if (used <= C) {
            // this request closes chunk cid (its last C - used slots; none for
            // the empty chunk 0 of the pass) and opens chunk cid + 1 with the rest
            const uint32_t split = used < C ? C - used : 0;
            const unsigned long long b1 = split ? *(volatile unsigned long long *)&c.base[cid & 7] + used : 0;
            const unsigned long long nb = atomicAdd(len, (unsigned long long)C);
            const uint32_t next = (cid + 1) & 0xffu;
            *(volatile unsigned long long *)&c.base[next & 7] = nb;
            __threadfence_block();
            atomicExch(&c.state, (next << 24) | (k - split));
            return EpSlots{b1, nb, split};
        }
        // another warp is opening the next chunk
        while ((*(volatile uint32_t *)&c.state >> 24) == cid)
            if (++spins >= kMbarSpinCap)
                break;
        old = atomicAdd(&c.state, k);
    }
    set_err(err, kErrLookback);
    return EpSlots{~0ull, ~0ull, 0};
}

// Reserves k (1..32) list slots; b1 = b2 = ~0 when a wait for a new chunk
// gave up (the status bit is set).  Lane 0 only.  No fence on the common
// path: the base read depends on the chunk number the atomic returned, and
// the closer publishes the base before it publishes that number.
__device__ __forceinline__ EpSlots chunk_reserve(EpChunks &c, unsigned long long *len, uint32_t k, uint32_t *err)
{
    const uint32_t old = atomicAdd(&c.state, k);
    const uint32_t cid = old >> 24, used = old & 0xffffffu;
    if (used + k <= c.size) {
        const unsigned long long b = *(volatile unsigned long long *)&c.base[cid & 7] + used;
        return EpSlots{b, b, k};
    }
    return chunk_reserve_slow(c, len, k, err, old);
}

// Writes the `cnt` (<= 32) oldest ring entries to the list and offers them.
template <int KIND>
__device__ __forceinline__ void ring_flush(const RoundArgs &a, uint4 *out, unsigned long long *len, EpChunks &ch,
                                           OfferCache &oc, EpWarp &w, uint32_t &flushed, uint32_t cnt,
                                           uint32_t lane)
{
    __syncwarp();  // the lanes' ring writes are visible
    const bool on = lane < cnt;
    const uint4 rec = on ? w.ring[(flushed + lane) & (kRing - 1)] : make_uint4(0, 0, 0, 0);
    flushed += cnt;
    EpSlots sl{0, 0, 0};
    if (lane == 0)
        sl = chunk_reserve(ch, len, cnt, &a.ctl->err);
    const unsigned long long b1 = __shfl_sync(0xffffffffu, sl.b1, 0), b2 = __shfl_sync(0xffffffffu, sl.b2, 0);
    const uint32_t split = __shfl_sync(0xffffffffu, sl.split, 0);
    if (b2 != ~0ull) {
        const unsigned long long key =
            KIND == kKindMsf ? (((unsigned long long)rec.z << 32) | rec.w) : (unsigned long long)rec.w;
        const uint32_t may = offer_pair(a.best, oc, rec.x, rec.y, key, on);
        // the hook only looks at the roots where the record may have won
        // (the top bit of a root is free when n <= 2^31)
        uint4 r = rec;
        if (a.n <= kMarkMaxN) {
            r.x |= (may & 1u) << 31;
            r.y |= (may & 2u) << 30;
        }
        if (on)
            out[lane < split ? b1 + lane : b2 + (lane - split)] = r;
    }
    __syncwarp();  // the ring slots just read may be written again
}

// Bounded wait of the whole warp for a stage's bulk copy.
__device__ __forceinline__ bool ep_wait(unsigned long long *bar, uint32_t parity, uint32_t *err)
{
    bool ok = mbar_wait(reinterpret_cast<uint64_t *>(bar), parity, err);
    return __all_sync(0xffffffffu, ok);
}

// Input tile (the caller's records): rows of 32 records, lane-striped.
// LIGHT keeps key < threshold with the endpoints as roots (round 0: every
// vertex is its own root); otherwise keeps key >= threshold between different
// components after relabelling both endpoints (the heavy pass: parent[] is
// fully compressed, so one hop reaches the root).
template <int KIND, bool LIGHT>
__device__ __forceinline__ void ep_input_tile(const RoundArgs &a, const unsigned char *stage, bool bulk,
                                              uint64_t tbase, uint32_t rem, unsigned long long thr, EpWarp &w, uint32_t &filled, uint32_t &flushed, uint4 *out,
                                              unsigned long long *len, EpChunks &ch, OfferCache &oc,
                                              uint32_t lane, bool &any_bad)
{
    constexpr uint32_t REC = KIND == kKindMsf ? 12u : 8u;
    constexpr int ROWS = (int)(ep_tile_recs<REC>() / 32);
    uint32_t u[ROWS], v[ROWS], wt[ROWS];
    bool keep[ROWS];
    const uint32_t id0 = (uint32_t)tbase;
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
        const uint32_t idx = j * 32 + lane;
        const bool inb = idx < rem;
        uint32_t x = 0, y = 0, z = 0;
        if (KIND == kKindMsf) {
            if (bulk) {
                const uint32_t *p = reinterpret_cast<const uint32_t *>(stage) + 3 * idx;
                x = p[0];
                y = p[1];
                z = p[2];
            } else if (inb) {
                const uint32_t *p = static_cast<const uint32_t *>(a.e0) + 3 * (tbase + idx);
                x = __ldcs(p);
                y = __ldcs(p + 1);
                z = __ldcs(p + 2);
            }
        } else {
            unsigned long long e = 0;
            if (bulk)
                e = reinterpret_cast<const unsigned long long *>(stage)[idx];
            else if (inb)
                e = __ldcs(static_cast<const unsigned long long *>(a.e0) + tbase + idx);
            x = (uint32_t)(e >> 32);
            y = (uint32_t)e;
        }
        const uint32_t id = id0 + idx;
        const bool live = inb && e0_live<KIND>(x, y);
        const bool bad = live && max(x, y) >= a.n;
        any_bad |= bad;
        const bool light = e0_key<KIND>(z, id) < thr;
        keep[j] = live && !bad && (LIGHT ? light : !light);
        u[j] = x;
        v[j] = y;
        wt[j] = z;
    }
    if (!LIGHT) {
        // all rows' gathers in flight together
#pragma unroll
        for (int j = 0; j < ROWS; j++)
            if (keep[j]) {
                u[j] = __ldg(a.parent + u[j]);
                v[j] = __ldg(a.parent + v[j]);
            }
#pragma unroll
        for (int j = 0; j < ROWS; j++)
            keep[j] = keep[j] && u[j] != v[j];
    }
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
        ring_append(w, filled, keep[j], make_uint4(u[j], v[j], wt[j], id0 + j * 32 + lane), lane);
        if (filled - flushed >= 32)
            ring_flush<KIND>(a, out, len, ch, oc, w, flushed, 32, lane);
    }
}

// List tile (the previous round's survivors {root_u, root_v, w, id}): both
// roots are relabelled by one hop (the compress pointed every root that
// hooked at its new root) and records inside one component are dropped.
template <int KIND>
__device__ __forceinline__ void ep_list_tile(const RoundArgs &a, const uint4 *in, const unsigned char *stage,
                                             bool bulk, uint64_t tbase, uint32_t rem, EpWarp &w, uint32_t &filled,
                                             uint32_t &flushed, uint4 *out, unsigned long long *len, EpChunks &ch,
                                             OfferCache &oc, uint32_t lane)
{
    constexpr int ROWS = (int)(ep_tile_recs<16>() / 32);
    uint4 rec[ROWS];
    bool keep[ROWS];
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
        const uint32_t idx = j * 32 + lane;
        keep[j] = idx < rem;
        rec[j] = make_uint4(0, 0, 0, 0);
        if (bulk)
            rec[j] = reinterpret_cast<const uint4 *>(stage)[idx];
        else if (keep[j])
            rec[j] = __ldcs(in + tbase + idx);
    }
    const uint32_t rmask = a.n <= kMarkMaxN ? kRootMask : 0xffffffffu;  // drop the last round's marks
#pragma unroll
    for (int j = 0; j < ROWS; j++)
        if (keep[j]) {
            rec[j].x = __ldg(a.parent + (rec[j].x & rmask));
            rec[j].y = __ldg(a.parent + (rec[j].y & rmask));
        }
#pragma unroll
    for (int j = 0; j < ROWS; j++) {
        ring_append(w, filled, keep[j] && rec[j].x != rec[j].y, rec[j], lane);
        if (filled - flushed >= 32)
            ring_flush<KIND>(a, out, len, ch, oc, w, flushed, 32, lane);
    }
}

template <int KIND>
__global__ void __launch_bounds__(kEpThreads, kEpMaxCtasPerSm) edge_pass_kernel(RoundArgs a)
{
    __shared__ EpWarp s_warp[kEpWarps];
    __shared__ EpChunks s_chunks;
    __shared__ OfferCache s_offers;
    Ctl *ctl = a.ctl;
    if (!*(volatile uint32_t *)&ctl->go)
        return;
    const uint32_t r = *(volatile uint32_t *)&ctl->round;
    const uint32_t src = *(volatile uint32_t *)&ctl->src;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    EpWarp &w = s_warp[warp];
    const bool from_e0 = src != kSrcList;
    const uint32_t rec_bytes = from_e0 ? (KIND == kKindMsf ? 12u : 8u) : 16u;
    const uint32_t tile_recs = kEpStageBytes / rec_bytes;
    const uint64_t count = from_e0 ? a.m : ctl->wl_len[r - 1];
    const uint4 *in = (r & 1) ? a.wl0 : a.wl1;  // WL[(r - 1) & 1]
    uint4 *out = (r & 1) ? a.wl1 : a.wl0;       // WL[r & 1]
    unsigned long long *len = &ctl->wl_len[r];
    const char *src_base = from_e0 ? static_cast<const char *>(a.e0) : reinterpret_cast<const char *>(in);
    const uint64_t ntiles = (count + tile_recs - 1) / tile_recs;
    const uint64_t full_tiles = count / tile_recs;  // the partial last tile is read directly
    const uint64_t gw = (uint64_t)blockIdx.x * kEpWarps + warp, GW = (uint64_t)gridDim.x * kEpWarps;
    const unsigned long long thr = *(volatile unsigned long long *)&ctl->threshold;
    const uint64_t policy = l2_evict_first();  // inputs and lists are read once per pass
    if (threadIdx.x == 0) {
        // chunks of about a quarter of a CTA's expected survivors (a power of
        // two in [128, 2048]): few global atomics, and on average half a chunk
        // of padding per CTA.  Expected: the light edges in round 0, an eighth
        // of the input in the heavy pass, the whole list in list rounds.
        const uint64_t expect = src == kSrcLight ? a.light_k : (src == kSrcHeavy ? a.m / 8 : count);
        const uint64_t per = expect / ((uint64_t)gridDim.x * 4);
        uint32_t c = 128;
        while (c < 2048 && (uint64_t)c * 2 <= per)
            c *= 2;
        s_chunks.size = c;
        s_chunks.state = c;  // chunk 0 "full" (and empty): the first request opens chunk 1
    }
    for (int i = threadIdx.x; i < kOfferSlots; i += kEpThreads) {
        s_offers.tag[i] = kNoTag;
        s_offers.key[i] = kKeyNone;
    }
    __syncthreads();

    if (lane == 0) {
        for (int s = 0; s < kEpStages; s++)
            mbar_init(reinterpret_cast<uint64_t *>(&w.bar[s]), 1);
        fence_mbar_init();
    }
    __syncwarp();
    auto issue = [&](uint64_t t, int s) {  // lane 0 only
        mbar_arrive_expect_tx(reinterpret_cast<uint64_t *>(&w.bar[s]), kEpStageBytes);
        bulk_copy_g2s_hint(w.stage[s], src_base + t * kEpStageBytes, kEpStageBytes,
                           reinterpret_cast<uint64_t *>(&w.bar[s]), policy);
    };
    if (lane == 0 && gw < full_tiles)
        issue(gw, 0);
    uint32_t filled = 0, flushed = 0;  // ring cursors (warp-uniform)
    uint32_t parity = 0;               // bit s: phase of stage s's barrier to wait for
    uint32_t pending = gw < full_tiles ? 1u : 0u;  // bit s: a copy into stage s is in flight
    bool any_bad = false, failed = false;
    int s = 0;
    for (uint64_t t = gw; t < ntiles; t += GW, s ^= 1) {
        // tile t + GW goes into the other stage, which the previous tile left
        // (its reads were fenced against the async proxy before the warp
        // synchronised at the end of that tile)
        const uint64_t t2 = t + GW;
        if (t2 < full_tiles) {
            if (lane == 0)
                issue(t2, s ^ 1);
            pending |= 1u << (s ^ 1);
        }
        const bool bulk = t < full_tiles;
        if (bulk) {
            if (!ep_wait(&w.bar[s], (parity >> s) & 1u, &ctl->err)) {
                failed = true;
                break;
            }
            parity ^= 1u << s;
            pending &= ~(1u << s);
        }
        const uint64_t tbase = t * tile_recs;
        const uint64_t left = count - tbase;
        const uint32_t rem = left < tile_recs ? (uint32_t)left : tile_recs;
        if (src == kSrcList)
            ep_list_tile<KIND>(a, in, w.stage[s], bulk, tbase, rem, w, filled, flushed, out, len, s_chunks,
                               s_offers, lane);
        else if (src == kSrcLight)
            ep_input_tile<KIND, true>(a, w.stage[s], bulk, tbase, rem, thr, w, filled, flushed, out,
                                      len, s_chunks, s_offers, lane, any_bad);
        else
            ep_input_tile<KIND, false>(a, w.stage[s], bulk, tbase, rem, thr, w, filled, flushed, out,
                                       len, s_chunks, s_offers, lane, any_bad);
        fence_proxy_async_smem();  // this lane's reads of the stage precede its refill
        __syncwarp();
    }
    if (failed) {
        // a copy never completed (the status bit is set): wait, bounded, for
        // every copy still in flight into this warp's stages
        for (int q = 0; q < kEpStages; q++)
            if (pending & (1u << q))
                ep_wait(&w.bar[q], (parity >> q) & 1u, &ctl->err);
    } else {
        if (filled != flushed)
            ring_flush<KIND>(a, out, len, s_chunks, s_offers, w, flushed, filled - flushed, lane);
        if (__any_sync(0xffffffffu, any_bad) && lane == 0 && src == kSrcLight)
            set_err(&ctl->err, kErrRange);
        if (lane == 0 && filled)
            atomicAdd(&ctl->m_r[r], (unsigned long long)filled);
    }
    // the CTA's last chunk: pad its unused tail; the offer table goes to best[]
    __syncthreads();
    for (int i = threadIdx.x; i < kOfferSlots; i += kEpThreads) {
        const uint32_t t = s_offers.tag[i];
        if (t != kNoTag)
            atomicMin(a.best + t, s_offers.key[i]);
    }
    const uint32_t st = s_chunks.state;
    const uint32_t cid = st >> 24, used = min(st & 0xffffffu, s_chunks.size);
    if (s_chunks.state != s_chunks.size)  // a chunk was opened
        for (uint32_t i = used + threadIdx.x; i < s_chunks.size; i += kEpThreads)
            out[s_chunks.base[cid & 7] + i] = make_uint4(0, 0, 0, 0);
}

// Hook, over this round's survivor records: a record whose key is the
// minimum at an endpoint's component is that component's chosen edge (keys
// are unique, so each component finds exactly one).  A component hooks onto
// the far one and marks the edge; when both endpoints chose the same record
// (a mutual pair) the lower id stays root and the higher one hooks
// (new_grafting_edges, MST/src/kernels.cu:73-134).  Dead padding records
// (equal roots) are skipped.  The list was just written, so it is mostly read
// from L2.
// Chooser ids staged per warp before they go to the chooser list: a warp
// flushes once more than 256 are pending (an iteration adds at most 256),
// with one atomicAdd per flush and no barrier between warps.
constexpr uint32_t kHookBuf = 512;
constexpr int kHookCtasPerSm = 4;

template <int KIND>
__global__ void __launch_bounds__(kBlock) hook_kernel(RoundArgs a)
{
    __shared__ uint32_t s_buf[kWarps][kHookBuf];
    Ctl *ctl = a.ctl;
    if (!*(volatile uint32_t *)&ctl->go)
        return;
    const uint32_t r = *(volatile uint32_t *)&ctl->round;
    const uint64_t len = ctl->wl_len[r];
    const uint4 *wl = (r & 1) ? a.wl1 : a.wl0;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const unsigned below = (1u << lane) - 1u;
    const bool marks = a.n <= kMarkMaxN;
    const uint32_t rmask = marks ? kRootMask : 0xffffffffu;
    uint32_t *buf = s_buf[warp];
    uint32_t pend = 0;  // warp-uniform
    auto flush = [&]() {
        __syncwarp();
        unsigned long long base = 0;
        if (lane == 0)
            base = atomicAdd(&ctl->n_r[r], (unsigned long long)pend);
        base = __shfl_sync(0xffffffffu, base, 0);
        for (uint32_t i = lane; i < pend; i += 32)
            a.cand0[base + i] = buf[i];
        __syncwarp();
        pend = 0;
    };
    const uint64_t step = (uint64_t)gridDim.x * kBlock * 4;
    for (uint64_t i0 = (uint64_t)blockIdx.x * kBlock * 4; i0 < len; i0 += step) {
        uint4 rec[4];
        unsigned long long ka[4], kb[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const uint64_t i = i0 + q * kBlock + threadIdx.x;
            rec[q] = i < len ? __ldcg(wl + i) : make_uint4(0, 0, 0, 0);
            // only the roots where the record's offer may have won (marked by
            // the edge pass; every root when n is too large for marks)
            const bool ma = marks ? (rec[q].x >> 31) != 0 : rec[q].x != rec[q].y;
            const bool mb = marks ? (rec[q].y >> 31) != 0 : rec[q].x != rec[q].y;
            rec[q].x &= rmask;
            rec[q].y &= rmask;
            // best is read-only during this kernel: cached loads let the
            // few hub components of late rounds hit in L1
            ka[q] = ma ? __ldg(a.best + rec[q].x) : 0ull;
            kb[q] = mb ? __ldg(a.best + rec[q].y) : 0ull;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const unsigned long long key = ((unsigned long long)rec[q].z << 32) | rec[q].w;
            const bool real = rec[q].x != rec[q].y;
            const bool A = real && ka[q] == key, B = real && kb[q] == key;
            if (A || B) {
                uint32_t hk, tgt;
                if (A && B) {
                    hk = rec[q].x > rec[q].y ? rec[q].x : rec[q].y;
                    tgt = rec[q].x > rec[q].y ? rec[q].y : rec[q].x;
                } else if (A) {
                    hk = rec[q].x;
                    tgt = rec[q].y;
                } else {
                    hk = rec[q].y;
                    tgt = rec[q].x;
                }
                const uint32_t id = rec[q].w;
                a.parent[hk] = tgt;
                atomicOr(a.bitmap + (id >> 5), 1u << (id & 31));
                atomicAdd(a.chunk_cnt + (id >> 10), 1u);
                if (KIND == kKindPacked && a.forest)
                    a.forest[hk] = __ldg(reinterpret_cast<const unsigned long long *>(a.e0) + id);
            }
            // the round's choosers (each component finds its one record) go
            // to the chooser list, which the compress walks instead of all
            // vertices
            const unsigned ma = __ballot_sync(0xffffffffu, A);
            if (A)
                buf[pend + __popc(ma & below)] = rec[q].x;
            pend += __popc(ma);
            const unsigned mb = __ballot_sync(0xffffffffu, B);
            if (B)
                buf[pend + __popc(mb & below)] = rec[q].y;
            pend += __popc(mb);
        }
        if (pend > kHookBuf - 256)
            flush();
    }
    if (pend)
        flush();
}

// compress grid: four CTAs per SM, enough walks in flight for the
// all-vertex rounds and a short launch for the late rounds' few choosers
constexpr int kCompressCtasPerSm = 4;
constexpr int kVItems = 4;  // candidates per thread per iteration of the vertex kernels

// Pointer jumping over this round's choosers (the hook's list): each is
// pointed at its root and its best key is reset.  In the round where the
// light phase runs dry (no survivors, no choosers) every vertex is compressed
// to its root instead, so the heavy pass relabels original endpoints in one
// hop.
__device__ void advance_round(Ctl *ctl);

// `loop`: when the rounds run as a CUDA graph's while-node, the handle of its
// condition, which the block that decides the next round sets to the continue
// flag (use_loop 0: rounds queued on a stream).
__global__ void __launch_bounds__(kBlock) compress_kernel(RoundArgs a, cudaGraphConditionalHandle loop,
                                                          int use_loop)
{
    Ctl *ctl = a.ctl;
    if (!*(volatile uint32_t *)&ctl->go) {
        if (use_loop && blockIdx.x == 0 && threadIdx.x == 0)
            cudaGraphSetConditional(loop, 0);
        return;
    }
    const uint32_t r = *(volatile uint32_t *)&ctl->round;
    const bool full = *(volatile uint32_t *)&ctl->phase == 0 && ctl->m_r[r] == 0;
    const uint64_t count = full ? a.n : ctl->n_r[r];
    const uint64_t step = (uint64_t)gridDim.x * kBlock * kVItems;
    for (uint64_t i0 = (uint64_t)blockIdx.x * kBlock * kVItems; i0 < count; i0 += step) {
        bool walking[kVItems];
        uint32_t x[kVItems], y[kVItems], y0[kVItems];
        // the candidates' loads and root walks advance in lockstep, so their
        // dependent loads are in flight together
#pragma unroll
        for (int k = 0; k < kVItems; k++) {
            const uint64_t i = i0 + k * kBlock + threadIdx.x;
            walking[k] = i < count;
            x[k] = walking[k] ? (full ? (uint32_t)i : __ldcg(a.cand0 + i)) : 0;
        }
#pragma unroll
        for (int k = 0; k < kVItems; k++)
            y0[k] = y[k] = walking[k] ? a.parent[x[k]] : x[k];
        const bool active[kVItems] = {walking[0], walking[1], walking[2], walking[3]};
        static_assert(kVItems == 4, "active[] lists kVItems entries");
        for (uint32_t steps = 0;; steps++) {
            uint32_t p[kVItems];
#pragma unroll
            for (int k = 0; k < kVItems; k++)
                p[k] = walking[k] ? a.parent[y[k]] : y[k];
            bool any = false;
#pragma unroll
            for (int k = 0; k < kVItems; k++) {
                walking[k] = walking[k] && p[k] != y[k];
                y[k] = p[k];
                any |= walking[k];
            }
            if (!any)
                break;
            if (steps > a.n) {
                set_err(&ctl->err, kErrChase);
                break;
            }
        }
#pragma unroll
        for (int k = 0; k < kVItems; k++) {
            if (active[k]) {
                if (y0[k] != y[k])
                    a.parent[x[k]] = y[k];
                if (!full)
                    a.best[x[k]] = kKeyNone;
            }
        }
    }
    // the last block to finish decides the next round (no separate launch)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctl->misc[6], 1ull) == gridDim.x - 1) {
            __threadfence();
            ctl->misc[6] = 0;
            advance_round(ctl);
            if (use_loop)
                cudaGraphSetConditional(loop, ctl->go);
        }
    }
}

// Ends a round.  Live edges left -> another round on the survivor list.  No
// light edge left -> switch to the heavy pass (if there is a threshold).  No
// heavy edge left -> done.
// Decides the next round from this round's counters (one thread).
__device__ void advance_round(Ctl *ctl)
{
    if (!ctl->go)
        return;
    const uint32_t r = ctl->round;
    bool again;
    if (ctl->m_r[r] > 0) {
        ctl->src = kSrcList;
        ctl->cand_all = 0;
        again = true;
    } else if (ctl->phase == 0) {
        ctl->phase = 1;
        ctl->light_rounds = r + 1;
        ctl->src = kSrcHeavy;
        ctl->cand_all = 1;
        again = ctl->threshold != kKeyNone;
    } else {
        again = false;
    }
    if (again && r + 1 >= PHEM_MAX_ROUNDS) {
        ctl->err |= kErrRounds;
        again = false;
    }
    ctl->round = r + 1;
    ctl->go = again ? 1u : 0u;
}



// Ordered gather: MSF records ascending by id from the bitmap, plus count and
// uint64 total weight, without a block waiting for another.  The hook counts
// the edges it marks per chunk of 1024 edge ids (32 bitmap words); one block
// scans the chunk counts into offsets; then every warp takes whole chunks,
// ranks its 32 words' bits with a warp scan and gathers its records (12-byte
// random reads of the input) to out[offset + rank].
constexpr int kGatherWarps = kWarps;

// Offsets of the chunks' records: every block scans one tile of 4096 counts
// in place (exclusive, within the tile; one uint4 per thread) and publishes
// the tile's total; the last block to finish scans the totals into the
// tiles' offsets and the forest size.  No block waits for another.
__global__ void __launch_bounds__(1024) gather_scan_kernel(uint32_t *cnt, uint64_t tiles, Ctl *ctl)
{
    __shared__ uint32_t s_warp[33];
    __shared__ bool s_last;
    uint32_t *tile_total = cnt + tiles * 4096, *tile_off = tile_total + tiles;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    auto block_scan = [&](uint32_t v, uint32_t *total) {  // exclusive scan over the block
        uint32_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= (uint32_t)d)
                x += y;
        }
        if (lane == 31)
            s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            const uint32_t w = s_warp[lane];
            uint32_t wi = w;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, wi, d);
                if (lane >= (uint32_t)d)
                    wi += y;
            }
            s_warp[lane] = wi - w;
            if (lane == 31)
                s_warp[32] = wi;
        }
        __syncthreads();
        *total = s_warp[32];
        const uint32_t r = s_warp[warp] + x - v;
        __syncthreads();  // s_warp is reused
        return r;
    };
    uint4 *c4 = reinterpret_cast<uint4 *>(cnt + (uint64_t)blockIdx.x * 4096) + threadIdx.x;
    const uint4 v = *c4;
    uint32_t total;
    const uint32_t run = block_scan(v.x + v.y + v.z + v.w, &total);
    *c4 = make_uint4(run, run + v.x, run + v.x + v.y, run + v.x + v.y + v.z);
    if (threadIdx.x == 0) {
        tile_total[blockIdx.x] = total;
        __threadfence();
        s_last = atomicAdd(&ctl->misc[5], 1ull) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    if (threadIdx.x == 0)
        ctl->misc[5] = 0;
    uint32_t carry = 0;
    for (uint64_t t0 = 0; t0 < tiles; t0 += 1024) {
        const uint64_t t = t0 + threadIdx.x;
        const uint32_t tv = t < tiles ? __ldcg(tile_total + t) : 0u;
        uint32_t sum;
        const uint32_t ex = block_scan(tv, &sum);
        if (t < tiles)
            tile_off[t] = carry + ex;
        carry += sum;
    }
    if (threadIdx.x == 0)
        ctl->msf_count = carry;
}

__global__ void __launch_bounds__(kBlock) gather_kernel(RoundArgs a, phem_edge *out)
{
    __shared__ unsigned long long s_red[kWarps];
    const uint64_t words = (a.m + 31) / 32;
    const uint64_t chunks = (words + 31) / 32;
    const uint32_t lane = lane_id();
    const uint64_t gw = (uint64_t)blockIdx.x * kGatherWarps + (threadIdx.x >> 5);
    const uint64_t GW = (uint64_t)gridDim.x * kGatherWarps;
    const uint32_t *E = reinterpret_cast<const uint32_t *>(a.e0);
    unsigned long long wsum = 0;
    const uint32_t *tile_off = a.chunk_cnt + gather_chunks(a.m) + gather_tiles(a.m);
    for (uint64_t c = gw; c < chunks; c += GW) {
        const uint64_t wd = c * 32 + lane;
        uint32_t bits = wd < words ? __ldcs(a.bitmap + wd) : 0u;
        const uint32_t k = __popc(bits);
        uint32_t incl = k;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (uint32_t)d)
                incl += y;
        }
        uint64_t pos = (uint64_t)__ldcs(a.chunk_cnt + c) + __ldcg(tile_off + c / 4096) + (incl - k);
        // four of the lane's records per step, their loads in flight together
        while (bits) {
            uint32_t id[4];
            int cntq = 0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                id[q] = 0xffffffffu;
                if (bits) {
                    id[q] = (uint32_t)(wd * 32 + (__ffs(bits) - 1));
                    bits &= bits - 1;
                    cntq++;
                }
            }
            phem_edge e[4];
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (id[q] != 0xffffffffu) {
                    const uint64_t i3 = (uint64_t)id[q] * 3;
                    e[q].u = __ldg(E + i3);
                    e[q].v = __ldg(E + i3 + 1);
                    e[q].w = __ldg(E + i3 + 2);
                }
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (q < cntq) {
                    if (out)
                        out[pos] = e[q];
                    pos++;
                    wsum += e[q].w;
                }
        }
    }
    const unsigned long long bs = block_sum_u64(wsum, s_red);
    if (threadIdx.x == 0 && bs)
        atomicAdd(&a.ctl->msf_total, bs);
}

RoundArgs make_args(phem_context *ctx, const MsfPlan &p)
{
    RoundArgs a;
    std::memset(&a, 0, sizeof(a));  // no stray padding bytes: the graph cache compares args bytewise
    a.e0 = p.e0;
    a.m = p.m;
    a.n = p.n;
    a.parent = p.parent;
    a.best = p.best;
    a.cand0 = p.cand;
    a.bitmap = p.bitmap;
    a.chunk_cnt = p.chunk_cnt;
    a.wl0 = p.wl[0];
    a.wl1 = p.wl[1];
    a.status = p.status;
    a.forest = reinterpret_cast<unsigned long long *>(p.forest);
    a.ctl = ctx->ctl;
    a.light_k = p.m;
    return a;
}

int vertex_blocks(phem_context *ctx, uint64_t count)
{
    uint64_t b = (count + kBlock - 1) / kBlock;
    uint64_t cap = (uint64_t)ctx->sm_count * 8;
    return (int)std::max<uint64_t>(1, std::min(b, cap));
}

template <int KIND>
phem_status queue_round(phem_context *ctx, const RoundArgs &a)
{
    const int vb = vertex_blocks(ctx, a.n);
    {
        KernelScope k(ctx, kKEdgePass);
        edge_pass_kernel<KIND><<<ctx->edge_pass_blocks, kEpThreads, 0, ctx->stream>>>(a);
    }
    {
        KernelScope k(ctx, kKHook);
        hook_kernel<KIND><<<ctx->sm_count * kHookCtasPerSm, kBlock, 0, ctx->stream>>>(a);
    }
    {
        KernelScope k(ctx, kKCompress);
        compress_kernel<<<std::min(vb, ctx->sm_count * kCompressCtasPerSm), kBlock, 0, ctx->stream>>>(a, 0, 0);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

template <int KIND>
phem_status setup_kernels(phem_context *ctx)
{
    int per_sm = 0;
    PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, edge_pass_kernel<KIND>, kEpThreads, 0));
    const int want = std::min(ctx->tune_edge_ctas, kEpMaxCtasPerSm);
    ctx->edge_pass_blocks = ctx->sm_count * std::max(1, std::min(per_sm, want));
    PHEM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gather_kernel, kBlock, 0));
    ctx->gather_blocks = ctx->sm_count * std::max(1, per_sm);
    return PHEM_OK;
}

// The round loop as a CUDA graph: memsets, init, threshold select, then a
// while-node whose body is one round (edge pass, hook, compress) and whose
// condition the compress's deciding block sets to the continue flag.  The
// device runs exactly the rounds the solve needs, with no host round trip and
// no round queued after convergence.  The executable graph is cached in the
// context and rebuilt when anything baked into its nodes changes (buffers,
// sizes, grids, threshold).
struct GraphKey {
    RoundArgs a;
    unsigned long long thr;
    uint64_t k;
    int select, ep_blocks, vb_init, vb_comp, hook_blocks, kind;
};

template <class... Args>
phem_status add_kernel(cudaGraphNode_t *node, cudaGraph_t g, const cudaGraphNode_t *dep, void (*fn)(Args...),
                       dim3 grid, dim3 block, void **args)
{
    cudaKernelNodeParams p{};
    p.func = reinterpret_cast<void *>(fn);
    p.gridDim = grid;
    p.blockDim = block;
    p.sharedMemBytes = 0;
    p.kernelParams = args;
    PHEM_CUDA_TRY(cudaGraphAddKernelNode(node, g, dep, dep ? 1 : 0, &p));
    return PHEM_OK;
}

phem_status add_memset(cudaGraphNode_t *node, cudaGraph_t g, const cudaGraphNode_t *dep, void *dst, size_t bytes)
{
    cudaMemsetParams p{};
    p.dst = dst;
    p.value = 0;
    p.elementSize = 1;
    p.width = bytes;
    p.height = 1;
    p.pitch = bytes;
    PHEM_CUDA_TRY(cudaGraphAddMemsetNode(node, g, dep, dep ? 1 : 0, &p));
    return PHEM_OK;
}

template <int KIND>
phem_status build_graph(phem_context *ctx, const MsfPlan &plan, const GraphKey &key, cudaGraphExec_t *exec)
{
    cudaGraph_t g = nullptr;
    PHEM_CUDA_TRY(cudaGraphCreate(&g, 0));
    struct Drop {
        cudaGraph_t g;
        ~Drop() { cudaGraphDestroy(g); }
    } drop{g};
    // Before the round loop, as a DAG: the control block's reset, then the
    // vertex init and the threshold select side by side; the bitmap and
    // chunk-count resets run beside all of them.
    cudaGraphNode_t pre[4], n_ctl;
    int npre = 0;
    RoundArgs a = key.a;
    unsigned long long thr = key.thr;
    int set_thr = key.select ? 0 : 1;
    PHEM_TRY(add_memset(&n_ctl, g, nullptr, ctx->ctl, sizeof(Ctl)));
    const size_t bitmap_bytes = ((plan.m + 31) / 32) * sizeof(uint32_t);
    if (bitmap_bytes)  // a memset node of zero bytes is invalid
        PHEM_TRY(add_memset(&pre[npre++], g, nullptr, plan.bitmap, bitmap_bytes));
    PHEM_TRY(add_memset(&pre[npre++], g, nullptr, plan.chunk_cnt, gather_chunks(plan.m) * sizeof(uint32_t)));
    {
        void *args[] = {&a, &thr, &set_thr};
        PHEM_TRY(add_kernel(&pre[npre++], g, &n_ctl, init_kernel, dim3(key.vb_init), dim3(kBlock), args));
    }
    const uint32_t *e0w = static_cast<const uint32_t *>(plan.e0);
    uint64_t m = plan.m, k = key.k;
    Ctl *ctl = ctx->ctl;
    if (key.select) {
        uint32_t *samp = plan.samples;
        void *args[] = {&e0w, &m, &k, &samp, &ctl};
        PHEM_TRY(add_kernel(&pre[npre++], g, &n_ctl, select_threshold_kernel, dim3(kSelectBlocks),
                            dim3(kSelectThreads), args));
    }
    cudaGraphConditionalHandle loop;
    PHEM_CUDA_TRY(cudaGraphConditionalHandleCreate(&loop, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t nc;
    PHEM_CUDA_TRY(cudaGraphAddNode(&nc, g, pre, npre, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaGraphNode_t b0, b1, b2;
    {
        void *args[] = {&a};
        PHEM_TRY(add_kernel(&b0, body, nullptr, edge_pass_kernel<KIND>, dim3(key.ep_blocks), dim3(kEpThreads), args));
        PHEM_TRY(add_kernel(&b1, body, &b0, hook_kernel<KIND>, dim3(key.hook_blocks), dim3(kBlock), args));
    }
    {
        int use = 1;
        void *args[] = {&a, &loop, &use};
        PHEM_TRY(add_kernel(&b2, body, &b1, compress_kernel, dim3(key.vb_comp), dim3(kBlock), args));
    }
    if (*exec) {
        // same topology (the cached graph had a select node iff this one has):
        // update the instantiated graph's parameters in place, which costs
        // far less than instantiating again
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(*exec, g, &info) == cudaSuccess)
            return PHEM_OK;
        cudaGetLastError();
        cudaGraphExecDestroy(*exec);
        *exec = nullptr;
    }
    PHEM_CUDA_TRY(cudaGraphInstantiate(exec, g, 0));
    return PHEM_OK;
}

template <int KIND>
phem_status run_impl(phem_context *ctx, MsfPlan &plan, uint32_t *rounds_out, bool deferred)
{
    cudaStream_t s = ctx->stream;
    if (!(ctx->kernels_ready & (1u << KIND))) {
        PHEM_TRY(setup_kernels<KIND>(ctx));
        ctx->kernels_ready |= 1u << KIND;
    }
    RoundArgs a = make_args(ctx, plan);
    // light/heavy split: about light_per_vertex * n light edges, and only when
    // the input is at least filter_min_ratio times that large
    // the canonical forest's light edges are the first ones by index, which
    // start forming the large components only at about two per vertex
    const double lpv = KIND == kKindPacked ? ctx->tune_canonical_light : ctx->tune_light_per_vertex;
    const uint64_t k = (uint64_t)(lpv * (double)plan.n);
    const bool filter = lpv > 0 && k > 0 && (double)plan.m >= ctx->tune_filter_min_ratio * (double)k;
    a.light_k = filter ? k : plan.m;
    unsigned long long thr = kKeyNone;
    if (filter && KIND == kKindPacked)
        thr = k;  // canonical forest: the first k edges by index are light
    if (!ctx->profiling && ctx->tune_graph) {
        // the graph form (per-launch event timing needs the stream form)
        GraphKey key;
        std::memset(&key, 0, sizeof(key));
        key.a = a;
        key.thr = thr;
        key.k = k;
        key.select = filter && KIND == kKindMsf;
        key.ep_blocks = ctx->edge_pass_blocks;
        key.vb_init = vertex_blocks(ctx, plan.n);
        key.vb_comp = std::min(vertex_blocks(ctx, plan.n), ctx->sm_count * kCompressCtasPerSm);
        key.hook_blocks = ctx->sm_count * kHookCtasPerSm;
        key.kind = KIND;
        const bool cached = ctx->msf_exec[KIND] && std::memcmp(ctx->msf_key[KIND], &key, sizeof(key)) == 0;
        // a graph is built only for a solve seen twice in a row (same
        // buffers, sizes and grids): one-off shapes take the stream form
        // instead of paying for a graph they would use once
        const bool repeat = std::memcmp(ctx->msf_seen[KIND], &key, sizeof(key)) == 0;
        std::memcpy(ctx->msf_seen[KIND], &key, sizeof(key));
        if (!cached && !repeat)
            goto stream_form;
        if (!cached) {
            GraphKey old;
            std::memcpy(&old, ctx->msf_key[KIND], sizeof(old));
            if (ctx->msf_exec[KIND] && old.select != key.select) {
                cudaGraphExecDestroy(ctx->msf_exec[KIND]);
                ctx->msf_exec[KIND] = nullptr;
            }
            std::memset(ctx->msf_key[KIND], 0, sizeof(ctx->msf_key[KIND]));
            PHEM_TRY(build_graph<KIND>(ctx, plan, key, &ctx->msf_exec[KIND]));
            static_assert(sizeof(GraphKey) <= sizeof(ctx->msf_key[0]), "graph key storage");
            std::memcpy(ctx->msf_key[KIND], &key, sizeof(key));
        }
        PHEM_CUDA_TRY(cudaGraphLaunch(ctx->msf_exec[KIND], s));
        ctx->msf_graph_select = key.select;
        ctx->msf_graph_pending = true;
        if (deferred)
            return PHEM_OK;  // msf_finish waits and checks, after the caller queued more work
        return msf_finish(ctx, rounds_out);
    }
stream_form:
    PHEM_CUDA_TRY(cudaMemsetAsync(ctx->ctl, 0, sizeof(Ctl), s));
    PHEM_CUDA_TRY(cudaMemsetAsync(plan.bitmap, 0, ((plan.m + 31) / 32) * sizeof(uint32_t), s));
    PHEM_CUDA_TRY(cudaMemsetAsync(plan.chunk_cnt, 0, gather_chunks(plan.m) * sizeof(uint32_t), s));
    {
        KernelScope ks(ctx, kKInit);
        init_kernel<<<vertex_blocks(ctx, plan.n), kBlock, 0, s>>>(a, thr, 1);
    }
    if (filter && KIND == kKindMsf) {
        KernelScope ks(ctx, kKSelect);
        select_threshold_kernel<<<kSelectBlocks, kSelectThreads, 0, s>>>(static_cast<const uint32_t *>(plan.e0),
                                                                         plan.m, k, plan.samples, ctx->ctl);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    // Rounds are queued in batches; the host reads the continue flag between
    // batches.  Rounds queued after convergence return immediately.
    int queued = 0;
    int batch = ctx->tune_first_batch;
    while (queued < PHEM_MAX_ROUNDS) {
        for (int b = 0; b < batch && queued < PHEM_MAX_ROUNDS; b++, queued++)
            PHEM_TRY(queue_round<KIND>(ctx, a));
        PHEM_CUDA_TRY(cudaMemcpyAsync(&ctx->h_ctl->go, &ctx->ctl->go, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        PHEM_TRY(stream_wait(ctx));
        if (!*(volatile uint32_t *)&ctx->h_ctl->go)
            break;
        batch = ctx->tune_next_batch;
    }
    ctx->msf_graph_pending = false;
    if (deferred)
        return PHEM_OK;
    return msf_finish(ctx, rounds_out);
}

}  // namespace

phem_status msf_finish(phem_context *ctx, uint32_t *rounds_out)
{
    PHEM_CUDA_TRY(cudaMemcpyAsync(ctx->h_ctl, ctx->ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, ctx->stream));
    PHEM_TRY(stream_wait(ctx));
    const Ctl &h = *ctx->h_ctl;
    if (ctx->msf_graph_pending) {
        // launches the graph made: init, select, three per round
        ctx->launches[kKInit] += 1;
        ctx->launches[kKSelect] += ctx->msf_graph_select ? 1 : 0;
        ctx->launches[kKEdgePass] += h.round;
        ctx->launches[kKHook] += h.round;
        ctx->launches[kKCompress] += h.round;
        ctx->msf_graph_pending = false;
    }
    if (h.go)
        return ctl_status(h.err | kErrRounds, "msf");
    if (rounds_out)
        *rounds_out = h.round;
    return ctl_status(h.err, "msf");
}

// Records a survivor list may need: every edge, plus dead padding of at most
// one list chunk (2048 records) per edge-pass CTA (at most kEpMaxCtasPerSm
// per SM).
uint64_t wl_capacity(uint64_t m, int sm_count) { return m + (uint64_t)sm_count * kEpMaxCtasPerSm * 2048; }

// Workspace of one solve: parent (4n), best (8n), two candidate lists (4n
// each), the MSF bitmap (m / 8) and two survivor lists (16 bytes per record
// each).  The carve order is fixed;
// msf_plan repeats it.
size_t msf_workspace_bytes(uint64_t m, uint32_t n, int sm_count)
{
    Carve c;
    c.take<uint32_t>(n);
    c.take<unsigned long long>(n);
    c.take<uint32_t>(n);
    c.take<uint32_t>(kSample);
    c.take<uint32_t>((m + 31) / 32 + 4);
    c.take<uint32_t>(gather_words(m));
    c.take<uint4>(wl_capacity(m, sm_count));
    c.take<uint4>(wl_capacity(m, sm_count));
    return c.off;
}

phem_status msf_plan(phem_context *ctx, int kind, const void *d_e0, uint64_t m, uint32_t n, size_t extra_bytes,
                     MsfPlan *plan, size_t *extra_off)
{
    const size_t core = msf_workspace_bytes(m, n, ctx->sm_count);
    Carve c;
    c.off = core;
    const size_t extra_at = c.take<uint8_t>(extra_bytes);
    PHEM_TRY(ws_reserve(ctx, c.off));
    char *base = static_cast<char *>(ctx->ws);
    Carve k;
    plan->status = ctx->status;
    plan->parent = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(n));
    plan->best = reinterpret_cast<unsigned long long *>(base + k.take<unsigned long long>(n));
    plan->cand = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(n));
    plan->samples = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(kSample));
    plan->bitmap = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>((m + 31) / 32 + 4));
    plan->chunk_cnt = reinterpret_cast<uint32_t *>(base + k.take<uint32_t>(gather_words(m)));
    plan->wl[0] = reinterpret_cast<uint4 *>(base + k.take<uint4>(wl_capacity(m, ctx->sm_count)));
    plan->wl[1] = reinterpret_cast<uint4 *>(base + k.take<uint4>(wl_capacity(m, ctx->sm_count)));
    plan->e0 = d_e0;
    plan->m = m;
    plan->n = n;
    plan->forest = nullptr;
    plan->epoch_base = next_epochs(ctx, PHEM_MAX_ROUNDS + 4);
    (void)kind;
    if (extra_off)
        *extra_off = extra_at;
    return PHEM_OK;
}

phem_status msf_run(phem_context *ctx, int kind, MsfPlan &plan, uint32_t *rounds_out, bool deferred)
{
    if (kind == kKindMsf)
        return run_impl<kKindMsf>(ctx, plan, rounds_out, deferred);
    return run_impl<kKindPacked>(ctx, plan, rounds_out, deferred);
}

phem_status msf_gather(phem_context *ctx, MsfPlan &plan, phem_edge *d_out)
{
    const RoundArgs a = make_args(ctx, plan);
    const uint64_t chunks = gather_chunks(plan.m);
    {
        KernelScope k(ctx, kKGather);
        gather_scan_kernel<<<(unsigned)gather_tiles(plan.m), 1024, 0, ctx->stream>>>(plan.chunk_cnt,
                                                                                  gather_tiles(plan.m), ctx->ctl);
    }
    const uint64_t blocks_needed = (chunks + kGatherWarps - 1) / kGatherWarps;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(blocks_needed, (uint64_t)ctx->gather_blocks));
    {
        KernelScope k(ctx, kKGather);
        gather_kernel<<<blocks, kBlock, 0, ctx->stream>>>(a, d_out);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

}  // namespace phem
