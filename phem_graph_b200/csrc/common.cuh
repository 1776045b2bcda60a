// common.cuh -- device helpers shared by the CC and MSF kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/phem.h"

namespace phem {

// ---------------------------------------------------------------- status word
// Kernels never trap: a failed check sets a bit here and the host maps it to a
// phem_status after the solve.
enum : uint32_t {
    kErrRange = 1u << 0,        // an endpoint >= n
    kErrChase = 1u << 1,        // a root walk exceeded its bound
    kErrRetry = 1u << 2,        // a union retried more than its bound
    kErrLookback = 1u << 3,     // a look-back wait exceeded its bound
    kErrRounds = 1u << 4,       // Boruvka ran out of rounds
    kErrCapacity = 1u << 5,     // an output exceeded its capacity
};

constexpr uint64_t kKeyNone = ~0ull;           // "no candidate edge" (w = id = all ones)
constexpr uint64_t kForestEmpty = 0x7fffffffull;
constexpr int kBlock = 256;                    // threads per block for the streaming kernels
constexpr int kWarps = kBlock / 32;
constexpr int kItems = 4;                      // records per thread per tile
constexpr int kTile = kBlock * kItems;         // records per tile
constexpr uint32_t kUnionRetryCap = 1u << 16;  // CAS retries per union
constexpr uint32_t kLookbackSpinCap = 1u << 20; // waits per look-back window (~1 s)

// ---------------------------------------------------------------- device control block
// Small per-context device structure, zeroed at the start of each solve.
struct Ctl {
    uint32_t err;
    uint32_t round;                                  // device-side round counter
    uint32_t go;                                     // 1 while another round is needed
    uint32_t phase;                                  // 0: light edges, 1: heavy edges
    uint32_t src;                                    // input of this round's edge pass (kSrc*)
    uint32_t cand_all;                               // this round's candidates are all n vertices
    uint32_t light_rounds;                           // rounds spent in the light phase
    uint32_t pad0;
    unsigned long long threshold;                    // light edge <=> key < threshold
    unsigned long long m_r[PHEM_MAX_ROUNDS + 1];     // live edges entering round r (exact)
    unsigned long long wl_len[PHEM_MAX_ROUNDS + 1];  // records written by round r's edge pass,
                                                     // including dead padding at chunk tails
    unsigned long long n_r[PHEM_MAX_ROUNDS + 1];     // components with a live edge in round r
    uint32_t roots[PHEM_MAX_ROUNDS + 2];             // |candidate roots| entering round r
    uint32_t ticket[PHEM_MAX_ROUNDS + 2];            // tile tickets of the round's edge pass
    uint32_t out_ticket;                             // tile tickets of the output gather
    uint32_t pad1;
    unsigned long long msf_count;
    unsigned long long msf_total;
    unsigned long long misc[8];
};

// Input of an edge pass.
enum : uint32_t {
    kSrcLight = 0,  // the caller's edges, keeping key < threshold; endpoints are their own roots
    kSrcList = 1,   // the previous round's survivor records
    kSrcHeavy = 2,  // the caller's edges, keeping key >= threshold; endpoints relabelled by parent[]
};

// ---------------------------------------------------------------- memory helpers
__device__ __forceinline__ uint32_t ld_cg(const uint32_t *p) { return __ldcg(p); }
__device__ __forceinline__ int32_t ld_cg(const int32_t *p) { return __ldcg(p); }
__device__ __forceinline__ uint64_t ld_cg(const uint64_t *p)
{
    return (uint64_t)__ldcg(reinterpret_cast<const unsigned long long *>(p));
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t *p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t *p, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void set_err(uint32_t *err, uint32_t bit) { atomicOr(err, bit); }

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

// ---------------------------------------------------------------- warp-aggregated minimum
// Lanes with valid == true offer `key` to slot best[target]; lanes sharing a
// target are reduced first (__match_any_sync groups them; the 64-bit key is
// reduced as (high word, then low word among lanes holding the minimum high
// word) with __reduce_min_sync), then one guarded atomicMin per group.  Every
// lane of the warp must call this with the warp converged.
__device__ __forceinline__ void warp_min_to(unsigned long long *best, uint32_t target, uint64_t key,
                                            bool valid)
{
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (!valid)
        return;
    const unsigned peers = __match_any_sync(active, target);
    const uint32_t hi = (uint32_t)(key >> 32), lo = (uint32_t)key;
    const uint32_t mhi = __reduce_min_sync(peers, hi);
    const uint32_t mlo = __reduce_min_sync(peers, hi == mhi ? lo : 0xffffffffu);
    if ((int)lane_id() == __ffs(peers) - 1) {
        const unsigned long long k = ((unsigned long long)mhi << 32) | mlo;
        if (k < __ldcg(best + target))
            atomicMin(best + target, k);
    }
}


// ---------------------------------------------------------------- block scan
// Exclusive scan of one uint32 per thread over a kBlock-thread block.
// Returns the thread's exclusive prefix; *total gets the block sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *total, uint32_t *s_warp)
{
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d)
            x += y;
    }
    if (lane == 31)
        s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (uint32_t)kWarps ? s_warp[lane] : 0;
        uint32_t ws = w;
#pragma unroll
        for (int d = 1; d < kWarps; d <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, ws, d);
            if (lane >= (uint32_t)d)
                ws += y;
        }
        if (lane < (uint32_t)kWarps)
            s_warp[lane] = ws - w;  // exclusive warp offsets
        if (lane == kWarps - 1)
            s_warp[kWarps] = ws;  // block total
    }
    __syncthreads();
    *total = s_warp[kWarps];
    return s_warp[warp] + x - v;
}

// ---------------------------------------------------------------- decoupled look-back
// Single-pass stable prefix over tiles (Merrill & Garland, "Single-pass
// parallel prefix scan with decoupled look-back", 2016).  Tiles are numbered
// by a ticket taken when a block starts the tile, so every predecessor of a
// tile is already owned by a running block and the wait always ends; it is
// still bounded and reports kErrLookback if it does not.
//
// Status word per tile: bits 63..62 flag (1 = aggregate, 2 = inclusive prefix),
// bits 61..32 epoch (a word from an older launch never matches), bits 31..0
// value.  Called by warp 0 of the block; returns the tile's exclusive prefix.
constexpr uint64_t kFlagAgg = 1ull << 62, kFlagIncl = 2ull << 62;

__device__ __forceinline__ uint64_t lb_word(uint64_t flag, uint32_t epoch, uint32_t value)
{
    return flag | ((uint64_t)(epoch & 0x3fffffffu) << 32) | value;
}

// First half: publish the tile's aggregate (tile 0 publishes its inclusive
// prefix at once).  One lane calls it.
__device__ __forceinline__ void lookback_publish(uint64_t *status, uint32_t tile, uint32_t agg, uint32_t epoch)
{
    st_relaxed_u64(status + tile, lb_word(tile == 0 ? kFlagIncl : kFlagAgg, epoch, agg));
}

// Second half: wait for the predecessors, publish the inclusive prefix and
// return the exclusive one.  The whole warp calls it, after the publish.
__device__ __forceinline__ uint32_t lookback_resolve(uint64_t *status, uint32_t tile, uint32_t agg, uint32_t epoch,
                                                     uint32_t *err)
{
    const uint32_t lane = lane_id();
    if (tile == 0)
        return 0;
    const uint32_t ep = epoch & 0x3fffffffu;
    uint32_t excl = 0;
    int64_t top = (int64_t)tile - 1;  // nearest predecessor not yet folded in
    uint32_t spins = 0;
    while (top >= 0) {
        const int64_t idx = top - (int64_t)lane;
        uint64_t w = 0;
        bool ready;
        if (idx >= 0) {
            w = ld_relaxed_u64(status + idx);
            ready = ((uint32_t)(w >> 32) & 0x3fffffffu) == ep && (w >> 62) != 0;
        } else {
            w = kFlagIncl;  // before tile 0: inclusive prefix 0
            ready = true;
        }
        const bool incl = ready && (w >> 62) == 2;
        const unsigned incl_mask = __ballot_sync(0xffffffffu, incl);
        // lanes up to and including the nearest inclusive prefix must be ready
        const unsigned need = incl_mask ? ((incl_mask & (0u - incl_mask)) << 1) - 1 : 0xffffffffu;
        const unsigned ready_mask = __ballot_sync(0xffffffffu, ready);
        if ((ready_mask & need) != need) {
            // give up at the cap, or at once when another block already gave up
            bool give_up = ++spins > kLookbackSpinCap;
            if (!give_up && (spins & 255) == 0)
                give_up = (*(volatile uint32_t *)err & kErrLookback) != 0;
            if (give_up) {
                if (lane == 0)
                    set_err(err, kErrLookback);
                break;
            }
            __nanosleep(20);
            continue;
        }
        uint32_t v = ((need >> lane) & 1u) ? (uint32_t)w : 0u;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, d);
        excl += v;
        if (incl_mask)
            break;
        top -= 32;
    }
    if (lane == 0)
        st_relaxed_u64(status + tile, lb_word(kFlagIncl, epoch, excl + agg));
    return excl;
}

// Both halves back to back (warp-wide).
__device__ __forceinline__ uint32_t lookback_exclusive(uint64_t *status, uint32_t tile, uint32_t agg,
                                                       uint32_t epoch, uint32_t *err)
{
    if (lane_id() == 0)
        lookback_publish(status, tile, agg, epoch);
    __syncwarp();
    return lookback_resolve(status, tile, agg, epoch, err);
}

// Grid size for the persistent streaming kernels: whole waves over 148 SMs.
inline int persistent_blocks(int sm_count, int blocks_per_sm) { return sm_count * blocks_per_sm; }

// ---------------------------------------------------------------- bulk copies (TMA, sm_90+)
// 1-D cp.async.bulk global -> shared with mbarrier completion.  Plain loads
// only: no cluster multicast anywhere in this library.
constexpr uint32_t kMbarSpinCap = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders earlier generic-proxy accesses of shared memory before later
// async-proxy writes to it (a stage is refilled only after it was read).
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// L2 policy for data read once (streamed inputs): evict first, so the
// streams do not push small, reused arrays (parent, best) out of L2.
__device__ __forceinline__ uint64_t l2_evict_first()
{
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
    return policy;
}

// bulk_copy_g2s with an L2 cache policy for the source.
__device__ __forceinline__ void bulk_copy_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                                   uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of a barrier; false (and kErrLookback set)
// when the cap is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t *err)
{
    for (uint32_t i = 0; i < kMbarSpinCap; i++)
        if (mbar_try_wait(bar, parity))
            return true;
    set_err(err, kErrLookback);
    return false;
}

}  // namespace phem
