// csr.cu -- symmetrised CSR -> packed COO (or {u, v, w} records) on sm_100a.
//
// csr_to_coo (CC/graph.cu:149-196) walks rows in order and emits (i << 32 | col)
// for every entry with i < col.  Here the entries are cut into tiles of
// kCsrTile consecutive entries on a static grid-stride schedule (no block
// waits for another, so the loads of independent tiles overlap freely); a
// tile is kCsrWarps segments of 256 entries, one per warp, read lane-striped
// (step k of lane L holds entry 32k + L of the segment, so every load and
// store is one contiguous warp access):
//   1. csr_tile_rows_kernel, one thread per row, writes for every tile the row
//      that holds its first entry, so no tile searches the offsets;
//   2. csr_count_kernel marks, in shared memory, where each row inside the
//      tile starts (one coalesced pass over the tile's offsets) together with
//      the row each warp segment starts in; a warp then resolves the row of
//      every entry with one ballot per step (the latest mark at or before the
//      lane) and counts the entries with row < col;
//   3. csr_scan_kernel turns the tile counts into tile offsets: every block
//      scans a group of 4096 tiles and the last block to finish scans the
//      groups' totals (no block waits for another);
//   4. csr_write_kernel resolves the rows again and writes the kept entries in
//      order: group offset + tile offset + the warps before + the lanes before
//      (ballot).
// Every entry keeps its place in the reference's row walk, so the output order
// (and therefore the edge numbering) is exactly the reference's.  The record
// form fuses the MSF CSR input's packing: the kept entry at position p becomes
// {row, col, w[p]}.  Passes 2 and 4 load the next tile's columns and row
// range while they work on the current one.
#include <algorithm>

#include "internal.h"

namespace phem {
namespace {

constexpr int kCsrThreads = 256;                  // threads per block of passes 2 and 4
constexpr int kCsrWarps = kCsrThreads / 32;
constexpr int kCsrItems = 8;                      // entries per lane per tile
constexpr int kCsrSeg = 32 * kCsrItems;           // 256 entries per warp segment
constexpr int kCsrTile = kCsrWarps * kCsrSeg;     // 2048 entries per tile
constexpr int kCsrBlocksPerSm = 6;                // resident blocks per SM: 48 warps (registers <= 42)
constexpr int kScanBlock = 1024;
constexpr int kScanItems = 4;
constexpr int kScanGroup = kScanBlock * kScanItems;  // tiles per block of pass 3

// tile_rows[t] = the row i with offsets[i] <= t * kCsrTile < offsets[i + 1].
// Malformed offsets leave tiles unwritten; the conversion clamps what it reads.
__global__ void __launch_bounds__(kBlock) csr_tile_rows_kernel(const int64_t *offsets, int32_t n, uint32_t ntiles,
                                                               uint32_t *tile_rows)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int64_t a = std::max<int64_t>(__ldg(offsets + i), 0), b = __ldg(offsets + i + 1);
        if (a >= b)
            continue;
        const int64_t t1 = std::min<int64_t>((b - 1) / kCsrTile, (int64_t)ntiles - 1);
        for (int64_t t = (a + kCsrTile - 1) / kCsrTile; t <= t1; t++)
            tile_rows[t] = (uint32_t)i;
    }
}

// The columns of this lane's kCsrItems entries of tile t (lane-striped).
__device__ __forceinline__ void load_cols(const uint32_t *cols, int64_t nnz, uint32_t t, uint32_t ntiles,
                                          uint32_t (&c)[kCsrItems])
{
    if (t >= ntiles)
        return;
    const int64_t j0 = (int64_t)t * kCsrTile + (threadIdx.x >> 5) * kCsrSeg + lane_id();
#pragma unroll
    for (int k = 0; k < kCsrItems; k++)
        c[k] = j0 + 32 * k < nnz ? __ldcs(cols + j0 + 32 * k) : 0u;
}

// Thread 0: the row range of tile t into s_row[0..1] (the rows holding its
// first and its last entry, clamped to [0, n)).
__device__ __forceinline__ void load_row_range(const uint32_t *tile_rows, int32_t n, uint32_t t, uint32_t ntiles,
                                               int32_t *s_row)
{
    if (t >= ntiles)
        return;
    const int32_t r0 = (int32_t)min(__ldg(tile_rows + t), (uint32_t)(n - 1));
    const int32_t r1 = t + 1 < ntiles ? (int32_t)min(__ldg(tile_rows + t + 1), (uint32_t)(n - 1)) : n - 1;
    s_row[0] = r0;
    s_row[1] = max(r0, r1);
}

// Row marks of tile t: s_mark[o - first] = r for every non-empty row r that
// starts inside the tile, and s_seg[w] = the row holding the first entry of
// warp segment w when that row starts inside the tile (both stay 0 where the
// row is row0).
__device__ __forceinline__ void mark_rows(const int64_t *offsets, int64_t first, uint32_t len, int32_t row0,
                                          int32_t row1, uint32_t *s_mark, uint32_t *s_seg)
{
    for (int64_t r = (int64_t)row0 + 1 + threadIdx.x; r <= row1; r += kCsrThreads) {
        const int64_t o = __ldg(offsets + r);
        if (o >= first + len)
            break;
        const int64_t on = __ldg(offsets + r + 1);
        if (o > first && on > o) {
            s_mark[o - first] = (uint32_t)r;
            // warp segments whose first entry lies in [o, on)
            const int64_t lo = (o - first + kCsrSeg - 1) / kCsrSeg, hi = (on - 1 - first) / kCsrSeg;
            for (int64_t w = lo; w <= min(hi, (int64_t)kCsrWarps - 1); w++)
                s_seg[w] = (uint32_t)r;
        }
    }
}

// Rows of this lane's entries and their keep flags (bit k: entry k has
// row < col), after mark_rows and a __syncthreads.  Each lane zeroes the
// marks it reads (lane 0 its warp's segment row), so both are all zero again
// once every warp has returned.  *kept: the warp's kept entries.
__device__ __forceinline__ uint32_t resolve_rows(int64_t first, int64_t nnz, int32_t row0,
                                                 const uint32_t (&col)[kCsrItems], uint32_t (&row)[kCsrItems],
                                                 uint32_t *s_mark, uint32_t *s_seg, uint32_t *kept)
{
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t le = 0xffffffffu >> (31 - lane);  // lanes 0..lane
    const int64_t j0 = first + warp * kCsrSeg + lane;
    uint32_t *mk = s_mark + warp * kCsrSeg + lane;
    uint32_t carry = max(s_seg[warp], (uint32_t)row0), keep = 0;
    __syncwarp();
    if (lane == 0)
        s_seg[warp] = 0;
#pragma unroll
    for (int k = 0; k < kCsrItems; k++) {
        const uint32_t m = mk[32 * k];
        mk[32 * k] = 0;
        const uint32_t b = __ballot_sync(0xffffffffu, m != 0) & le;
        const uint32_t v = __shfl_sync(0xffffffffu, m, b ? 31 - __clz(b) : 0);
        row[k] = b ? v : carry;
        carry = __shfl_sync(0xffffffffu, row[k], 31);
        keep |= (uint32_t)(j0 + 32 * k < nnz && (int64_t)row[k] < (int64_t)col[k]) << k;
    }
    uint32_t n_kept = __popc(keep);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1)
        n_kept += __shfl_xor_sync(0xffffffffu, n_kept, d);
    *kept = n_kept;
    return keep;
}

// Pass 2: counts[t] += kept entries of tile t (counts zeroed beforehand).
__global__ void __launch_bounds__(kCsrThreads, kCsrBlocksPerSm)
    csr_count_kernel(const int64_t *offsets, const uint32_t *cols, int32_t n, int64_t nnz,
                     const uint32_t *tile_rows, uint32_t *counts)
{
    __shared__ uint32_t s_mark[kCsrTile];
    __shared__ uint32_t s_seg[kCsrWarps];
    __shared__ int32_t s_row[2][2];
    const uint32_t ntiles = (uint32_t)((nnz + kCsrTile - 1) / kCsrTile);
    for (uint32_t i = threadIdx.x; i < kCsrTile; i += kCsrThreads)
        s_mark[i] = 0;
    if (threadIdx.x < kCsrWarps)
        s_seg[threadIdx.x] = 0;
    uint32_t t = blockIdx.x;
    if (threadIdx.x == 0)
        load_row_range(tile_rows, n, t, ntiles, s_row[0]);
    uint32_t nc[kCsrItems];
    load_cols(cols, nnz, t, ntiles, nc);
    __syncthreads();
    for (int buf = 0; t < ntiles; t += gridDim.x, buf ^= 1) {
        uint32_t col[kCsrItems], row[kCsrItems], kept;
#pragma unroll
        for (int k = 0; k < kCsrItems; k++)
            col[k] = nc[k];
        const int32_t row0 = s_row[buf][0], row1 = s_row[buf][1];
        const uint32_t tn = t + gridDim.x;
        if (threadIdx.x == 0)
            load_row_range(tile_rows, n, tn, ntiles, s_row[buf ^ 1]);
        load_cols(cols, nnz, tn, ntiles, nc);  // in flight while this tile resolves
        const int64_t first = (int64_t)t * kCsrTile;
        const uint32_t len = (uint32_t)min((int64_t)kCsrTile, nnz - first);
        mark_rows(offsets, first, len, row0, row1, s_mark, s_seg);
        __syncthreads();
        resolve_rows(first, nnz, row0, col, row, s_mark, s_seg, &kept);
        if (lane_id() == 0 && kept)
            atomicAdd(counts + t, kept);
        __syncthreads();  // marks read (and zeroed) before the next tile writes them
    }
}

// Pass 3: prefix[t] = kept entries before tile t within its group of
// kScanGroup tiles (one block per group, kScanItems tiles per thread); the
// last block to finish scans the group totals into group_off[] and writes
// the whole count to *kept.
__global__ void __launch_bounds__(kScanBlock) csr_scan_kernel(const uint32_t *counts, uint32_t ntiles,
                                                              uint32_t *prefix, uint32_t *group_tot,
                                                              uint32_t *group_off, unsigned long long *kept,
                                                              unsigned long long *ticket)
{
    __shared__ uint32_t s_w[kScanBlock / 32 + 1];
    __shared__ bool s_last;
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    // exclusive scan of one value per thread over the block; *total = the sum
    auto block_scan = [&](uint32_t x, uint32_t *total) {
        uint32_t inc = x;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= (uint32_t)d)
                inc += y;
        }
        if (lane == 31)
            s_w[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const uint32_t a = s_w[lane];
            uint32_t z = a;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
                if (lane >= (uint32_t)d)
                    z += y;
            }
            s_w[lane] = z - a;
            if (lane == 31)
                s_w[32] = z;
        }
        __syncthreads();
        *total = s_w[32];
        const uint32_t r = s_w[warp] + inc - x;
        __syncthreads();  // s_w is reused
        return r;
    };
    const uint64_t i0 = (uint64_t)blockIdx.x * kScanGroup + (uint64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems], sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = i0 + k < ntiles ? counts[i0 + k] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t run = block_scan(sum, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (i0 + k < ntiles) {
            prefix[i0 + k] = run;
            run += v[k];
        }
    if (threadIdx.x == 0) {
        group_tot[blockIdx.x] = total;
        __threadfence();
        s_last = atomicAdd(ticket, 1ull) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    if (threadIdx.x == 0)
        *ticket = 0;
    uint64_t carry = 0;
    for (uint32_t g0 = 0; g0 < gridDim.x; g0 += kScanBlock) {
        const uint32_t g = g0 + threadIdx.x;
        const uint32_t x = g < gridDim.x ? __ldcg(group_tot + g) : 0u;
        uint32_t s;
        const uint32_t ex = block_scan(x, &s);
        if (g < gridDim.x)
            group_off[g] = (uint32_t)carry + ex;
        carry += s;
    }
    if (threadIdx.x == 0)
        *kept = carry;
}

// Pass 4.  RECORDS: write {row, col, w[p]} to rec_out[p] for p < cap;
// otherwise packed pairs to out.
template <bool RECORDS>
__global__ void __launch_bounds__(kCsrThreads, kCsrBlocksPerSm)
    csr_write_kernel(const int64_t *offsets, const uint32_t *cols, int32_t n, int64_t nnz,
                     const uint32_t *tile_rows, const uint32_t *prefix, const uint32_t *group_off,
                     unsigned long long *out, const uint32_t *w, phem_edge *rec_out, uint64_t cap)
{
    __shared__ uint32_t s_mark[kCsrTile];
    __shared__ uint32_t s_seg[kCsrWarps];
    __shared__ uint32_t s_wsum[kCsrWarps];
    __shared__ int32_t s_row[2][2];
    const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;  // lanes before this one
    const uint32_t ntiles = (uint32_t)((nnz + kCsrTile - 1) / kCsrTile);
    for (uint32_t i = threadIdx.x; i < kCsrTile; i += kCsrThreads)
        s_mark[i] = 0;
    if (threadIdx.x < kCsrWarps)
        s_seg[threadIdx.x] = 0;
    uint32_t t = blockIdx.x;
    if (threadIdx.x == 0)
        load_row_range(tile_rows, n, t, ntiles, s_row[0]);
    uint32_t nc[kCsrItems];
    load_cols(cols, nnz, t, ntiles, nc);
    __syncthreads();
    for (int buf = 0; t < ntiles; t += gridDim.x, buf ^= 1) {
        uint32_t col[kCsrItems], row[kCsrItems], kept;
#pragma unroll
        for (int k = 0; k < kCsrItems; k++)
            col[k] = nc[k];
        const int32_t row0 = s_row[buf][0], row1 = s_row[buf][1];
        const uint32_t base = __ldg(prefix + t) + __ldg(group_off + t / kScanGroup);
        const uint32_t tn = t + gridDim.x;
        if (threadIdx.x == 0)
            load_row_range(tile_rows, n, tn, ntiles, s_row[buf ^ 1]);
        load_cols(cols, nnz, tn, ntiles, nc);  // in flight while this tile resolves
        const int64_t first = (int64_t)t * kCsrTile;
        const uint32_t len = (uint32_t)min((int64_t)kCsrTile, nnz - first);
        mark_rows(offsets, first, len, row0, row1, s_mark, s_seg);
        __syncthreads();
        const uint32_t keep = resolve_rows(first, nnz, row0, col, row, s_mark, s_seg, &kept);
        if (lane == 0)
            s_wsum[warp] = kept;
        __syncthreads();  // also: every mark is read (and zeroed) before the next tile writes them
        uint64_t pos = base;
        for (uint32_t k = 0; k < warp; k++)
            pos += s_wsum[k];
#pragma unroll
        for (int k = 0; k < kCsrItems; k++) {
            const bool kp = keep >> k & 1;
            const uint32_t b = __ballot_sync(0xffffffffu, kp);
            if (kp) {
                const uint64_t q = pos + __popc(b & lt);
                if (RECORDS) {
                    if (q < cap) {
                        phem_edge rc;
                        rc.u = row[k];
                        rc.v = col[k];
                        rc.w = __ldcs(w + q);
                        rec_out[q] = rc;
                    }
                } else {
                    out[q] = ((unsigned long long)row[k] << 32) | col[k];
                }
            }
            pos += __popc(b);
        }
        // No barrier here: s_wsum is rewritten only after the next tile's
        // first barrier, which every warp reaches after reading it.
    }
}

}  // namespace

size_t csr_scratch_bytes(int64_t nnz)
{
    const size_t tiles = (size_t)((nnz + kCsrTile - 1) / kCsrTile);
    const size_t groups = (tiles + kScanGroup - 1) / kScanGroup;
    return align256((3 * tiles + 1 + 2 * groups) * sizeof(uint32_t));
}

phem_status csr_launch_to_coo(phem_context *ctx, const int64_t *offsets, const uint32_t *cols, int32_t n,
                              int64_t nnz, uint32_t *scratch, uint64_t *out, const uint32_t *w, phem_edge *records,
                              uint64_t cap)
{
    if (nnz < 0 || (uint64_t)nnz >= (1ull << 32)) {
        set_error("csr: %lld entries (must be < 2^32)", (long long)nnz);
        return PHEM_ERR_INVALID;
    }
    const uint64_t tiles = ((uint64_t)nnz + kCsrTile - 1) / kCsrTile;
    if (tiles == 0 || n <= 0) {
        PHEM_CUDA_TRY(cudaMemsetAsync(&ctx->ctl->misc[2], 0, sizeof(unsigned long long), ctx->stream));
        return PHEM_OK;
    }
    const uint64_t groups = (tiles + kScanGroup - 1) / kScanGroup;
    uint32_t *tile_rows = scratch, *counts = scratch + tiles + 1, *prefix = counts + tiles;
    uint32_t *group_tot = prefix + tiles, *group_off = group_tot + groups;
    const int blocks = (int)std::min<uint64_t>(tiles, (uint64_t)ctx->sm_count * kCsrBlocksPerSm);
    {
        KernelScope k(ctx, kKCsrCoo);
        const int rblocks = (int)std::max<int64_t>(1, std::min<int64_t>(((int64_t)n + kBlock - 1) / kBlock,
                                                                         (int64_t)ctx->sm_count * 8));
        csr_tile_rows_kernel<<<rblocks, kBlock, 0, ctx->stream>>>(offsets, n, (uint32_t)tiles, tile_rows);
    }
    PHEM_CUDA_TRY(cudaMemsetAsync(counts, 0, tiles * sizeof(uint32_t), ctx->stream));
    {
        KernelScope k(ctx, kKCsrCoo);
        csr_count_kernel<<<blocks, kCsrThreads, 0, ctx->stream>>>(offsets, cols, n, nnz, tile_rows, counts);
    }
    PHEM_CUDA_TRY(cudaMemsetAsync(&ctx->ctl->misc[3], 0, sizeof(unsigned long long), ctx->stream));  // scan ticket
    {
        KernelScope k(ctx, kKCsrCoo);
        csr_scan_kernel<<<(unsigned)groups, kScanBlock, 0, ctx->stream>>>(counts, (uint32_t)tiles, prefix, group_tot,
                                                                         group_off, &ctx->ctl->misc[2],
                                                                         &ctx->ctl->misc[3]);
    }
    if (records || out) {
        KernelScope k(ctx, kKCsrCoo);
        auto *o = reinterpret_cast<unsigned long long *>(out);
        (records ? csr_write_kernel<true> : csr_write_kernel<false>)<<<blocks, kCsrThreads, 0, ctx->stream>>>(
            offsets, cols, n, nnz, tile_rows, prefix, group_off, o, w, records, cap);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

}  // namespace phem
