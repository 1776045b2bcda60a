// csr.cu -- symmetrised CSR -> packed COO on sm_100a.
//
// csr_to_coo (CC/graph.cu:149-196) walks rows in order and emits (i << 32 | col)
// for every entry with i < col.  Here every entry is a thread item: a tile of
// kTile consecutive entries finds its row range once (binary search on the
// int64 offsets), each entry finds its row inside that range, and kept entries
// are written with the same stable single-pass compaction the MSF edge pass
// uses, so the output order (and therefore the edge numbering) is exactly the
// reference's.
#include <algorithm>

#include "internal.h"

namespace phem {
namespace {

// Largest row i in [lo, hi] with offsets[i] <= j (the row that holds entry j).
__device__ __forceinline__ int32_t row_of(const int64_t *offsets, int32_t lo, int32_t hi, int64_t j)
{
    while (lo < hi) {
        const int32_t mid = lo + (hi - lo + 1) / 2;
        if (__ldg(offsets + mid) <= j)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kBlock) csr_coo_kernel(const int64_t *offsets, const uint32_t *cols, int32_t n,
                                                         int64_t nnz, unsigned long long *out, uint64_t *status,
                                                         uint32_t epoch, Ctl *ctl)
{
    __shared__ uint32_t s_tile, s_base;
    __shared__ int32_t s_row0, s_row1;
    __shared__ uint32_t s_warp[kWarps + 1];
    const uint32_t ntiles = (uint32_t)((nnz + kTile - 1) / kTile);
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t t = atomicAdd(&ctl->out_ticket, 1u);
            s_tile = t;
            if (t < ntiles) {
                const int64_t first = (int64_t)t * kTile;
                const int64_t last = std::min<int64_t>(first + kTile, nnz) - 1;
                s_row0 = row_of(offsets, 0, n - 1, first);
                s_row1 = row_of(offsets, s_row0, n - 1, last);
            }
        }
        __syncthreads();
        const uint32_t t = s_tile;
        if (t >= ntiles)
            break;
        const int64_t base = (int64_t)t * kTile + (int64_t)threadIdx.x * kItems;
        unsigned long long rec[4];
        bool keep[4];
        uint32_t c = 0;
        int32_t row = s_row0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int64_t j = base + k;
            keep[k] = false;
            rec[k] = 0;
            if (j < nnz) {
                row = row_of(offsets, row, s_row1, j);
                const uint32_t col = __ldcs(cols + j);
                keep[k] = (int64_t)row < (int64_t)col;
                rec[k] = ((unsigned long long)(uint32_t)row << 32) | col;
            }
            c += keep[k];
        }
        uint32_t total;
        const uint32_t off = block_exclusive_scan(c, &total, s_warp);
        if (threadIdx.x < 32) {
            const uint32_t ex = lookback_exclusive(status, t, total, epoch, &ctl->err);
            if (threadIdx.x == 0) {
                s_base = ex;
                if (t == ntiles - 1)
                    ctl->misc[2] = (unsigned long long)ex + total;
            }
        }
        __syncthreads();
        uint32_t pos = s_base + off;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (keep[k]) {
                if (out)
                    out[pos] = rec[k];
                pos++;
            }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock) pack_records_kernel(const unsigned long long *pairs, const uint32_t *w,
                                                              uint64_t m, phem_edge *out)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
        const unsigned long long e = __ldcs(pairs + i);
        phem_edge r;
        r.u = (uint32_t)(e >> 32);
        r.v = (uint32_t)e;
        r.w = __ldcs(w + i);
        out[i] = r;
    }
}

}  // namespace

phem_status csr_launch_pack_records(phem_context *ctx, const uint64_t *pairs, const uint32_t *w, uint64_t m,
                                    phem_edge *out)
{
    if (!m)
        return PHEM_OK;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((m + kBlock - 1) / kBlock,
                                                                      (uint64_t)ctx->sm_count * 8));
    KernelScope k(ctx, kKPack);
    pack_records_kernel<<<blocks, kBlock, 0, ctx->stream>>>(reinterpret_cast<const unsigned long long *>(pairs), w,
                                                            m, out);
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

phem_status csr_launch_to_coo(phem_context *ctx, const int64_t *offsets, const uint32_t *cols, int32_t n,
                              int64_t nnz, uint64_t *out)
{
    if (nnz < 0 || (uint64_t)nnz >= (1ull << 32)) {
        set_error("csr: %lld entries (must be < 2^32)", (long long)nnz);
        return PHEM_ERR_INVALID;
    }
    const uint64_t tiles = ((uint64_t)nnz + kTile - 1) / kTile;
    PHEM_TRY(status_reserve(ctx, tiles + 2));
    PHEM_CUDA_TRY(cudaMemsetAsync(&ctx->ctl->out_ticket, 0, sizeof(uint32_t), ctx->stream));
    PHEM_CUDA_TRY(cudaMemsetAsync(&ctx->ctl->misc[2], 0, sizeof(unsigned long long), ctx->stream));
    const uint32_t epoch = (uint32_t)next_epochs(ctx, 1);
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(tiles, (uint64_t)ctx->sm_count * 4));
    if (tiles > 0 && n > 0) {
        KernelScope k(ctx, kKCsrCoo);
        csr_coo_kernel<<<blocks, kBlock, 0, ctx->stream>>>(offsets, cols, n, nnz,
                                                           reinterpret_cast<unsigned long long *>(out),
                                                           ctx->status, epoch, ctx->ctl);
    }
    PHEM_CUDA_TRY(cudaGetLastError());
    return PHEM_OK;
}

}  // namespace phem
