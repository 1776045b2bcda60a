// noalloc.cu -- connected components + spanning forest without allocating.
//
// phem_cc_solve_noalloc runs phem_cc_solve's union-find (the same union
// steps, uf.cuh, and the same prefix / compress / rest schedule), so its
// labels and forest mean the same (the reference's
// init_parent_label_T1edges + union_find_gpu_COO + cc,
// CC/ExternalSpanningTree.cu:77-116, CC/GPUSpanningTree.cu:122-128), with its
// parent array in a fixed-size file-scope device array instead of a context
// workspace.  It exists for callers that cannot allocate device memory when
// they need a solve:
//   * a serving process whose device memory is already committed to resident
//     state and memory pools under a budget: a cudaMalloc there fails, or
//     takes memory that the budget has promised to someone else;
//   * latency-critical loops: cudaMalloc and cudaFree may synchronise the
//     whole device, stalling every other stream of the process;
//   * code that must not create a phem_context, which allocates its control
//     block, workspace, streams and events.
// Nothing here calls cudaMalloc, cudaFree or any allocating library routine.
//
// Rules a caller must follow:
//   * n <= PHEM_CC_NOALLOC_MAX_VERTICES (2^20).  The scratch is 4 MiB of
//     parent words plus one status word, reserved when the CUDA module of this
//     file is loaded; larger n is rejected with PHEM_ERR_INVALID.
//   * Every call looks the scratch address up with the call's device current
//     (cudaGetSymbolAddress: a table lookup, no allocation), so an address is
//     never carried over from an earlier CUDA context of that device (after a
//     cudaDeviceReset, or under a different driver context).  The first call
//     on a device also loads this file's module.
//   * Every call on one device uses the same scratch.  Calls that overlap in
//     time (two host threads, or two streams with work in flight at once)
//     race on it and corrupt each other's results; serialise them.
//   * The status word must start at zero; the init kernel clears it at the
//     start of every call, before any other kernel of the call can set it.
#include <cuda_runtime.h>

#include "internal.h"
#include "uf.cuh"

namespace phem {
namespace {

constexpr int32_t kNoallocMaxVertices = PHEM_CC_NOALLOC_MAX_VERTICES;

static_assert(kNoallocMaxVertices == (1 << 20), "scratch size is part of the documented limit");

// The scratch: union-find parents and one status word (error bits).
static __device__ __align__(256) int32_t g_noalloc_parent[kNoallocMaxVertices];
static __device__ __align__(256) uint32_t g_noalloc_status;

__global__ void __launch_bounds__(kBlock) na_init_kernel(int32_t n, int32_t *parent, unsigned long long *forest,
                                                         uint32_t *status)
{
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *status = 0;
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        parent[i] = i;
        if (forest)
            forest[i] = kForestEmpty;
    }
}

// Two packed edges per 128-bit streaming load (edges 16-byte aligned), the
// odd last edge alone; the union is phem_cc_solve's (uf.cuh).
__global__ void __launch_bounds__(kBlock) na_unite_kernel(const unsigned long long *edges, int64_t m, int32_t n,
                                                          int32_t *parent, unsigned long long *forest,
                                                          uint32_t *status)
{
    const int64_t pairs = m / 2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const uint4 *q = reinterpret_cast<const uint4 *>(edges);
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < pairs; g += stride) {
        const uint4 a = __ldcs(q + g);
        unite_packed(parent, forest, ((unsigned long long)a.y << 32) | a.x, n, status);
        unite_packed(parent, forest, ((unsigned long long)a.w << 32) | a.z, n, status);
    }
    if ((m & 1) && blockIdx.x == 0 && threadIdx.x == 0)
        unite_packed(parent, forest, __ldcs(edges + m - 1), n, status);
}

// Every vertex pointed at its root, so the next unions settle most edges
// with two loads.
__global__ void __launch_bounds__(kBlock) na_compress_kernel(int32_t n, int32_t *parent, uint32_t *status)
{
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const int32_t r = uf_find<true>(parent, i, n, status);
        if (parent[i] != r)
            parent[i] = r;
    }
}

// label[i] = root(i), which is the smallest id of i's component.
__global__ void __launch_bounds__(kBlock) na_label_kernel(int32_t n, int32_t *parent, int32_t *label,
                                                          uint32_t *status)
{
    const int32_t stride = gridDim.x * blockDim.x;
    for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        label[i] = uf_find<false>(parent, i, n, status);
}

struct NoallocScratch {
    int32_t *parent = nullptr;
    uint32_t *status = nullptr;
};

// Scratch addresses in the CUDA context current on this thread (the call's
// device), looked up on every call.
phem_status noalloc_scratch(NoallocScratch *out)
{
    void *parent = nullptr, *status = nullptr;
    PHEM_CUDA_TRY(cudaGetSymbolAddress(&parent, g_noalloc_parent));
    PHEM_CUDA_TRY(cudaGetSymbolAddress(&status, g_noalloc_status));
    out->parent = static_cast<int32_t *>(parent);
    out->status = static_cast<uint32_t *>(status);
    return PHEM_OK;
}

// True when p is device or managed memory that device `dev` owns.
bool on_device(const void *p, int dev)
{
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) && attr.device == dev;
}

int na_grid(int sm_count, int64_t work)
{
    const int64_t blocks = (work + kBlock - 1) / kBlock;
    const int64_t cap = (int64_t)sm_count * 8;
    return (int)(blocks < 1 ? 1 : (blocks < cap ? blocks : cap));
}

}  // namespace
}  // namespace phem

using namespace phem;

extern "C" phem_status phem_cc_solve_noalloc(const uint64_t *d_edges, int64_t m, int32_t n, int32_t *d_labels,
                                             uint64_t *d_forest, void *stream)
{
    if (n <= 0 || n > kNoallocMaxVertices) {
        set_error("cc_solve_noalloc: n = %d is outside [1, %d], the size of the fixed scratch "
                  "(use phem_cc_solve for larger graphs)", n, kNoallocMaxVertices);
        return PHEM_ERR_INVALID;
    }
    if (m < 0 || (m > 0 && !d_edges) || !d_labels) {
        set_error("cc_solve_noalloc: need m >= 0, device edges when m > 0, and device labels");
        return PHEM_ERR_INVALID;
    }
    int dev = 0, sm_count = 0;
    PHEM_CUDA_TRY(cudaGetDevice(&dev));
    PHEM_CUDA_TRY(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev));
    if ((m > 0 && (!on_device(d_edges, dev) || ((uintptr_t)d_edges & 15))) || !on_device(d_labels, dev) ||
        (d_forest && !on_device(d_forest, dev))) {
        set_error("cc_solve_noalloc: edges (16-byte aligned), labels and forest must be memory of the "
                  "current device %d", dev);
        return PHEM_ERR_INVALID;
    }
    NoallocScratch s;
    PHEM_TRY(noalloc_scratch(&s));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long *forest = reinterpret_cast<unsigned long long *>(d_forest);

    na_init_kernel<<<na_grid(sm_count, n), kBlock, 0, st>>>(n, s.parent, forest, s.status);
    PHEM_CUDA_TRY(cudaGetLastError());
    // phem_cc_solve's schedule: a prefix of about one edge per vertex builds
    // the big components, a compress points every vertex at its root, then
    // the rest of the edges (an even prefix keeps the rest 16-byte aligned)
    const unsigned long long *e = reinterpret_cast<const unsigned long long *>(d_edges);
    const int64_t pre = m > n ? (int64_t)n & ~int64_t(1) : m;
    if (pre > 0) {
        na_unite_kernel<<<na_grid(sm_count, (pre + 1) / 2), kBlock, 0, st>>>(e, pre, n, s.parent, forest, s.status);
        PHEM_CUDA_TRY(cudaGetLastError());
    }
    if (pre < m) {
        na_compress_kernel<<<na_grid(sm_count, n), kBlock, 0, st>>>(n, s.parent, s.status);
        na_unite_kernel<<<na_grid(sm_count, (m - pre + 1) / 2), kBlock, 0, st>>>(e + pre, m - pre, n, s.parent,
                                                                                 forest, s.status);
        PHEM_CUDA_TRY(cudaGetLastError());
    }
    na_label_kernel<<<na_grid(sm_count, n), kBlock, 0, st>>>(n, s.parent, d_labels, s.status);
    PHEM_CUDA_TRY(cudaGetLastError());
    uint32_t status = 0;
    PHEM_CUDA_TRY(cudaMemcpyAsync(&status, s.status, sizeof(status), cudaMemcpyDeviceToHost, st));
    PHEM_CUDA_TRY(cudaStreamSynchronize(st));
    return ctl_status(status, "cc_solve_noalloc");
}
