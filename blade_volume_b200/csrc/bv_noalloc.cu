// Allocation-free variant of the start-cell search (power-nearest site of a
// set of query points), for callers that cannot call cudaMalloc.
//
// Some hosts own every byte of device memory through their own pool: a
// renderer that carves all buffers out of one frame arena, a framework whose
// caching allocator holds the GPU's memory, an embedding under a hard memory
// budget.  cudaMalloc/cudaFree behind such a pool's back would break its
// accounting, and both calls may synchronise the device in the middle of a
// frame.  bv_containing_points_noalloc() therefore allocates nothing: the
// caller passes the site table and the output array, and the per-block
// partial results and ticket counters that the search needs live in the
// fixed-size device array below, which every GPU that loads this library
// holds until the process exits.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "bv_internal.h"

namespace {

using namespace bv;

// Largest blocks-per-query start_cell_blocks() ever returns.
constexpr int kNoAllocMaxBlocks = 296;

struct NoAllocScratch {
    double partial_dist[kMaxStartQueries * kNoAllocMaxBlocks];
    uint32_t partial_index[kMaxStartQueries * kNoAllocMaxBlocks];
    uint32_t counters[kMaxStartQueries];
};

// 113,792 bytes per device.  In host code `g_noalloc_scratch` is only a
// host-side stand-in for the symbol: the device address comes from
// cudaGetSymbolAddress() in noalloc_scratch_for_current_device().
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
// Per device: the context the address was looked up in, and the address.  A
// cudaDeviceReset (or a primary context torn down and made again) loads the
// module anew, and the array may then sit elsewhere, so the address is only
// reused while the current context is the one it was looked up in.
struct NoAllocSlot {
    CUcontext ctx;
    NoAllocScratch *ptr;
};
NoAllocSlot g_noalloc_slot[kMaxDevices] = {};
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
CtxGetCurrentFn g_ctx_get_current = nullptr;

bv_status noalloc_fail(bv_status code, const std::string &msg) {
    set_last_error(msg.c_str());  // read back through bv_last_error()
    return code;
}

// Once per device and context, with that device current: look up the device
// address of the scratch array.
bv_status noalloc_scratch_for_current_device(NoAllocScratch **out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return noalloc_fail(BV_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices)
        return noalloc_fail(BV_ERR_NOT_SUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_ctx_get_current) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return noalloc_fail(BV_ERR_CUDA, "cuCtxGetCurrent is not available from the driver");
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
    }
    // The context the launch will use: the thread's current one, or, when
    // the runtime has not made one current yet, the device's primary
    // context (cudaSetDevice initialises it and makes it current).
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS)
        return noalloc_fail(BV_ERR_CUDA, "cuCtxGetCurrent failed");
    if (!ctx) {
        e = cudaSetDevice(device);
        if (e != cudaSuccess)
            return noalloc_fail(BV_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
        if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx)
            return noalloc_fail(BV_ERR_CUDA, "no current CUDA context");
    }
    NoAllocSlot &slot = g_noalloc_slot[device];
    if (!slot.ptr || slot.ctx != ctx) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            return noalloc_fail(BV_ERR_CUDA,
                                std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        slot.ctx = ctx;
        slot.ptr = static_cast<NoAllocScratch *>(ptr);
    }
    *out = slot.ptr;
    return BV_OK;
}

}  // namespace

extern "C" {

bv_status bv_containing_points_noalloc(const float *sites_dev, uint32_t num_sites,
                                       const float *positions, uint32_t n_queries,
                                       uint32_t *out_index_dev, bv_stream stream) {
    if (!sites_dev || !positions || !out_index_dev)
        return noalloc_fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (num_sites == 0) return noalloc_fail(BV_ERR_INVALID_ARGUMENT, "no sites");
    if (n_queries == 0) return BV_OK;
    if (n_queries > (uint32_t)kMaxStartQueries)
        return noalloc_fail(BV_ERR_INVALID_ARGUMENT,
                            "bv_containing_points_noalloc takes at most 32 queries per call");
    if ((reinterpret_cast<uintptr_t>(sites_dev) & 15u) != 0)
        return noalloc_fail(BV_ERR_INVALID_ARGUMENT, "sites_dev must be 16-byte aligned");
    const int blocks = start_cell_blocks(num_sites);
    if (blocks > kNoAllocMaxBlocks)
        return noalloc_fail(BV_ERR_INVALID_ARGUMENT, "site count exceeds the scratch capacity");
    StartCellQueries q;
    std::memset(&q, 0, sizeof(q));
    q.count = n_queries;
    for (uint32_t i = 0; i < n_queries; ++i)
        for (int k = 0; k < 3; ++k) q.position[i][k] = positions[3 * i + k];
    NoAllocScratch *scratch = nullptr;
    bv_status st = noalloc_scratch_for_current_device(&scratch);
    if (st != BV_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // The ticket counters must start at zero; the partials are written before
    // they are read.  The array keeps the last call's contents otherwise.
    cudaError_t e = cudaMemsetAsync(scratch->counters, 0, sizeof(scratch->counters), s);
    if (e != cudaSuccess)
        return noalloc_fail(BV_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    StartCellScratch sc{scratch->partial_dist, scratch->partial_index, scratch->counters, blocks};
    e = launch_start_cells(reinterpret_cast<const float4 *>(sites_dev), num_sites, q, sc,
                           out_index_dev, s);
    if (e != cudaSuccess)
        return noalloc_fail(BV_ERR_CUDA, std::string("start-cell launch: ") + cudaGetErrorString(e));
    return BV_OK;
}

}  // extern "C"
