// Heaviest-first tile scheduling shared by the BVH tracers (splat render and
// training, SH Gaussians, relight).  A warp traces one 8x4 tile; tile costs
// span orders of magnitude (rays through a dense core against rays that
// leave the scene), and a heavy tile that starts in a launch's last wave
// runs alone.  A launch therefore records each tile's duration, two small
// kernels order the tiles heaviest first, and the next launch of the same
// shape takes them in that order.  Every per-ray index follows from the
// tile a warp is given, so the order changes no result.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "bv_internal.h"

namespace bv {
namespace {

// The work item of thread `slot`: its warp slot's tile (tile_order, a
// permutation of the launch's tiles, or the slot itself) and its lane.
// Every per-ray and per-tile index (pixel, ray state, interval record)
// follows from it, so the order tiles are taken in changes no result.
__device__ __forceinline__ uint32_t tile_item(const uint32_t *order, uint32_t slot) {
    return order ? (__ldg(order + (slot >> 5)) << 5) | (slot & 31u) : slot;
}

constexpr uint32_t kNoTile = 0xffffffffu;

// Lane 0 of a warp stores its tile's duration since `begin` (clock64).
__device__ __forceinline__ void store_tile_cost(uint32_t *cost, uint32_t w, long long begin) {
    if (cost && (threadIdx.x & 31u) == 0) {
        const unsigned long long d = (unsigned long long)(clock64() - begin) >> 6;
        cost[w >> 5] = d > 0xffffffffull ? 0xffffffffu : (uint32_t)d;
    }
}

// Heaviest-first tile order from a launch's tile durations: tiles go to
// 32 classes by floor(log2(cost)) and the classes are laid out from the
// heaviest down (the order inside a class is whatever the atomics give).
// counts[0..31] per class, counts[32..63] the classes' fill cursors, both
// zero on entry.
constexpr int kOrderClasses = 32;

__device__ __forceinline__ uint32_t order_class(uint32_t cost) {
    return 31u - (uint32_t)__clz(cost | 1u);
}

__global__ void tile_cost_histogram_kernel(const uint32_t *__restrict__ cost, uint32_t tiles,
                                           uint32_t *__restrict__ counts) {
    __shared__ uint32_t h[kOrderClasses];
    if (threadIdx.x < kOrderClasses) h[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < tiles; i += gridDim.x * blockDim.x)
        atomicAdd(&h[order_class(cost[i])], 1u);
    __syncthreads();
    if (threadIdx.x < kOrderClasses && h[threadIdx.x]) atomicAdd(&counts[threadIdx.x], h[threadIdx.x]);
}

__global__ void tile_order_scatter_kernel(const uint32_t *__restrict__ cost, uint32_t tiles,
                                          uint32_t *__restrict__ counts,
                                          uint32_t *__restrict__ order) {
    __shared__ uint32_t start[kOrderClasses];
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int c = kOrderClasses - 1; c >= 0; --c) {
            start[c] = acc;
            acc += counts[c];
        }
    }
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < tiles; i += gridDim.x * blockDim.x) {
        const uint32_t c = order_class(cost[i]);
        order[start[c] + atomicAdd(&counts[kOrderClasses + c], 1u)] = i;
    }
}

cudaError_t launch_tile_order(const uint32_t *cost, uint32_t tiles, uint32_t *counts,
                              uint32_t *order, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(counts, 0, 2 * kOrderClasses * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    const int blocks = (int)std::min<uint32_t>(296u, (tiles + 255u) / 256u);
    tile_cost_histogram_kernel<<<blocks, 256, 0, s>>>(cost, tiles, counts);
    tile_order_scatter_kernel<<<blocks, 256, 0, s>>>(cost, tiles, counts, order);
    return cudaGetLastError();
}

// Heaviest-first scheduling of one kind of launch from frame to frame: a launch times its tiles into `cost`, the order is
// built from those times after it, and the next launch of the same shape
// (views, width, height: the same tiles) takes its tiles in that order.
// Frames of a moving camera keep most of their heavy tiles where they were;
// the order changes no result, only when each tile starts.
struct TileScheduler {
    uint32_t *cost = nullptr, *order = nullptr, *counts = nullptr;
    size_t capacity = 0;
    uint32_t views = 0, width = 0, height = 0;
    bool valid = false;

    void release() {
        cudaFree(cost);
        cudaFree(order);
        cudaFree(counts);
        cost = order = counts = nullptr;
        capacity = 0;
        valid = false;
    }
    // Before a launch of `tiles` tiles: whether it times them (buffers to
    // hand) and the order to take them in (null: launch order).
    bool begin(bool enabled, size_t tiles, uint32_t n_views, uint32_t w, uint32_t h,
               const uint32_t *&use) {
        use = nullptr;
        if (!enabled || n_views > (uint32_t)kMaxViewsPerLaunch) return false;
        if (tiles > capacity) {
            release();
            if (cudaMalloc(&counts, 2 * kOrderClasses * sizeof(uint32_t)) != cudaSuccess ||
                cudaMalloc(&cost, tiles * sizeof(uint32_t)) != cudaSuccess ||
                cudaMalloc(&order, tiles * sizeof(uint32_t)) != cudaSuccess) {
                (void)cudaGetLastError();  // no room: launch order
                release();
                return false;
            }
            capacity = tiles;
        }
        if (valid && views == n_views && width == w && height == h) use = order;
        valid = false;
        return true;
    }
    // After the launch (same stream): the order for the next one.
    cudaError_t end(size_t tiles, uint32_t n_views, uint32_t w, uint32_t h, cudaStream_t s) {
        const cudaError_t e = launch_tile_order(cost, (uint32_t)tiles, counts, order, s);
        if (e != cudaSuccess) return e;
        views = n_views;
        width = w;
        height = h;
        valid = true;
        return cudaSuccess;
    }
};


}  // namespace
}  // namespace bv
