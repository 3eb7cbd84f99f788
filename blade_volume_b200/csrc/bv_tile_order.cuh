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



// The class of a tile time: floor(log2(cost)) >> shift (shift 0: classes a
// factor of 2 apart; larger shifts merge them, so that fewer, wider classes
// keep more tiles in launch order).
__device__ __forceinline__ uint32_t order_class(uint32_t cost, uint32_t shift = 0) {
    return (31u - (uint32_t)__clz(cost | 1u)) >> shift;
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

// The same order, stable: inside a class the tiles keep their launch order,
// so tiles that run at the same time stay neighbours on screen and share
// cache lines.  Block b of kOrderBlocks takes a contiguous range of tiles:
// pass 1 counts each class in each block, pass 2 (one warp) turns the counts
// into each (block, class) start, pass 3 ranks the tiles of a block within
// their class in order (a warp's tiles of one class through a match mask,
// the warps of a 1024-tile chunk through a per-class prefix).  `counts`
// holds kOrderBlocks x kOrderClasses words.
constexpr int kOrderBlocks = 148;
constexpr int kOrderThreads = 1024;

__device__ __forceinline__ void order_block_range(uint32_t tiles, uint32_t &lo, uint32_t &hi) {
    const uint32_t per = (tiles + gridDim.x - 1) / gridDim.x;
    lo = min(tiles, blockIdx.x * per);
    hi = min(tiles, lo + per);
}

__global__ void __launch_bounds__(kOrderThreads)
tile_class_count_kernel(const uint32_t *__restrict__ cost, uint32_t tiles, uint32_t shift,
                        uint32_t *__restrict__ counts) {
    __shared__ uint32_t h[kOrderClasses];
    if (threadIdx.x < kOrderClasses) h[threadIdx.x] = 0;
    __syncthreads();
    uint32_t lo, hi;
    order_block_range(tiles, lo, hi);
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x)
        atomicAdd(&h[order_class(cost[i], shift)], 1u);
    __syncthreads();
    if (threadIdx.x < kOrderClasses) counts[blockIdx.x * kOrderClasses + threadIdx.x] = h[threadIdx.x];
}

// One warp: lane c owns class c.  counts[b][c] becomes the first position
// of block b's tiles of class c (classes from the heaviest, 31, down).
__global__ void tile_class_offsets_kernel(uint32_t *__restrict__ counts, uint32_t blocks) {
    const uint32_t c = threadIdx.x;
    uint32_t total = 0;
    for (uint32_t b = 0; b < blocks; ++b) total += counts[b * kOrderClasses + c];
    // exclusive sum over the heavier classes c + 1 .. 31
    __shared__ uint32_t tot[kOrderClasses];
    tot[c] = total;
    __syncwarp();
    uint32_t above = 0;
    for (uint32_t k = c + 1; k < (uint32_t)kOrderClasses; ++k) above += tot[k];
    uint32_t run = above;
    for (uint32_t b = 0; b < blocks; ++b) {
        const uint32_t n = counts[b * kOrderClasses + c];
        counts[b * kOrderClasses + c] = run;
        run += n;
    }
}

__global__ void __launch_bounds__(kOrderThreads)
tile_class_scatter_kernel(const uint32_t *__restrict__ cost, uint32_t tiles, uint32_t shift,
                          const uint32_t *__restrict__ offsets, uint32_t *__restrict__ order) {
    __shared__ uint32_t next[kOrderClasses];                       // next free position per class
    __shared__ uint32_t warp_n[kOrderThreads / 32][kOrderClasses];  // class counts per warp
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x < kOrderClasses) next[threadIdx.x] = offsets[blockIdx.x * kOrderClasses + threadIdx.x];
    uint32_t lo, hi;
    order_block_range(tiles, lo, hi);
    for (uint32_t base = lo; base < hi; base += blockDim.x) {
        for (uint32_t k = threadIdx.x; k < (kOrderThreads / 32) * kOrderClasses; k += blockDim.x)
            (&warp_n[0][0])[k] = 0;
        __syncthreads();
        const uint32_t i = base + threadIdx.x;
        const bool have = i < hi;
        const uint32_t c = have ? order_class(cost[i], shift) : kOrderClasses;  // none
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
        if (have && rank == 0) warp_n[warp][c] = __popc(peers);
        __syncthreads();
        if (have) {
            uint32_t before = 0;  // this class's tiles in the chunk's earlier warps
            for (uint32_t v = 0; v < warp; ++v) before += warp_n[v][c];
            order[next[c] + before + rank] = i;
        }
        __syncthreads();
        if (threadIdx.x < kOrderClasses) {
            uint32_t n = 0;
            for (uint32_t v = 0; v < kOrderThreads / 32; ++v) n += warp_n[v][threadIdx.x];
            next[threadIdx.x] += n;
        }
        __syncthreads();
    }
}

// stable: the order above, or classes in the order the atomics give (tiles
// running at the same time then come from anywhere on screen, which spreads
// the walk replay's gradient atomics: measured faster there).  Three
// launches when stable, two otherwise.
cudaError_t launch_tile_order(const uint32_t *cost, uint32_t tiles, uint32_t *counts,
                              uint32_t *order, bool stable, uint32_t shift, cudaStream_t s) {
    if (stable) {
        tile_class_count_kernel<<<kOrderBlocks, kOrderThreads, 0, s>>>(cost, tiles, shift, counts);
        tile_class_offsets_kernel<<<1, 32, 0, s>>>(counts, kOrderBlocks);
        tile_class_scatter_kernel<<<kOrderBlocks, kOrderThreads, 0, s>>>(cost, tiles, shift, counts,
                                                                        order);
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(counts, 0, 2 * kOrderClasses * sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    const int blocks = (int)std::min<uint32_t>(296u, (tiles + 255u) / 256u);
    tile_cost_histogram_kernel<<<blocks, 256, 0, s>>>(cost, tiles, counts);
    tile_order_scatter_kernel<<<blocks, 256, 0, s>>>(cost, tiles, counts, order);
    return cudaGetLastError();
}

// Heaviest-first scheduling of one kind of launch from frame to frame: a
// launch times its tiles into `cost`, the order is
// built from those times after it, and the next launch of the same shape
// (views, width, height: the same tiles) takes its tiles in that order.
// Frames of a moving camera keep most of their heavy tiles where they were;
// the order changes no result, only when each tile starts.
struct TileScheduler {
    uint32_t *cost = nullptr, *order = nullptr, *counts = nullptr;
    size_t capacity = 0;
    uint32_t views = 0, width = 0, height = 0;
    bool valid = false;
    bool stable = true;  // launch order kept inside a cost class (launch_tile_order)
    // an optional second order from the same tile times (second_shift >= 0):
    // stable, classes floor(log2(cost)) >> second_shift
    int second_shift = -1;
    uint32_t *order2 = nullptr;

    uint32_t order_launches() const {
        return (stable ? 3u : 2u) + (second_shift >= 0 ? 3u : 0u);
    }

    void release() {
        cudaFree(cost);
        cudaFree(order);
        cudaFree(order2);
        cudaFree(counts);
        cost = order = order2 = counts = nullptr;
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
            if (cudaMalloc(&counts, kOrderBlocks * kOrderClasses * sizeof(uint32_t)) != cudaSuccess ||
                cudaMalloc(&cost, tiles * sizeof(uint32_t)) != cudaSuccess ||
                cudaMalloc(&order, tiles * sizeof(uint32_t)) != cudaSuccess ||
                (second_shift >= 0 &&
                 cudaMalloc(&order2, tiles * sizeof(uint32_t)) != cudaSuccess)) {
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
    // The second order for the next launch of the shape begin() was given
    // (null: launch order); call after begin().
    const uint32_t *second(const uint32_t *first) const { return first ? order2 : nullptr; }
    // After the launch (same stream): the order(s) for the next one.
    cudaError_t end(size_t tiles, uint32_t n_views, uint32_t w, uint32_t h, cudaStream_t s) {
        cudaError_t e = launch_tile_order(cost, (uint32_t)tiles, counts, order, stable, 0u, s);
        if (e == cudaSuccess && second_shift >= 0)
            e = launch_tile_order(cost, (uint32_t)tiles, counts, order2, true, (uint32_t)second_shift, s);
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
