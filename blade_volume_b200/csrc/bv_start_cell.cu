// Start-cell location on the device: the site whose power cell contains a
// query point, argmin_i |q - p_i|^2 - r_i^2 with ties to the lowest index.
//
// The reference finds it on the host with a kiddo kd-tree in FP32
// (blade-volume/src/gpu/radfoam.rs:77-112, lib.rs:526-541).  Here every site
// is scored in FP64 (the differences and squares of FP32 inputs are exact in
// FP64), which makes the choice exact except for true ties.  Compiled with
// -fmad=false so the FP64 expression is the same sequence of rounded
// operations as the CPU check.
//
// One launch handles up to kMaxStartQueries queries: blockIdx.y selects the
// query, each block reduces a slice of the sites to (distance, index), and
// the last block of each query (ticket counter) reduces the per-block
// partials and re-arms the counter for the next launch.

#include <cfloat>

#include "bv_internal.h"

namespace bv {
namespace {

constexpr int kStartBlock = 256;
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ bool better(double d, uint32_t i, double bd, uint32_t bi) {
    return d < bd || (d == bd && i < bi);
}

__device__ __forceinline__ void warp_argmin(double &d, uint32_t &i) {
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) {
        const double od = __shfl_xor_sync(kFull, d, s);
        const uint32_t oi = __shfl_xor_sync(kFull, i, s);
        if (better(od, oi, d, i)) {
            d = od;
            i = oi;
        }
    }
}

__device__ __forceinline__ void block_argmin(double &d, uint32_t &i) {
    __shared__ double sd[kStartBlock / 32];
    __shared__ uint32_t si[kStartBlock / 32];
    warp_argmin(d, i);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        sd[warp] = d;
        si[warp] = i;
    }
    __syncthreads();
    if (warp == 0) {
        d = lane < kStartBlock / 32 ? sd[lane] : DBL_MAX;
        i = lane < kStartBlock / 32 ? si[lane] : 0xffffffffu;
        warp_argmin(d, i);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kStartBlock)
start_cell_kernel(const float4 *__restrict__ geom, uint32_t n,
                  const __grid_constant__ StartCellQueries Q, double *partial_dist,
                  uint32_t *partial_index, uint32_t *counters, uint32_t *out) {
    const uint32_t q = blockIdx.y;
    const double qx = Q.position[q][0], qy = Q.position[q][1], qz = Q.position[q][2];
    double best = DBL_MAX;
    uint32_t best_i = 0xffffffffu;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float4 g = __ldg(geom + i);
        const double dx = qx - (double)g.x;
        const double dy = qy - (double)g.y;
        const double dz = qz - (double)g.z;
        const double r = (double)g.w;
        const double dist = (dx * dx + dy * dy + dz * dz) - r * r;
        if (dist < best) {  // i increases per thread: strict < keeps the lowest
            best = dist;
            best_i = i;
        }
    }
    block_argmin(best, best_i);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        partial_dist[q * gridDim.x + blockIdx.x] = best;
        partial_index[q * gridDim.x + blockIdx.x] = best_i;
        __threadfence();
        const uint32_t ticket = atomicAdd(counters + q, 1u);
        last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double d = DBL_MAX;
    uint32_t i = 0xffffffffu;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const double od = __ldcg(partial_dist + q * gridDim.x + b);
        const uint32_t oi = __ldcg(partial_index + q * gridDim.x + b);
        if (better(od, oi, d, i)) {
            d = od;
            i = oi;
        }
    }
    block_argmin(d, i);
    if (threadIdx.x == 0) {
        out[q] = i == 0xffffffffu ? 0u : i;
        counters[q] = 0u;
    }
}

// Start cells of a served batch: blockIdx.y strides over the frames of the
// batch (the frame count is read from the device table, so the grid is
// fixed and the launch can live in a captured graph); kServeStartBlocks
// blocks search each frame's scene.  Same scoring and tie rule as above.
__global__ void __launch_bounds__(kStartBlock) serve_start_cells_kernel(const __grid_constant__ ServeParams P) {
    const uint32_t n_views = P.header->n_views;
    __shared__ bool last;
    for (uint32_t v = blockIdx.y; v < n_views; v += gridDim.y) {
        ServeView *sv = P.views + v;
        const uint32_t scene = sv->scene;
        const float4 *geom = P.scenes[scene].geom;
        const uint32_t n = P.scenes[scene].n;
        const double qx = sv->v.origin[0], qy = sv->v.origin[1], qz = sv->v.origin[2];
        double best = DBL_MAX;
        uint32_t best_i = 0xffffffffu;
        const uint32_t stride = gridDim.x * blockDim.x;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const float4 g = __ldg(geom + i);
            const double dx = qx - (double)g.x;
            const double dy = qy - (double)g.y;
            const double dz = qz - (double)g.z;
            const double r = (double)g.w;
            const double dist = (dx * dx + dy * dy + dz * dz) - r * r;
            if (dist < best) {
                best = dist;
                best_i = i;
            }
        }
        block_argmin(best, best_i);
        double *pd = P.partial_dist + (size_t)v * gridDim.x;
        uint32_t *pi = P.partial_index + (size_t)v * gridDim.x;
        if (threadIdx.x == 0) {
            pd[blockIdx.x] = best;
            pi[blockIdx.x] = best_i;
            __threadfence();
            last = atomicAdd(P.counters + v, 1u) == gridDim.x - 1;
        }
        __syncthreads();
        if (last) {
            __threadfence();
            double d = DBL_MAX;
            uint32_t i = 0xffffffffu;
            for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
                const double od = __ldcg(pd + b);
                const uint32_t oi = __ldcg(pi + b);
                if (better(od, oi, d, i)) {
                    d = od;
                    i = oi;
                }
            }
            block_argmin(d, i);
            if (threadIdx.x == 0) {
                sv->start_cell = i == 0xffffffffu ? 0u : i;
                P.counters[v] = 0u;
            }
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_serve_start_cells(const ServeParams &p, cudaStream_t s) {
    dim3 grid(kServeStartBlocks, kServeStartRows);
    serve_start_cells_kernel<<<grid, kStartBlock, 0, s>>>(p);
    return cudaGetLastError();
}

int start_cell_blocks(uint32_t n) {
    const uint32_t per_block = kStartBlock * 8u;
    uint32_t b = (n + per_block - 1) / per_block;
    if (b < 1) b = 1;
    if (b > 296) b = 296;
    return (int)b;
}

cudaError_t launch_start_cells(const float4 *geom, uint32_t n, const StartCellQueries &queries,
                               const StartCellScratch &scratch, uint32_t *out, cudaStream_t s) {
    if (queries.count == 0) return cudaSuccess;
    if (queries.count > (uint32_t)kMaxStartQueries) return cudaErrorInvalidValue;
    dim3 grid((unsigned)scratch.blocks_per_query, queries.count);
    start_cell_kernel<<<grid, kStartBlock, 0, s>>>(geom, n, queries, scratch.partial_dist,
                                                   scratch.partial_index, scratch.counters, out);
    return cudaGetLastError();
}

}  // namespace bv
