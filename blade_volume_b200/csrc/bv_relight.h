// Device layout and launch descriptor of the relightable-Gaussian tracer.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "blade_volume_b200.h"
#include "bv_bvh.h"

namespace bv {

// One prepared particle (gpu/relight.rs:178-253), in BVH leaf order, 80 B.
// The first three vectors are all the candidate test reads.
struct __align__(16) GaussPrim {
    float4 center_opacity;  // mean, opacity
    float4 qinv;            // inverse rotation (-x, -y, -z, w)
    float4 scale_support;   // scale, support^2 = 2 ln(opacity / 0.03)
    float4 normal_radius;   // PBR normal, surfel radius 3 cbrt(sx sy sz)
    uint4 ids;              // filtered index, material, 0, 0
};

struct RelightLight {  // PointLight (relight.rs:176-181)
    float position[3];
    float direction[3];  // unit, used when exponent != 0
    float intensity[3];
    float exponent;
};

struct __align__(16) RelightMaterial {  // Material (relight.rs:77-86)
    float4 a;  // albedo, roughness
    float4 b;  // specular_f0, pad
};

constexpr int kMaxRelightLights = 64;
// Traversal stack entries per ray; the BVH depth must stay below it.
constexpr int kRelightStack = 64;

// Per-view table of each particle's camera-origin terms (local origin and
// squared distance), formed once per dispatch instead of in every lane for
// every candidate test.
#ifndef BV_RELIGHT_LOCAL
#define BV_RELIGHT_LOCAL 1
#endif

struct RelightParams {
    const GaussPrim *prims;
    float4 *local;      // per table position, for this view's camera: R^-1 (o - mu) / s, |mu - o|^2
    uint32_t n_prims;
    const BvhNode *nodes;
    const RelightMaterial *materials;
    float4 *out;
    unsigned long long *stats;  // [3] rays, composited hits, nodes visited (or null)
    float origin[3];
    float depth;
    float q[4];
    float tan_half[2];
    float principal[2];
    uint32_t width, height, tiles_x, total_work;
    const uint32_t *tile_order;  // [tiles] tile of warp slot i, or null (bv_tile_order.cuh)
    uint32_t *tile_cost;         // [tiles] each tile's duration, or null
    float background[3];
    uint32_t n_lights;
    RelightLight lights[kMaxRelightLights];
};

// launches: kernels enqueued (the origin-term kernel is skipped for an empty
// scene, both for an empty image).
cudaError_t launch_relight(const RelightParams &p, cudaStream_t s, uint32_t &launches);

}  // namespace bv
