// C ABI of the relightable-Gaussian tracer: validation, particle
// preparation (gpu/relight.rs:178-253), the host-built BVH and the
// dispatch (RelightTracer::new_gaussian / set_point_light / dispatch,
// gpu/relight.rs:313, :841-866, :905-934).  Host code only.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bv_internal.h"
#include "bv_relight.h"
#include "bv_tile_order.cuh"

// Relight tiles heaviest first by the previous dispatch's tile times (1) or
// in launch order (0).
#ifndef BV_RELIGHT_TILE_ORDER
#define BV_RELIGHT_TILE_ORDER 1
#endif

using namespace bv;

struct bv_relight_tracer {
    uint32_t n_input = 0;
    uint32_t n_kept = 0;
    uint32_t n_nodes = 0;
    uint32_t n_materials = 0;
    GaussPrim *prims = nullptr;
    float4 *local = nullptr;  // per-view camera-origin terms, refilled by each dispatch
    BvhNode *nodes = nullptr;
    RelightMaterial *materials = nullptr;
    unsigned long long *stats = nullptr;
    std::vector<RelightLight> lights;
    float background[3] = {0.f, 0.f, 0.f};
    bool stats_enabled = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool last_has_stats = false;
    // The per-view origin table is rewritten by every dispatch: a dispatch on
    // another stream than the previous one first waits for the previous one.
    cudaEvent_t done = nullptr;
    cudaStream_t last_stream = nullptr;
    bool dispatched = false;
    uint32_t last_launches = 0;
    TileScheduler tile_sched;  // heaviest-first tile order between dispatches
};

namespace {

bv_status rfail(bv_status code, const char *msg) {
    set_last_error(msg);
    return code;
}

void free_relight(bv_relight_tracer *t) {
    if (!t) return;
    cudaFree(t->prims);
    cudaFree(t->local);
    t->tile_sched.release();
    cudaFree(t->nodes);
    cudaFree(t->materials);
    cudaFree(t->stats);
    for (auto &e : t->ev)
        if (e) cudaEventDestroy(e);
    if (t->done) cudaEventDestroy(t->done);
    delete t;
}

inline bool finite3(const float *v) {
    return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

// PointCloudModel::validate, transforms and PBR parts (lib.rs:246-340).
bv_status validate_gaussians(const bv_gaussian_desc *g) {
    if (!g || !g->points || !g->rotations || !g->scales || !g->normals || !g->material_indices ||
        !g->materials)
        return rfail(BV_ERR_INVALID_MODEL, "Gaussian model arrays are required");
    if (g->num_points == 0) return rfail(BV_ERR_INVALID_MODEL, "model has no points");
    if (g->num_materials == 0)
        return rfail(BV_ERR_INVALID_MODEL, "PBR attributes require at least one material");
    for (uint32_t i = 0; i < g->num_points; ++i) {
        const float *p = g->points + 4 * (size_t)i;
        if (!finite3(p) || !std::isfinite(p[3]) || p[3] < 0.0f)
            return rfail(BV_ERR_INVALID_MODEL,
                         "points must have finite coordinates and non-negative opacity");
        const float *q = g->rotations + 4 * (size_t)i;
        const float ql = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (!finite3(q) || !std::isfinite(q[3]) || std::fabs(ql - 1.0f) > 1.0e-3f)
            return rfail(BV_ERR_INVALID_MODEL, "transform rotations must be finite and unit length");
        const float *s = g->scales + 3 * (size_t)i;
        if (!finite3(s) || std::min(std::min(s[0], s[1]), s[2]) <= 0.0f)
            return rfail(BV_ERR_INVALID_MODEL, "transform scales must be finite and positive");
        const float *n = g->normals + 3 * (size_t)i;
        const float nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (!finite3(n) || std::fabs(nl - 1.0f) > 1.0e-3f)
            return rfail(BV_ERR_INVALID_MODEL, "PBR normals must be finite and unit length");
        if (g->material_indices[i] >= g->num_materials)
            return rfail(BV_ERR_INVALID_MODEL, "PBR point refers to a missing material");
    }
    for (uint32_t m = 0; m < g->num_materials; ++m) {
        const bv_material &mt = g->materials[m];
        if (!std::isfinite(mt.roughness) || mt.roughness < 0.0f || mt.roughness > 1.0f ||
            !finite3(mt.albedo) || !finite3(mt.specular_f0))
            return rfail(BV_ERR_INVALID_MODEL,
                         "PBR materials must be finite with roughness in [0, 1]");
    }
    return BV_OK;
}

}  // namespace

extern "C" {

bv_status bv_relight_tracer_new_gaussian(const bv_gaussian_desc *g,
                                         const bv_relight_settings *settings,
                                         bv_relight_tracer **out) {
    if (!out) return rfail(BV_ERR_INVALID_ARGUMENT, "out handle pointer is null");
    *out = nullptr;
    bv_status st = validate_gaussians(g);
    if (st != BV_OK) return st;
    if (settings && settings->diffuse_samples != 0)
        return rfail(BV_ERR_NOT_SUPPORTED,
                     "visibility rays (diffuse_samples > 0) are not implemented on this path");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return rfail(BV_ERR_NO_DEVICE, "no CUDA device");

    // prepare_geometry (gpu/relight.rs:205-246): opacity > 0.03 only
    std::vector<GaussPrim> prims;
    std::vector<BvhBox> boxes;
    std::vector<float> centers;
    prims.reserve(g->num_points);
    boxes.reserve(g->num_points);
    uint32_t kept = 0;
    for (uint32_t i = 0; i < g->num_points; ++i) {
        const float *p = g->points + 4 * (size_t)i;
        if (p[3] <= 0.03f) continue;
        const float *q = g->rotations + 4 * (size_t)i;
        const float *s = g->scales + 3 * (size_t)i;
        const float *n = g->normals + 3 * (size_t)i;
        GaussPrim gp;
        gp.center_opacity = make_float4(p[0], p[1], p[2], p[3]);
        gp.qinv = make_float4(-q[0], -q[1], -q[2], q[3]);
        const float support_sq = 2.0f * logf(p[3] / 0.03f);
        gp.scale_support = make_float4(s[0], s[1], s[2], support_sq);
        gp.normal_radius = make_float4(n[0], n[1], n[2], 3.0f * cbrtf(s[0] * s[1] * s[2]));
        gp.ids = make_uint4(kept, g->material_indices[i], 0u, 0u);
        prims.push_back(gp);
        // conservative box of the support ellipsoid: half extent along world
        // axis k is support * |row k of R diag(s)|, inflated
        const double x = q[0], y = q[1], z = q[2], w = q[3];
        const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)},
                                {2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)},
                                {2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)}};
        const double sup = std::sqrt(std::max((double)support_sq, 0.0));
        BvhBox bx;
        for (int k = 0; k < 3; ++k) {
            double e2 = 0.0;
            for (int j = 0; j < 3; ++j) {
                const double a = R[k][j] * (double)s[j];
                e2 += a * a;
            }
            const double ext = sup * std::sqrt(e2) * (1.0 + 1e-4) + 1e-6 * (1.0 + std::fabs(p[k]));
            bx.lo[k] = std::nextafter((float)((double)p[k] - ext), -INFINITY);
            bx.hi[k] = std::nextafter((float)((double)p[k] + ext), INFINITY);
        }
        boxes.push_back(bx);
        centers.insert(centers.end(), {p[0], p[1], p[2]});
        kept += 1;
    }
    if (kept == 0)
        return rfail(BV_ERR_INVALID_MODEL, "PBR Gaussian geometry has no particles above alpha 0.03");

    // BVH over the support boxes, particles stored in leaf order
    BvhBuild bvh = build_bvh(boxes, centers, BvhMethod::kMorton);
    if (bvh_depth(bvh.nodes) >= (uint32_t)kRelightStack)
        return rfail(BV_ERR_NOT_SUPPORTED, "BVH deeper than the traversal stack");
    std::vector<GaussPrim> sorted_prims(kept);
    for (uint32_t i = 0; i < kept; ++i) sorted_prims[i] = prims[bvh.order[i]];

    bv_relight_tracer *t = new bv_relight_tracer();
    t->n_input = g->num_points;
    t->n_kept = kept;
    t->n_nodes = (uint32_t)bvh.nodes.size();
    t->n_materials = g->num_materials;
    std::vector<RelightMaterial> mats(g->num_materials);
    for (uint32_t m = 0; m < g->num_materials; ++m) {
        const bv_material &s = g->materials[m];
        mats[m].a = make_float4(s.albedo[0], s.albedo[1], s.albedo[2], s.roughness);
        mats[m].b = make_float4(s.specular_f0[0], s.specular_f0[1], s.specular_f0[2], 0.f);
    }
    auto cleanup = [&](cudaError_t e, const char *what) {
        free_relight(t);
        set_last_error(what);
        return e == cudaErrorMemoryAllocation ? BV_ERR_OUT_OF_MEMORY : BV_ERR_CUDA;
    };
#define BV_RTRY(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cleanup(e_, what); \
    } while (0)
    BV_RTRY(cudaMalloc(&t->prims, sizeof(GaussPrim) * kept), "cudaMalloc particles");
    BV_RTRY(cudaMalloc(&t->local, sizeof(float4) * kept), "cudaMalloc particle origin terms");
    BV_RTRY(cudaMalloc(&t->nodes, sizeof(BvhNode) * t->n_nodes), "cudaMalloc nodes");
    BV_RTRY(cudaMalloc(&t->materials, sizeof(RelightMaterial) * mats.size()), "cudaMalloc materials");
    BV_RTRY(cudaMalloc(&t->stats, sizeof(unsigned long long) * 4), "cudaMalloc stats");
    BV_RTRY(cudaMemcpy(t->prims, sorted_prims.data(), sizeof(GaussPrim) * kept, cudaMemcpyHostToDevice),
            "upload particles");
    BV_RTRY(cudaMemcpy(t->nodes, bvh.nodes.data(), sizeof(BvhNode) * t->n_nodes,
                       cudaMemcpyHostToDevice), "upload nodes");
    BV_RTRY(cudaMemcpy(t->materials, mats.data(), sizeof(RelightMaterial) * mats.size(),
                       cudaMemcpyHostToDevice), "upload materials");
    for (auto &e : t->ev) BV_RTRY(cudaEventCreate(&e), "cudaEventCreate");
    BV_RTRY(cudaEventCreateWithFlags(&t->done, cudaEventDisableTiming), "cudaEventCreate");
#undef BV_RTRY
    if (settings) std::memcpy(t->background, settings->background, sizeof(t->background));
    *out = t;
    return BV_OK;
}

void bv_relight_tracer_destroy(bv_relight_tracer *t) {
    if (!t) return;
    cudaDeviceSynchronize();
    free_relight(t);
}

bv_status bv_relight_tracer_set_point_lights(bv_relight_tracer *t, const bv_point_light *lights,
                                             uint32_t n_lights) {
    if (!t || (!lights && n_lights)) return rfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (n_lights > (uint32_t)kMaxRelightLights)
        return rfail(BV_ERR_INVALID_ARGUMENT, "at most 64 point lights per tracer");
    std::vector<RelightLight> ls(n_lights);
    for (uint32_t i = 0; i < n_lights; ++i) {
        const bv_point_light &L = lights[i];
        const float dl2 = L.direction[0] * L.direction[0] + L.direction[1] * L.direction[1] +
                          L.direction[2] * L.direction[2];
        // RelightTracer::set_point_light (gpu/relight.rs:841-866)
        if (!finite3(L.position) || !finite3(L.intensity) || L.intensity[0] < 0.f ||
            L.intensity[1] < 0.f || L.intensity[2] < 0.f || !std::isfinite(L.exponent) ||
            L.exponent < 0.f || (L.exponent != 0.f && !(dl2 > 1.1920929e-7f)))
            return rfail(BV_ERR_INVALID_ARGUMENT, "invalid point light");
        std::memcpy(ls[i].position, L.position, 12);
        std::memcpy(ls[i].intensity, L.intensity, 12);
        ls[i].exponent = L.exponent;
        if (L.exponent == 0.f) {
            ls[i].direction[0] = 0.f;
            ls[i].direction[1] = 0.f;
            ls[i].direction[2] = 1.f;
        } else {
            const float inv = 1.0f / std::sqrt(dl2);
            for (int k = 0; k < 3; ++k) ls[i].direction[k] = L.direction[k] * inv;
        }
    }
    t->lights = ls;
    return BV_OK;
}

bv_status bv_relight_tracer_set_background(bv_relight_tracer *t, const float rgb[3]) {
    if (!t || !rgb) return rfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::memcpy(t->background, rgb, sizeof(t->background));
    return BV_OK;
}

bv_status bv_relight_tracer_dispatch(bv_relight_tracer *t, float *out_rgba_dev,
                                     const bv_camera *c, uint32_t width, uint32_t height,
                                     bv_stream stream) {
    if (!t || !out_rgba_dev || !c) return rfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (width == 0 || height == 0)
        return rfail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (t->lights.empty())
        return rfail(BV_ERR_INVALID_ARGUMENT, "set at least one point light before dispatch");
    if (!finite3(c->cam_position) || !std::isfinite(c->depth) || !(c->depth > 0.f))
        return rfail(BV_ERR_INVALID_ARGUMENT, "camera must be finite with positive depth");
    RelightParams p;
    std::memset(&p, 0, sizeof(p));
    p.prims = t->prims;
    p.local = t->local;
    p.n_prims = t->n_kept;
    p.nodes = t->nodes;
    p.materials = t->materials;
    p.out = reinterpret_cast<float4 *>(out_rgba_dev);
    p.stats = t->stats_enabled ? t->stats : nullptr;
    for (int k = 0; k < 3; ++k) p.origin[k] = c->cam_position[k];
    p.depth = c->depth;
    for (int k = 0; k < 4; ++k) p.q[k] = c->cam_orientation[k];
    p.tan_half[0] = (float)std::tan((double)(0.5f * c->fov[0]));
    p.tan_half[1] = (float)std::tan((double)(0.5f * c->fov[1]));
    p.principal[0] = c->principal[0];
    p.principal[1] = c->principal[1];
    p.width = width;
    p.height = height;
    p.tiles_x = (width + 7) / 8;
    const uint64_t work = (uint64_t)p.tiles_x * ((height + 3) / 4) * 32u;
    if (work >= (1ull << 31)) return rfail(BV_ERR_INVALID_ARGUMENT, "image too large");
    p.total_work = (uint32_t)work;
    std::memcpy(p.background, t->background, sizeof(p.background));
    p.n_lights = (uint32_t)t->lights.size();
    std::memcpy(p.lights, t->lights.data(), sizeof(RelightLight) * t->lights.size());
    cudaStream_t s = (cudaStream_t)stream;
    t->last_has_stats = t->stats_enabled;
    if (t->stats_enabled) {
        if (cudaMemsetAsync(t->stats, 0, sizeof(unsigned long long) * 4, s) != cudaSuccess ||
            cudaEventRecord(t->ev[0], s) != cudaSuccess)
            return rfail(BV_ERR_CUDA, "stats setup failed");
    }
    if (t->dispatched && t->last_stream != s && cudaStreamWaitEvent(s, t->done, 0) != cudaSuccess)
        return rfail(BV_ERR_CUDA, "stream wait on the previous dispatch failed");
    uint32_t launches = 0;
    const size_t tiles = work / 32u;
    const bool time_tiles =
        t->tile_sched.begin(BV_RELIGHT_TILE_ORDER, tiles, 1, width, height, p.tile_order);
    p.tile_cost = time_tiles ? t->tile_sched.cost : nullptr;
    cudaError_t e = launch_relight(p, s, launches);
    if (e == cudaSuccess && time_tiles) {
        e = t->tile_sched.end(tiles, 1, width, height, s);
        launches += t->tile_sched.order_launches();
    }
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return BV_ERR_CUDA;
    }
    t->last_launches = launches;
    if (cudaEventRecord(t->done, s) != cudaSuccess) return rfail(BV_ERR_CUDA, "event record failed");
    t->last_stream = s;
    t->dispatched = true;
    if (t->stats_enabled && cudaEventRecord(t->ev[1], s) != cudaSuccess)
        return rfail(BV_ERR_CUDA, "event record failed");
    return BV_OK;
}

uint32_t bv_relight_tracer_num_particles(const bv_relight_tracer *t) { return t ? t->n_kept : 0; }

bv_status bv_relight_tracer_enable_stats(bv_relight_tracer *t, uint32_t enabled) {
    if (!t) return rfail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->stats_enabled = enabled != 0;
    return BV_OK;
}

bv_status bv_relight_tracer_last_stats(bv_relight_tracer *t, bv_launch_stats *out) {
    if (!t || !out) return rfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->launches = t->last_launches;  // origin terms, trace
    if (!t->last_has_stats) return BV_OK;
    if (cudaEventSynchronize(t->ev[1]) != cudaSuccess)
        return rfail(BV_ERR_CUDA, "event sync failed");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t->ev[0], t->ev[1]);
    out->kernel_ms = ms;
    unsigned long long h[4] = {0, 0, 0, 0};
    if (cudaMemcpy(h, t->stats, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
        return rfail(BV_ERR_CUDA, "stats read failed");
    out->rays = h[0];
    out->steps = h[1];  // composited hits
    out->faces = h[2];  // BVH nodes visited
    return BV_OK;
}

}  // extern "C"
