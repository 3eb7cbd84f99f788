// Gaussian ray tracing with SH colour on sm_100a: per ray, every particle
// whose maximum response along the ray reaches min_opacity, composited
// front to back in strict (depth, index) order until the transmittance
// falls to min_transmittance.
//
// Restates trace_gaussians (blade-volume/src/trace.rs:695-773), the CPU
// oracle of the reference's hardware-ray-query tracer
// (shaders/gaussian_trace.wgsl:66-177 under shaders/gaussian.wgsl), with the
// local ray formed as the shader forms it (qrot of the inverse rotation,
// then a per-axis division by the scale, gaussian_trace.wgsl:147-151).
// Candidates come from a BVH over the support ellipsoids (the proxies of
// gpu/gaussian.rs:175-200 scale the unit sphere by sqrt(2 ln(opacity /
// min_opacity))), gathered in windows of kWindow keys (bv_window.cuh).
//
// Host side: GaussianGpuCloud::new (gpu/gaussian.rs:94-280) — validation,
// the opacity filter, the particle table in BVH leaf order — and the draw
// pass as one dispatch per camera.
//
// Compiled with -fmad=false: the arithmetic is the CPU oracle's, operation
// for operation, so images are bit-identical to it.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "bv_device.cuh"
#include "bv_internal.h"
#include "bv_tile_order.cuh"
#include "bv_window.cuh"

namespace bv {
namespace {

constexpr int kGaussBlock = 128;
// resident blocks per SM requested from the register allocator
// Tiles heaviest first by the previous dispatch's tile times (1) or in
// launch order (0).
#ifndef BV_GAUSS_TILE_ORDER
#define BV_GAUSS_TILE_ORDER 1
#endif
#ifndef BV_MINB_GAUSS
#define BV_MINB_GAUSS 4
#endif
// Per-view table of each particle's camera-origin terms (local origin and
// squared distance), formed once per dispatch instead of in every lane for
// every candidate test.
#ifndef BV_GAUSS_LOCAL
#define BV_GAUSS_LOCAL 1
#endif
// Window keys per lane, in registers (BV_GAUSS_SMEM_WINDOW 0) or in dynamic
// shared memory (1).  Measured (1M particles, 1024 x 768): 16 keys in
// registers 91.4 Mrays/s (128 registers), in shared memory 16 / 20 / 24 /
// 28 / 32 keys 95.0 / 104.9-106.9 / 104.7-105.4 / 98.0 / 96.8 (96 registers; 24
// keys make most rays one pass over the BVH, 416 -> 355 nodes per ray).
#ifndef BV_GAUSS_WINDOW
#define BV_GAUSS_WINDOW 24
#endif
#ifndef BV_GAUSS_SMEM_WINDOW
#define BV_GAUSS_SMEM_WINDOW 1
#endif
constexpr int kWindow = BV_GAUSS_WINDOW;
constexpr int kStack = 64;
// Each window's hits evaluated (alpha and SH colour) spread over the warp in
// rounds of BV_GAUSS_SPREAD_KEYS keys per lane, then composited by their own
// lane in order (1), or each lane evaluates its own hits (0).  Measured: 105.5
// Mrays/s in place, 106.2 / 107.0 spread with 24 / 20 keys: the hits are a
// small part of this kernel (25.6 of 32 lanes already active; the traversal
// is the rest), so the relight tracer's gain does not carry over.
#ifndef BV_GAUSS_SPREAD
#define BV_GAUSS_SPREAD 0
#endif
#ifndef BV_GAUSS_SPREAD_KEYS
#define BV_GAUSS_SPREAD_KEYS 4
#endif
#if BV_GAUSS_SPREAD
constexpr int kGSpread = BV_GAUSS_SPREAD_KEYS;
#endif

// One particle in BVH leaf order, 48 B: all a candidate test reads.
struct __align__(16) GaussShPrim {
    float4 center_opacity;  // mean, opacity
    float4 qinv;            // inverse rotation (-x, -y, -z, w)
    float4 scale_cut;       // scale, |local hit|^2 bound past which alpha < min_opacity
};

struct GaussianParams {
    const GaussShPrim *prims;
    const float4 *local;  // per table position, for this view's camera: R^-1 (o - mu) / s, |mu - o|^2
    const uint32_t *ids;  // filtered model index per table position
    const BvhNode *nodes;
    const float *sh;      // [n][sh_stride] in table order
    float4 *out;
    unsigned long long *stats;  // [3] rays, composited hits, nodes visited (or null)
    uint32_t sh_stride;
    float origin[3];
    float depth;
    float q[4];
    float tan_half[2];
    float principal[2];
    uint32_t width, height, tiles_x, total_work;
    const uint32_t *tile_order;  // [tiles] tile of warp slot i, or null (bv_tile_order.cuh)
    uint32_t *tile_cost;         // [tiles] each tile's duration, or null
    float min_opacity, min_transmittance;
    float background[3];
};

__device__ __forceinline__ float gdot(float ax, float ay, float az, float bx, float by, float bz) {
    return ax * bx + ay * by + az * bz;
}

// qrot (common.wgsl:386-390)
__device__ __forceinline__ float3 gqrot(float4 q, float vx, float vy, float vz) {
    const float t0 = 2.0f * (q.y * vz - q.z * vy);
    const float t1 = 2.0f * (q.z * vx - q.x * vz);
    const float t2 = 2.0f * (q.x * vy - q.y * vx);
    return make_float3((vx + q.w * t0) + (q.y * t2 - q.z * t1),
                       (vy + q.w * t1) + (q.z * t0 - q.x * t2),
                       (vz + q.w * t2) + (q.x * t1 - q.y * t0));
}

// Conservative pre-test: a hit lies inside the support ellipsoid, so within
// sqrt(cut) * max(scale) of the mean; rays passing farther from the mean than
// that (with a margin for the rounding of |oc|^2 - b^2) cannot hit.  d is unit.
__device__ __forceinline__ bool support_sphere_hit(const float4 &co, const float4 &sc,
                                                   const float4 &local, const WinRay &r) {
    const float ox = co.x - r.ox, oy = co.y - r.oy, oz = co.z - r.oz;
    const float b = gdot(ox, oy, oz, r.dx, r.dy, r.dz);
#if BV_GAUSS_LOCAL
    const float oo = local.w;
#else
    (void)local;
    const float oo = gdot(ox, oy, oz, ox, oy, oz);
#endif
    const float smax = fmaxf(fmaxf(sc.x, sc.y), sc.z);
    const float r2 = sc.w * (smax * smax);
    return oo - b * b <= r2 * 1.001f + 1e-6f * oo + 1e-30f;
}

// Maximum-response depth and alpha (trace.rs:731-747); false when the
// depth is outside (0, t_end) or alpha < min_opacity.
__device__ __forceinline__ bool response(const GaussianParams &P, uint32_t pos, const WinRay &r,
                                         float &t_out, float &alpha_out) {
    const float4 co = __ldg(&P.prims[pos].center_opacity);
    const float4 sc = __ldg(&P.prims[pos].scale_cut);
#if BV_GAUSS_LOCAL
    const float4 local = __ldg(&P.local[pos]);
#else
    const float4 local = make_float4(0.f, 0.f, 0.f, 0.f);
#endif
    if (!support_sphere_hit(co, sc, local, r)) return false;
    const float4 qi = __ldg(&P.prims[pos].qinv);
    const float3 ld0 = gqrot(qi, r.dx, r.dy, r.dz);
#if BV_GAUSS_LOCAL
    const float lox = local.x, loy = local.y, loz = local.z;
#else
    const float3 lo0 = gqrot(qi, r.ox - co.x, r.oy - co.y, r.oz - co.z);
    const float lox = lo0.x / sc.x, loy = lo0.y / sc.y, loz = lo0.z / sc.z;
#endif
    const float ldx = ld0.x / sc.x, ldy = ld0.y / sc.y, ldz = ld0.z / sc.z;
    const float t = -gdot(lox, loy, loz, ldx, ldy, ldz) / gdot(ldx, ldy, ldz, ldx, ldy, ldz);
    if (!(t > 0.0f && t < P.depth)) return false;
    const float px = lox + t * ldx, py = loy + t * ldy, pz = loz + t * ldz;
    const float sq = gdot(px, py, pz, px, py, pz);
    if (sq > sc.w) return false;  // alpha would be below min_opacity by a margin
    const float alpha = co.w * bv_expf(-0.5f * sq);
    if (!(alpha >= P.min_opacity)) return false;
    t_out = t;
    alpha_out = alpha;
    return true;
}

// Alpha and clamped SH colour of a windowed hit (the key's particle passed
// response() for this ray when it was gathered, so it passes again).
template <int DEG>
__device__ __forceinline__ void hit_colour(const GaussianParams &P, uint32_t pos, const WinRay &r,
                                           float &a, float &cr, float &cg, float &cb) {
    float tt;
    a = 0.f;
    response(P, pos, r, tt, a);
    float coef[ShDims<DEG>::N];
    const float4 *row = reinterpret_cast<const float4 *>(P.sh + (size_t)pos * P.sh_stride);
#pragma unroll
    for (int qd = 0; qd < (ShDims<DEG>::N + 3) / 4; ++qd) {
        const float4 v = __ldg(row + qd);
        const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (qd * 4 + e < ShDims<DEG>::N) coef[qd * 4 + e] = vv[e];
    }
    eval_sh<DEG>(coef, r.dx, r.dy, r.dz, cr, cg, cb);
    cr = fmaxf(cr, 0.0f);
    cg = fmaxf(cg, 0.0f);
    cb = fmaxf(cb, 0.0f);
}

template <int DEG>
__global__ void __launch_bounds__(kGaussBlock, BV_MINB_GAUSS) gaussian_kernel(const __grid_constant__ GaussianParams P) {
    // whole warps past the last tile leave together; lanes of a partial edge
    // tile stay (inactive) because the traversal is warp-cooperative
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if ((slot & ~31u) >= P.total_work) return;
    const long long clock_begin = clock64();
    const uint32_t w = tile_item(P.tile_order, slot);
    const uint32_t tile = w / 32u, in = w % 32u;
    const uint32_t x = (tile % P.tiles_x) * 8u + in % 8u;
    const uint32_t y = (tile / P.tiles_x) * 4u + in / 8u;
    const bool active = x < P.width && y < P.height;

    // pixel -> ray: radfoam.wgsl:44-52 mapping, one normalisation
    WinRay ray;
    {
        const float px = ((float)x + 0.5f) / (float)P.width;
        const float py = ((float)y + 0.5f) / (float)P.height;
        const float vx = (px * 2.0f - 1.0f - P.principal[0]) * P.tan_half[0];
        const float vy = (py * 2.0f - 1.0f - P.principal[1]) * P.tan_half[1];
        const float4 q = make_float4(P.q[0], P.q[1], P.q[2], P.q[3]);
        const float3 rv = gqrot(q, vx, vy, 1.0f);
        const float len = sqrtf(gdot(rv.x, rv.y, rv.z, rv.x, rv.y, rv.z));
        const float inv = 1.0f / len;
        ray.dx = rv.x * inv;
        ray.dy = rv.y * inv;
        ray.dz = rv.z * inv;
        ray.ox = P.origin[0];
        ray.oy = P.origin[1];
        ray.oz = P.origin[2];
        ray.ix = win_inverse(ray.dx);
        ray.iy = win_inverse(ray.dy);
        ray.iz = win_inverse(ray.dz);
    }

#if BV_GAUSS_SPREAD
#if !BV_GAUSS_SMEM_WINDOW
#error "spread evaluation reads other lanes' window keys from shared memory"
#endif
    __shared__ float s_gdir[kGaussBlock / 32][32][3];
    __shared__ int s_gfirst[kGaussBlock / 32][32];
    __shared__ float4 s_ghit[kGaussBlock / 32][32][kGSpread];  // alpha, colour
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    s_gdir[warp][lane][0] = ray.dx;
    s_gdir[warp][lane][1] = ray.dy;
    s_gdir[warp][lane][2] = ray.dz;
    __syncwarp();
#endif
    float rad_r = 0.f, rad_g = 0.f, rad_b = 0.f, T = 1.0f;
    bool cursor_valid = false, finished = !active;
    float cur_t = 0.f;
    uint32_t cur_idx = 0, hits_used = 0, nodes_visited = 0;
    auto hit = [&](uint32_t p, bool mine, float, WinKey &k) -> bool {
        float &t = k.t;
        uint32_t &id = k.idx;
        float a;
        if (!mine || !response(P, p, ray, t, a)) return false;
        id = __ldg(&P.ids[p]);
        return true;
    };
#if BV_GAUSS_SMEM_WINDOW
    TRACE_WINDOW_DECL(BV_GAUSS_SMEM_WINDOW, kWindow, kGaussBlock);
#endif
    for (;;) {
        const bool want = !finished && T > P.min_transmittance;
        if (!__any_sync(0xffffffffu, want)) break;
#if !BV_GAUSS_SMEM_WINDOW
        TRACE_WINDOW_DECL(BV_GAUSS_SMEM_WINDOW, kWindow, kGaussBlock);
#endif
        const int count = TRACE_WINDOW_PASS(BV_GAUSS_SMEM_WINDOW, kWindow, kStack, P.nodes, ray,
                                            P.depth, want, cursor_valid, cur_t, cur_idx,
                                            nodes_visited, hit);
#if BV_GAUSS_SPREAD
        // rounds of kGSpread keys per lane: the round's hits of all lanes are
        // evaluated one per lane, then each lane composites its own in order
        {
            const int cnt = want ? count : 0;
            const int n_max = __reduce_max_sync(0xffffffffu, cnt);
            bool lane_done = cnt == 0 || T <= P.min_transmittance;
            for (int i0 = 0; i0 < n_max; i0 += kGSpread) {
                const int mine = lane_done ? 0 : max(0, min(cnt - i0, kGSpread));
                int incl = mine;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if ((int)lane >= o) incl += v;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                s_gfirst[warp][lane] = incl - mine;
                __syncwarp();
                for (int j = (int)lane; j < total; j += 32) {
                    int lo = 0, hi = 31;  // owner: the last lane whose first job is at or before j
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (s_gfirst[warp][mid] <= j)
                            lo = mid;
                        else
                            hi = mid - 1;
                    }
                    const int kk = j - s_gfirst[warp][lo];
                    const uint32_t key = (uint32_t)(i0 + kk) * kGaussBlock + (warp << 5) + (uint32_t)lo;
                    WinRay r = ray;
                    r.dx = s_gdir[warp][lo][0];
                    r.dy = s_gdir[warp][lo][1];
                    r.dz = s_gdir[warp][lo][2];
                    float a, cr, cg, cb;
                    hit_colour<DEG>(P, s_trace_win[2u * kWindow * kGaussBlock + key], r, a, cr, cg, cb);
                    s_ghit[warp][lo][kk] = make_float4(a, cr, cg, cb);
                }
                __syncwarp();
#pragma unroll 1
                for (int kk = 0; kk < mine; ++kk) {
                    if (T <= P.min_transmittance) {
                        lane_done = true;
                        break;
                    }
                    const float4 hc = s_ghit[warp][lane][kk];
                    const float a = hc.x;
                    const float wt = a * T;
                    rad_r += wt * hc.y;
                    rad_g += wt * hc.z;
                    rad_b += wt * hc.w;
                    T *= 1.0f - a;
                    hits_used += 1;
                }
                __syncwarp();
            }
        }
        if (!want) continue;
#else
        if (!want) continue;
#pragma unroll 1
        for (int i = 0; i < count; ++i) {
            if (T <= P.min_transmittance) break;
            const WinKey h = TRACE_WINDOW_KEY(BV_GAUSS_SMEM_WINDOW, kWindow, i);
            float a, cr, cg, cb;
            hit_colour<DEG>(P, h.pos, ray, a, cr, cg, cb);
            const float wt = a * T;
            rad_r += wt * cr;
            rad_g += wt * cg;
            rad_b += wt * cb;
            T *= 1.0f - a;
            hits_used += 1;
        }
#endif
        if (count < kWindow) {
            finished = true;
        } else {
            cursor_valid = true;
            const WinKey last = TRACE_WINDOW_KEY(BV_GAUSS_SMEM_WINDOW, kWindow, kWindow - 1);
            cur_t = last.t;
            cur_idx = last.idx;
        }
    }
    if (active) {
        const size_t o = (size_t)y * P.width + x;
        P.out[o] = make_float4(rad_r + T * P.background[0], rad_g + T * P.background[1],
                               rad_b + T * P.background[2], 1.0f - T);
        if (P.stats) {
            atomicAdd(P.stats + 0, 1ull);
            atomicAdd(P.stats + 1, (unsigned long long)hits_used);
            atomicAdd(P.stats + 2, (unsigned long long)nodes_visited);
        }
    }
    store_tile_cost(P.tile_cost, w, clock_begin);
}

// The camera-origin terms of every particle for one view, with the
// operations response() and support_sphere_hit() would apply per lane.
__global__ void __launch_bounds__(256) gauss_local_kernel(const GaussShPrim *prims, uint32_t n,
                                                          float ox, float oy, float oz,
                                                          float4 *local) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 co = __ldg(&prims[i].center_opacity);
    const float4 sc = __ldg(&prims[i].scale_cut);
    const float4 qi = __ldg(&prims[i].qinv);
    const float3 lo0 = gqrot(qi, ox - co.x, oy - co.y, oz - co.z);
    const float cx = co.x - ox, cy = co.y - oy, cz = co.z - oz;
    local[i] = make_float4(lo0.x / sc.x, lo0.y / sc.y, lo0.z / sc.z, gdot(cx, cy, cz, cx, cy, cz));
}

cudaError_t launch_gaussian(const GaussianParams &p, uint32_t n, uint32_t deg, cudaStream_t s,
                            uint32_t &launches) {
    launches = 0;
#if BV_GAUSS_LOCAL
    if (n) {
        gauss_local_kernel<<<(n + 255) / 256, 256, 0, s>>>(p.prims, n, p.origin[0], p.origin[1],
                                                           p.origin[2], const_cast<float4 *>(p.local));
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        launches += 1;
    }
#else
    (void)n;
#endif
    const int blocks = (int)((p.total_work + kGaussBlock - 1) / kGaussBlock);
    if (blocks == 0) return cudaSuccess;
    launches += 1;
    const size_t smem = BV_GAUSS_SMEM_WINDOW ? (size_t)3 * kWindow * kGaussBlock * 4u : 0u;
    void (*kernel)(GaussianParams) = deg == 0   ? gaussian_kernel<0>
                                     : deg == 1 ? gaussian_kernel<1>
                                     : deg == 2 ? gaussian_kernel<2>
                                                : gaussian_kernel<3>;
    if (smem > (size_t)32 * 1024) {
        const cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kernel<<<blocks, kGaussBlock, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace
}  // namespace bv

using namespace bv;

struct bv_gaussian_tracer {
    uint32_t n_input = 0, n_kept = 0, n_nodes = 0, sh_degree = 0, sh_stride = 0;
    float min_opacity = 0.01f, min_transmittance = 0.01f;
    float background[3] = {0.f, 0.f, 0.f};
    GaussShPrim *prims = nullptr;
    float4 *local = nullptr;  // per-view camera-origin terms, refilled by each dispatch
    uint32_t *ids = nullptr;
    BvhNode *nodes = nullptr;
    float *sh = nullptr;
    unsigned long long *stats = nullptr;
    bool stats_enabled = false, last_has_stats = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    TileScheduler tile_sched;  // heaviest-first tile order between dispatches
    // The per-view origin table is rewritten by every dispatch: a dispatch on
    // another stream than the previous one first waits for the previous one.
    cudaEvent_t done = nullptr;
    cudaStream_t last_stream = nullptr;
    bool dispatched = false;
    uint32_t last_launches = 0;
};

namespace {

bv_status gfail(bv_status code, const char *msg) {
    set_last_error(msg);
    return code;
}

void free_gaussian(bv_gaussian_tracer *t) {
    if (!t) return;
    cudaFree(t->prims);
    cudaFree(t->local);
    t->tile_sched.release();
    cudaFree(t->ids);
    cudaFree(t->nodes);
    cudaFree(t->sh);
    cudaFree(t->stats);
    for (auto &e : t->ev)
        if (e) cudaEventDestroy(e);
    if (t->done) cudaEventDestroy(t->done);
    delete t;
}

inline bool gfinite3(const float *v) {
    return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]);
}

// PointCloudModel::validate for a Gaussian model (lib.rs:246-340) and the
// asserts of GaussianGpuCloud::new / trace_gaussians (gpu/gaussian.rs:100-112,
// trace.rs:704-727).
bv_status validate_gaussian_sh(const bv_gaussian_sh_desc *g, const bv_gaussian_trace_settings *s) {
    if (!g || !g->points || !g->rotations || !g->scales || !g->sh_coefficients)
        return gfail(BV_ERR_INVALID_MODEL, "Gaussian model arrays are required");
    if (g->num_points == 0) return gfail(BV_ERR_INVALID_MODEL, "model has no points");
    if (g->sh_degree > 3) return gfail(BV_ERR_INVALID_MODEL, "sh_degree must be at most 3");
    if (!(std::isfinite(s->min_opacity) && s->min_opacity > 0.0f))
        return gfail(BV_ERR_INVALID_ARGUMENT, "Gaussian min_opacity must be finite and positive");
    if (!(std::isfinite(s->min_transmittance) && s->min_transmittance >= 0.0f &&
          s->min_transmittance <= 1.0f))
        return gfail(BV_ERR_INVALID_ARGUMENT, "min_transmittance must be finite and in [0, 1]");
    if (!gfinite3(s->background))
        return gfail(BV_ERR_INVALID_ARGUMENT, "background must be finite");
    const uint32_t n3k = 3u * (g->sh_degree + 1) * (g->sh_degree + 1);
    for (uint32_t i = 0; i < g->num_points; ++i) {
        const float *p = g->points + 4 * (size_t)i;
        if (!gfinite3(p) || !std::isfinite(p[3]) || p[3] < 0.0f)
            return gfail(BV_ERR_INVALID_MODEL,
                         "points must have finite coordinates and non-negative opacity");
        const float *q = g->rotations + 4 * (size_t)i;
        const float ql = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (!gfinite3(q) || !std::isfinite(q[3]) || std::fabs(ql - 1.0f) > 1.0e-3f)
            return gfail(BV_ERR_INVALID_MODEL, "transform rotations must be finite and unit length");
        const float *sc = g->scales + 3 * (size_t)i;
        if (!gfinite3(sc) || std::min(std::min(sc[0], sc[1]), sc[2]) <= 0.0f)
            return gfail(BV_ERR_INVALID_MODEL, "transform scales must be finite and positive");
        const float *c = g->sh_coefficients + (size_t)n3k * i;
        for (uint32_t k = 0; k < n3k; ++k)
            if (!std::isfinite(c[k]))
                return gfail(BV_ERR_INVALID_MODEL, "SH coefficients must be finite");
    }
    return BV_OK;
}

}  // namespace

extern "C" {

bv_status bv_gaussian_tracer_new(const bv_gaussian_sh_desc *g,
                                 const bv_gaussian_trace_settings *settings,
                                 bv_gaussian_tracer **out) {
    if (!out) return gfail(BV_ERR_INVALID_ARGUMENT, "out handle pointer is null");
    *out = nullptr;
    bv_gaussian_trace_settings st;
    if (settings) {
        st = *settings;
    } else {
        st.min_opacity = 0.01f;
        st.min_transmittance = 0.01f;
        st.background[0] = st.background[1] = st.background[2] = 0.0f;
    }
    bv_status vs = validate_gaussian_sh(g, &st);
    if (vs != BV_OK) return vs;
    // visible_point_indices (gpu/gaussian.rs:19-27): opacity > min_opacity
    const uint32_t K = (g->sh_degree + 1) * (g->sh_degree + 1);
    const uint32_t n3k = 3 * K;
    const uint32_t stride = (n3k + 3) & ~3u;
    std::vector<GaussShPrim> prims;
    std::vector<uint32_t> kept_model;
    std::vector<BvhBox> boxes;
    std::vector<float> centers;
    for (uint32_t i = 0; i < g->num_points; ++i) {
        const float *p = g->points + 4 * (size_t)i;
        if (!(p[3] > st.min_opacity)) continue;
        const float *q = g->rotations + 4 * (size_t)i;
        const float *s = g->scales + 3 * (size_t)i;
        // alpha >= min_opacity  <=>  |local|^2 <= 2 ln(opacity / min_opacity);
        // the cut is widened so that rounding never rejects a hit
        const double support = 2.0 * std::log((double)p[3] / (double)st.min_opacity);
        GaussShPrim gp;
        gp.center_opacity = make_float4(p[0], p[1], p[2], p[3]);
        gp.qinv = make_float4(-q[0], -q[1], -q[2], q[3]);
        gp.scale_cut = make_float4(s[0], s[1], s[2], (float)(support * (1.0 + 1e-3) + 1e-5));
        prims.push_back(gp);
        const double x = q[0], y = q[1], z = q[2], w = q[3];
        const double R[3][3] = {{1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)},
                                {2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)},
                                {2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)}};
        const double sup = std::sqrt(support * (1.0 + 1e-3) + 1e-5);
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
        kept_model.push_back(i);
    }
    const uint32_t kept = (uint32_t)prims.size();
    if (kept == 0)
        return gfail(BV_ERR_INVALID_MODEL, "Gaussian model has no points above min_opacity");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return gfail(BV_ERR_NO_DEVICE, "no CUDA device");

    BvhBuild bvh = build_bvh(boxes, centers, BvhMethod::kSah);
    if (bvh_depth(bvh.nodes) >= (uint32_t)kStack)
        return gfail(BV_ERR_NOT_SUPPORTED, "BVH deeper than the traversal stack");
    std::vector<GaussShPrim> sorted(kept);
    std::vector<uint32_t> ids(kept);
    std::vector<float> sh((size_t)kept * stride, 0.0f);
    for (uint32_t i = 0; i < kept; ++i) {
        const uint32_t f = bvh.order[i];  // filtered index
        sorted[i] = prims[f];
        ids[i] = f;
        std::memcpy(&sh[(size_t)i * stride], g->sh_coefficients + (size_t)n3k * kept_model[f],
                    sizeof(float) * n3k);
    }

    bv_gaussian_tracer *t = new bv_gaussian_tracer();
    t->n_input = g->num_points;
    t->n_kept = kept;
    t->n_nodes = (uint32_t)bvh.nodes.size();
    t->sh_degree = g->sh_degree;
    t->sh_stride = stride;
    t->min_opacity = st.min_opacity;
    t->min_transmittance = st.min_transmittance;
    std::memcpy(t->background, st.background, sizeof(t->background));
    auto cleanup = [&](cudaError_t e, const char *what) {
        free_gaussian(t);
        set_last_error(what);
        return e == cudaErrorMemoryAllocation ? BV_ERR_OUT_OF_MEMORY : BV_ERR_CUDA;
    };
#define BV_GTRY(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cleanup(e_, what); \
    } while (0)
    BV_GTRY(cudaMalloc(&t->prims, sizeof(GaussShPrim) * kept), "cudaMalloc particles");
    BV_GTRY(cudaMalloc(&t->local, sizeof(float4) * kept), "cudaMalloc particle origin terms");
    BV_GTRY(cudaMalloc(&t->ids, sizeof(uint32_t) * kept), "cudaMalloc ids");
    BV_GTRY(cudaMalloc(&t->nodes, sizeof(BvhNode) * t->n_nodes), "cudaMalloc nodes");
    BV_GTRY(cudaMalloc(&t->sh, sizeof(float) * sh.size()), "cudaMalloc SH");
    BV_GTRY(cudaMalloc(&t->stats, sizeof(unsigned long long) * 4), "cudaMalloc stats");
    BV_GTRY(cudaMemcpy(t->prims, sorted.data(), sizeof(GaussShPrim) * kept, cudaMemcpyHostToDevice),
            "upload particles");
    BV_GTRY(cudaMemcpy(t->ids, ids.data(), sizeof(uint32_t) * kept, cudaMemcpyHostToDevice),
            "upload ids");
    BV_GTRY(cudaMemcpy(t->nodes, bvh.nodes.data(), sizeof(BvhNode) * t->n_nodes,
                       cudaMemcpyHostToDevice), "upload nodes");
    BV_GTRY(cudaMemcpy(t->sh, sh.data(), sizeof(float) * sh.size(), cudaMemcpyHostToDevice),
            "upload SH");
    for (auto &e : t->ev) BV_GTRY(cudaEventCreate(&e), "cudaEventCreate");
    BV_GTRY(cudaEventCreateWithFlags(&t->done, cudaEventDisableTiming), "cudaEventCreate");
#undef BV_GTRY
    *out = t;
    return BV_OK;
}

void bv_gaussian_tracer_destroy(bv_gaussian_tracer *t) {
    if (!t) return;
    cudaDeviceSynchronize();
    free_gaussian(t);
}

bv_status bv_gaussian_tracer_set_min_transmittance(bv_gaussian_tracer *t, float v) {
    if (!t) return gfail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    if (!(std::isfinite(v) && v >= 0.0f && v <= 1.0f))
        return gfail(BV_ERR_INVALID_ARGUMENT, "min_transmittance must be finite and in [0, 1]");
    t->min_transmittance = v;
    return BV_OK;
}

bv_status bv_gaussian_tracer_set_background(bv_gaussian_tracer *t, const float rgb[3]) {
    if (!t || !rgb) return gfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (!gfinite3(rgb)) return gfail(BV_ERR_INVALID_ARGUMENT, "background must be finite");
    std::memcpy(t->background, rgb, sizeof(t->background));
    return BV_OK;
}

uint32_t bv_gaussian_tracer_num_points(const bv_gaussian_tracer *t) { return t ? t->n_kept : 0; }

bv_status bv_gaussian_tracer_dispatch(bv_gaussian_tracer *t, float *out_rgba_dev,
                                      const bv_camera *c, uint32_t width, uint32_t height,
                                      bv_stream stream) {
    if (!t || !out_rgba_dev || !c) return gfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (width == 0 || height == 0)
        return gfail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (!gfinite3(c->cam_position) || !std::isfinite(c->depth) || !(c->depth > 0.f))
        return gfail(BV_ERR_INVALID_ARGUMENT, "camera must be finite with positive depth");
    GaussianParams p;
    std::memset(&p, 0, sizeof(p));
    p.prims = t->prims;
    p.local = t->local;
    p.ids = t->ids;
    p.nodes = t->nodes;
    p.sh = t->sh;
    p.sh_stride = t->sh_stride;
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
    if (work >= (1ull << 31)) return gfail(BV_ERR_INVALID_ARGUMENT, "image too large");
    p.total_work = (uint32_t)work;
    p.min_opacity = t->min_opacity;
    p.min_transmittance = t->min_transmittance;
    std::memcpy(p.background, t->background, sizeof(p.background));
    cudaStream_t s = (cudaStream_t)stream;
    t->last_has_stats = t->stats_enabled;
    if (t->stats_enabled) {
        if (cudaMemsetAsync(t->stats, 0, sizeof(unsigned long long) * 4, s) != cudaSuccess ||
            cudaEventRecord(t->ev[0], s) != cudaSuccess)
            return gfail(BV_ERR_CUDA, "stats setup failed");
    }
    if (t->dispatched && t->last_stream != s && cudaStreamWaitEvent(s, t->done, 0) != cudaSuccess)
        return gfail(BV_ERR_CUDA, "stream wait on the previous dispatch failed");
    uint32_t launches = 0;
    const size_t tiles = work / 32u;
    const bool time_tiles =
        t->tile_sched.begin(BV_GAUSS_TILE_ORDER, tiles, 1, width, height, p.tile_order);
    p.tile_cost = time_tiles ? t->tile_sched.cost : nullptr;
    cudaError_t e = launch_gaussian(p, t->n_kept, t->sh_degree, s, launches);
    if (e == cudaSuccess && time_tiles) {
        e = t->tile_sched.end(tiles, 1, width, height, s);
        launches += t->tile_sched.order_launches();
    }
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return BV_ERR_CUDA;
    }
    t->last_launches = launches;
    if (cudaEventRecord(t->done, s) != cudaSuccess)
        return gfail(BV_ERR_CUDA, "event record failed");
    t->last_stream = s;
    t->dispatched = true;
    if (t->stats_enabled && cudaEventRecord(t->ev[1], s) != cudaSuccess)
        return gfail(BV_ERR_CUDA, "event record failed");
    return BV_OK;
}

bv_status bv_gaussian_tracer_enable_stats(bv_gaussian_tracer *t, uint32_t enabled) {
    if (!t) return gfail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->stats_enabled = enabled != 0;
    return BV_OK;
}

bv_status bv_gaussian_tracer_last_stats(bv_gaussian_tracer *t, bv_launch_stats *out) {
    if (!t || !out) return gfail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->launches = t->last_launches;
    if (!t->last_has_stats) return BV_OK;
    if (cudaEventSynchronize(t->ev[1]) != cudaSuccess)
        return gfail(BV_ERR_CUDA, "event sync failed");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t->ev[0], t->ev[1]);
    out->kernel_ms = ms;
    unsigned long long h[4] = {0, 0, 0, 0};
    if (cudaMemcpy(h, t->stats, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
        return gfail(BV_ERR_CUDA, "stats read failed");
    out->rays = h[0];
    out->steps = h[1];  // composited hits
    out->faces = h[2];  // BVH nodes visited
    return BV_OK;
}

}  // extern "C"
