// Relightable Gaussians with finite point lights on sm_100a: per-ray gather
// of every particle whose support ellipsoid the ray crosses, strict
// (depth, index) order, surface-band grouping and GGX point-light shading.
//
// Restates blade-volume/shaders/relight.wgsl (kernel 2 = learned volumetric
// Gaussian, point light, no visibility ray): intersect_surfel :419-441,
// point_light_shade :190-261, surface_group_response :606-624,
// trace_blended :626-744, trace_main :747-780.  The reference enumerates
// candidates with hardware ray queries over icosahedron proxies; here a BVH
// over the support ellipsoids' boxes is traversed front to back in windows
// of kWindow hits: a pass keeps the kWindow smallest (t, index) keys above
// the cursor, pruning boxes that end before the cursor or start after the
// window's last key, so every pass touches only a thin slab of the tree.
// The result does not depend on the window size (groups carry across
// windows), which is what the reference's own tests establish.
//
// Compiled with -fmad=false: the arithmetic is the CPU oracle's, operation
// for operation, so images are bit-identical.

#include "bv_device.cuh"
#include "bv_relight.h"
#include "bv_tile_order.cuh"
#include "bv_window.cuh"

namespace bv {
namespace {

constexpr int kRelightBlock = 128;
// resident blocks per SM requested from the register allocator (unset: the
// allocator's choice, 128 registers)
#ifdef BV_MINB_RELIGHT
#define BV_RELIGHT_BOUNDS __launch_bounds__(kRelightBlock, BV_MINB_RELIGHT)
#else
#define BV_RELIGHT_BOUNDS __launch_bounds__(kRelightBlock)
#endif
// Window keys per lane, in registers (BV_RELIGHT_SMEM_WINDOW 0) or in
// dynamic shared memory (1).  Measured (1M Gaussians, 16 lights, 1024 x
// 768), shading in place: 16 keys in registers 62.3 Mrays/s, in shared
// memory 16 / 24 / 32 keys 61.8 / 65.4 / 64.9 (303 -> 251 nodes per ray at
// 24 keys); shading spread over the warp (below): 16 / 20 / 24 / 28 / 32
// keys 71.2 / 76.3 / 82.1-83.3 / 93.4 / 92.2.
#ifndef BV_RELIGHT_WINDOW
#define BV_RELIGHT_WINDOW 28
#endif
#ifndef BV_RELIGHT_SMEM_WINDOW
#define BV_RELIGHT_SMEM_WINDOW 1
#endif
constexpr int kWindow = BV_RELIGHT_WINDOW;
// Shading of a window's hits spread over the warp (1): in rounds of
// BV_RELIGHT_SPREAD_KEYS keys per lane, the warp's hits are shaded one per
// lane whoever's ray they are on, into shared memory, and each lane then
// composites its own in order; or each lane shades its own hits (0).  The
// lanes of a tile hold different numbers of hits, so shading in place runs
// the 16 lights in a third of the lanes (10.6 of 32 active per instruction).
// Measured (1M Gaussians, 16 lights, 1024 x 768, 24-key windows): in place
// 65.0 Mrays/s; spread with 2 / 4 / 8 keys per shading round 80.7 / 82.1 /
// 83.4.  A hit's shading is the same expression in whichever lane evaluates
// it, so the image is unchanged bit for bit.
#ifndef BV_RELIGHT_SPREAD
#define BV_RELIGHT_SPREAD 1
#endif
#ifndef BV_RELIGHT_SPREAD_KEYS
#define BV_RELIGHT_SPREAD_KEYS 4
#endif
constexpr int kSpread = BV_RELIGHT_SPREAD_KEYS;

// qrot (common.wgsl:386-390)
__device__ __forceinline__ float3 qrot(float4 q, float vx, float vy, float vz) {
    const float t0 = 2.0f * (q.y * vz - q.z * vy);
    const float t1 = 2.0f * (q.z * vx - q.x * vz);
    const float t2 = 2.0f * (q.x * vy - q.y * vx);
    return make_float3((vx + q.w * t0) + (q.y * t2 - q.z * t1),
                       (vy + q.w * t1) + (q.z * t0 - q.x * t2),
                       (vz + q.w * t2) + (q.x * t1 - q.y * t0));
}

// intersect_surfel, kernel 2 (relight.wgsl:419-441).
__device__ __forceinline__ bool intersect(const GaussPrim *__restrict__ prims,
                                          const float4 *__restrict__ local_terms, uint32_t pos,
                                          const WinRay &r, float t_end, float &t_out,
                                          float &alpha_out) {
    const float4 co = __ldg(&prims[pos].center_opacity);
    const float4 ss = __ldg(&prims[pos].scale_support);
#if BV_RELIGHT_LOCAL
    const float4 local = __ldg(&local_terms[pos]);
#else
    (void)local_terms;
#endif
    {
        // conservative pre-test: a hit lies inside the support ellipsoid, so
        // within support * max(scale) of the mean (d is unit; the margin
        // covers the rounding of |oc|^2 - b^2)
        const float ox = co.x - r.ox, oy = co.y - r.oy, oz = co.z - r.oz;
        const float b = dot3(ox, oy, oz, r.dx, r.dy, r.dz);
#if BV_RELIGHT_LOCAL
        const float oo = local.w;
#else
        const float oo = dot3(ox, oy, oz, ox, oy, oz);
#endif
        const float smax = fmaxf(fmaxf(ss.x, ss.y), ss.z);
        if (oo - b * b > ss.w * (smax * smax) * 1.001f + 1e-6f * oo + 1e-30f) return false;
    }
    const float4 qi = __ldg(&prims[pos].qinv);
    const float3 ld0 = qrot(qi, r.dx, r.dy, r.dz);
#if BV_RELIGHT_LOCAL
    const float lox = local.x, loy = local.y, loz = local.z;
#else
    const float3 lo0 = qrot(qi, r.ox - co.x, r.oy - co.y, r.oz - co.z);
    const float lox = lo0.x / ss.x, loy = lo0.y / ss.y, loz = lo0.z / ss.z;
#endif
    const float ldx = ld0.x / ss.x, ldy = ld0.y / ss.y, ldz = ld0.z / ss.z;
    const float t = -dot3(lox, loy, loz, ldx, ldy, ldz) / dot3(ldx, ldy, ldz, ldx, ldy, ldz);
    if (t <= 0.0f || t >= t_end) return false;
    const float px = lox + t * ldx, py = loy + t * ldy, pz = loz + t * ldz;
    const float sq = dot3(px, py, pz, px, py, pz);
    if (sq > ss.w) return false;
    const float response = fminf(0.999f, co.w * bv_expf(-0.5f * sq));
    t_out = t;
    alpha_out = 1.0f - bv_powf(1.0f - response, 1.1f);
    return true;
}

// point_light_shade (relight.wgsl:190-261), diffuse_samples = 0; result is
// added to acc.
__device__ __forceinline__ void shade_light(const RelightLight &L, float px, float py, float pz,
                                            float nx, float ny, float nz, float vx, float vy,
                                            float vz, const float4 &m0, const float4 &m1,
                                            float &ar, float &ag, float &ab) {
    const float flx = px - L.position[0], fly = py - L.position[1], flz = pz - L.position[2];
    const float d2 = dot3(flx, fly, flz, flx, fly, flz);
    if (d2 <= 1.1920929e-7f) return;
    const float inv = 1.0f / sqrtf(d2);
    const float awx = flx * inv, awy = fly * inv, awz = flz * inv;
    float angular = 1.0f;
    if (L.exponent != 0.0f)
        angular = bv_powf(fmaxf(dot3(L.direction[0], L.direction[1], L.direction[2], awx, awy, awz),
                               0.0f),
                         L.exponent);
    const float tx = -awx, ty = -awy, tz = -awz;
    const float ndl = fmaxf(dot3(nx, ny, nz, tx, ty, tz), 0.0f);
    if (ndl == 0.0f) return;
    const float a_d2 = angular / d2;
    const float rr = L.intensity[0] * a_d2, rg = L.intensity[1] * a_d2, rb = L.intensity[2] * a_d2;
    float outr = m0.x * rr * ndl, outg = m0.y * rg * ndl, outb = m0.z * rb * ndl;
    if (!(m1.x == 0.0f && m1.y == 0.0f && m1.z == 0.0f)) {
        const float ndv = fmaxf(dot3(nx, ny, nz, vx, vy, vz), 0.0f);
        const float hx = tx + vx, hy = ty + vy, hz = tz + vz;
        const float hs2 = dot3(hx, hy, hz, hx, hy, hz);
        if (!(ndv == 0.0f || hs2 <= 1.1920929e-7f)) {
            const float hinv = 1.0f / sqrtf(hs2);
            const float ux = hx * hinv, uy = hy * hinv, uz = hz * hinv;
            const float ndh = fmaxf(dot3(nx, ny, nz, ux, uy, uz), 0.0f);
            const float vdh = fminf(fmaxf(dot3(vx, vy, vz, ux, uy, uz), 0.0f), 1.0f);
            const float rc = fminf(fmaxf(m0.w, 0.045f), 1.0f);
            const float alpha = rc * rc;
            const float a2 = alpha * alpha;
            const float den = ndh * ndh * (a2 - 1.0f) + 1.0f;
            const float pi = 3.14159265f;
            const float dist = a2 / fmaxf(pi * den * den, 1.1754944e-38f);
            const float sl = 2.0f * ndl / (ndl + sqrtf(a2 + (1.0f - a2) * ndl * ndl));
            const float sv = 2.0f * ndv / (ndv + sqrtf(a2 + (1.0f - a2) * ndv * ndv));
            const float g1 = 1.0f - vdh;
            const float g2 = g1 * g1;
            const float grazing = (g2 * g2) * g1;
            const float scale = pi * dist * sl * sv / (4.0f * ndv);
            outr += rr * scale * (m1.x + (1.0f - m1.x) * grazing);
            outg += rg * scale * (m1.y + (1.0f - m1.y) * grazing);
            outb += rb * scale * (m1.z + (1.0f - m1.z) * grazing);
        }
    }
    ar += outr;
    ag += outg;
    ab += outb;
}

// The 16-light shading of one hit at depth t of a ray with direction d
// from the camera origin: relight.wgsl's trace_blended body for one hit
// (the normal faces the viewer), summed over the lights in order.
__device__ __forceinline__ void shade_hit(const RelightParams &P, uint32_t pos, float t, float dx,
                                          float dy, float dz, float &sr, float &sg, float &sb) {
    const float ptx = P.origin[0] + t * dx, pty = P.origin[1] + t * dy, ptz = P.origin[2] + t * dz;
    const float4 nr = __ldg(&P.prims[pos].normal_radius);
    float nx = nr.x, ny = nr.y, nz = nr.z;
    if (dot3(nx, ny, nz, dx, dy, dz) > 0.0f) {
        nx = -nx;
        ny = -ny;
        nz = -nz;
    }
    const uint32_t mat = __ldg(&P.prims[pos].ids.y);
    const float4 m0 = __ldg(&P.materials[mat].a);
    const float4 m1 = __ldg(&P.materials[mat].b);
    sr = sg = sb = 0.f;
    for (uint32_t l = 0; l < P.n_lights; ++l)
        shade_light(P.lights[l], ptx, pty, ptz, nx, ny, nz, -dx, -dy, -dz, m0, m1, sr, sg, sb);
}

__global__ void BV_RELIGHT_BOUNDS
relight_kernel(const __grid_constant__ RelightParams P) {
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

    // trace_main ray mapping (relight.wgsl:760-766): one normalisation
    WinRay ray;
    {
        const float px = ((float)x + 0.5f) / (float)P.width;
        const float py = ((float)y + 0.5f) / (float)P.height;
        const float vx = (px * 2.0f - 1.0f - P.principal[0]) * P.tan_half[0];
        const float vy = (py * 2.0f - 1.0f - P.principal[1]) * P.tan_half[1];
        const float4 q = make_float4(P.q[0], P.q[1], P.q[2], P.q[3]);
        const float3 rv = qrot(q, vx, vy, 1.0f);
        const float len = sqrtf(dot3(rv.x, rv.y, rv.z, rv.x, rv.y, rv.z));
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
    const float t_end = P.depth;
#if BV_RELIGHT_SPREAD
#if !BV_RELIGHT_SMEM_WINDOW
#error "spread shading reads other lanes' window keys from shared memory"
#endif
    // per warp: each lane's ray direction, the first job of each lane in a
    // round, and each lane's shaded keys of the round
    __shared__ float s_dir[kRelightBlock / 32][32][3];
    __shared__ int s_first[kRelightBlock / 32][32];
    __shared__ float s_shade[kRelightBlock / 32][32][kSpread][3];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    s_dir[warp][lane][0] = ray.dx;
    s_dir[warp][lane][1] = ray.dy;
    s_dir[warp][lane][2] = ray.dz;
    __syncwarp();
#endif

    float rad_r = 0.f, rad_g = 0.f, rad_b = 0.f, T = 1.0f;
    bool group = false, stopped = false;
    float limit = 0.f, sc_r = 0.f, sc_g = 0.f, sc_b = 0.f, sum_w = 0.f, group_T = 1.f;
    bool cursor_valid = false;
    float cur_t = 0.f;
    uint32_t cur_idx = 0;
    uint32_t hits_used = 0, nodes_visited = 0;
    auto hit = [&](uint32_t p, bool mine, float, WinKey &k) -> bool {
        float &t = k.t;
        uint32_t &id = k.idx;
        float a;
        if (!mine || !intersect(P.prims, P.local, p, ray, t_end, t, a) || !(a > 0.0f)) return false;
        id = __ldg(&P.prims[p].ids.x);
        return true;
    };

    bool finished = !active;
#if BV_RELIGHT_SMEM_WINDOW
    TRACE_WINDOW_DECL(BV_RELIGHT_SMEM_WINDOW, kWindow, kRelightBlock);
#endif
    for (;;) {
        // ---- gather the next window of keys above the cursor (whole warp)
        const bool want = !finished;
        if (!__any_sync(0xffffffffu, want)) break;
#if !BV_RELIGHT_SMEM_WINDOW
        TRACE_WINDOW_DECL(BV_RELIGHT_SMEM_WINDOW, kWindow, kRelightBlock);
#endif
        const int count =
            TRACE_WINDOW_PASS(BV_RELIGHT_SMEM_WINDOW, kWindow, kRelightStack, P.nodes, ray, t_end,
                              want, cursor_valid, cur_t, cur_idx, nodes_visited, hit);
#if BV_RELIGHT_SPREAD
        // ---- shade and composite the window in rounds of kSpread keys per
        // lane (trace_blended :693-728): the round's hits of all lanes are
        // shaded one per lane, then each lane composites its own in order
        {
            const int cnt = (want && count > 0) ? count : 0;
            const int n_max = __reduce_max_sync(0xffffffffu, cnt);
            bool lane_done = cnt == 0;
            for (int i0 = 0; i0 < n_max; i0 += kSpread) {
                const int mine = lane_done ? 0 : max(0, min(cnt - i0, kSpread));
                int incl = mine;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, o);
                    if ((int)lane >= o) incl += v;
                }
                const int total = __shfl_sync(0xffffffffu, incl, 31);
                s_first[warp][lane] = incl - mine;
                __syncwarp();
                for (int j = (int)lane; j < total; j += 32) {
                    // owner: the last lane whose first job is at or before j
                    int lo = 0, hi = 31;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (s_first[warp][mid] <= j)
                            lo = mid;
                        else
                            hi = mid - 1;
                    }
                    const int kk = j - s_first[warp][lo];
                    const uint32_t otid = (warp << 5) + (uint32_t)lo;
                    const uint32_t key = (uint32_t)(i0 + kk) * kRelightBlock + otid;
                    const float t = __uint_as_float(s_trace_win[key]);
                    const uint32_t pos = s_trace_win[2u * kWindow * kRelightBlock + key];
                    shade_hit(P, pos, t, s_dir[warp][lo][0], s_dir[warp][lo][1], s_dir[warp][lo][2],
                              s_shade[warp][lo][kk][0], s_shade[warp][lo][kk][1],
                              s_shade[warp][lo][kk][2]);
                }
                __syncwarp();
#pragma unroll 1
                for (int kk = 0; kk < mine; ++kk) {
                    const WinKey h = TRACE_WINDOW_KEY(BV_RELIGHT_SMEM_WINDOW, kWindow, i0 + kk);
                    if (!group || h.t > limit) {
                        if (group) {
                            const float a_sum = fminf(1.0f, sum_w);
                            const float a_union = 1.0f - group_T;
                            const float alpha = a_union * (1.0f - 0.75f) + a_sum * 0.75f;
                            const float wmax = fmaxf(sum_w, 1.0e-6f);
                            rad_r += T * (alpha * sc_r / wmax);
                            rad_g += T * (alpha * sc_g / wmax);
                            rad_b += T * (alpha * sc_b / wmax);
                            T *= 1.0f - alpha;
                            group = false;
                            if (T <= 0.003f) {
                                stopped = true;
                                lane_done = true;
                                break;
                            }
                        }
                        group = true;
                        limit = h.t + 0.5f * __ldg(&P.prims[h.pos].normal_radius.w);
                        sc_r = sc_g = sc_b = 0.f;
                        sum_w = 0.f;
                        group_T = 1.f;
                    }
                    float tt, a;
                    intersect(P.prims, P.local, h.pos, ray, t_end, tt, a);
                    hits_used += 1;
                    const float sr = s_shade[warp][lane][kk][0], sg = s_shade[warp][lane][kk][1],
                                sb = s_shade[warp][lane][kk][2];
                    sc_r += a * sr;
                    sc_g += a * sg;
                    sc_b += a * sb;
                    sum_w += a;
                    group_T *= 1.0f - a;
                }
                __syncwarp();
            }
        }
        if (!want) continue;
        if (count == 0) {
            finished = true;
            continue;
        }
#else
        if (!want) continue;
        if (count == 0) {
            finished = true;
            continue;
        }
        // ---- composite the window in order (trace_blended :693-728)
#pragma unroll 1
        for (int i = 0; i < count; ++i) {
            const WinKey h = TRACE_WINDOW_KEY(BV_RELIGHT_SMEM_WINDOW, kWindow, i);
            if (!group || h.t > limit) {
                if (group) {
                    const float a_sum = fminf(1.0f, sum_w);
                    const float a_union = 1.0f - group_T;
                    const float alpha = a_union * (1.0f - 0.75f) + a_sum * 0.75f;
                    const float wmax = fmaxf(sum_w, 1.0e-6f);
                    rad_r += T * (alpha * sc_r / wmax);
                    rad_g += T * (alpha * sc_g / wmax);
                    rad_b += T * (alpha * sc_b / wmax);
                    T *= 1.0f - alpha;
                    group = false;
                    if (T <= 0.003f) {
                        stopped = true;
                        break;
                    }
                }
                group = true;
                limit = h.t + 0.5f * __ldg(&P.prims[h.pos].normal_radius.w);
                sc_r = sc_g = sc_b = 0.f;
                sum_w = 0.f;
                group_T = 1.f;
            }
            float tt, a;
            intersect(P.prims, P.local, h.pos, ray, t_end, tt, a);
            hits_used += 1;
            const float ptx = ray.ox + h.t * ray.dx, pty = ray.oy + h.t * ray.dy,
                        ptz = ray.oz + h.t * ray.dz;
            const float4 nr = __ldg(&P.prims[h.pos].normal_radius);
            float nx = nr.x, ny = nr.y, nz = nr.z;
            if (dot3(nx, ny, nz, ray.dx, ray.dy, ray.dz) > 0.0f) {
                nx = -nx;
                ny = -ny;
                nz = -nz;
            }
            const uint32_t mat = __ldg(&P.prims[h.pos].ids.y);
            const float4 m0 = __ldg(&P.materials[mat].a);
            const float4 m1 = __ldg(&P.materials[mat].b);
            float sr = 0.f, sg = 0.f, sb = 0.f;
            for (uint32_t l = 0; l < P.n_lights; ++l)
                shade_light(P.lights[l], ptx, pty, ptz, nx, ny, nz, -ray.dx, -ray.dy, -ray.dz, m0,
                            m1, sr, sg, sb);
            sc_r += a * sr;
            sc_g += a * sg;
            sc_b += a * sb;
            sum_w += a;
            group_T *= 1.0f - a;
        }
#endif
        if (stopped) {
            finished = true;
            continue;
        }
        if (count < kWindow) {
            if (group) {
                const float a_sum = fminf(1.0f, sum_w);
                const float a_union = 1.0f - group_T;
                const float alpha = a_union * (1.0f - 0.75f) + a_sum * 0.75f;
                const float wmax = fmaxf(sum_w, 1.0e-6f);
                rad_r += T * (alpha * sc_r / wmax);
                rad_g += T * (alpha * sc_g / wmax);
                rad_b += T * (alpha * sc_b / wmax);
                T *= 1.0f - alpha;
                group = false;
            }
            finished = true;
            continue;
        }
        cursor_valid = true;
        const WinKey last = TRACE_WINDOW_KEY(BV_RELIGHT_SMEM_WINDOW, kWindow, kWindow - 1);
        cur_t = last.t;
        cur_idx = last.idx;
    }
    if (group && !stopped) {
        const float a_sum = fminf(1.0f, sum_w);
        const float a_union = 1.0f - group_T;
        const float alpha = a_union * (1.0f - 0.75f) + a_sum * 0.75f;
        const float wmax = fmaxf(sum_w, 1.0e-6f);
        rad_r += T * (alpha * sc_r / wmax);
        rad_g += T * (alpha * sc_g / wmax);
        rad_b += T * (alpha * sc_b / wmax);
        T *= 1.0f - alpha;
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
// operations intersect() would apply per lane.
__global__ void __launch_bounds__(256) relight_local_kernel(const GaussPrim *prims, uint32_t n,
                                                            float ox, float oy, float oz,
                                                            float4 *local) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 co = __ldg(&prims[i].center_opacity);
    const float4 ss = __ldg(&prims[i].scale_support);
    const float4 qi = __ldg(&prims[i].qinv);
    const float3 lo0 = qrot(qi, ox - co.x, oy - co.y, oz - co.z);
    const float cx = co.x - ox, cy = co.y - oy, cz = co.z - oz;
    local[i] = make_float4(lo0.x / ss.x, lo0.y / ss.y, lo0.z / ss.z, dot3(cx, cy, cz, cx, cy, cz));
}

}  // namespace

cudaError_t launch_relight(const RelightParams &p, cudaStream_t s, uint32_t &launches) {
    launches = 0;
    const int blocks = (int)((p.total_work + kRelightBlock - 1) / kRelightBlock);
    if (blocks == 0) return cudaSuccess;
#if BV_RELIGHT_LOCAL
    if (p.n_prims) {
        relight_local_kernel<<<(p.n_prims + 255) / 256, 256, 0, s>>>(p.prims, p.n_prims, p.origin[0],
                                                                     p.origin[1], p.origin[2], p.local);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        launches += 1;
    }
#endif
    const size_t smem = BV_RELIGHT_SMEM_WINDOW ? (size_t)3 * kWindow * kRelightBlock * 4u : 0u;
    if (smem > (size_t)32 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(relight_kernel,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess) return e;
    }
    relight_kernel<<<blocks, kRelightBlock, smem, s>>>(p);
    launches += 1;
    return cudaGetLastError();
}

}  // namespace bv
