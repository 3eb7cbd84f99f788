// RadFoam / PowerFoam cell walk for sm_100a: forward render, path recorder,
// and the fused forward + loss + replay backward.
//
// The arithmetic of one walk step restates blade-volume/src/trace.rs
// (find_exit_face :170-205, support_interval :209-238, trace_one_ray
// :1680-1820, record_path_jacobians :1573-1676) in the same operation order.
// This file is compiled with -fmad=false, so every float expression below is
// a sequence of IEEE-rounded single operations exactly as written, matching
// the FP32 CPU restatement bit for bit (cells, t values, colours, alpha).
// The only fused operations are the explicit __fmaf_rn calls in bv_expf.
//
// Scheduling: one ray per lane, persistent warps.  A warp refills idle lanes
// from a global ray dispenser (one atomic per refill, ballot + popc to rank
// the idle lanes), so rays that finish early do not leave lanes idle while
// their neighbours walk long paths.  Work items are tile-ordered (8x4
// pixels) so that lanes refilled together start on neighbouring pixels.

#include <cuda_bf16.h>

#include "bv_internal.h"

namespace bv {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNone = 0xffffffffu;
constexpr int kWalkBlock = 256;
constexpr int kRefillMin = 8;

// ---------------------------------------------------------------------------
// exp(x): Cody & Waite reduction x = k ln2 + r (ln2 split into a high part
// with 12 trailing zero bits and a low part), degree-7 Taylor polynomial of
// e^r in Horner form with fused multiply-adds, exact scaling by 2^k.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float bv_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283935546875f) return __int_as_float(0x7f800000);
    if (x < -103.972084045410156f) return 0.0f;
    const float k = rintf(x * 1.44269502162933349609375f);
    float r = __fmaf_rn(k, -0.693115234375f, x);
    r = __fmaf_rn(k, -3.19461832987144589424133e-05f, r);
    float p = 1.98412701138295233249664e-04f;
    p = __fmaf_rn(p, r, 1.38888892251998186111450e-03f);
    p = __fmaf_rn(p, r, 8.33333376795053482055664e-03f);
    p = __fmaf_rn(p, r, 4.16666679084300994873047e-02f);
    p = __fmaf_rn(p, r, 1.66666671633720397949219e-01f);
    p = __fmaf_rn(p, r, 0.5f);
    p = __fmaf_rn(p, r, 1.0f);
    p = __fmaf_rn(p, r, 1.0f);
    int ki = (int)k;
    if (ki > 127) {
        p = p * 2.0f;
        ki -= 1;
    }
    if (ki < -126) {
        p = p * __int_as_float((ki + 64 + 127) << 23);
        return p * 5.42101086242752217004e-20f;
    }
    return p * __int_as_float((ki + 127) << 23);
}

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return ax * bx + ay * by + az * bz;
}

// SH constants (trace.rs:242-261).
__device__ __constant__ float kSH[16] = {
    0.2820948f,  -0.48860252f, 0.48860252f, -0.48860252f, 1.0925485f,  -1.0925485f,
    0.31539157f, -1.0925485f,  0.54627424f, -0.5900436f,  2.8906114f,  -0.4570458f,
    0.37317634f, -0.4570458f,  1.4453057f,  -0.5900436f,
};

template <int DEG>
struct ShDims {
    static constexpr int K = (DEG + 1) * (DEG + 1);
    static constexpr int N = 3 * K;
};

// Row of SH coefficients for one site into registers (float or bf16 table).
template <int DEG, bool BF16>
__device__ __forceinline__ void load_sh_row(const DeviceModel &m, uint32_t cell,
                                            float (&c)[ShDims<DEG>::N]) {
    constexpr int N = ShDims<DEG>::N;
    if (BF16) {
        const uint4 *row = reinterpret_cast<const uint4 *>(
            static_cast<const __nv_bfloat16 *>(m.sh) + (size_t)cell * m.sh_stride);
        constexpr int Q = (N + 7) / 8;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const uint4 v = __ldg(row + q);
            const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int i0 = q * 8 + 2 * h;
                if (i0 < N) c[i0] = __uint_as_float(w[h] << 16);
                if (i0 + 1 < N) c[i0 + 1] = __uint_as_float(w[h] & 0xffff0000u);
            }
        }
    } else {
        const float4 *row =
            reinterpret_cast<const float4 *>(static_cast<const float *>(m.sh) + (size_t)cell * m.sh_stride);
        constexpr int Q = (N + 3) / 4;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float4 v = __ldg(row + q);
            const float w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int h = 0; h < 4; ++h)
                if (q * 4 + h < N) c[q * 4 + h] = w[h];
        }
    }
}

// eval_rgb_sh_unclamped + clamp (trace.rs:264-402), same operation order.
template <int DEG>
__device__ __forceinline__ void eval_sh(const float (&c)[ShDims<DEG>::N], float x, float y, float z,
                                        float &r, float &g, float &b) {
    const float xx = x * x, yy = y * y, zz = z * z;
    r = 0.0f;
    g = 0.0f;
    b = 0.0f;
    r += kSH[0] * c[0];
    g += kSH[0] * c[1];
    b += kSH[0] * c[2];
    if (DEG >= 1) {
        r += kSH[1] * c[3] * y;  g += kSH[1] * c[4] * y;  b += kSH[1] * c[5] * y;
        r += kSH[2] * c[6] * z;  g += kSH[2] * c[7] * z;  b += kSH[2] * c[8] * z;
        r += kSH[3] * c[9] * x;  g += kSH[3] * c[10] * x; b += kSH[3] * c[11] * x;
    }
    if (DEG >= 2) {
        r += kSH[4] * c[12] * x * y; g += kSH[4] * c[13] * x * y; b += kSH[4] * c[14] * x * y;
        r += kSH[5] * c[15] * y * z; g += kSH[5] * c[16] * y * z; b += kSH[5] * c[17] * y * z;
        const float t6 = 3.0f * zz - 1.0f;
        r += kSH[6] * c[18] * t6; g += kSH[6] * c[19] * t6; b += kSH[6] * c[20] * t6;
        r += kSH[7] * c[21] * x * z; g += kSH[7] * c[22] * x * z; b += kSH[7] * c[23] * x * z;
        const float t8 = xx - yy;
        r += kSH[8] * c[24] * t8; g += kSH[8] * c[25] * t8; b += kSH[8] * c[26] * t8;
    }
    if (DEG >= 3) {
        const float t9 = y * (3.0f * xx - yy);
        r += kSH[9] * c[27] * t9; g += kSH[9] * c[28] * t9; b += kSH[9] * c[29] * t9;
        const float t10 = x * y * z;
        r += kSH[10] * c[30] * t10; g += kSH[10] * c[31] * t10; b += kSH[10] * c[32] * t10;
        const float t11 = y * (5.0f * zz - 1.0f);
        r += kSH[11] * c[33] * t11; g += kSH[11] * c[34] * t11; b += kSH[11] * c[35] * t11;
        const float t12 = z * (5.0f * zz - 3.0f);
        r += kSH[12] * c[36] * t12; g += kSH[12] * c[37] * t12; b += kSH[12] * c[38] * t12;
        const float t13 = x * (5.0f * zz - 1.0f);
        r += kSH[13] * c[39] * t13; g += kSH[13] * c[40] * t13; b += kSH[13] * c[41] * t13;
        const float t14 = z * (xx - yy);
        r += kSH[14] * c[42] * t14; g += kSH[14] * c[43] * t14; b += kSH[14] * c[44] * t14;
        const float t15 = x * (xx - 3.0f * yy);
        r += kSH[15] * c[45] * t15; g += kSH[15] * c[46] * t15; b += kSH[15] * c[47] * t15;
    }
    r = 0.5f + r;
    g = 0.5f + g;
    b = 0.5f + b;
}

// SH basis values Y_m(dir) (derivative of the colour w.r.t. coefficient m).
template <int DEG>
__device__ __forceinline__ void sh_basis(float x, float y, float z, float (&Y)[ShDims<DEG>::K]) {
    Y[0] = kSH[0];
    if (DEG >= 1) {
        Y[1] = kSH[1] * y;
        Y[2] = kSH[2] * z;
        Y[3] = kSH[3] * x;
    }
    if (DEG >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        Y[4] = kSH[4] * x * y;
        Y[5] = kSH[5] * y * z;
        Y[6] = kSH[6] * (3.0f * zz - 1.0f);
        Y[7] = kSH[7] * x * z;
        Y[8] = kSH[8] * (xx - yy);
        if (DEG >= 3) {
            Y[9] = kSH[9] * y * (3.0f * xx - yy);
            Y[10] = kSH[10] * x * y * z;
            Y[11] = kSH[11] * y * (5.0f * zz - 1.0f);
            Y[12] = kSH[12] * z * (5.0f * zz - 3.0f);
            Y[13] = kSH[13] * x * (5.0f * zz - 1.0f);
            Y[14] = kSH[14] * z * (xx - yy);
            Y[15] = kSH[15] * x * (xx - 3.0f * yy);
        }
    }
}

// ---------------------------------------------------------------------------
// ray generation: radfoam.wgsl:44-52 (qrot, common.wgsl:386-390), glam's
// normalize, then trace_one_ray's own dir /= |dir| (trace.rs:1692-1705).
// ---------------------------------------------------------------------------
struct Ray {
    float ox, oy, oz;
    float dx, dy, dz;
};

__device__ __forceinline__ bool make_ray(const ViewDesc &v, uint32_t x, uint32_t y, Ray &ray) {
    const float px = ((float)x + 0.5f) / (float)v.width;
    const float py = ((float)y + 0.5f) / (float)v.height;
    const float ndc_x = px * 2.0f - 1.0f;
    const float ndc_y = py * 2.0f - 1.0f;
    const float vx = (ndc_x - v.principal[0]) * v.tan_half[0];
    const float vy = (ndc_y - v.principal[1]) * v.tan_half[1];
    const float vz = 1.0f;
    const float qx = v.q[0], qy = v.q[1], qz = v.q[2], qw = v.q[3];
    const float tx = 2.0f * (qy * vz - qz * vy);
    const float ty = 2.0f * (qz * vx - qx * vz);
    const float tz = 2.0f * (qx * vy - qy * vx);
    const float rx = (vx + qw * tx) + (qy * tz - qz * ty);
    const float ry = (vy + qw * ty) + (qz * tx - qx * tz);
    const float rz = (vz + qw * tz) + (qx * ty - qy * tx);
    const float len = sqrtf(dot3(rx, ry, rz, rx, ry, rz));
    const float inv = 1.0f / len;
    const float ux = rx * inv, uy = ry * inv, uz = rz * inv;
    const float dl = sqrtf(dot3(ux, uy, uz, ux, uy, uz));
    ray.ox = v.origin[0];
    ray.oy = v.origin[1];
    ray.oz = v.origin[2];
    if (!(dl > 0.0f) || !isfinite(dl)) {
        ray.dx = ray.dy = ray.dz = 0.0f;
        return false;
    }
    ray.dx = ux / dl;
    ray.dy = uy / dl;
    ray.dz = uz / dl;
    return true;
}

// Tile-ordered work index -> (view, pixel).  Returns false for the padding
// lanes of partial edge tiles.
template <typename Params>
__device__ __forceinline__ bool work_item(const Params &P, uint32_t w, uint32_t &view,
                                          uint32_t &x, uint32_t &y) {
    uint32_t v = 0;
    while (v + 1 < P.n_views && w >= P.views[v + 1].ray_begin) ++v;
    const ViewDesc &vd = P.views[v];
    const uint32_t local = w - vd.ray_begin;
    const uint32_t tile = local / kTileRays, in = local % kTileRays;
    x = (tile % vd.tiles_x) * kTileW + in % kTileW;
    y = (tile / vd.tiles_x) * kTileH + in / kTileW;
    view = v;
    return x < vd.width && y < vd.height;
}

// Output index of pixel (view, x, y) in a [views][H][W] image stack.
template <typename Params>
__device__ __forceinline__ size_t pixel_index(const Params &P, uint32_t view, uint32_t x,
                                              uint32_t y) {
    return (size_t)P.views[view].pixel_begin + (size_t)y * P.views[view].width + x;
}

// ---------------------------------------------------------------------------
// find_exit_face (trace.rs:170-205): the first face in CSR order with the
// smallest t in (t0, best).  Neighbour indices and site records are fetched
// four at a time so that four independent gathers are in flight.
// ---------------------------------------------------------------------------
template <bool BOUNDED>
__device__ __forceinline__ void find_exit(const DeviceModel &m, uint32_t cur, float cpx, float cpy,
                                          float cpz, float cr, const Ray &ray, float t0,
                                          float depth, float &best, uint32_t &best_j,
                                          float4 &best_g, uint32_t &faces) {
    const uint32_t begin = __ldg(m.offsets + cur);
    const uint32_t end = __ldg(m.offsets + cur + 1);
    best = depth;
    best_j = kNone;
    best_g = make_float4(0.f, 0.f, 0.f, 0.f);
    const float ri2 = cr * cr;
    for (uint32_t k = begin; k < end; k += 4) {
        uint32_t j[4];
        float4 g[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) j[u] = (k + u < end) ? __ldg(m.neighbors + k + u) : cur;
#pragma unroll
        for (int u = 0; u < 4; ++u) g[u] = __ldg(m.geom + j[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (k + u < end) {
                const float offx = g[u].x - cpx, offy = g[u].y - cpy, offz = g[u].z - cpz;
                float shift;
                if (BOUNDED) {
                    const float rj = g[u].w;
                    const float dsq = fmaxf(dot3(offx, offy, offz, offx, offy, offz), 1e-20f);
                    shift = 0.5f + 0.5f * (ri2 - rj * rj) / dsq;
                } else {
                    shift = 0.5f;
                }
                const float fox = cpx + shift * offx;
                const float foy = cpy + shift * offy;
                const float foz = cpz + shift * offz;
                const float dp = dot3(offx, offy, offz, ray.dx, ray.dy, ray.dz);
                if (dp > 0.0f) {
                    const float t =
                        dot3(fox - ray.ox, foy - ray.oy, foz - ray.oz, offx, offy, offz) / dp;
                    if (isfinite(t) && t > t0 && t < best) {
                        best = t;
                        best_j = j[u];
                        best_g = g[u];
                    }
                }
            }
        }
    }
    faces = end - begin;
}

// support_interval (trace.rs:209-238).
template <bool BOUNDED>
__device__ __forceinline__ bool support(const Ray &ray, float cx, float cy, float cz, float radius,
                                        float t0, float t1, float &s, float &e) {
    if (!BOUNDED) {
        s = t0;
        e = t1;
        return t1 > t0;
    }
    const float ocx = ray.ox - cx, ocy = ray.oy - cy, ocz = ray.oz - cz;
    const float a = dot3(ray.dx, ray.dy, ray.dz, ray.dx, ray.dy, ray.dz);
    if (!isfinite(a) || a <= 0.0f) return false;
    const float b = dot3(ocx, ocy, ocz, ray.dx, ray.dy, ray.dz);
    const float c = dot3(ocx, ocy, ocz, ocx, ocy, ocz) - radius * radius;
    const float disc = b * b - a * c;
    if (disc <= 0.0f) return false;
    const float root = sqrtf(disc);
    const float nt = (-b - root) / a;
    const float ft = (-b + root) / a;
    s = fmaxf(t0, nt);
    e = fminf(t1, ft);
    return e > s;
}

// sphere_intersection_jacobians (trace.rs:1101-1124), direction normalized.
__device__ __forceinline__ bool sphere_hit(const Ray &ray, float cx, float cy, float cz,
                                           float radius, float &nt, float &ft, float &root,
                                           float &b) {
    const float ocx = ray.ox - cx, ocy = ray.oy - cy, ocz = ray.oz - cz;
    b = dot3(ocx, ocy, ocz, ray.dx, ray.dy, ray.dz);
    const float disc = b * b - (dot3(ocx, ocy, ocz, ocx, ocy, ocz) - radius * radius);
    if (disc <= 0.0f || !isfinite(disc)) return false;
    root = sqrtf(disc);
    nt = -b - root;
    ft = -b + root;
    return true;
}

__device__ __forceinline__ float3 heatmap(float t) {
    const float tc = fminf(fmaxf(t, 0.0f), 1.0f);
    if (tc < 0.25f) return make_float3(0.0f, tc / 0.25f, 1.0f);
    if (tc < 0.5f) return make_float3(0.0f, 1.0f, 1.0f - (tc - 0.25f) / 0.25f);
    if (tc < 0.75f) return make_float3((tc - 0.5f) / 0.25f, 1.0f, 0.0f);
    return make_float3(1.0f, 1.0f - (tc - 0.75f) / 0.25f, 0.0f);
}

// Persistent ray dispenser: refills idle lanes of the calling warp.  Returns
// the updated "active" flag for this lane; sets drained when the dispenser
// has run out.  Work index w is assigned to a lane that was idle.
__device__ __forceinline__ bool refill(uint32_t *counter, uint32_t total, bool active,
                                       bool &drained, uint32_t &w) {
    const unsigned idle = __ballot_sync(kFull, !active);
    if (drained || idle == 0) return false;
    const int cnt = __popc(idle);
    if (idle != kFull && cnt < kRefillMin) return false;
    const unsigned lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, (uint32_t)cnt);
    base = __shfl_sync(kFull, base, 0);
    if (base + (uint32_t)cnt >= total) drained = true;
    if (active) return false;
    const uint32_t rank = __popc(idle & ((1u << lane) - 1u));
    w = base + rank;
    return w < total;
}

// ---------------------------------------------------------------------------
// forward render: trace_one_ray per pixel
// ---------------------------------------------------------------------------
template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock)
walk_forward_kernel(const __grid_constant__ WalkParams P) {
    const DeviceModel &m = P.m;
    bool drained = false, active = false;
    Ray ray;
    float t0 = 0.f, T = 1.f, ar = 0.f, ag = 0.f, ab = 0.f, depth = 0.f;
    float cpx = 0.f, cpy = 0.f, cpz = 0.f, cr = 0.f;
    uint32_t cur = 0, steps = 0, visited = 0;
    size_t out_index = 0;
    unsigned long long n_rays = 0, n_steps = 0, n_faces = 0;
    for (;;) {
        uint32_t w;
        if (refill(P.work_counter, P.total_work, active, drained, w)) {
            uint32_t view, x, y;
            if (work_item(P, w, view, x, y)) {
                const ViewDesc &vd = P.views[view];
                out_index = pixel_index(P, view, x, y);
                const uint32_t start = P.start_cells[view];
                const bool ok = make_ray(vd, x, y, ray);
                cur = start;
                const float4 g = __ldg(m.geom + cur);
                cpx = g.x;
                cpy = g.y;
                cpz = g.z;
                cr = g.w;
                t0 = 0.f;
                T = 1.f;
                ar = ag = ab = 0.f;
                depth = vd.depth;
                steps = 0;
                visited = 0;
                n_rays += 1;
                if (ok) {
                    active = true;
                } else {
                    P.out_rgba[out_index] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (drained) break;
            continue;
        }
        if (!active) continue;
        // one iteration of trace_one_ray's loop (trace.rs:1722-1809)
        bool done = false;
        if (steps >= P.max_steps) {
            done = true;
        } else {
            steps += 1;
            if (T <= P.weight_threshold || t0 > depth) {
                done = true;
            } else {
                float best;
                uint32_t nj, faces;
                float4 ng;
                find_exit<BOUNDED>(m, cur, cpx, cpy, cpz, cr, ray, t0, depth, best, nj, ng, faces);
                n_steps += 1;
                n_faces += faces;
                float ss, se;
                if (support<BOUNDED>(ray, cpx, cpy, cpz, cr, t0, best, ss, se)) {
                    visited += 1;
                    const float dens = __ldg(m.density + cur) * 1.0f;
                    if (dens > 1e-6f) {
                        const float dt = se - ss;
                        const float alpha = 1.0f - bv_expf(-dens * dt);
                        const float wgt = T * alpha;
                        float c[ShDims<DEG>::N];
                        load_sh_row<DEG, BF16>(m, cur, c);
                        float r, g, b;
                        eval_sh<DEG>(c, ray.dx, ray.dy, ray.dz, r, g, b);
                        ar += wgt * fmaxf(r, 0.0f);
                        ag += wgt * fmaxf(g, 0.0f);
                        ab += wgt * fmaxf(b, 0.0f);
                        T *= 1.0f - alpha;
                    }
                }
                if (nj == kNone) {
                    t0 = best;
                    done = true;
                } else {
                    t0 = fmaxf(t0, best);
                    cur = nj;
                    cpx = ng.x;
                    cpy = ng.y;
                    cpz = ng.z;
                    cr = ng.w;
                }
            }
        }
        if (done) {
            float4 o = make_float4(ar, ag, ab, 1.0f - T);
            if (P.debug_cell_density) {
                const float3 h = heatmap((float)visited / 100.0f);
                o = make_float4(h.x, h.y, h.z, 1.0f);
            }
            P.out_rgba[out_index] = o;
            active = false;
        }
    }
    if (P.stats) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            n_rays += __shfl_xor_sync(kFull, n_rays, s);
            n_steps += __shfl_xor_sync(kFull, n_steps, s);
            n_faces += __shfl_xor_sync(kFull, n_faces, s);
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicAdd(P.stats + 0, n_rays);
            atomicAdd(P.stats + 1, n_steps);
            atomicAdd(P.stats + 2, n_faces);
        }
    }
}

// ---------------------------------------------------------------------------
// path recorder: record_path_jacobians (trace.rs:1573-1676) per pixel
// ---------------------------------------------------------------------------
__device__ __forceinline__ void face_jacobian(const Ray &ray, float cpx, float cpy, float cpz,
                                              float cr, float apx, float apy, float apz, float ar,
                                              float t, float4 &cj, float4 &aj) {
    const float nx = apx - cpx, ny = apy - cpy, nz = apz - cpz;
    const float den = dot3(ray.dx, ray.dy, ray.dz, nx, ny, nz);
    if (!isfinite(den) || fabsf(den) <= 1e-20f) {
        cj = make_float4(0.f, 0.f, 0.f, 0.f);
        aj = cj;
        return;
    }
    cj = make_float4((ray.ox - cpx + t * ray.dx) / den, (ray.oy - cpy + t * ray.dy) / den,
                     (ray.oz - cpz + t * ray.dz) / den, cr / den);
    aj = make_float4((apx - ray.ox - t * ray.dx) / den, (apy - ray.oy - t * ray.dy) / den,
                     (apz - ray.oz - t * ray.dz) / den, -ar / den);
}

__device__ __forceinline__ float4 f4add(float4 a, float4 b) {
    return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 f4sub(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}

// One recorded segment with its dt Jacobians (path_interval_jacobian,
// trace.rs:1199-1325, without oriented surfaces).
struct Segment {
    float start, end;
    float4 jp, jc, jn;  // d dt / d (x, y, z, r) of previous, current, next
};

template <bool BOUNDED>
__device__ __forceinline__ bool interval_jacobian(const Ray &ray, uint32_t prev, uint32_t cur,
                                                  uint32_t next, float ppx, float ppy, float ppz,
                                                  float pr, float cpx, float cpy, float cpz,
                                                  float cr, float4 ng, float t0, float t1,
                                                  bool want_jac, Segment &sg) {
    float start = t0, end = t1;
    bool start_sphere = false, end_sphere = false;
    float4 nj = make_float4(0.f, 0.f, 0.f, 0.f), fj = nj;
    float4 qprev = nj, qcur = nj;
    if (BOUNDED) {
        float nt, ft, root, b;
        if (!sphere_hit(ray, cpx, cpy, cpz, cr, nt, ft, root, b)) return false;
        if (nt > start) {
            start = nt;
            start_sphere = true;
        }
        if (ft < end) {
            end = ft;
            end_sphere = true;
        }
        if (want_jac) {
            const float ocx = ray.ox - cpx, ocy = ray.oy - cpy, ocz = ray.oz - cpz;
            const float px = ocx - b * ray.dx, py = ocy - b * ray.dy, pz = ocz - b * ray.dz;
            const float rx = px / root, ry = py / root, rz = pz / root;
            const float rr = cr / root;
            nj = make_float4(ray.dx - rx, ray.dy - ry, ray.dz - rz, -rr);
            fj = make_float4(ray.dx + rx, ray.dy + ry, ray.dz + rz, rr);
        }
    }
    if (end <= start || !isfinite(start) || !isfinite(end)) return false;
    sg.start = start;
    sg.end = end;
    if (!want_jac) return true;
    if (start_sphere) {
        qcur = nj;
    } else if (prev != cur) {
        face_jacobian(ray, cpx, cpy, cpz, cr, ppx, ppy, ppz, pr, t0, qcur, qprev);
    }
    float4 jp = make_float4(0.f, 0.f, 0.f, 0.f), jc = jp, jn = jp;
    jc = f4sub(jc, qcur);
    jp = f4sub(jp, qprev);
    if (end_sphere) {
        jc = f4add(jc, fj);
    } else if (next != cur) {
        float4 cj, aj;
        face_jacobian(ray, cpx, cpy, cpz, cr, ng.x, ng.y, ng.z, ng.w, t1, cj, aj);
        jc = f4add(jc, cj);
        jn = f4add(jn, aj);
    }
    sg.jp = jp;
    sg.jc = jc;
    sg.jn = jn;
    return true;
}

template <bool BOUNDED>
__global__ void __launch_bounds__(kWalkBlock)
record_paths_kernel(const __grid_constant__ RecordParams P) {
    const DeviceModel &m = P.m;
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= P.total_work) return;
    uint32_t view, x, y;
    if (!work_item(P, w, view, x, y)) return;
    const ViewDesc &vd = P.views[view];
    const size_t pix = pixel_index(P, view, x, y);
    const size_t row = pix * P.buf.max_steps;
    Ray ray;
    uint32_t count = 0, status = 0;
    if (make_ray(vd, x, y, ray)) {
        float t0 = 0.0f;
        uint32_t cur = P.start_cells[view], prev = cur;
        float4 g = __ldg(m.geom + cur);
        float cpx = g.x, cpy = g.y, cpz = g.z, cr = g.w;
        float ppx = cpx, ppy = cpy, ppz = cpz, pr = cr;
        const bool want_jac = P.buf.dt_grad_current_dev || P.buf.dt_grad_previous_dev ||
                              P.buf.dt_grad_next_dev;
        uint32_t steps = 0;
        bool finished = false;
        while (steps < P.max_steps) {
            steps += 1;
            if (t0 > vd.depth) {
                finished = true;
                break;
            }
            float best;
            uint32_t nj, faces;
            float4 ng;
            find_exit<BOUNDED>(m, cur, cpx, cpy, cpz, cr, ray, t0, vd.depth, best, nj, ng, faces);
            const uint32_t next = nj == kNone ? cur : nj;
            Segment sg;
            if (interval_jacobian<BOUNDED>(ray, prev, cur, next, ppx, ppy, ppz, pr, cpx, cpy, cpz,
                                           cr, ng, t0, best, want_jac, sg)) {
                if (count < P.buf.max_steps) {
                    const size_t k = row + count;
                    if (P.buf.previous_cells_dev) P.buf.previous_cells_dev[k] = prev;
                    if (P.buf.cells_dev) P.buf.cells_dev[k] = cur;
                    if (P.buf.next_cells_dev) P.buf.next_cells_dev[k] = next;
                    if (P.buf.dts_dev) P.buf.dts_dev[k] = sg.end - sg.start;
                    if (P.buf.dt_grad_previous_dev)
                        reinterpret_cast<float4 *>(P.buf.dt_grad_previous_dev)[k] = sg.jp;
                    if (P.buf.dt_grad_current_dev)
                        reinterpret_cast<float4 *>(P.buf.dt_grad_current_dev)[k] = sg.jc;
                    if (P.buf.dt_grad_next_dev)
                        reinterpret_cast<float4 *>(P.buf.dt_grad_next_dev)[k] = sg.jn;
                }
                count += 1;
            }
            if (nj == kNone) {
                finished = true;
                break;
            }
            t0 = fmaxf(t0, best);
            prev = cur;
            ppx = cpx;
            ppy = cpy;
            ppz = cpz;
            pr = cr;
            cur = nj;
            cpx = ng.x;
            cpy = ng.y;
            cpz = ng.z;
            cr = ng.w;
        }
        if (!finished) status = BV_PATH_TRUNCATED;
    }
    if (P.buf.path_status_dev)
        P.buf.path_status_dev[pix] = (count < P.buf.max_steps ? count : P.buf.max_steps) | status;
}

// ---------------------------------------------------------------------------
// fused forward + loss + replay backward
// ---------------------------------------------------------------------------
// Error-free sum a + b = s + e (Knuth's two-sum).
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
    s = a + b;
    const float bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// Compensated accumulator: hi + lo carries the running sum to about twice
// FP32 precision, so that the suffix C - P_k of the replay stays accurate.
__device__ __forceinline__ void acc_add(float &hi, float &lo, float v) {
    float s, e;
    two_sum(hi, v, s, e);
    hi = s;
    lo = lo + e;
}

template <int DEG>
__device__ __forceinline__ void scatter_sh(float *d_sh, uint32_t cell, float gw0, float gw1,
                                           float gw2, const float (&Y)[ShDims<DEG>::K],
                                           bool m0, bool m1, bool m2) {
    constexpr int K = ShDims<DEG>::K;
    constexpr int N = 3 * K;
    float *row = d_sh + (size_t)cell * N;
    const float gw[3] = {m0 ? gw0 : 0.f, m1 ? gw1 : 0.f, m2 ? gw2 : 0.f};
    if (N % 4 == 0) {
        float4 *row4 = reinterpret_cast<float4 *>(row);
#pragma unroll
        for (int q = 0; q < N / 4; ++q) {
            float v[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int i = q * 4 + h;
                v[h] = gw[i % 3] * Y[i / 3];
            }
            atomicAdd(row4 + q, make_float4(v[0], v[1], v[2], v[3]));
        }
    } else {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const float v = gw[i % 3] * Y[i / 3];
            if (v != 0.0f) atomicAdd(row + i, v);
        }
    }
}

__device__ __forceinline__ void scatter_pos(float *d_pos, float *d_radius, uint32_t cell,
                                            float gdt, float4 j) {
    if (d_pos) {
        float *p = d_pos + 3 * (size_t)cell;
        atomicAdd(p + 0, gdt * j.x);
        atomicAdd(p + 1, gdt * j.y);
        atomicAdd(p + 2, gdt * j.z);
    }
    if (d_radius && j.w != 0.0f) atomicAdd(d_radius + cell, gdt * j.w);
}

template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock)
forward_backward_kernel(const __grid_constant__ TrainParams P) {
    const DeviceModel &m = P.m;
    constexpr int K = ShDims<DEG>::K;
    bool drained = false, active = false;
    bool replay = false;
    Ray ray;
    float t0 = 0.f, T = 1.f, depth = 0.f;
    uint32_t cur = 0, prev = 0, steps = 0, start_cell = 0;
    float cpx = 0.f, cpy = 0.f, cpz = 0.f, cr = 0.f, ppx = 0.f, ppy = 0.f, ppz = 0.f, pr = 0.f;
    float Ch[3] = {0.f, 0.f, 0.f}, Cl[3] = {0.f, 0.f, 0.f};  // forward colour
    float Ph[3] = {0.f, 0.f, 0.f}, Pl[3] = {0.f, 0.f, 0.f};  // replay prefix
    float gC[3] = {0.f, 0.f, 0.f};                          // dL/dC
    size_t pix = 0;
    float loss_acc = 0.f;
    unsigned long long n_rays = 0, n_steps = 0, n_faces = 0;
    for (;;) {
        uint32_t w;
        if (refill(P.work_counter, P.total_work, active, drained, w)) {
            uint32_t view, x, y;
            if (work_item(P, w, view, x, y)) {
                const ViewDesc &vd = P.views[view];
                pix = pixel_index(P, view, x, y);
                make_ray(vd, x, y, ray);
                start_cell = P.start_cells[view];
                depth = vd.depth;
                replay = false;
                active = true;
                n_rays += 1;
                for (int c = 0; c < 3; ++c) {
                    Ch[c] = Cl[c] = Ph[c] = Pl[c] = 0.f;
                }
                // (re)start of the walk is done below when steps == 0
                steps = 0;
                cur = kNone;
            }
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (drained) break;
            continue;
        }
        if (!active) continue;
        if (cur == kNone) {
            cur = start_cell;
            prev = cur;
            const float4 g = __ldg(m.geom + cur);
            cpx = ppx = g.x;
            cpy = ppy = g.y;
            cpz = ppz = g.z;
            cr = pr = g.w;
            t0 = 0.f;
            T = 1.f;
            steps = 0;
        }
        bool done = false;
        const bool dir_ok = ray.dx != 0.f || ray.dy != 0.f || ray.dz != 0.f;
        if (!dir_ok || steps >= P.max_steps) {
            done = true;
        } else {
            steps += 1;
            if (T <= P.weight_threshold || t0 > depth) {
                done = true;
            } else {
                float best;
                uint32_t nj, faces;
                float4 ng;
                find_exit<BOUNDED>(m, cur, cpx, cpy, cpz, cr, ray, t0, depth, best, nj, ng, faces);
                if (!replay) {
                    n_steps += 1;
                    n_faces += faces;
                }
                const uint32_t next = nj == kNone ? cur : nj;
                Segment sg;
                if (interval_jacobian<BOUNDED>(ray, prev, cur, next, ppx, ppy, ppz, pr, cpx, cpy,
                                               cpz, cr, ng, t0, best, replay, sg)) {
                    const float dens = __ldg(m.density + cur);
                    if (dens > 1e-6f) {
                        const float dt_raw = sg.end - sg.start;
                        const float dt = fminf(dt_raw, P.max_dt);
                        const float alpha = 1.0f - bv_expf(-dens * dt);
                        const float wgt = T * alpha;
                        const float Tn = T * (1.0f - alpha);
                        float c[ShDims<DEG>::N];
                        load_sh_row<DEG, BF16>(m, cur, c);
                        float cu[3];
                        eval_sh<DEG>(c, ray.dx, ray.dy, ray.dz, cu[0], cu[1], cu[2]);
                        const float cc[3] = {fmaxf(cu[0], 0.f), fmaxf(cu[1], 0.f),
                                             fmaxf(cu[2], 0.f)};
                        if (!replay) {
#pragma unroll
                            for (int ch = 0; ch < 3; ++ch) acc_add(Ch[ch], Cl[ch], wgt * cc[ch]);
                        } else {
                            float gs = 0.f;
#pragma unroll
                            for (int ch = 0; ch < 3; ++ch) {
                                acc_add(Ph[ch], Pl[ch], wgt * cc[ch]);
                                const float suffix = (Ch[ch] - Ph[ch]) + (Cl[ch] - Pl[ch]);
                                gs += gC[ch] * (Tn * cc[ch] - suffix);
                            }
                            atomicAdd(P.d_density + cur, dt * gs);
                            float Y[K];
                            sh_basis<DEG>(ray.dx, ray.dy, ray.dz, Y);
                            scatter_sh<DEG>(P.d_sh, cur, gC[0] * wgt, gC[1] * wgt, gC[2] * wgt, Y,
                                            cu[0] > 0.f, cu[1] > 0.f, cu[2] > 0.f);
                            if ((P.d_pos || P.d_radius) && dt_raw < P.max_dt) {
                                const float gdt = dens * gs;
                                if (prev != cur) scatter_pos(P.d_pos, P.d_radius, prev, gdt, sg.jp);
                                scatter_pos(P.d_pos, P.d_radius, cur, gdt, sg.jc);
                                if (next != cur) scatter_pos(P.d_pos, P.d_radius, next, gdt, sg.jn);
                            }
                        }
                        T = Tn;
                    }
                }
                if (nj == kNone) {
                    done = true;
                } else {
                    t0 = fmaxf(t0, best);
                    prev = cur;
                    ppx = cpx;
                    ppy = cpy;
                    ppz = cpz;
                    pr = cr;
                    cur = nj;
                    cpx = ng.x;
                    cpy = ng.y;
                    cpz = ng.z;
                    cr = ng.w;
                }
            }
        }
        if (done) {
            if (!replay) {
                const float *tg = P.target + 3 * pix;
                float l = 0.f;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    const float col = Ch[ch] + Cl[ch];
                    const float diff = col - __ldg(tg + ch);
                    if (P.loss_kind == BV_LOSS_L2) {
                        l += diff * diff;
                        gC[ch] = 2.0f * diff * P.inv_count;
                    } else {
                        l += fabsf(diff);
                        gC[ch] = (diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f)) * P.inv_count;
                    }
                    if (P.rgb_out) P.rgb_out[3 * pix + ch] = col;
                }
                loss_acc += l;
                replay = true;
                cur = kNone;  // restart the same ray for the replay
            } else {
                active = false;
            }
        }
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) loss_acc += __shfl_xor_sync(kFull, loss_acc, s);
    if ((threadIdx.x & 31u) == 0 && loss_acc != 0.f) atomicAdd(P.loss, loss_acc * P.inv_count);
    if (P.stats) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            n_rays += __shfl_xor_sync(kFull, n_rays, s);
            n_steps += __shfl_xor_sync(kFull, n_steps, s);
            n_faces += __shfl_xor_sync(kFull, n_faces, s);
        }
        if ((threadIdx.x & 31u) == 0) {
            atomicAdd(P.stats + 0, n_rays);
            atomicAdd(P.stats + 1, n_steps);
            atomicAdd(P.stats + 2, n_faces);
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers: pick the instantiation for (SH degree, bounded, bf16)
// ---------------------------------------------------------------------------
#define BV_SELECT(KERNEL, PARAMS, GRID, STREAM)                                                 \
    do {                                                                                        \
        const DeviceModel &mm = (PARAMS).m;                                                     \
        const int key = (int)mm.sh_degree * 4 + (mm.bounded ? 2 : 0) + (mm.sh_bf16 ? 1 : 0);    \
        switch (key) {                                                                          \
            case 0: KERNEL<0, false, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;     \
            case 1: KERNEL<0, false, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            case 2: KERNEL<0, true, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            case 3: KERNEL<0, true, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;       \
            case 4: KERNEL<1, false, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;     \
            case 5: KERNEL<1, false, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            case 6: KERNEL<1, true, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            case 7: KERNEL<1, true, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;       \
            case 8: KERNEL<2, false, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;     \
            case 9: KERNEL<2, false, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            case 10: KERNEL<2, true, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;     \
            case 11: KERNEL<2, true, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            case 12: KERNEL<3, false, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;    \
            case 13: KERNEL<3, false, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;     \
            case 14: KERNEL<3, true, false><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;     \
            case 15: KERNEL<3, true, true><<<GRID, kWalkBlock, 0, STREAM>>>(PARAMS); break;      \
            default: return cudaErrorInvalidValue;                                              \
        }                                                                                       \
    } while (0)

cudaError_t launch_walk_forward(const WalkParams &p, int grid, cudaStream_t s) {
    BV_SELECT(walk_forward_kernel, p, grid, s);
    return cudaGetLastError();
}

cudaError_t launch_forward_backward(const TrainParams &p, int grid, cudaStream_t s) {
    BV_SELECT(forward_backward_kernel, p, grid, s);
    return cudaGetLastError();
}

cudaError_t launch_record_paths(const RecordParams &p, int grid, cudaStream_t s) {
    (void)grid;
    const int blocks = (int)((p.total_work + kWalkBlock - 1) / kWalkBlock);
    if (blocks == 0) return cudaSuccess;
    if (p.m.bounded)
        record_paths_kernel<true><<<blocks, kWalkBlock, 0, s>>>(p);
    else
        record_paths_kernel<false><<<blocks, kWalkBlock, 0, s>>>(p);
    return cudaGetLastError();
}

// Persistent grid: enough resident blocks to fill every SM.
int walk_grid_size(int device, int kind) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    int per_sm = 1;
    if (kind == 0)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, walk_forward_kernel<3, false, false>,
                                                      kWalkBlock, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
                                                      forward_backward_kernel<3, false, false>,
                                                      kWalkBlock, 0);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

}  // namespace bv
