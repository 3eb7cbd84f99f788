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
// Scheduling: one ray per lane, persistent warps.  A warp takes a whole 8x4
// pixel tile (32 tile-ordered work items) from a global ray dispenser and
// keeps it until every lane is done (BV_REFILL_MIN = 32: refilling single
// lanes was measured slower, because lockstep rays of one tile share cells,
// which the L1 and the gradient aggregation exploit).

#include <cuda_bf16.h>

#include "bv_internal.h"
#include "bv_device.cuh"
#include "bv_segment.cuh"
#include "bv_tile_order.cuh"

namespace bv {
namespace {

constexpr int kWalkBlock = 256;

// Tuning knobs (measured on B200; see the profiles): face entries in flight
// per lane, idle lanes that trigger a refill, and resident blocks per SM
// requested from the register allocator for each kernel.
#ifndef BV_FACE_UNROLL
#define BV_FACE_UNROLL 4
#endif
#ifndef BV_MINB_RENDER
#define BV_MINB_RENDER 4
#endif
#ifndef BV_MINB_TRAIN_FWD
#define BV_MINB_TRAIN_FWD 4
#endif
#ifndef BV_MINB_TRAIN_BWD
#define BV_MINB_TRAIN_BWD 3
#endif
#ifndef BV_REC_PREFETCH
#define BV_REC_PREFETCH 1
#endif
// Exit search: skip the division of faces that provably cannot win (1).
#ifndef BV_EXIT_DIV_SAVER
#define BV_EXIT_DIV_SAVER 1
#endif
constexpr int kFaceUnroll = BV_FACE_UNROLL;


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

// Exit distance through a face (neighbour site s) of cell c in FP64 from the
// FP32 inputs: the re-evaluation of the exit-face tie-break.
template <bool BOUNDED>
__device__ __noinline__ double face_t_f64(const Cell &c, const float4 &s, const Ray &ray) {
    const double offx = (double)s.x - (double)c.x, offy = (double)s.y - (double)c.y,
                 offz = (double)s.z - (double)c.z;
    double shift = 0.5;
    if (BOUNDED) {
        const double ri = c.r, rj = s.w;
        shift = 0.5 + 0.5 * (ri * ri - rj * rj) / fmax(offx * offx + offy * offy + offz * offz, 1e-20);
    }
    const double rx = ((double)c.x + shift * offx) - (double)ray.ox;
    const double ry = ((double)c.y + shift * offy) - (double)ray.oy;
    const double rz = ((double)c.z + shift * offz) - (double)ray.oz;
    return (rx * offx + ry * offy + rz * offz) /
           (offx * (double)ray.dx + offy * (double)ray.dy + offz * (double)ray.dz);
}

// Runner-up distances within this many FP32 ulps of the winner are re-evaluated.
constexpr float kTieUlps = 4.0f;

// ---------------------------------------------------------------------------
// Exit distance through the face of cell c towards neighbour site s
// (find_exit_face's per-face arithmetic, trace.rs:170-205): the radical
// plane's point c + shift (s - c), shift = 0.5 + 0.5 (r_c^2 - r_s^2) / |s - c|^2
// (0.5 for RadFoam), and t = <point - o, s - c> / <s - c, d>.  False when the
// ray does not move towards the face (<s - c, d> <= 0).  The search and the
// replay of a recorded exit both evaluate a face through this function, so a
// recorded face reproduces the searched t bit for bit.
template <bool BOUNDED>
__device__ __forceinline__ bool face_exit_nd(const Cell &c, float ri2, const float4 &site,
                                             const Ray &ray, float &num, float &dp) {
    const float offx = site.x - c.x, offy = site.y - c.y, offz = site.z - c.z;
    float shift;
    if (BOUNDED) {
        const float rj = site.w;
        const float dsq = fmaxf(dot3(offx, offy, offz, offx, offy, offz), 1e-20f);
        shift = 0.5f + 0.5f * (ri2 - rj * rj) / dsq;
    } else {
        shift = 0.5f;
    }
    const float fox = c.x + shift * offx;
    const float foy = c.y + shift * offy;
    const float foz = c.z + shift * offz;
    dp = dot3(offx, offy, offz, ray.dx, ray.dy, ray.dz);
    if (!(dp > 0.0f)) return false;
    num = dot3(fox - ray.ox, foy - ray.oy, foz - ray.oz, offx, offy, offz);
    return true;
}

template <bool BOUNDED>
__device__ __forceinline__ bool face_exit_t(const Cell &c, float ri2, const float4 &site,
                                            const Ray &ray, float &t) {
    float num, dp;
    if (!face_exit_nd<BOUNDED>(c, ri2, site, ray, num, dp)) return false;
    t = num / dp;
    return true;
}

// True when num / dp >= best holds exactly (dp > 0, best > 0), so that the
// rounded quotient cannot be below best and the face cannot win: a division
// saved.  p = fl(best dp) is within one rounding of best dp, so
// fl(p (1 + 2^-21)) >= best dp whenever p is a normal number.  Otherwise (and
// for NaN) the caller divides, which keeps the search's result bit for bit.
__device__ __forceinline__ bool quotient_not_below(float num, float dp, float best) {
    const float p = best * dp;
    return p > 1.0e-30f && num >= p * 1.000000476837158203125f;
}

// find_exit_face (trace.rs:170-205): the first face in CSR order with the
// smallest t in (t0, best).  The face entries of the current cell are read
// four at a time so that four independent loads are in flight; the winner's
// entry already carries the next cell's site, CSR range and density.
// TIE: the runner-up is tracked too, and when its FP32 distance is within
// kTieUlps ulps of the winner's both are re-evaluated in FP64 and the smaller
// wins (equal: the earlier face in CSR order, the reference's own rule).
// ---------------------------------------------------------------------------
template <bool BOUNDED, bool TIE = false>
__device__ __forceinline__ bool find_exit(const DeviceModel &m, const Cell &c, const Ray &ray,
                                          float t0, float depth, float &best, FaceEntry &win,
                                          uint32_t &face) {
    best = depth;
    uint32_t best_k = 0xffffffffu;
    float4 best_site = make_float4(0.f, 0.f, 0.f, 0.f);
    float second = depth;
    uint32_t second_k = 0xffffffffu;
    float4 second_site = best_site;
    const float ri2 = c.r * c.r;
    for (uint32_t k = c.begin; k < c.end; k += kFaceUnroll) {
        float4 site[kFaceUnroll];
#pragma unroll
        for (int u = 0; u < kFaceUnroll; ++u) site[u] = __ldg(&m.faces[min(k + u, c.end - 1)].site);
#pragma unroll
        for (int u = 0; u < kFaceUnroll; ++u) {
            if (k + u < c.end) {
                float num, dp;
                if (face_exit_nd<BOUNDED>(c, ri2, site[u], ray, num, dp) &&
                    (TIE || !BV_EXIT_DIV_SAVER || !quotient_not_below(num, dp, best))) {
                    const float t = num / dp;
                    if (isfinite(t) && t > t0 && t < best) {
                        if (TIE) {
                            second = best;
                            second_k = best_k;
                            second_site = best_site;
                        }
                        best = t;
                        best_k = k + u;
                        best_site = site[u];
                    } else if (TIE && isfinite(t) && t > t0 && t < second && t < depth) {
                        second = t;
                        second_k = k + u;
                        second_site = site[u];
                    }
                }
            }
        }
    }
    if (best_k == 0xffffffffu) return false;
    if (TIE && second_k != 0xffffffffu) {
        const float ab = fabsf(best);
        const float ulp = __uint_as_float(__float_as_uint(ab) + 1u) - ab;
        if (second - best <= kTieUlps * ulp) {
            const double tb = face_t_f64<BOUNDED>(c, best_site, ray);
            const double t2 = face_t_f64<BOUNDED>(c, second_site, ray);
            if (t2 < tb || (t2 == tb && second_k < best_k)) {
                best = second;
                best_k = second_k;
                best_site = second_site;
            }
        }
    }
    // The winner's link shares the 32-byte sector of the site just read.
    win.site = best_site;
    win.link = __ldg(&m.faces[best_k].link);
    face = best_k;
    return true;
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

__device__ __forceinline__ float3 heatmap(float t) {
    const float tc = fminf(fmaxf(t, 0.0f), 1.0f);
    if (tc < 0.25f) return make_float3(0.0f, tc / 0.25f, 1.0f);
    if (tc < 0.5f) return make_float3(0.0f, 1.0f, 1.0f - (tc - 0.25f) / 0.25f);
    if (tc < 0.75f) return make_float3((tc - 0.5f) / 0.25f, 1.0f, 0.0f);
    return make_float3(1.0f, 1.0f - (tc - 0.75f) / 0.25f, 0.0f);
}


// ---------------------------------------------------------------------------
// forward render: trace_one_ray per pixel
// ---------------------------------------------------------------------------
template <int DEG, bool BOUNDED, bool BF16, bool TIE>
__device__ __forceinline__ void walk_forward_body(const WalkParams &P) {
    const DeviceModel &m = P.m;
    bool drained = false, active = false;
    Ray ray;
    Cell c;
    float t0 = 0.f, T = 1.f, ar = 0.f, ag = 0.f, ab = 0.f, depth = 0.f;
    uint32_t steps = 0, visited = 0;
    size_t out_index = 0;
    uint32_t n_rays = 0, n_steps = 0, n_faces = 0;
    for (;;) {
        uint32_t w;
        if (refill(P.work_counter, P.total_work, active, drained, w)) {
            uint32_t view, x, y;
            if (work_item(P, w, view, x, y)) {
                const ViewDesc &vd = P.views[view];
                out_index = pixel_index(P, view, x, y);
                const bool ok = make_ray(vd, x, y, ray);
                c = load_cell(m, P.start_cells[view]);
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
                FaceEntry win;
                uint32_t face;
                const bool has_exit =
                    find_exit<BOUNDED, TIE>(m, c, ray, t0, depth, best, win, face);
                n_steps += 1;
                n_faces += c.end - c.begin;
                float ss, se;
                if (support<BOUNDED>(ray, c.x, c.y, c.z, c.r, t0, best, ss, se)) {
                    visited += 1;
                    const float dens = c.density * 1.0f;
                    if (dens > 1e-6f) {
                        const float dt = se - ss;
                        const float alpha = 1.0f - bv_expf(-dens * dt);
                        const float wgt = T * alpha;
                        float coef[ShDims<DEG>::N];
                        load_sh_row<DEG, BF16>(m, c.id, coef);
                        float r, g, b;
                        eval_sh<DEG>(coef, ray.dx, ray.dy, ray.dz, r, g, b);
                        ar += wgt * fmaxf(r, 0.0f);
                        ag += wgt * fmaxf(g, 0.0f);
                        ab += wgt * fmaxf(b, 0.0f);
                        T *= 1.0f - alpha;
                    }
                }
                if (!has_exit) {
                    t0 = best;
                    done = true;
                } else {
                    t0 = fmaxf(t0, best);
                    c = cell_from_face(win);
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
            atomicAdd(P.stats + 0, (unsigned long long)n_rays);
            atomicAdd(P.stats + 1, (unsigned long long)n_steps);
            atomicAdd(P.stats + 2, (unsigned long long)n_faces);
        }
    }
}

template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock, BV_MINB_RENDER)
walk_forward_kernel(const __grid_constant__ WalkParams P) {
    walk_forward_body<DEG, BOUNDED, BF16, false>(P);
}

// The render walk with the FP64 exit-face tie-break.
template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock, BV_MINB_RENDER)
walk_forward_tb_kernel(const __grid_constant__ WalkParams P) {
    walk_forward_body<DEG, BOUNDED, BF16, true>(P);
}

// ---------------------------------------------------------------------------
// path recorder: record_path_jacobians (trace.rs:1573-1676) per pixel
// ---------------------------------------------------------------------------
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
        Cell c = load_cell(m, P.start_cells[view]);
        uint32_t prev = c.id;
        float4 pp = make_float4(c.x, c.y, c.z, c.r);
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
            FaceEntry win;
            uint32_t face;
            const bool has_exit = find_exit<BOUNDED>(m, c, ray, t0, vd.depth, best, win, face);
            const uint32_t next = has_exit ? win.link.x : c.id;
            Interval iv;
            if (record_interval<BOUNDED>(ray, c, t0, best, iv)) {
                if (count < P.buf.max_steps) {
                    const size_t k = row + count;
                    if (P.buf.previous_cells_dev) P.buf.previous_cells_dev[k] = prev;
                    if (P.buf.cells_dev) P.buf.cells_dev[k] = c.id;
                    if (P.buf.next_cells_dev) P.buf.next_cells_dev[k] = next;
                    if (P.buf.dts_dev) P.buf.dts_dev[k] = iv.end - iv.start;
                    if (want_jac) {
                        const Jacobians J = interval_jacobians(ray, iv, prev, pp, c, has_exit,
                                                               win.site, t0, best);
                        if (P.buf.dt_grad_previous_dev)
                            reinterpret_cast<float4 *>(P.buf.dt_grad_previous_dev)[k] = J.jp;
                        if (P.buf.dt_grad_current_dev)
                            reinterpret_cast<float4 *>(P.buf.dt_grad_current_dev)[k] = J.jc;
                        if (P.buf.dt_grad_next_dev)
                            reinterpret_cast<float4 *>(P.buf.dt_grad_next_dev)[k] = J.jn;
                    }
                }
                count += 1;
            }
            if (!has_exit) {
                finished = true;
                break;
            }
            t0 = fmaxf(t0, best);
            prev = c.id;
            pp = make_float4(c.x, c.y, c.z, c.r);
            c = cell_from_face(win);
        }
        if (!finished) status = BV_PATH_TRUNCATED;
    }
    if (P.buf.path_status_dev)
        P.buf.path_status_dev[pix] = (count < P.buf.max_steps ? count : P.buf.max_steps) | status;
}

// ---------------------------------------------------------------------------
// training: forward + loss kernel, then the replay backward kernel
// ---------------------------------------------------------------------------
// The walk of the training contract: record_path_jacobians' loop
// (trace.rs:1573-1676) with trace_one_ray's transmittance cut (trace.rs:1724)
// evaluated on dt clamped to max_dt (MAX_PATH_DT, diff_render.rs:2484).
// Shared operation for operation by the forward and the replay kernels.
struct TrainWalk {
    Ray ray;
    Cell c;
    uint32_t prev;
    float4 pp;
    float t0, T, depth;
    uint32_t steps;
    uint32_t work;  // dispenser index of the ray
};

// Step record of the training forward, read back by the replay: for ray w
// and step s < rec_steps a block of 4 x 32 words at ((w / 32) rec_steps + s)
// 128 holds, at lane w % 32 of each row, the exit face (kNoExitFace: the cell
// has none) and the unclamped SH colour r, g, b of the step (written when
// the step composites), so the 32 rays of a tile, which step together, write
// and read whole 128-byte lines.
// The host bounds the record to 2^31 words, so its index is 32-bit.
constexpr uint32_t kNoExitFace = 0xffffffffu;
constexpr uint32_t kNotRecorded = 0xffffffffu;
__device__ __forceinline__ uint32_t step_rec_index(const TrainParams &P, uint32_t w, uint32_t s) {
    return s < P.rec_steps ? ((w >> 5) * P.rec_steps + s) * 128u + (w & 31u) : kNotRecorded;
}

template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock, BV_MINB_TRAIN_FWD)
train_forward_kernel(const __grid_constant__ TrainParams P) {
    const DeviceModel &m = P.m;
    bool drained = false, active = false;
    TrainWalk W = {};
    float Ch[3] = {0.f, 0.f, 0.f}, Cl[3] = {0.f, 0.f, 0.f};
    size_t pix = 0;
    float loss_acc = 0.f;
    uint32_t n_rays = 0, n_steps = 0, n_faces = 0;
    // the warp's current tile and when it took it (tile times for the next
    // call's heaviest-first order)
    uint32_t tile_id = kNoTile;
    long long tile_begin = 0;
    for (;;) {
        if (P.tile_cost && tile_id != kNoTile && __ballot_sync(kFull, active) == 0) {
            store_tile_cost(P.tile_cost, tile_id << 5, tile_begin);
            tile_id = kNoTile;
        }
        uint32_t w;
        if (refill(P.work_counter, P.total_work, active, drained, w)) {
            uint32_t view, x, y;
            const uint32_t item = tile_item(P.tile_order, w);
            if (work_item(P, P.work_begin + item, view, x, y)) {
                const ViewDesc &vd = P.views[view];
                pix = pixel_index(P, view, x, y);
                const bool ok = make_ray(vd, x, y, W.ray);
                W.c = load_cell(m, P.start_cells[view]);
                W.prev = W.c.id;
                W.t0 = 0.f;
                W.T = 1.f;
                W.depth = ok ? vd.depth : -1.0f;  // a failed direction records nothing
                W.steps = 0;
                W.work = item;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) Ch[ch] = Cl[ch] = 0.f;
                active = true;
                n_rays += 1;
            }
        }
        if (P.tile_cost && tile_id == kNoTile) {
            const unsigned act = __ballot_sync(kFull, active);
            if (act) {
                tile_id = __shfl_sync(kFull, W.work >> 5, __ffs(act) - 1);
                tile_begin = clock64();
            }
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (drained) break;
            continue;
        }
        if (!active) continue;
        bool done = false;
        if (W.steps >= P.max_steps) {
            done = true;
        } else {
            W.steps += 1;
            if (W.T <= P.weight_threshold || W.t0 > W.depth) {
                done = true;
            } else {
                float best;
                FaceEntry win;
                uint32_t face = kNoExitFace;
                const bool has_exit =
                    find_exit<BOUNDED>(m, W.c, W.ray, W.t0, W.depth, best, win, face);
                if (W.steps <= P.rec_steps)
                    __stcs(P.step_rec + step_rec_index(P, W.work, W.steps - 1),
                           has_exit ? face : kNoExitFace);
                n_steps += 1;
                n_faces += W.c.end - W.c.begin;
                Interval iv;
                if (record_interval<BOUNDED>(W.ray, W.c, W.t0, best, iv)) {
                    const float dens = W.c.density;
                    if (dens > 1e-6f) {
                        const float dt = fminf(iv.end - iv.start, P.max_dt);
                        const float alpha = 1.0f - bv_expf(-dens * dt);
                        const float wgt = W.T * alpha;
                        float coef[ShDims<DEG>::N];
                        load_sh_row<DEG, BF16>(m, W.c.id, coef);
                        float cu[3];
                        eval_sh<DEG>(coef, W.ray.dx, W.ray.dy, W.ray.dz, cu[0], cu[1], cu[2]);
                        if (W.steps <= P.rec_steps) {
                            uint32_t *col = P.step_rec + step_rec_index(P, W.work, W.steps - 1);
#pragma unroll
                            for (int ch = 0; ch < 3; ++ch)
                                __stcs(col + 32u * (ch + 1), __float_as_uint(cu[ch]));
                        }
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch)
                            acc_add(Ch[ch], Cl[ch], wgt * fmaxf(cu[ch], 0.f));
                        W.T = W.T * (1.0f - alpha);
                    }
                }
                if (!has_exit) {
                    done = true;
                } else {
                    W.t0 = fmaxf(W.t0, best);
                    W.c = cell_from_face(win);
                }
            }
        }
        if (done) {
            const float *tg = P.target + 3 * pix;
            float l = 0.f, gC[3];
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
            RayState st;
            st.c_hi = make_float4(Ch[0], Ch[1], Ch[2], gC[0]);
            st.c_lo = make_float4(Cl[0], Cl[1], Cl[2], gC[1]);
            st.g = make_float4(gC[2], 0.f, 0.f, 0.f);
            P.ray_state[pix] = st;
            active = false;
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
            atomicAdd(P.stats + 0, (unsigned long long)n_rays);
            atomicAdd(P.stats + 1, (unsigned long long)n_steps);
            atomicAdd(P.stats + 2, (unsigned long long)n_faces);
        }
    }
}

// Replay: walk each ray again front to back, recompute T, w and the colour
// of every segment, form the suffix S_{k+1} = C - P_k from the compensated
// prefix, and scatter
//   dL/dsigma_k = dt_k sum_c g_c (T_{k+1} c_kc - S_{k+1,c})
//   dL/dSH_kmc  = g_c w_k Y_m(d) [c_kc unclamped > 0]
//   dL/ddt_k    = sigma_k sum_c g_c (T_{k+1} c_kc - S_{k+1,c})  -> sites
// through the exact dt Jacobians of the fixed path (trace.rs:1077-1124).
template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock, BV_MINB_TRAIN_BWD)
train_backward_kernel(const __grid_constant__ TrainParams P) {
    const DeviceModel &m = P.m;
    constexpr int K = ShDims<DEG>::K;
    constexpr int N = 3 * K;
    bool drained = false, active = false;
    TrainWalk W = {};
    float Ch[3] = {0.f, 0.f, 0.f}, Cl[3] = {0.f, 0.f, 0.f};
    float Ph[3] = {0.f, 0.f, 0.f}, Pl[3] = {0.f, 0.f, 0.f};
    float gC[3] = {0.f, 0.f, 0.f};
    for (;;) {
        uint32_t w;
        if (refill(P.work_counter + 1, P.total_work, active, drained, w)) {
            uint32_t view, x, y;
            const uint32_t item = tile_item(P.tile_order, w);
            if (work_item(P, P.work_begin + item, view, x, y)) {
                const ViewDesc &vd = P.views[view];
                const size_t pix = pixel_index(P, view, x, y);
                const bool ok = make_ray(vd, x, y, W.ray);
                W.c = load_cell(m, P.start_cells[view]);
                W.prev = W.c.id;
                W.pp = make_float4(W.c.x, W.c.y, W.c.z, W.c.r);
                W.t0 = 0.f;
                W.T = 1.f;
                W.depth = ok ? vd.depth : -1.0f;
                W.steps = 0;
                W.work = item;
                const RayState st = P.ray_state[pix];
                Ch[0] = st.c_hi.x;
                Ch[1] = st.c_hi.y;
                Ch[2] = st.c_hi.z;
                Cl[0] = st.c_lo.x;
                Cl[1] = st.c_lo.y;
                Cl[2] = st.c_lo.z;
                gC[0] = st.c_hi.w;
                gC[1] = st.c_lo.w;
                gC[2] = st.g.x;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) Ph[ch] = Pl[ch] = 0.f;
                active = (gC[0] != 0.f || gC[1] != 0.f || gC[2] != 0.f);
            }
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (drained) break;
            continue;
        }
        // one replay step per active lane; the current cell's contribution
        // is scattered below at a point all 32 lanes reach
        bool done = false, contrib = false;
        uint32_t cell = 0;
        float g_density = 0.f, gw[3] = {0.f, 0.f, 0.f};
        float4 g_site = make_float4(0.f, 0.f, 0.f, 0.f);
        if (active) {
            if (W.steps >= P.max_steps) {
                done = true;
            } else {
                W.steps += 1;
                if (W.T <= P.weight_threshold || W.t0 > W.depth) {
                    done = true;
                } else {
                    float best;
                    FaceEntry win;
                    bool has_exit;
                    const uint32_t rec = step_rec_index(P, W.work, W.steps - 1);
                    if (rec != kNotRecorded) {
#if BV_REC_PREFETCH
                        // the record streams from DRAM: start the next
                        // step's four lines on their way to L2 now
                        if (W.steps < P.rec_steps) {
                            const uint32_t *nx =
                                P.step_rec + step_rec_index(P, W.work, W.steps);
#pragma unroll
                            for (int f = 0; f < 4; ++f)
                                asm volatile("prefetch.global.L2 [%0];" ::"l"(nx + 32 * f));
                        }
#endif
                        // the forward's exit face of this step: one entry
                        // instead of the cell's row
                        const uint32_t face = __ldcs(P.step_rec + rec);
                        has_exit = face != kNoExitFace;
                        best = W.depth;
                        if (has_exit) {
                            win.site = __ldg(&m.faces[face].site);
                            win.link = __ldg(&m.faces[face].link);
                            face_exit_t<BOUNDED>(W.c, W.c.r * W.c.r, win.site, W.ray, best);
                        }
                    } else {
                        uint32_t face;
                        has_exit = find_exit<BOUNDED>(m, W.c, W.ray, W.t0, W.depth, best, win, face);
                    }
                    Interval iv;
                    if (record_interval<BOUNDED>(W.ray, W.c, W.t0, best, iv)) {
                        const float dens = W.c.density;
                        if (dens > 1e-6f) {
                            const float dt_raw = iv.end - iv.start;
                            const float dt = fminf(dt_raw, P.max_dt);
                            const float alpha = 1.0f - bv_expf(-dens * dt);
                            const float wgt = W.T * alpha;
                            const float Tn = W.T * (1.0f - alpha);
                            float cu[3];
                            if (rec != kNotRecorded) {
                                // the forward's colour of this step
#pragma unroll
                                for (int ch = 0; ch < 3; ++ch)
                                    cu[ch] = __uint_as_float(__ldcs(P.step_rec + rec + 32u * (ch + 1)));
                            } else {
                                float coef[ShDims<DEG>::N];
                                load_sh_row<DEG, BF16>(m, W.c.id, coef);
                                eval_sh<DEG>(coef, W.ray.dx, W.ray.dy, W.ray.dz, cu[0], cu[1], cu[2]);
                            }
                            float gs = 0.f;
#pragma unroll
                            for (int ch = 0; ch < 3; ++ch) {
                                const float cc = fmaxf(cu[ch], 0.f);
                                acc_add(Ph[ch], Pl[ch], wgt * cc);
                                const float suffix = (Ch[ch] - Ph[ch]) + (Cl[ch] - Pl[ch]);
                                gs += gC[ch] * (Tn * cc - suffix);
                                gw[ch] = cu[ch] > 0.f ? gC[ch] * wgt : 0.f;
                            }
                            contrib = true;
                            cell = W.c.id;
                            g_density = dt * gs;
                            if (P.d_site && dt_raw < P.max_dt) {
                                const float gdt = dens * gs;
                                const Jacobians J = interval_jacobians(
                                    W.ray, iv, W.prev, W.pp, W.c, has_exit, win.site, W.t0, best);
                                g_site = make_float4(gdt * J.jc.x, gdt * J.jc.y, gdt * J.jc.z,
                                                     gdt * J.jc.w);
                                if (W.prev != W.c.id && !iv.start_sphere)
                                    scatter_site(P.d_site, W.prev, gdt, J.jp);
                                if (has_exit && !iv.end_sphere)
                                    scatter_site(P.d_site, win.link.x, gdt, J.jn);
                            }
                            W.T = Tn;
                        }
                    }
                    if (!has_exit) {
                        done = true;
                    } else {
                        W.t0 = fmaxf(W.t0, best);
                        W.prev = W.c.id;
                        W.pp = make_float4(W.c.x, W.c.y, W.c.z, W.c.r);
                        W.c = cell_from_face(win);
                    }
                }
            }
        }
        // warp-aggregated scatter of the current cells' gradients
        const PeerTree tree = peer_tree(contrib, cell);
        float Y[K];
        sh_basis<DEG>(W.ray.dx, W.ray.dy, W.ray.dz, Y);
        if (P.d_site) {
            float v[5] = {g_density, g_site.x, g_site.y, g_site.z, g_site.w};
            group_sum(tree, v);
            if (contrib && tree.leader) {
                atomicAdd(P.d_density + cell, v[0]);
                atomicAdd(P.d_site + cell, make_float4(v[1], v[2], v[3], v[4]));
            }
        } else {
            float v[1] = {g_density};
            group_sum(tree, v);
            if (contrib && tree.leader) atomicAdd(P.d_density + cell, v[0]);
        }
        if (N % 4 == 0) {
            // eight coefficients per tree pass (four for N = 12)
            constexpr int Q = N % 8 == 0 ? 8 : 4;
            float4 *row4 = reinterpret_cast<float4 *>(P.d_sh + (size_t)cell * N);
#pragma unroll
            for (int q = 0; q < N / Q; ++q) {
                float v[Q];
#pragma unroll
                for (int h = 0; h < Q; ++h) v[h] = gw[(q * Q + h) % 3] * Y[(q * Q + h) / 3];
                group_sum(tree, v);
                if (contrib && tree.leader) {
#pragma unroll
                    for (int h = 0; h < Q; h += 4)
                        atomicAdd(row4 + (q * Q + h) / 4, make_float4(v[h], v[h + 1], v[h + 2], v[h + 3]));
                }
            }
        } else {
            float *row = P.d_sh + (size_t)cell * N;
#pragma unroll
            for (int i = 0; i < N; i += 3) {
                float v[3] = {gw[0] * Y[i / 3], gw[1] * Y[i / 3], gw[2] * Y[i / 3]};
                group_sum(tree, v);
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    if (contrib && tree.leader && v[c] != 0.0f) atomicAdd(row + i + c, v[c]);
            }
        }
        if (done) active = false;
    }
}

// ---------------------------------------------------------------------------
// serving: one persistent traversal over the frames of many requests (any
// resident scene, any resolution) listed in a device-side table.  Per ray
// the arithmetic is walk_forward_kernel's, so a frame renders bit for bit
// the same in any batch.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t serve_view_of(const ServeView *views, uint32_t n,
                                                  uint32_t w) {
    uint32_t lo = 0, hi = n - 1;  // last frame with ray_begin <= w
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) / 2;
        if (__ldg(&views[mid].v.ray_begin) <= w)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <int DEG, bool BOUNDED, bool BF16>
__global__ void __launch_bounds__(kWalkBlock, BV_MINB_RENDER)
serve_walk_kernel(const __grid_constant__ ServeParams P) {
    __shared__ DeviceModel s_scenes[kMaxServeScenes];
    if (threadIdx.x < P.n_scenes) s_scenes[threadIdx.x] = P.scenes[threadIdx.x];
    __syncthreads();
    const uint32_t n_views = P.header->n_views;
    const uint32_t total = P.header->total_work;
    bool drained = n_views == 0, active = false;
    Ray ray;
    Cell c;
    uint32_t scene = 0;
    float t0 = 0.f, T = 1.f, ar = 0.f, ag = 0.f, ab = 0.f, depth = 0.f;
    uint32_t steps = 0;
    float4 *out = nullptr;
    for (;;) {
        uint32_t w;
        if (refill(P.work_counter, total, active, drained, w)) {
            const ServeView *sv = P.views + serve_view_of(P.views, n_views, w);
            const ViewDesc vd = sv->v;
            const uint32_t local = w - vd.ray_begin;
            const uint32_t tile = local / kTileRays, in = local % kTileRays;
            const uint32_t x = (tile % vd.tiles_x) * kTileW + in % kTileW;
            const uint32_t y = (tile / vd.tiles_x) * kTileH + in / kTileW;
            if (x < vd.width && y < vd.height) {
                scene = sv->scene;
                out = reinterpret_cast<float4 *>(sv->out) + (size_t)y * vd.width + x;
                const bool ok = make_ray(vd, x, y, ray);
                c = load_cell(s_scenes[scene], sv->start_cell);
                t0 = 0.f;
                T = 1.f;
                ar = ag = ab = 0.f;
                depth = vd.depth;
                steps = 0;
                if (ok)
                    active = true;
                else
                    *out = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        if (__ballot_sync(kFull, active) == 0) {
            if (drained) break;
            continue;
        }
        if (!active) continue;
        const DeviceModel &m = s_scenes[scene];
        bool done = false;
        if (steps >= P.max_steps) {
            done = true;
        } else {
            steps += 1;
            if (T <= P.weight_threshold || t0 > depth) {
                done = true;
            } else {
                float best;
                FaceEntry win;
                uint32_t face;
                const bool has_exit = find_exit<BOUNDED>(m, c, ray, t0, depth, best, win, face);
                float ss, se;
                if (support<BOUNDED>(ray, c.x, c.y, c.z, c.r, t0, best, ss, se)) {
                    const float dens = c.density * 1.0f;
                    if (dens > 1e-6f) {
                        const float dt = se - ss;
                        const float alpha = 1.0f - bv_expf(-dens * dt);
                        const float wgt = T * alpha;
                        float coef[ShDims<DEG>::N];
                        load_sh_row<DEG, BF16>(m, c.id, coef);
                        float r, g, b;
                        eval_sh<DEG>(coef, ray.dx, ray.dy, ray.dz, r, g, b);
                        ar += wgt * fmaxf(r, 0.0f);
                        ag += wgt * fmaxf(g, 0.0f);
                        ab += wgt * fmaxf(b, 0.0f);
                        T *= 1.0f - alpha;
                    }
                }
                if (!has_exit) {
                    t0 = best;
                    done = true;
                } else {
                    t0 = fmaxf(t0, best);
                    c = cell_from_face(win);
                }
            }
        }
        if (done) {
            *out = make_float4(ar, ag, ab, 1.0f - T);
            active = false;
        }
    }
}

// d_pos[i] += site[i].xyz, d_radius[i] += site[i].w (scatter-add semantics
// of the caller's tables), then clears the site table for the next call.
__global__ void fold_site_grads_kernel(float4 *site, uint32_t n, float *d_pos, float *d_radius) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 g = site[i];
    if (d_pos) {
        d_pos[3 * (size_t)i + 0] += g.x;
        d_pos[3 * (size_t)i + 1] += g.y;
        d_pos[3 * (size_t)i + 2] += g.z;
    }
    if (d_radius) d_radius[i] += g.w;
    site[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

}  // namespace

cudaError_t launch_fold_site_grads(float4 *site, uint32_t n, float *d_pos, float *d_radius,
                                   cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    fold_site_grads_kernel<<<(n + 255) / 256, 256, 0, s>>>(site, n, d_pos, d_radius);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// launchers: pick the instantiation for (SH degree, bounded, bf16)
// ---------------------------------------------------------------------------
#define BV_SELECT(KERNEL, PARAMS, GRID, STREAM) BV_SELECT_M(KERNEL, (PARAMS).m, PARAMS, GRID, STREAM)
#define BV_SELECT_M(KERNEL, MODEL, PARAMS, GRID, STREAM)                                        \
    do {                                                                                        \
        const DeviceModel &mm = (MODEL);                                                        \
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
    if (p.tie_break)
        BV_SELECT(walk_forward_tb_kernel, p, grid, s);
    else
        BV_SELECT(walk_forward_kernel, p, grid, s);
    return cudaGetLastError();
}

cudaError_t launch_train_forward(const TrainParams &p, int grid, cudaStream_t s) {
    BV_SELECT(train_forward_kernel, p, grid, s);
    return cudaGetLastError();
}

cudaError_t launch_train_backward(const TrainParams &p, int grid, cudaStream_t s) {
    BV_SELECT(train_backward_kernel, p, grid, s);
    return cudaGetLastError();
}

// Every scene of a served batch shares (SH degree, bounded, bf16): the
// instantiation is picked from scene 0.
cudaError_t launch_serve_walk(const ServeParams &p, int grid, cudaStream_t s) {
    if (p.n_scenes == 0 || p.n_scenes > (uint32_t)kMaxServeScenes) return cudaErrorInvalidValue;
    BV_SELECT_M(serve_walk_kernel, p.scenes[0], p, grid, s);
    return cudaGetLastError();
}

int serve_grid_size(int device) {
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, serve_walk_kernel<3, false, false>,
                                                  kWalkBlock, 0);
    return sms * (per_sm < 1 ? 1 : per_sm);
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
    else if (kind == 1)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, train_forward_kernel<3, false, false>,
                                                      kWalkBlock, 0);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, train_backward_kernel<3, false, false>,
                                                      kWalkBlock, 0);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

}  // namespace bv
