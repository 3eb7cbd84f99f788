// PowerFoam splat render on sm_100a: per ray, every support sphere the ray
// crosses (spheres within 4 r of the camera excluded) is clipped by its Cech
// row into [face_near, face_far] intersected with the sphere, the clipped
// intervals are taken in (entry depth, cell) order, truncated to max_steps
// and composited front to back.
//
// Restates blade-volume/src/trace.rs: powerfoam_splat_interval :1331-1389,
// sorted_powerfoam_splat_intervals :1391-1411, trace_powerfoam_splats
// :1456-1546 (the reference's GPU path, gpu/powerfoam_splat.rs:51-343,
// records bounded candidate rows and sorts them).  Here a BVH over the
// support spheres is walked front to back in windows of W intervals (32
// for the render, 20 for training): a pass keeps the W smallest (t, cell)
// keys above the cursor, pruning boxes and spheres that end at or before the cursor or
// start after the window's last key, so there is no per-ray candidate
// scratch and no capacity to overflow.  The order equals the full sort, so
// the image is the oracle's bit for bit (-fmad=false; every expression is
// the CPU restatement's sequence of IEEE-rounded operations).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <thread>
#include <utility>
#include <vector>

#include "bv_bvh.h"
#include "bv_device.cuh"
#include "bv_internal.h"
#include "bv_segment.cuh"
#include "bv_tile_order.cuh"
#include "bv_window.cuh"

namespace bv {
namespace {

// Tuning knobs (measured on B200, 1M-site mixture at 4 x 1024^2): keys per
// lane per window pass, for the render (12-byte keys) and for training
// (16-byte keys with the interval's plane offsets).  A larger window means
// fewer passes over the BVH and fewer supports clipped again in the next
// pass, most of all for the heavy tiles, against fewer resident blocks:
// render 16 / 24 / 28 / 32 / 40 keys 47.7 / 55.7 / 58.0 / 59.6 / 54.5 Mrays/s
// (with the stable tile order: 32 keys 64.1, 40 keys 54.5); training
// 16 / 20 / 24 / 28 / 32 keys 51.0 / 54.3 / 48.9 / 40.4 / 41.6 (20 keys
// still fit 5 blocks per SM, 24 and more only 4 or 3).  And the resident
// blocks per SM requested for the render kernel (4: 128 registers, 19.4
// Mrays/s; without the bound 162 registers, 16.3).
#ifndef BV_SPLAT_WINDOW
#define BV_SPLAT_WINDOW 32
#endif
#ifndef BV_SPLAT_TRAIN_WINDOW
#define BV_SPLAT_TRAIN_WINDOW 20
#endif
#ifndef BV_MINB_SPLAT
#define BV_MINB_SPLAT 4
#endif
// Resident blocks per SM asked of the training forward (0: no minimum; the
// compiler then takes 80 registers and spills, 6 blocks by registers and
// shared memory; 5: 94 registers without spills, 50.6 vs 49.6 Mrays/s for
// config-2 training; 4: 42.6).
#ifndef BV_MINB_SPLAT_TRAIN
#define BV_MINB_SPLAT_TRAIN 5
#endif
#if BV_MINB_SPLAT_TRAIN
#define SPLAT_TRAIN_BOUNDS __launch_bounds__(kSplatBlock, BV_MINB_SPLAT_TRAIN)
#else
#define SPLAT_TRAIN_BOUNDS __launch_bounds__(kSplatBlock)
#endif
#ifndef BV_SPLAT_SHARED_NUM
#define BV_SPLAT_SHARED_NUM 1
#endif
// Window keys in shared memory (1) or registers (0).
#ifndef BV_SPLAT_SMEM_WINDOW
#define BV_SPLAT_SMEM_WINDOW 1
#endif
// Cech-row clip: each chunk of a row staged in the warp's shared memory (1)
// or broadcast lane to lane with shuffles (0); entries read from shared
// memory per iteration of the clip loop, 1, 2 or 4 (config-2 training
// 30.4 / 32.7 / 33.2 Mrays/s, its render 23.8 / 26.4 / 27.3 before tile
// ordering and 37.0 / 38.1 for 2 / 4 with it).
#ifndef BV_SPLAT_SMEM_ROWS
#define BV_SPLAT_SMEM_ROWS 1
#endif
#ifndef BV_SPLAT_CLIP_ILP
#define BV_SPLAT_CLIP_ILP 4
#endif
// Each Cech row's clip planes stored nearest to the site first (1), so that
// a support the clip empties is left after fewer planes, or in CSR order (0).
#ifndef BV_SPLAT_ROW_SORT
#define BV_SPLAT_ROW_SORT 1
#endif
// Training launches take tiles heaviest first (1), ordered by the time each
// tile's forward took in the previous call over the same views, or in
// launch order (0).
#ifndef BV_SPLAT_TILE_ORDER
#define BV_SPLAT_TILE_ORDER 1
#endif
// Training: one stable order for the forward and the replay (0), or the
// replay on an unstable order of the same times, whose concurrent tiles
// from all over the screen spread the gradient atomics (1; measured 57.4 vs
// 57.8 Mrays/s: the splat replay, 7 ms of the 73 ms step, gains nothing).
#ifndef BV_SPLAT_SPLIT_ORDER
#define BV_SPLAT_SPLIT_ORDER 0
#endif
constexpr int kSplatBlock = 128;
constexpr int kSplatWindow = BV_SPLAT_WINDOW;            // render
constexpr int kSplatTrainWindow = BV_SPLAT_TRAIN_WINDOW;  // training forward and replay
constexpr int kSplatStack = 80;  // > BVH depth, checked at tracer creation

// Dynamic shared memory of a splat kernel's window: `fields` words per key
// (3 for WinKey, 4 for WinKey2), `keys` keys per thread.
constexpr size_t splat_window_bytes(int fields, int keys) {
    return (BV_SPLAT_SMEM_WINDOW ? (size_t)fields * keys * kSplatBlock * 4u : 0u);
}

// The window of a splat kernel: SPLAT_WINDOW(Key, W) declares it (W keys
// per thread in shared memory, or a register array), SPLAT_GATHER runs one
// pass into it and SPLAT_KEY(i) reads key i.
#if BV_SPLAT_SMEM_WINDOW
// in dynamic shared memory (splat_window_bytes per block, set at launch), so
// that windows of more than 20 keys fit: field f of key i of thread tid at
// word (f W + i) 128 + tid
#define SPLAT_WINDOW(KEY, W)                                                      \
    constexpr int kWin = (W);                                                     \
    extern __shared__ uint32_t s_win_dyn[];                                       \
    SmemWindow<kWin, KEY> win{                                                    \
        reinterpret_cast<float *>(s_win_dyn) + threadIdx.x,                       \
        s_win_dyn + 1 * kWin * kSplatBlock + threadIdx.x,                         \
        s_win_dyn + 2 * kWin * kSplatBlock + threadIdx.x,                         \
        s_win_dyn + (sizeof(KEY) == sizeof(WinKey2) ? 3 * kWin * kSplatBlock + threadIdx.x : 0), \
        kSplatBlock}
#define SPLAT_GATHER(...) win_gather_warp_smem<kWin, kSplatStack>(__VA_ARGS__, win, nodes_visited, hit)
#define SPLAT_KEY(i) win.get(i)
#else
#define SPLAT_WINDOW(KEY, W)  \
    constexpr int kWin = (W); \
    KEY buf[kWin]
#define SPLAT_GATHER(...) win_gather_warp<kWin, kSplatStack>(__VA_ARGS__, buf, nodes_visited, hit)
#define SPLAT_KEY(i) win_at(buf, i)
#endif
// Entry / exit plane of an interval as an offset in its Cech row (16 bits
// each in the key; rows are at most 65,534 entries, checked at creation).
constexpr uint32_t kNoPlane = 0xffffu;

// One support sphere in BVH leaf order, 32 B.
struct __align__(16) SplatPrim {
    float4 site;  // x, y, z, power radius
    uint4 link;   // cell (model index), Cech row begin, row end, 0
};

// One Cech entry of a support's row: the clip plane's point f = s_i + shift n
// and normal n = s_j - s_i (shift = 0.5 + 0.5 (r_i^2 - r_j^2) / max(|n|^2,
// 1e-20)), formed on the host in the kernel's FP32 operation order
// (trace.rs:1351-1389), so each ray evaluates only (f - o).n and d.n.  A
// row's entries may be stored in any order (nearest plane first, see
// BV_SPLAT_ROW_SORT): each carries its offset in the CSR row, which breaks
// ties between planes at the same depth as the CSR order does, and its
// neighbour.  Interval keys and records name an entry by its stored
// position.
struct __align__(16) SplatFace {
    float4 point;   // f, CSR offset in the row (uint bits)
    float4 normal;  // n, neighbour j (uint bits)
};

struct SplatParams {
    DeviceModel m;                 // density, SH rows (model order)
    const SplatPrim *prims;        // [N] leaf order
    const BvhNode *nodes;
    const SplatFace *row_faces;    // [M] CSR order: clip plane of each Cech entry
    uint32_t max_steps;
    float weight_threshold;
    uint32_t n_views;
    uint32_t total_work;
    float4 *out;                   // [n_views][H][W]
    unsigned long long *stats;     // [3] rays, composited intervals, Cech entries clipped (or null)
    uint32_t *max_candidates;      // counting pass: max over rays of the support hits
    unsigned long long *count_totals;  // counting pass: [2] support hits, their Cech row entries
    uint32_t count_only;
    const uint32_t *tile_order;    // [tiles] tile taken by warp slot i, or null: slot i takes tile i
    uint32_t *tile_cost;           // [tiles] the tile's duration in 64-cycle units, or null
    ViewDesc views[kMaxViewsPerLaunch];
};


// Slab test for the counting pass (per-lane traversal).
__device__ __forceinline__ bool slab(const float4 &lo, const float4 &hi, const WinRay &r, float t_end,
                                     float &tn, float &tf) {
    return win_slab(lo, hi, r, t_end, tn, tf);
}

// Support-sphere test of powerfoam_splat_interval (trace.rs:1331-1350):
// false when the camera is within 4 r of the site, the ray misses the sphere,
// or the sphere lies behind the camera or beyond depth.
__device__ __forceinline__ bool splat_sphere(const WinRay &ray, const float4 &s, float depth,
                                             float &sn, float &sf) {
    const float cx = s.x - ray.ox, cy = s.y - ray.oy, cz = s.z - ray.oz;
    const float excl = 4.0f * s.w;
    if (dot3(cx, cy, cz, cx, cy, cz) < excl * excl) return false;
    const float ocx = ray.ox - s.x, ocy = ray.oy - s.y, ocz = ray.oz - s.z;
    const float b = dot3(ocx, ocy, ocz, ray.dx, ray.dy, ray.dz);
    const float disc = b * b - (dot3(ocx, ocy, ocz, ocx, ocy, ocz) - s.w * s.w);
    if (disc <= 0.0f || !isfinite(disc)) return false;
    const float root = sqrtf(disc);
    sn = -b - root;
    sf = -b + root;
    return !(sf <= 0.0f || sn >= depth);
}

// Division savers of the clip, exact: true only when the plane's rounded
// quotient num / den cannot move the bound.  For a far plane (den > 0) that
// is num / den >= face_far; for a near plane (den < 0) num / den <=
// face_near, i.e. num >= face_near den.  p = fl(bound den) is within one
// rounding of the exact product, so fl(p (1 +- 2^-21)) (the factor that moves
// p away from zero's side the product could lie on) bounds it whenever p is
// normal; otherwise the caller divides.
__device__ __forceinline__ bool clip_far_cannot_tighten(float num, float den, float face_far) {
    const float p = face_far * den;
    return p > 1.0e-30f && num >= p * 1.000000476837158203125f;
}

__device__ __forceinline__ bool clip_near_cannot_tighten(float num, float den, float face_near) {
    if (face_near == 0.0f) return num >= 0.0f;  // num / den <= 0 exactly
    const float p = face_near * den;            // face_near > 0, den < 0
    return p < -1.0e-30f && num >= p * 0.999999523162841796875f;
}

// Cech-row clip of one support (trace.rs:1351-1389, path_interval_jacobian
// :1199-1325 for the bounded clip), warp-cooperative: every lane calls it
// for the same support; the row's clip planes are read 32 at a time (one
// coalesced load per chunk) and each is broadcast to the lanes that clip
// (need).  face_near / face_far are a max / min over the row and a parallel
// face with num < 0 empties the interval, so the result does not depend on
// the order the entries are taken in; once a lane's interval is empty it
// stays empty (face_near only grows, face_far only shrinks), and the warp
// leaves the row when every lane's is.  False for lanes whose interval is
// empty.
__device__ __forceinline__ bool splat_clip_warp(const SplatParams &P, const WinRay &ray,
                                                uint32_t begin, uint32_t end, float depth,
                                                float sn, float sf, bool need, float &start,
                                                float &dt, uint32_t &links) {
    const uint32_t lane = threadIdx.x & 31u;
    float face_near = 0.0f, face_far = depth;
    uint32_t near_k = kNoPlane, far_k = kNoPlane;  // stored positions in the row
    bool empty = !need;
    // CSR offset of the entry stored at position k (ties only: rare)
    auto csr_offset = [&](uint32_t k) {
        return __float_as_uint(__ldg(&P.row_faces[begin + k].point.w));
    };
    // One Cech entry (stored position k, CSR offset o, numerator <f - o, n>,
    // denominator <d, n>) applied to this lane's interval.  The bounds are a
    // min / max over the row; of planes at the same depth the one earliest
    // in CSR order bounds the interval, as the reference's scan in CSR order
    // keeps the first, whatever order the entries are taken in.  A plane
    // whose quotient provably cannot reach the bound is passed without
    // dividing (clip_*_cannot_tighten: the rounded quotient is then
    // strictly beyond it, so no tie is passed either); the planes that can
    // are divided and compared, so the interval and the planes that bound it
    // are the same bit for bit.
    auto clip_entry = [&](float num, float den, uint32_t k, uint32_t o) {
        bool moved = false;
        if (den > 1.0e-20f) {
            if (!clip_far_cannot_tighten(num, den, face_far)) {
                const float t = num / den;
                if (t < face_far || (t == face_far && far_k != kNoPlane && o < csr_offset(far_k))) {
                    face_far = t;
                    far_k = k;
                    moved = true;
                }
            }
        } else if (den < -1.0e-20f) {
            if (!clip_near_cannot_tighten(num, den, face_near)) {
                const float t = num / den;
                if (t > face_near ||
                    (t == face_near && near_k != kNoPlane && o < csr_offset(near_k))) {
                    face_near = t;
                    near_k = k;
                    moved = true;
                }
            }
        } else if (num < 0.0f) {
            empty = true;
        }
        if (moved) {
            const float st = sn > face_near ? sn : face_near;
            const float en = sf < face_far ? sf : face_far;
            if (en <= st) empty = true;
        }
    };
    for (uint32_t base = begin; base < end; base += 32u) {
        if (!__any_sync(0xffffffffu, !empty)) break;
        const uint32_t n = min(32u, end - base);
        float4 fp = make_float4(0.f, 0.f, 0.f, 0.f), fn = fp;
        if (base + lane < end) {
            fp = __ldg(&P.row_faces[base + lane].point);
            fn = __ldg(&P.row_faces[base + lane].normal);
        }
#if BV_SPLAT_SHARED_NUM
        // The warp's rays share one camera origin, so <p - o, n> of an entry
        // is the same in every lane: the lane that loaded it evaluates it
        // (the same operations each lane would apply) and broadcasts it
        // with the normal.
        const float num_own = dot3(fp.x - ray.ox, fp.y - ray.oy, fp.z - ray.oz, fn.x, fn.y, fn.z);
#endif
#if BV_SPLAT_SMEM_ROWS && BV_SPLAT_SHARED_NUM
        // The chunk (numerator and normal of each entry) goes to the warp's
        // slice of shared memory once; every lane that still clips then
        // reads the entries it needs (broadcast reads) and leaves the row
        // alone as soon as its interval is empty.
        __shared__ float4 s_row[kSplatBlock];
        __shared__ uint32_t s_row_off[kSplatBlock];
        float4 *row = s_row + (threadIdx.x & ~31u);
        uint32_t *row_off = s_row_off + (threadIdx.x & ~31u);
        __syncwarp();
        row[lane] = make_float4(num_own, fn.x, fn.y, fn.z);
        row_off[lane] = __float_as_uint(fp.w);
        __syncwarp();
#if BV_SPLAT_CLIP_ILP > 1
        // BV_SPLAT_CLIP_ILP entries per iteration: their denominators are
        // formed before any is applied, then they are applied in row order
        // (slots past the last entry are read but not applied; lanes past
        // the row's end wrote zeros there, and the slot index stays below 32)
        constexpr uint32_t kIlp = BV_SPLAT_CLIP_ILP;
        for (uint32_t j = 0; j < n && !empty; j += kIlp) {
            float4 e[kIlp];
            float den[kIlp];
#pragma unroll
            for (uint32_t u = 0; u < kIlp; ++u) {
                e[u] = row[min(j + u, 31u)];
                den[u] = dot3(ray.dx, ray.dy, ray.dz, e[u].y, e[u].z, e[u].w);
            }
            clip_entry(e[0].x, den[0], base + j - begin, row_off[j]);
#pragma unroll
            for (uint32_t u = 1; u < kIlp; ++u)
                if (j + u < n && !empty)
                    clip_entry(e[u].x, den[u], base + j + u - begin, row_off[j + u]);
        }
#else
        for (uint32_t j = 0; j < n && !empty; ++j) {
            const float4 e = row[j];
            clip_entry(e.x, dot3(ray.dx, ray.dy, ray.dz, e.y, e.z, e.w), base + j - begin,
                       row_off[j]);
        }
#endif
#else
        for (uint32_t j = 0; j < n; ++j) {
#if BV_SPLAT_SHARED_NUM
            const float num = __shfl_sync(0xffffffffu, num_own, j);
#else
            const float fx = __shfl_sync(0xffffffffu, fp.x, j);
            const float fy = __shfl_sync(0xffffffffu, fp.y, j);
            const float fz = __shfl_sync(0xffffffffu, fp.z, j);
#endif
            const float nx = __shfl_sync(0xffffffffu, fn.x, j);
            const float ny = __shfl_sync(0xffffffffu, fn.y, j);
            const float nz = __shfl_sync(0xffffffffu, fn.z, j);
            const uint32_t o = __shfl_sync(0xffffffffu, __float_as_uint(fp.w), j);
            if (empty) continue;
#if !BV_SPLAT_SHARED_NUM
            const float num = dot3(fx - ray.ox, fy - ray.oy, fz - ray.oz, nx, ny, nz);
#endif
            clip_entry(num, dot3(ray.dx, ray.dy, ray.dz, nx, ny, nz), base + j - begin, o);
        }
#endif
    }
    if (empty) return false;
    float st = face_near, en = face_far;
    if (sn > st) st = sn;
    if (sf < en) en = sf;
    if (en <= st || !isfinite(st) || !isfinite(en)) return false;
    start = st;
    dt = en - st;
    links = near_k | (far_k << 16);
    return true;
}

// Window candidate test of support p for win_gather_warp (every lane calls
// it): the sphere test per lane, then the warp clips the support's Cech row
// for the lanes whose sphere interval can still enter their window; the key
// is (clipped entry depth, cell), pos carries the interval length and a
// WinKey2's aux the row offsets of its entry / exit planes.
__device__ __forceinline__ void set_links(WinKey &, uint32_t) {}
__device__ __forceinline__ void set_links(WinKey2 &k, uint32_t links) { k.aux = links; }

template <class Key>
__device__ __forceinline__ bool splat_hit(const SplatParams &P, const WinRay &ray, float depth,
                                          bool cursor_valid, float cur_t, uint32_t p, bool mine,
                                          float limit, Key &k, uint32_t &clipped) {
    const float4 s = __ldg(&P.prims[p].site);
    float sn = 0.f, sf = 0.f;
    bool need = mine && splat_sphere(ray, s, depth, sn, sf);
    // the clipped start lies in [sn, sf): skip supports whose every key is at
    // or below the cursor or past the window end
    if (need && cursor_valid && sf <= cur_t) need = false;
    if (need && sn > limit) need = false;
    if (!__any_sync(0xffffffffu, need)) return false;
    const uint4 link = __ldg(&P.prims[p].link);
    if (need) clipped += link.z - link.y;
    float st, dt;
    uint32_t links;
    if (!splat_clip_warp(P, ray, link.y, link.z, depth, sn, sf, need, st, dt, links)) return false;
    k.t = st;
    k.idx = link.x;
    k.pos = __float_as_uint(dt);
    set_links(k, links);
    return true;
}

// The tile / view of work item w and its camera ray (radfoam.wgsl:44-52).
// active: the lane has a pixel and a valid direction.
struct SplatLane {
    WinRay ray;
    Ray r0;
    const ViewDesc *vd;
    uint32_t x, y;
    bool inside, active;
};

template <typename Params>
__device__ __forceinline__ SplatLane splat_lane(const Params &P, uint32_t w) {
    SplatLane L;
    uint32_t view = 0;
    while (view + 1 < P.n_views && w >= P.views[view + 1].ray_begin) ++view;
    L.vd = &P.views[view];
    const uint32_t local = w - L.vd->ray_begin;
    const uint32_t tile = local / kTileRays, in = local % kTileRays;
    L.x = (tile % L.vd->tiles_x) * kTileW + in % kTileW;
    L.y = (tile / L.vd->tiles_x) * kTileH + in / kTileW;
    L.inside = L.x < L.vd->width && L.y < L.vd->height;
    L.r0 = Ray{0.f, 0.f, 0.f, 1.f, 0.f, 0.f};
    L.active = L.inside && make_ray(*L.vd, L.x, L.y, L.r0);
    // every lane, inside the image or not, carries its view's camera origin
    // (make_ray's own value for the active ones), which the clip relies on
    L.ray.ox = L.vd->origin[0];
    L.ray.oy = L.vd->origin[1];
    L.ray.oz = L.vd->origin[2];
    L.ray.dx = L.active ? L.r0.dx : 1.0f;
    L.ray.dy = L.active ? L.r0.dy : 0.0f;
    L.ray.dz = L.active ? L.r0.dz : 0.0f;
    L.ray.ix = win_inverse(L.ray.dx);
    L.ray.iy = win_inverse(L.ray.dy);
    L.ray.iz = win_inverse(L.ray.dz);
    return L;
}

template <int DEG, bool BF16>
__global__ void __launch_bounds__(kSplatBlock, BV_MINB_SPLAT)
splat_kernel(const __grid_constant__ SplatParams P) {
    // A view's work is whole 8x4 tiles, so a warp is one tile of one view;
    // whole warps past the end leave together, lanes of a partial edge tile
    // stay (inactive) because the main pass is warp-cooperative.
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if ((slot & ~31u) >= P.total_work) return;
    const long long clock_begin = clock64();
    const uint32_t w = tile_item(P.tile_order, slot);
    const SplatLane L = splat_lane(P, w);
    const WinRay &ray = L.ray;
    const bool active = L.active;
    float4 *out = P.out + (size_t)L.vd->pixel_begin + (size_t)L.y * L.vd->width + L.x;
    if (L.inside && !active && !P.count_only) *out = make_float4(0.f, 0.f, 0.f, 0.f);
    const float depth = L.vd->depth;

    if (P.count_only) {
        // every support hit, no window pruning, one ray per thread
        if (!active) return;
        uint32_t hits = 0, entries = 0;
        uint32_t stack[kSplatStack];
        int sp = 0;
        stack[sp++] = 0u;
        while (sp > 0) {
            const BvhNode nd = P.nodes[stack[--sp]];
            const float4 lo[2] = {nd.l_lo, nd.r_lo}, hi[2] = {nd.l_hi, nd.r_hi};
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const uint32_t cnt = __float_as_uint(hi[c].w);
                float tn, tf;
                if (cnt == kBvhNoChild || !slab(lo[c], hi[c], ray, depth, tn, tf)) continue;
                const uint32_t ref = __float_as_uint(lo[c].w);
                if (cnt == 0u) {
                    if (sp < kSplatStack) stack[sp++] = ref;
                    continue;
                }
                for (uint32_t p = ref; p < ref + cnt; ++p) {
                    float sn, sf;
                    if (!splat_sphere(ray, __ldg(&P.prims[p].site), depth, sn, sf)) continue;
                    const uint4 link = __ldg(&P.prims[p].link);
                    hits += 1;
                    entries += link.z - link.y;
                }
            }
        }
        atomicMax(P.max_candidates, hits);
        atomicAdd(P.count_totals + 0, (unsigned long long)hits);
        atomicAdd(P.count_totals + 1, (unsigned long long)entries);
        return;
    }

    float T = 1.0f, ar = 0.f, ag = 0.f, ab = 0.f;
    uint32_t steps = 0, clipped = 0, nodes_visited = 0;
    bool cursor_valid = false, finished = !active;
    float cur_t = 0.f;
    uint32_t cur_cell = 0;
    auto hit = [&](uint32_t p, bool mine, float limit, auto &k) -> bool {
        return splat_hit(P, ray, depth, cursor_valid, cur_t, p, mine, limit, k, clipped);
    };
    SPLAT_WINDOW(WinKey, kSplatWindow);
    for (;;) {
        const bool want = !finished;
        if (!__any_sync(0xffffffffu, want)) break;
        const int count = SPLAT_GATHER(P.nodes, ray, depth, want, cursor_valid, cur_t, cur_cell);
        if (!want) continue;
        // ---- composite the window in order (trace.rs:1490-1530)
#pragma unroll 1
        for (int i = 0; i < count; ++i) {
            const WinKey e = SPLAT_KEY(i);
            if (T <= P.weight_threshold || steps >= P.max_steps) {
                finished = true;
                break;
            }
            steps += 1;
            const float dens = __ldg(P.m.density + e.idx) * 1.0f;
            if (dens <= 1.0e-6f) continue;
            const float alpha = 1.0f - bv_expf(-dens * __uint_as_float(e.pos));
            const float wgt = T * alpha;
            float coef[ShDims<DEG>::N];
            load_sh_row<DEG, BF16>(P.m, e.idx, coef);
            float r, g, b;
            eval_sh<DEG>(coef, ray.dx, ray.dy, ray.dz, r, g, b);
            ar += wgt * fmaxf(r, 0.0f);
            ag += wgt * fmaxf(g, 0.0f);
            ab += wgt * fmaxf(b, 0.0f);
            T *= 1.0f - alpha;
        }
        if (finished) continue;
        if (count < kWin) {
            finished = true;
        } else {
            const auto last = SPLAT_KEY(kWin - 1);
            cursor_valid = true;
            cur_t = last.t;
            cur_cell = last.idx;
        }
    }
    if (active) {
        *out = make_float4(ar, ag, ab, 1.0f - T);
        if (P.stats) {
            atomicAdd(P.stats + 0, 1ull);
            atomicAdd(P.stats + 1, (unsigned long long)steps);
            atomicAdd(P.stats + 2, (unsigned long long)clipped);
        }
    }
    store_tile_cost(P.tile_cost, w, clock_begin);
}

// ---------------------------------------------------------------------------
// training with splat semantics: record_powerfoam_splats_jacobians
// (trace.rs:1421-1452) integrated like the walk's training contract
// ---------------------------------------------------------------------------
struct SplatTrainParams {
    SplatParams base;           // traversal, density / SH tables, views
    const float4 *geom;         // [N] model order: site, radius
    const uint32_t *offsets;    // [N+1] CSR
    const uint32_t *neighbors;  // [M] CSR neighbour ids
    float max_dt;
    uint32_t loss_kind;
    float inv_count;            // 1 / (3 * rays of the whole call)
    const float *target;        // [pixels][3] of this launch's views
    float *rgb_out;             // [pixels][3] or null
    float *loss;
    RayState *ray_state;        // [pixels]
    float *d_density, *d_sh;
    float4 *d_site;             // [N] or null
    uint32_t *rec_pool;         // interval-record chunks, or null
    uint32_t *rec_table;        // [tiles][rec_chunks] chunk of each (tile, chunk rank)
    uint32_t *rec_next;         // next free chunk of the pool
    uint32_t rec_chunks;        // chunk ranks per tile; 0: the replay traverses every ray
    uint32_t rec_limit;         // intervals recorded per ray at most
    uint32_t pool_chunks;       // chunks in the pool
};

// Interval record of the training forward, read back by the replay.  The
// i-th composited interval of ray w (the cell, the raw interval length as
// float bits, the entry / exit plane offsets of its WinKey2 and the
// unclamped SH colour r, g, b) sits in the chunk that the tile of w (the 32
// rays w / 32) holds for ranks 16 (i / 16) .. +15: a chunk is 16 ranks x 6
// rows x 32 lanes of words, so the rays of a tile, which composite together,
// write and read whole 128-byte rows.  Chunks are taken from a pool when a
// ray of the tile first needs that rank (an atomic counter; a CAS publishes
// the chunk in the tile's table, and a lane that loses the race uses the
// winner's), so the record grows with the intervals actually composited.  A
// ray that finds the pool empty, or composites more than rec_limit
// intervals, stops recording and is marked kRecOverflow in its RayState; the
// replay traverses it again.
#ifndef BV_SPLAT_REC_ENTRIES
#define BV_SPLAT_REC_ENTRIES 1024
#endif
#ifndef BV_SPLAT_REC_GIB
#define BV_SPLAT_REC_GIB 12
#endif
constexpr uint32_t kRecWords = 6;
constexpr uint32_t kChunkEntries = 16;
constexpr uint32_t kChunkWords = kChunkEntries * kRecWords * 32u;  // 12 KiB
constexpr uint32_t kSplatRecEntries = BV_SPLAT_REC_ENTRIES;
constexpr size_t kSplatRecBytes = size_t(BV_SPLAT_REC_GIB) << 30;
constexpr uint32_t kNoChunk = 0xffffffffu;
constexpr uint32_t kRecOverflow = 0xffffffffu;

__device__ __forceinline__ uint32_t *rec_entry(const SplatTrainParams &TP, uint32_t chunk,
                                               uint32_t w, uint32_t i) {
    return TP.rec_pool + (size_t)chunk * kChunkWords + (i % kChunkEntries) * (kRecWords * 32u) +
           (w & 31u);
}

// The chunk for rank i of ray w's tile (i a multiple of 16), taken from the
// pool if no ray of the tile holds it yet; kNoChunk when none can be had.
// The lanes of the tile that reach rank i together (the calling lanes that
// ask for the same chunk) elect one of them to take it, so a tile takes one
// chunk per rank; a lane that asks later finds it in the table.
__device__ __forceinline__ uint32_t rec_chunk_for_write(const SplatTrainParams &TP, uint32_t w,
                                                        uint32_t i) {
    const uint32_t c = i / kChunkEntries;
    const unsigned active = __activemask();
    const unsigned group = __match_any_sync(active, c);
    const int leader = __ffs(group) - 1;
    uint32_t id = kNoChunk;
    if ((int)(threadIdx.x & 31u) == leader && c < TP.rec_chunks) {
        uint32_t *slot = TP.rec_table + (size_t)(w >> 5) * TP.rec_chunks + c;
        id = *reinterpret_cast<volatile uint32_t *>(slot);
        if (id == kNoChunk) {
            const uint32_t mine = atomicAdd(TP.rec_next, 1u);
            if (mine < TP.pool_chunks) {
                const uint32_t prev = atomicCAS(slot, kNoChunk, mine);
                id = prev == kNoChunk ? mine : prev;
            } else {
                id = *reinterpret_cast<volatile uint32_t *>(slot);
            }
        }
    }
    return __shfl_sync(group, id, leader);
}

// The entry / exit planes of a windowed interval from the row offsets its
// key carries (kNoPlane: no plane bounds that side): their depths before
// the sphere clip, evaluated as splat_clip_warp evaluates them, and the
// neighbours across them (the cell itself when none).
__device__ __forceinline__ float splat_plane_t(const SplatTrainParams &TP, const WinRay &ray,
                                               uint32_t k, uint32_t &neighbour) {
    const float4 fp = __ldg(&TP.base.row_faces[k].point);
    const float4 fn = __ldg(&TP.base.row_faces[k].normal);
    neighbour = __float_as_uint(fn.w);
    const float rx = fp.x - ray.ox, ry = fp.y - ray.oy, rz = fp.z - ray.oz;
    const float num = dot3(rx, ry, rz, fn.x, fn.y, fn.z);
    const float den = dot3(ray.dx, ray.dy, ray.dz, fn.x, fn.y, fn.z);
    return num / den;
}

__device__ __forceinline__ void splat_planes_of(const SplatTrainParams &TP, const WinRay &ray,
                                                uint32_t cell, float depth, uint32_t links,
                                                float &face_near, float &face_far,
                                                uint32_t &prev, uint32_t &next) {
    const uint32_t b = __ldg(TP.offsets + cell);
    const uint32_t nk = links & 0xffffu, fk = links >> 16;
    face_near = 0.0f;
    face_far = depth;
    prev = next = cell;
    if (nk != kNoPlane) face_near = splat_plane_t(TP, ray, b + nk, prev);
    if (fk != kNoPlane) face_far = splat_plane_t(TP, ray, b + fk, next);
}

template <int DEG, bool BF16>
__global__ void SPLAT_TRAIN_BOUNDS
splat_train_forward_kernel(const __grid_constant__ SplatTrainParams TP) {
    const SplatParams &P = TP.base;
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if ((slot & ~31u) >= P.total_work) return;
    const long long clock_begin = clock64();
    const uint32_t w = tile_item(P.tile_order, slot);
    const SplatLane L = splat_lane(P, w);
    const WinRay &ray = L.ray;
    const float depth = L.vd->depth;
    const size_t pix = (size_t)L.vd->pixel_begin + (size_t)L.y * L.vd->width + L.x;
    float Ch[3] = {0.f, 0.f, 0.f}, Cl[3] = {0.f, 0.f, 0.f};
    float T = 1.0f;
    uint32_t steps = 0, clipped = 0, nodes_visited = 0, composited = 0;
    bool rec_ok = TP.rec_chunks != 0;
    uint32_t rec_chunk = kNoChunk;
    bool cursor_valid = false, finished = !L.active;
    float cur_t = 0.f;
    uint32_t cur_cell = 0;
    auto hit = [&](uint32_t p, bool mine, float limit, auto &k) -> bool {
        return splat_hit(P, ray, depth, cursor_valid, cur_t, p, mine, limit, k, clipped);
    };
    SPLAT_WINDOW(WinKey2, kSplatTrainWindow);
    for (;;) {
        const bool want = !finished;
        if (!__any_sync(0xffffffffu, want)) break;
        const int count = SPLAT_GATHER(P.nodes, ray, depth, want, cursor_valid, cur_t, cur_cell);
        if (!want) continue;
#pragma unroll 1
        for (int i = 0; i < count; ++i) {
            const WinKey2 e = SPLAT_KEY(i);
            if (T <= P.weight_threshold || steps >= P.max_steps) {
                finished = true;
                break;
            }
            steps += 1;
            const float dens = __ldg(P.m.density + e.idx) * 1.0f;
            if (dens <= 1.0e-6f) continue;
            const float dt = fminf(__uint_as_float(e.pos), TP.max_dt);
            const float alpha = 1.0f - bv_expf(-dens * dt);
            const float wgt = T * alpha;
            float coef[ShDims<DEG>::N];
            load_sh_row<DEG, BF16>(P.m, e.idx, coef);
            float cu[3];
            eval_sh<DEG>(coef, ray.dx, ray.dy, ray.dz, cu[0], cu[1], cu[2]);
            if (composited >= TP.rec_limit) rec_ok = false;
            if (rec_ok && composited % kChunkEntries == 0) {
                rec_chunk = rec_chunk_for_write(TP, w, composited);
                rec_ok = rec_chunk != kNoChunk;
            }
            if (rec_ok) {
                uint32_t *rec = rec_entry(TP, rec_chunk, w, composited);
                __stcs(rec, e.idx);
                __stcs(rec + 32, e.pos);
                __stcs(rec + 64, e.aux);
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) __stcs(rec + 96 + 32 * ch, __float_as_uint(cu[ch]));
            }
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) acc_add(Ch[ch], Cl[ch], wgt * fmaxf(cu[ch], 0.f));
            T = T * (1.0f - alpha);
            composited += 1;
        }
        if (finished) continue;
        if (count < kWin) {
            finished = true;
        } else {
            const auto last = SPLAT_KEY(kWin - 1);
            cursor_valid = true;
            cur_t = last.t;
            cur_cell = last.idx;
        }
    }
    // loss and dL/dC of the pixel (the walk's training epilogue)
    float l = 0.f;
    if (L.inside) {
        const float *tg = TP.target + 3 * pix;
        float gC[3];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) {
            const float col = Ch[ch] + Cl[ch];
            const float diff = col - __ldg(tg + ch);
            if (TP.loss_kind == BV_LOSS_L2) {
                l += diff * diff;
                gC[ch] = 2.0f * diff * TP.inv_count;
            } else {
                l += fabsf(diff);
                gC[ch] = (diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f)) * TP.inv_count;
            }
            if (TP.rgb_out) TP.rgb_out[3 * pix + ch] = col;
        }
        RayState st;
        st.c_hi = make_float4(Ch[0], Ch[1], Ch[2], gC[0]);
        st.c_lo = make_float4(Cl[0], Cl[1], Cl[2], gC[1]);
        const uint32_t recorded = rec_ok ? composited : kRecOverflow;
        st.g = make_float4(gC[2], __uint_as_float(recorded), 0.f, 0.f);
        TP.ray_state[pix] = st;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31u) == 0 && l != 0.f) atomicAdd(TP.loss, l * TP.inv_count);
    if (P.stats && L.active) {
        atomicAdd(P.stats + 0, 1ull);
        atomicAdd(P.stats + 1, (unsigned long long)composited);
        atomicAdd(P.stats + 2, (unsigned long long)clipped);
    }
    store_tile_cost(P.tile_cost, w, clock_begin);
}

// Gradient of one composited interval of the replay (cell, raw length,
// entry / exit plane offsets, unclamped colour cu), advancing T and the
// compensated prefix P:
//   dL/dsigma_k = dt_k sum_c g_c (T_{k+1} c_kc - S_{k+1,c})
//   dL/dSH_kmc  = g_c w_k Y_m(d) [c_kc unclamped > 0]
//   dL/ddt_k    = sigma_k sum_c g_c (T_{k+1} c_kc - S_{k+1,c})  -> sites, radii
// with S_{k+1} = C - P_k, through the interval's exact Jacobians
// (path_interval_jacobian of the entry / exit neighbours, trace.rs:1199-1325).
// The entry / exit neighbours' site gradients are scattered here; the
// cell's own terms are returned for the caller's scatter.
struct IntervalGrad {
    float g_density;
    float gw[3];     // dL/dSH_kmc = gw[c] Y_m
    float4 g_site;   // the cell's site / radius gradient (zero without one)
};

template <int DEG>
__device__ __forceinline__ IntervalGrad splat_interval_terms(
    const SplatTrainParams &TP, const WinRay &ray, const Ray &r, float depth, uint32_t cell,
    float dens, float dt_raw, uint32_t links, const float (&cu)[3], const float (&Ch)[3],
    const float (&Cl)[3], const float (&gC)[3], float &T, float (&Ph)[3], float (&Pl)[3]) {
    IntervalGrad G;
    const float dt = fminf(dt_raw, TP.max_dt);
    const float alpha = 1.0f - bv_expf(-dens * dt);
    const float wgt = T * alpha;
    const float Tn = T * (1.0f - alpha);
    float gs = 0.f;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        const float cc = fmaxf(cu[ch], 0.f);
        acc_add(Ph[ch], Pl[ch], wgt * cc);
        const float suffix = (Ch[ch] - Ph[ch]) + (Cl[ch] - Pl[ch]);
        gs += gC[ch] * (Tn * cc - suffix);
        G.gw[ch] = cu[ch] > 0.f ? gC[ch] * wgt : 0.f;
    }
    G.g_density = dt * gs;
    G.g_site = make_float4(0.f, 0.f, 0.f, 0.f);
    if (TP.d_site && dt_raw < TP.max_dt) {
        float face_near, face_far;
        uint32_t prev, next;
        splat_planes_of(TP, ray, cell, depth, links, face_near, face_far, prev, next);
        const float4 g = __ldg(TP.geom + cell);
        Cell c;
        c.id = cell;
        c.x = g.x;
        c.y = g.y;
        c.z = g.z;
        c.r = g.w;
        c.density = dens;
        Interval iv;
        record_interval<true>(r, c, face_near, face_far, iv);
        const float4 pp = __ldg(TP.geom + prev), np = __ldg(TP.geom + next);
        const Jacobians J =
            interval_jacobians(r, iv, prev, pp, c, next != cell, np, face_near, face_far);
        const float gdt = dens * gs;
        G.g_site = make_float4(gdt * J.jc.x, gdt * J.jc.y, gdt * J.jc.z, gdt * J.jc.w);
        if (prev != cell && !iv.start_sphere) scatter_site(TP.d_site, prev, gdt, J.jp);
        if (next != cell && !iv.end_sphere) scatter_site(TP.d_site, next, gdt, J.jn);
    }
    T = Tn;
    return G;
}

// The cell's terms of one interval, one lane's own atomics.
template <int DEG>
__device__ __forceinline__ void scatter_interval(const SplatTrainParams &TP,
                                                 const float (&Y)[ShDims<DEG>::K], uint32_t cell,
                                                 const IntervalGrad &G) {
    constexpr int N = 3 * ShDims<DEG>::K;
    atomicAdd(TP.d_density + cell, G.g_density);
    if (N % 4 == 0) {
        float4 *row4 = reinterpret_cast<float4 *>(TP.d_sh + (size_t)cell * N);
#pragma unroll
        for (int q = 0; q < N / 4; ++q) {
            float v[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) v[h] = G.gw[(q * 4 + h) % 3] * Y[(q * 4 + h) / 3];
            atomicAdd(row4 + q, make_float4(v[0], v[1], v[2], v[3]));
        }
    } else {
        float *row = TP.d_sh + (size_t)cell * N;
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const float v = G.gw[m % 3] * Y[m / 3];
            if (v != 0.0f) atomicAdd(row + m, v);
        }
    }
    if (TP.d_site) atomicAdd(TP.d_site + cell, G.g_site);
}

// The same, reduced over the lanes of the warp that scatter into the same
// cell at this point first (all 32 lanes call it; `valid` marks the lanes
// with an interval).
template <int DEG>
__device__ __forceinline__ void scatter_interval_warp(const SplatTrainParams &TP,
                                                      const float (&Y)[ShDims<DEG>::K],
                                                      bool valid, uint32_t cell,
                                                      const IntervalGrad &G) {
    constexpr int N = 3 * ShDims<DEG>::K;
    const PeerTree tree = peer_tree(valid, cell);
    const bool lead = valid && tree.leader;
    if (TP.d_site) {
        float v[5] = {G.g_density, G.g_site.x, G.g_site.y, G.g_site.z, G.g_site.w};
        group_sum(tree, v);
        if (lead) {
            atomicAdd(TP.d_density + cell, v[0]);
            atomicAdd(TP.d_site + cell, make_float4(v[1], v[2], v[3], v[4]));
        }
    } else {
        float v[1] = {G.g_density};
        group_sum(tree, v);
        if (lead) atomicAdd(TP.d_density + cell, v[0]);
    }
    if (N % 4 == 0) {
        constexpr int Q = N % 8 == 0 ? 8 : 4;
        float4 *row4 = reinterpret_cast<float4 *>(TP.d_sh + (size_t)cell * N);
#pragma unroll
        for (int q = 0; q < N / Q; ++q) {
            float v[Q];
#pragma unroll
            for (int h = 0; h < Q; ++h) v[h] = G.gw[(q * Q + h) % 3] * Y[(q * Q + h) / 3];
            group_sum(tree, v);
            if (lead) {
#pragma unroll
                for (int h = 0; h < Q; h += 4)
                    atomicAdd(row4 + (q * Q + h) / 4, make_float4(v[h], v[h + 1], v[h + 2], v[h + 3]));
            }
        }
    } else {
        float *row = TP.d_sh + (size_t)cell * N;
#pragma unroll
        for (int i = 0; i < N; i += 3) {
            float v[3] = {G.gw[0] * Y[i / 3], G.gw[1] * Y[i / 3], G.gw[2] * Y[i / 3]};
            group_sum(tree, v);
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (lead && v[c] != 0.0f) atomicAdd(row + i + c, v[c]);
        }
    }
}

// Replay.  A ray whose composited intervals all fit the forward's record
// walks that list: no traversal, no clip, no SH row.  The others (record
// overflow, or no record) gather the same windows in the same order again
// and recompute each interval's colour.  Both feed splat_interval_grad.
template <int DEG, bool BF16>
__global__ void __launch_bounds__(kSplatBlock, 5)
splat_train_backward_kernel(const __grid_constant__ SplatTrainParams TP) {
    const SplatParams &P = TP.base;
    constexpr int K = ShDims<DEG>::K;
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if ((slot & ~31u) >= P.total_work) return;
    const uint32_t w = tile_item(P.tile_order, slot);
    const SplatLane L = splat_lane(P, w);
    const WinRay &ray = L.ray;
    const float depth = L.vd->depth;
    const Ray r{ray.ox, ray.oy, ray.oz, ray.dx, ray.dy, ray.dz};
    float Ch[3] = {0.f, 0.f, 0.f}, Cl[3] = {0.f, 0.f, 0.f}, gC[3] = {0.f, 0.f, 0.f};
    uint32_t recorded = kRecOverflow;
    if (L.active) {
        const RayState st =
            TP.ray_state[(size_t)L.vd->pixel_begin + (size_t)L.y * L.vd->width + L.x];
        Ch[0] = st.c_hi.x;
        Ch[1] = st.c_hi.y;
        Ch[2] = st.c_hi.z;
        Cl[0] = st.c_lo.x;
        Cl[1] = st.c_lo.y;
        Cl[2] = st.c_lo.z;
        gC[0] = st.c_hi.w;
        gC[1] = st.c_lo.w;
        gC[2] = st.g.x;
        recorded = __float_as_uint(st.g.y);
    }
    float Ph[3] = {0.f, 0.f, 0.f}, Pl[3] = {0.f, 0.f, 0.f};
    float Y[K];
    sh_basis<DEG>(ray.dx, ray.dy, ray.dz, Y);
    float T = 1.0f;
    bool finished = !L.active || (gC[0] == 0.f && gC[1] == 0.f && gC[2] == 0.f);
    // recorded rays: entry i of every lane at once, so that lanes compositing
    // the same support at the same rank share one atomic per value
    const bool replay = !finished && recorded != kRecOverflow;
    const uint32_t rounds = __reduce_max_sync(0xffffffffu, replay ? recorded : 0u);
#pragma unroll 1
    for (uint32_t i = 0; i < rounds; ++i) {
        const bool valid = replay && i < recorded;
        uint32_t cell = 0;
        IntervalGrad G{};
        if (valid) {
            const uint32_t chunk =
                __ldg(TP.rec_table + (size_t)(w >> 5) * TP.rec_chunks + i / kChunkEntries);
            const uint32_t *rec = rec_entry(TP, chunk, w, i);
            cell = __ldcs(rec);
            const float dt_raw = __uint_as_float(__ldcs(rec + 32));
            const uint32_t links = __ldcs(rec + 64);
            float cu[3];
#pragma unroll
            for (int ch = 0; ch < 3; ++ch) cu[ch] = __uint_as_float(__ldcs(rec + 96 + 32 * ch));
            const float dens = __ldg(P.m.density + cell) * 1.0f;
            G = splat_interval_terms<DEG>(TP, ray, r, depth, cell, dens, dt_raw, links, cu, Ch,
                                          Cl, gC, T, Ph, Pl);
        }
        scatter_interval_warp<DEG>(TP, Y, valid, cell, G);
    }
    if (replay) finished = true;
    uint32_t steps = 0, clipped = 0, nodes_visited = 0;
    bool cursor_valid = false;
    float cur_t = 0.f;
    uint32_t cur_cell = 0;
    auto hit = [&](uint32_t p, bool mine, float limit, auto &k) -> bool {
        return splat_hit(P, ray, depth, cursor_valid, cur_t, p, mine, limit, k, clipped);
    };
    SPLAT_WINDOW(WinKey2, kSplatTrainWindow);
    for (;;) {
        const bool want = !finished;
        if (!__any_sync(0xffffffffu, want)) break;
        const int count = SPLAT_GATHER(P.nodes, ray, depth, want, cursor_valid, cur_t, cur_cell);
        if (!want) continue;
#pragma unroll 1
        for (int i = 0; i < count; ++i) {
            const WinKey2 e = SPLAT_KEY(i);
            if (T <= P.weight_threshold || steps >= P.max_steps) {
                finished = true;
                break;
            }
            steps += 1;
            const uint32_t cell = e.idx;
            const float dens = __ldg(P.m.density + cell) * 1.0f;
            if (dens <= 1.0e-6f) continue;
            float coef[ShDims<DEG>::N];
            load_sh_row<DEG, BF16>(P.m, cell, coef);
            float cu[3];
            eval_sh<DEG>(coef, ray.dx, ray.dy, ray.dz, cu[0], cu[1], cu[2]);
            const IntervalGrad G =
                splat_interval_terms<DEG>(TP, ray, r, depth, cell, dens, __uint_as_float(e.pos),
                                          e.aux, cu, Ch, Cl, gC, T, Ph, Pl);
            scatter_interval<DEG>(TP, Y, cell, G);
        }
        if (finished) continue;
        if (count < kWin) {
            finished = true;
        } else {
            const auto last = SPLAT_KEY(kWin - 1);
            cursor_valid = true;
            cur_t = last.t;
            cur_cell = last.idx;
        }
    }
}

// Launches KERNEL<DEG, BF16> with `smem` bytes of dynamic shared memory
// (raising the kernel's limit first when that with the kernel's static
// shared memory can pass the default 48 KB).
template <class K, class P>
cudaError_t launch_with_smem(K kernel, int blocks, size_t smem, cudaStream_t s, const P &p) {
    if (smem > (size_t)32 * 1024) {  // static + dynamic above 48 KB needs the opt-in
        const cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kernel<<<blocks, kSplatBlock, smem, s>>>(p);
    return cudaGetLastError();
}

#define BV_SPLAT_SELECT(KERNEL, PARAMS, DEGREE, BF, BLOCKS, SMEM, STREAM)                 \
    switch ((int)(DEGREE) * 2 + ((BF) ? 1 : 0)) {                                         \
        case 0: return launch_with_smem(KERNEL<0, false>, BLOCKS, SMEM, STREAM, PARAMS);  \
        case 1: return launch_with_smem(KERNEL<0, true>, BLOCKS, SMEM, STREAM, PARAMS);   \
        case 2: return launch_with_smem(KERNEL<1, false>, BLOCKS, SMEM, STREAM, PARAMS);  \
        case 3: return launch_with_smem(KERNEL<1, true>, BLOCKS, SMEM, STREAM, PARAMS);   \
        case 4: return launch_with_smem(KERNEL<2, false>, BLOCKS, SMEM, STREAM, PARAMS);  \
        case 5: return launch_with_smem(KERNEL<2, true>, BLOCKS, SMEM, STREAM, PARAMS);   \
        case 6: return launch_with_smem(KERNEL<3, false>, BLOCKS, SMEM, STREAM, PARAMS);  \
        case 7: return launch_with_smem(KERNEL<3, true>, BLOCKS, SMEM, STREAM, PARAMS);   \
        default: return cudaErrorInvalidValue;                                            \
    }

cudaError_t launch_splat_train(const SplatTrainParams &p, bool backward, cudaStream_t s) {
    const int blocks = (int)((p.base.total_work + kSplatBlock - 1) / kSplatBlock);
    if (blocks == 0) return cudaSuccess;
    const size_t smem = splat_window_bytes(4, kSplatTrainWindow);
    if (backward) {
        BV_SPLAT_SELECT(splat_train_backward_kernel, p, p.base.m.sh_degree, p.base.m.sh_bf16,
                        blocks, smem, s);
    }
    BV_SPLAT_SELECT(splat_train_forward_kernel, p, p.base.m.sh_degree, p.base.m.sh_bf16, blocks,
                    smem, s);
}

cudaError_t launch_splat(const SplatParams &p, cudaStream_t s) {
    const int blocks = (int)((p.total_work + kSplatBlock - 1) / kSplatBlock);
    if (blocks == 0) return cudaSuccess;
    BV_SPLAT_SELECT(splat_kernel, p, p.m.sh_degree, p.m.sh_bf16, blocks,
                    splat_window_bytes(3, kSplatWindow), s);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bv_status sp_fail(bv_status code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    set_last_error(buf);
    return code;
}

bv_status sp_cuda(cudaError_t e, const char *what) {
    return sp_fail(e == cudaErrorMemoryAllocation ? BV_ERR_OUT_OF_MEMORY : BV_ERR_CUDA, "%s: %s",
                   what, cudaGetErrorString(e));
}

#define SP_CUDA(call, what)                              \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return sp_cuda(e_, what); \
    } while (0)

}  // namespace
}  // namespace bv

using namespace bv;

struct bv_splat_tracer {
    uint32_t n = 0, m_edges = 0, sh_degree = 0, sh_stride = 0, n_nodes = 0;
    bool bf16 = false;
    bv_trace_settings settings{};
    uint32_t capacity = 0;
    // device
    SplatPrim *prims = nullptr;
    BvhNode *nodes = nullptr;
    SplatFace *row_faces = nullptr;
    float4 *geom = nullptr;          // [N] model order (training Jacobians)
    uint32_t *offsets = nullptr;     // [N+1] CSR
    uint32_t *neighbors = nullptr;   // [M] CSR
    float *density = nullptr;
    // training scratch
    RayState *ray_state = nullptr;
    size_t ray_state_capacity = 0;
    uint32_t *rec_pool = nullptr;      // training forward's interval-record chunks
    size_t rec_pool_chunks = 0;
    uint32_t *rec_table = nullptr;     // chunk of each (tile, chunk rank), then the pool counter
    size_t rec_table_words = 0;
    uint32_t *rec_demand = nullptr;    // pinned: the pool counter after the last forward
    cudaEvent_t rec_event = nullptr;   // that copy has landed
    uint32_t rec_entries = kSplatRecEntries;
    TileScheduler render_order, train_order;  // heaviest-first tile orders
    float4 *site_grads = nullptr;    // [N], kept zero between calls
    void *sh = nullptr;
    unsigned long long *stats = nullptr;
    uint32_t *max_candidates = nullptr;
    unsigned long long *count_totals = nullptr;
    // last dispatch (for the candidate count and stats)
    std::vector<bv_camera> last_cams;
    uint32_t last_w = 0, last_h = 0;
    cudaStream_t last_stream = nullptr;
    bool stats_enabled = false, last_has_stats = false;
    uint32_t last_launches = 0;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    // every dispatch and training call: its end, and the stream it ran on
    // (a call on another stream waits for it: the tile orders, ray state and
    // interval record are the tracer's)
    cudaEvent_t done = nullptr;
    cudaStream_t work_stream = nullptr;
    bool worked = false;

    DeviceModel model() const {
        DeviceModel m;
        std::memset(&m, 0, sizeof(m));
        m.density = density;
        m.sh = sh;
        m.n = n;
        m.sh_degree = sh_degree;
        m.sh_stride = sh_stride;
        m.sh_bf16 = bf16 ? 1u : 0u;
        m.bounded = 1u;
        return m;
    }
};

namespace {

void free_splat(bv_splat_tracer *t) {
    if (!t) return;
    cudaFree(t->prims);
    cudaFree(t->nodes);
    cudaFree(t->row_faces);
    cudaFree(t->geom);
    cudaFree(t->offsets);
    cudaFree(t->neighbors);
    cudaFree(t->ray_state);
    cudaFree(t->rec_pool);
    cudaFree(t->rec_table);
    t->render_order.release();
    t->train_order.release();
    cudaFreeHost(t->rec_demand);
    if (t->rec_event) cudaEventDestroy(t->rec_event);
    cudaFree(t->site_grads);
    cudaFree(t->density);
    cudaFree(t->sh);
    cudaFree(t->stats);
    cudaFree(t->max_candidates);
    cudaFree(t->count_totals);
    for (auto &e : t->ev)
        if (e) cudaEventDestroy(e);
    if (t->done) cudaEventDestroy(t->done);
    delete t;
}

uint16_t bf16_rne(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
    return (uint16_t)((u + ((u >> 16) & 1u) + 0x7fffu) >> 16);
}

// Enqueues the splat kernel for the cameras (chunks of kMaxViewsPerLaunch).
// The clip planes of rows [r0, r1) of the Cech CSR into `rows` (see
// SplatFace), each row in BV_SPLAT_ROW_SORT order.
void build_clip_rows_range(const bv_model_desc *md, uint32_t r0, uint32_t r1, SplatFace *rows) {
    std::vector<std::pair<double, uint32_t>> order;
    std::vector<SplatFace> faces;
    for (uint32_t i = r0; i < r1; ++i) {
        const float *si = md->points + 4 * (size_t)i;
        const float ri = md->radii[i];
        const uint32_t b = md->adjacency_offsets[i], e = md->adjacency_offsets[i + 1];
        order.clear();
        faces.resize(e - b);
        for (uint32_t k = b; k < e; ++k) {
            const uint32_t j = md->adjacency_neighbors[k];
            const float *a = md->points + 4 * (size_t)j;
            const float rj = md->radii[j];
            const float nx = a[0] - si[0], ny = a[1] - si[1], nz = a[2] - si[2];
            const float dsq = std::max((nx * nx + ny * ny) + nz * nz, 1.0e-20f);
            const float shift = 0.5f + 0.5f * (ri * ri - rj * rj) / dsq;
            SplatFace &f = faces[k - b];
            uint32_t off = k - b;
            float off_bits, nbr_bits;
            std::memcpy(&off_bits, &off, 4);
            std::memcpy(&nbr_bits, &j, 4);
            f.point = make_float4(si[0] + shift * nx, si[1] + shift * ny, si[2] + shift * nz, off_bits);
            f.normal = make_float4(nx, ny, nz, nbr_bits);
            double key = BV_SPLAT_ROW_SORT ? (double)shift * std::sqrt((double)dsq) : 0.0;
            if (!(key == key)) key = INFINITY;  // a NaN sorts last
            order.emplace_back(key, off);
        }
        std::sort(order.begin(), order.end());
        for (uint32_t p = 0; p < e - b; ++p) rows[b + p] = faces[order[p].second];
    }
}

void build_clip_rows(const bv_model_desc *md, uint32_t n, SplatFace *rows) {
    const uint32_t hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const uint32_t workers = std::min<uint32_t>(hw, std::max<uint32_t>(1u, n / 4096u));
    std::vector<std::thread> pool;
    for (uint32_t w = 0; w < workers; ++w) {
        const uint32_t r0 = (uint32_t)((uint64_t)n * w / workers);
        const uint32_t r1 = (uint32_t)((uint64_t)n * (w + 1) / workers);
        pool.emplace_back(build_clip_rows_range, md, r0, r1, rows);
    }
    for (auto &th : pool) th.join();
}

// Orders a call on stream s after the tracer's previous call when that ran
// on another stream; marks the call's end afterwards.
bv_status order_after_previous(bv_splat_tracer *t, cudaStream_t s) {
    if (t->worked && t->work_stream != s)
        SP_CUDA(cudaStreamWaitEvent(s, t->done, 0), "stream wait on the previous call");
    return BV_OK;
}

bv_status mark_call_end(bv_splat_tracer *t, cudaStream_t s) {
    SP_CUDA(cudaEventRecord(t->done, s), "event record");
    t->work_stream = s;
    t->worked = true;
    return BV_OK;
}

bv_status enqueue_splats(bv_splat_tracer *t, float4 *out, const bv_camera *cams, uint32_t n,
                         uint32_t w, uint32_t h, bool count_only, cudaStream_t s) {
    for (uint32_t c0 = 0; c0 < n; c0 += kMaxViewsPerLaunch) {
        const uint32_t nc = std::min<uint32_t>(kMaxViewsPerLaunch, n - c0);
        SplatParams p;
        std::memset(&p, 0, sizeof(p));
        p.m = t->model();
        p.prims = t->prims;
        p.nodes = t->nodes;
        p.row_faces = t->row_faces;
        p.max_steps = t->settings.max_steps;
        p.weight_threshold = t->settings.weight_threshold;
        p.n_views = nc;
        uint32_t work = 0;
        for (uint32_t v = 0; v < nc; ++v) {
            p.views[v] = view_desc(cams[c0 + v], w, h, work, (uint64_t)v * w * h);
            work += tile_padded_rays(w, h);
        }
        p.total_work = work;
        p.out = out ? out + (size_t)c0 * w * h : nullptr;
        p.stats = (t->stats_enabled && !count_only) ? t->stats : nullptr;
        p.max_candidates = t->max_candidates;
        p.count_totals = t->count_totals;
        p.count_only = count_only ? 1u : 0u;
        const size_t tiles = work / 32u;
        bool time_tiles = false;
        if (!count_only && n <= (uint32_t)kMaxViewsPerLaunch)
            time_tiles = t->render_order.begin(BV_SPLAT_TILE_ORDER, tiles, nc, w, h, p.tile_order);
        p.tile_cost = time_tiles ? t->render_order.cost : nullptr;
        SP_CUDA(launch_splat(p, s), "splat launch");
        t->last_launches += 1;
        if (time_tiles) {
            SP_CUDA(t->render_order.end(tiles, nc, w, h, s), "tile order");
            t->last_launches += t->render_order.order_launches();
        }
    }
    return BV_OK;
}

}  // namespace

extern "C" {

bv_status bv_powerfoam_splat_tracer_new(const bv_model_desc *md, const bv_trace_settings *settings,
                                        bv_splat_tracer **out) {
    if (!out) return sp_fail(BV_ERR_INVALID_ARGUMENT, "out handle pointer is null");
    *out = nullptr;
    if (!md) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null model");
    if (!md->radii) return sp_fail(BV_ERR_INVALID_ARGUMENT, "PowerFoam splat tracer requires radii");
    bv_trace_settings ts{};
    if (settings) {
        ts = *settings;
    } else {
        ts.max_steps = 1024;
        ts.weight_threshold = 0.001f;
    }
    if (ts.max_steps == 0) return sp_fail(BV_ERR_INVALID_ARGUMENT, "PowerFoam splat max_steps must be non-zero");
    if (ts.debug_cell_density)
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "PowerFoam splat tracer has no cell-density debug mode");
    if (bv_model_validate(md, nullptr, 0) != BV_OK) return BV_ERR_INVALID_MODEL;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return sp_fail(BV_ERR_NO_DEVICE, "no CUDA device");

    const uint32_t n = md->num_points, m_edges = md->adjacency_offsets[n];
    const uint32_t deg = md->sh_degree > 3 ? 3 : md->sh_degree;
    const uint32_t nsh = 3 * (deg + 1) * (deg + 1);
    const bool bf16 = (md->flags & BV_MODEL_SH_BF16) != 0;
    const uint32_t align = bf16 ? 8u : 4u;
    const uint32_t stride = (nsh + align - 1) / align * align;

    // supports: conservative boxes, Morton-ordered BVH
    std::vector<BvhBox> boxes(n);
    std::vector<float> centers(3 * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) {
        const float *p = md->points + 4 * (size_t)i;
        const double r = std::max((double)md->radii[i], 0.0);
        for (int k = 0; k < 3; ++k) {
            const double ext = r * (1.0 + 1e-4) + 1e-6 * (1.0 + std::fabs((double)p[k]));
            boxes[i].lo[k] = std::nextafter((float)((double)p[k] - ext), -INFINITY);
            boxes[i].hi[k] = std::nextafter((float)((double)p[k] + ext), INFINITY);
            centers[3 * (size_t)i + k] = p[k];
        }
    }
    for (uint32_t i = 0; i < n; ++i)
        if (md->adjacency_offsets[i + 1] - md->adjacency_offsets[i] >= kNoPlane)
            return sp_fail(BV_ERR_NOT_SUPPORTED, "a Cech row longer than 65,534 entries");
    BvhBuild bvh = build_bvh(boxes, centers, BvhMethod::kMorton);
    if (bvh_depth(bvh.nodes) >= (uint32_t)kSplatStack)
        return sp_fail(BV_ERR_NOT_SUPPORTED, "BVH deeper than the traversal stack");
    std::vector<SplatPrim> prims(n);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t c = bvh.order[i];
        const float *p = md->points + 4 * (size_t)c;
        prims[i].site = make_float4(p[0], p[1], p[2], md->radii[c]);
        prims[i].link = make_uint4(c, md->adjacency_offsets[c], md->adjacency_offsets[c + 1], 0u);
    }
    // clip planes of every Cech entry, FP32 in the per-ray order of
    // powerfoam_splat_interval (this file is built with FP contraction off);
    // each row stored nearest plane first (the plane's distance from the
    // site, shift |n|; ties by CSR offset), over the host's threads
    std::vector<SplatFace> rows(std::max<uint32_t>(m_edges, 1));
    build_clip_rows(md, n, rows.data());
    std::vector<float> dens(n);
    std::vector<float4> geom(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float *p = md->points + 4 * (size_t)i;
        dens[i] = p[3];
        geom[i] = make_float4(p[0], p[1], p[2], md->radii[i]);
    }

    bv_splat_tracer *t = new bv_splat_tracer();
    if (BV_SPLAT_SPLIT_ORDER) {
        t->train_order.stable = false;
        t->train_order.second_shift = 0;
    }
    t->n = n;
    t->m_edges = m_edges;
    t->sh_degree = deg;
    t->sh_stride = stride;
    t->bf16 = bf16;
    t->settings = ts;
    t->capacity = std::max(std::max(ts.max_steps > 0x3fffffffu ? 0xffffffffu : ts.max_steps * 4u, 1024u),
                           ts.powerfoam_candidate_capacity);
    t->n_nodes = (uint32_t)bvh.nodes.size();
    auto cleanup = [&](cudaError_t e, const char *what) {
        free_splat(t);
        return sp_cuda(e, what);
    };
#define SP_TRY(call, what)                                \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cleanup(e_, what);  \
    } while (0)
    SP_TRY(cudaMalloc(&t->prims, sizeof(SplatPrim) * n), "cudaMalloc supports");
    SP_TRY(cudaMalloc(&t->nodes, sizeof(BvhNode) * t->n_nodes), "cudaMalloc nodes");
    SP_TRY(cudaMalloc(&t->row_faces, sizeof(SplatFace) * rows.size()), "cudaMalloc rows");
    SP_TRY(cudaMalloc(&t->density, sizeof(float) * n), "cudaMalloc density");
    SP_TRY(cudaMalloc(&t->stats, sizeof(unsigned long long) * 4), "cudaMalloc stats");
    SP_TRY(cudaMalloc(&t->max_candidates, sizeof(uint32_t)), "cudaMalloc counter");
    SP_TRY(cudaMalloc(&t->count_totals, 2 * sizeof(unsigned long long)), "cudaMalloc counters");
    SP_TRY(cudaMemcpy(t->prims, prims.data(), sizeof(SplatPrim) * n, cudaMemcpyHostToDevice), "upload supports");
    SP_TRY(cudaMemcpy(t->nodes, bvh.nodes.data(), sizeof(BvhNode) * t->n_nodes, cudaMemcpyHostToDevice),
           "upload nodes");
    SP_TRY(cudaMemcpy(t->row_faces, rows.data(), sizeof(SplatFace) * rows.size(), cudaMemcpyHostToDevice),
           "upload rows");
    SP_TRY(cudaMemcpy(t->density, dens.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "upload density");
    SP_TRY(cudaMalloc(&t->geom, sizeof(float4) * n), "cudaMalloc sites");
    SP_TRY(cudaMalloc(&t->offsets, sizeof(uint32_t) * (n + 1)), "cudaMalloc offsets");
    SP_TRY(cudaMalloc(&t->neighbors, sizeof(uint32_t) * std::max<uint32_t>(m_edges, 1)),
           "cudaMalloc neighbours");
    SP_TRY(cudaMalloc(&t->site_grads, sizeof(float4) * n), "cudaMalloc site grads");
    SP_TRY(cudaMemset(t->site_grads, 0, sizeof(float4) * n), "memset site grads");
    SP_TRY(cudaMemcpy(t->geom, geom.data(), sizeof(float4) * n, cudaMemcpyHostToDevice),
           "upload sites");
    SP_TRY(cudaMemcpy(t->offsets, md->adjacency_offsets, sizeof(uint32_t) * (n + 1),
                      cudaMemcpyHostToDevice), "upload offsets");
    if (m_edges)
        SP_TRY(cudaMemcpy(t->neighbors, md->adjacency_neighbors, sizeof(uint32_t) * m_edges,
                          cudaMemcpyHostToDevice), "upload neighbours");
    if (bf16) {
        std::vector<uint16_t> row((size_t)n * stride, 0);
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t k = 0; k < nsh; ++k)
                row[(size_t)i * stride + k] = bf16_rne(md->sh_coefficients[(size_t)i * nsh + k]);
        SP_TRY(cudaMalloc(&t->sh, row.size() * 2), "cudaMalloc sh");
        SP_TRY(cudaMemcpy(t->sh, row.data(), row.size() * 2, cudaMemcpyHostToDevice), "upload sh");
    } else {
        std::vector<float> row((size_t)n * stride, 0.0f);
        for (uint32_t i = 0; i < n; ++i)
            std::memcpy(&row[(size_t)i * stride], md->sh_coefficients + (size_t)i * nsh, nsh * 4);
        SP_TRY(cudaMalloc(&t->sh, row.size() * 4), "cudaMalloc sh");
        SP_TRY(cudaMemcpy(t->sh, row.data(), row.size() * 4, cudaMemcpyHostToDevice), "upload sh");
    }
    for (auto &e : t->ev) SP_TRY(cudaEventCreate(&e), "cudaEventCreate");
    SP_TRY(cudaEventCreateWithFlags(&t->done, cudaEventDisableTiming), "cudaEventCreate");
#undef SP_TRY
    *out = t;
    return BV_OK;
}

void bv_powerfoam_splat_tracer_destroy(bv_splat_tracer *t) {
    if (!t) return;
    cudaDeviceSynchronize();
    free_splat(t);
}

bv_status bv_powerfoam_splat_tracer_dispatch_batch(bv_splat_tracer *t, float *out_rgba_dev,
                                                   const bv_camera *cams, uint32_t n_cams,
                                                   uint32_t width, uint32_t height, bv_stream stream) {
    if (!t || !out_rgba_dev || !cams) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (width == 0 || height == 0) return sp_fail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (n_cams == 0) return sp_fail(BV_ERR_INVALID_ARGUMENT, "no cameras");
    if ((uint64_t)tile_padded_rays(width, height) * kMaxViewsPerLaunch >= (1ull << 32))
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "image too large");
    for (uint32_t i = 0; i < n_cams; ++i) {
        const bv_status st = validate_camera(cams[i]);
        if (st != BV_OK) return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    bv_status st = order_after_previous(t, s);
    if (st != BV_OK) return st;
    t->last_cams.assign(cams, cams + n_cams);
    t->last_w = width;
    t->last_h = height;
    t->last_stream = s;
    t->last_launches = 0;
    t->last_has_stats = t->stats_enabled;
    if (t->stats_enabled) {
        SP_CUDA(cudaMemsetAsync(t->stats, 0, 4 * sizeof(unsigned long long), s), "stats reset");
        SP_CUDA(cudaEventRecord(t->ev[0], s), "event");
    }
    st = enqueue_splats(t, reinterpret_cast<float4 *>(out_rgba_dev), cams, n_cams, width, height,
                        false, s);
    if (st != BV_OK) return st;
    if (t->stats_enabled) SP_CUDA(cudaEventRecord(t->ev[1], s), "event");
    return mark_call_end(t, s);
}

bv_status bv_powerfoam_splat_tracer_dispatch(bv_splat_tracer *t, float *out_rgba_dev,
                                             const bv_camera *camera, uint32_t width, uint32_t height,
                                             bv_stream stream) {
    return bv_powerfoam_splat_tracer_dispatch_batch(t, out_rgba_dev, camera, 1, width, height, stream);
}

bv_status bv_powerfoam_splat_tracer_candidate_stats(bv_splat_tracer *t, uint32_t *max_hits,
                                                    uint64_t *total_hits, uint64_t *row_entries) {
    if (!t || !max_hits) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (t->last_cams.empty()) return sp_fail(BV_ERR_INVALID_ARGUMENT, "no dispatch to count");
    cudaStream_t s = t->last_stream;
    bv_status st = order_after_previous(t, s);
    if (st != BV_OK) return st;
    SP_CUDA(cudaMemsetAsync(t->max_candidates, 0, sizeof(uint32_t), s), "counter reset");
    SP_CUDA(cudaMemsetAsync(t->count_totals, 0, 2 * sizeof(unsigned long long), s), "counter reset");
    const uint32_t launches = t->last_launches;
    st = enqueue_splats(t, nullptr, t->last_cams.data(), (uint32_t)t->last_cams.size(), t->last_w,
                        t->last_h, true, s);
    t->last_launches = launches;
    if (st != BV_OK) return st;
    st = mark_call_end(t, s);
    if (st != BV_OK) return st;
    uint32_t h = 0;
    unsigned long long tot[2] = {0, 0};
    SP_CUDA(cudaMemcpyAsync(&h, t->max_candidates, sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "read");
    SP_CUDA(cudaMemcpyAsync(tot, t->count_totals, sizeof(tot), cudaMemcpyDeviceToHost, s), "read");
    SP_CUDA(cudaStreamSynchronize(s), "synchronize");
    *max_hits = h;
    if (total_hits) *total_hits = tot[0];
    if (row_entries) *row_entries = tot[1];
    return BV_OK;
}

bv_status bv_powerfoam_splat_tracer_validate_candidate_counts(bv_splat_tracer *t, uint32_t *observed) {
    if (!t || !observed) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    uint32_t h = 0;
    const bv_status st = bv_powerfoam_splat_tracer_candidate_stats(t, &h, nullptr, nullptr);
    if (st != BV_OK) return st;
    *observed = h;
    if (h > t->capacity)
        return sp_fail(BV_ERR_CANDIDATE_OVERFLOW,
                       "PowerFoam render needs %u candidates for one ray, but scratch capacity is %u", h,
                       t->capacity);
    return BV_OK;
}

uint32_t bv_powerfoam_splat_tracer_candidate_capacity(const bv_splat_tracer *t) {
    return t ? t->capacity : 0;
}
uint32_t bv_powerfoam_splat_tracer_max_steps(const bv_splat_tracer *t) {
    return t ? t->settings.max_steps : 0;
}
float bv_powerfoam_splat_tracer_weight_threshold(const bv_splat_tracer *t) {
    return t ? t->settings.weight_threshold : 0.0f;
}
bv_status bv_powerfoam_splat_tracer_set_weight_threshold(bv_splat_tracer *t, float w) {
    if (!t) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    if (!(w >= 0.0f)) return sp_fail(BV_ERR_INVALID_ARGUMENT, "weight threshold must be >= 0");
    t->settings.weight_threshold = w;
    return BV_OK;
}

bv_status bv_powerfoam_splat_tracer_set_interval_record(bv_splat_tracer *t, uint32_t entries) {
    if (!t) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->rec_entries = entries;
    if (entries == 0) {
        cudaFree(t->rec_pool);
        cudaFree(t->rec_table);
        t->rec_pool = t->rec_table = nullptr;
        t->rec_pool_chunks = t->rec_table_words = 0;
    }
    return BV_OK;
}

bv_status bv_powerfoam_splat_tracer_enable_stats(bv_splat_tracer *t, uint32_t enabled) {
    if (!t) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->stats_enabled = enabled != 0;
    return BV_OK;
}

bv_status bv_powerfoam_splat_tracer_last_stats(bv_splat_tracer *t, bv_launch_stats *out) {
    if (!t || !out) return sp_fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->launches = t->last_launches;
    if (!t->last_has_stats) return BV_OK;
    SP_CUDA(cudaEventSynchronize(t->ev[1]), "event sync");
    float ms = 0.f;
    SP_CUDA(cudaEventElapsedTime(&ms, t->ev[0], t->ev[1]), "elapsed");
    out->kernel_ms = ms;
    unsigned long long h[4] = {0, 0, 0, 0};
    SP_CUDA(cudaMemcpy(h, t->stats, sizeof(h), cudaMemcpyDeviceToHost), "stats read");
    out->rays = h[0];
    out->steps = h[1];
    out->faces = h[2];
    return BV_OK;
}

bv_status bv_powerfoam_splat_tracer_forward_backward(
    bv_splat_tracer *t, const bv_camera *cams, uint32_t n_cams, uint32_t width, uint32_t height,
    const float *target, const bv_train_settings *ts, const bv_grads *grads, float *loss,
    float *rgb_out, bv_stream stream) {
    if (!t || !cams || !target || !ts || !grads || !loss)
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (!grads->d_density_dev || !grads->d_sh_dev)
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "density and SH gradient tables are required");
    if (width == 0 || height == 0 || n_cams == 0)
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (ts->loss != BV_LOSS_L2 && ts->loss != BV_LOSS_L1)
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "unknown loss %u", ts->loss);
    if (!(ts->max_dt > 0.0f)) return sp_fail(BV_ERR_INVALID_ARGUMENT, "max_dt must be positive");
    if (ts->max_steps == 0) return sp_fail(BV_ERR_INVALID_ARGUMENT, "max_steps must be non-zero");
    const uint32_t nsh = 3 * (t->sh_degree + 1) * (t->sh_degree + 1);
    if ((nsh % 4) == 0 && (reinterpret_cast<uintptr_t>(grads->d_sh_dev) & 15u) != 0)
        return sp_fail(BV_ERR_INVALID_ARGUMENT, "d_sh table must be 16-byte aligned");
    const uint64_t chunk_rays = (uint64_t)std::min<uint32_t>(n_cams, kMaxViewsPerLaunch) * width * height;
    if (chunk_rays >= (1ull << 31)) return sp_fail(BV_ERR_INVALID_ARGUMENT, "batch too large");
    for (uint32_t i = 0; i < n_cams; ++i) {
        bv_status st = validate_camera(cams[i]);
        if (st != BV_OK) return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    {
        const bv_status st = order_after_previous(t, s);
        if (st != BV_OK) return st;
    }
    if (chunk_rays > t->ray_state_capacity) {
        cudaFree(t->ray_state);
        t->ray_state = nullptr;
        t->ray_state_capacity = 0;
        SP_CUDA(cudaMalloc(&t->ray_state, sizeof(RayState) * chunk_rays), "cudaMalloc ray state");
        t->ray_state_capacity = chunk_rays;
    }
    // interval record: up to rec_entries composited intervals of every ray,
    // in chunks from a pool (rays beyond the limit, or finding the pool
    // empty, are traversed again by the replay).  The pool starts at two
    // chunks per tile and grows to twice the demand the previous call
    // reported (the allocation counter, copied back after each forward),
    // up to kSplatRecBytes.
    uint32_t rec_chunks = 0;
    size_t tiles = 0;
    {
        const size_t chunk_work =
            (size_t)std::min<uint32_t>(n_cams, kMaxViewsPerLaunch) * tile_padded_rays(width, height);
        tiles = chunk_work / 32;
        const uint32_t entries = std::min<uint32_t>(t->rec_entries, ts->max_steps);
        rec_chunks = (entries + kChunkEntries - 1) / kChunkEntries;
        const size_t cap = std::min<size_t>(kSplatRecBytes / (kChunkWords * sizeof(uint32_t)),
                                            tiles * rec_chunks);
        size_t pool = std::min<size_t>(cap, tiles * 2);
        if (t->rec_event) {
            const cudaError_t q = cudaEventQuery(t->rec_event);
            if (q == cudaSuccess && *t->rec_demand > t->rec_pool_chunks)
                pool = std::min<size_t>(cap, std::max<size_t>(pool, 2 * (size_t)*t->rec_demand));
            else if (q == cudaErrorNotReady)
                (void)cudaGetLastError();  // still in flight: keep the current pool
        }
        const size_t table = tiles * rec_chunks + 1;
        bool ok = rec_chunks > 0;
        if (ok && !t->rec_demand) {
            if (cudaMallocHost(&t->rec_demand, sizeof(uint32_t)) != cudaSuccess ||
                cudaEventCreateWithFlags(&t->rec_event, cudaEventDisableTiming) != cudaSuccess) {
                (void)cudaGetLastError();
                ok = false;
            } else {
                *t->rec_demand = 0;
            }
        }
        if (ok && (pool > t->rec_pool_chunks || table > t->rec_table_words)) {
            cudaFree(t->rec_pool);
            cudaFree(t->rec_table);
            t->rec_pool = t->rec_table = nullptr;
            t->rec_pool_chunks = t->rec_table_words = 0;
            if (cudaMalloc(&t->rec_pool, pool * kChunkWords * sizeof(uint32_t)) == cudaSuccess &&
                cudaMalloc(&t->rec_table, table * sizeof(uint32_t)) == cudaSuccess) {
                t->rec_pool_chunks = pool;
                t->rec_table_words = table;
            } else {
                (void)cudaGetLastError();  // out of memory: the replay traverses
                cudaFree(t->rec_pool);
                cudaFree(t->rec_table);
                t->rec_pool = t->rec_table = nullptr;
                ok = false;
            }
        }
        if (!ok) rec_chunks = 0;
    }
    // heaviest-first tile order (calls of one launch): the forward times its
    // tiles, the order is built from those times after the backward
    const uint32_t *order = nullptr;
    const bool time_tiles = t->train_order.begin(BV_SPLAT_TILE_ORDER, tiles, n_cams, width, height, order);
    t->last_launches = 0;
    t->last_has_stats = t->stats_enabled;
    if (t->stats_enabled) {
        SP_CUDA(cudaMemsetAsync(t->stats, 0, sizeof(unsigned long long) * 4, s), "stats reset");
        SP_CUDA(cudaEventRecord(t->ev[0], s), "event");
    }
    SP_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s), "loss reset");
    const bool want_site = grads->d_positions_dev || grads->d_radii_dev;
    const double total_rays = (double)n_cams * width * height;
    for (uint32_t c0 = 0; c0 < n_cams; c0 += kMaxViewsPerLaunch) {
        const uint32_t nc = std::min<uint32_t>(kMaxViewsPerLaunch, n_cams - c0);
        SplatTrainParams p;
        std::memset(&p, 0, sizeof(p));
        p.base.m = t->model();
        p.base.prims = t->prims;
        p.base.nodes = t->nodes;
        p.base.row_faces = t->row_faces;
        p.base.max_steps = ts->max_steps;
        p.base.weight_threshold = ts->weight_threshold;
        p.base.n_views = nc;
        uint32_t work = 0;
        for (uint32_t v = 0; v < nc; ++v) {
            p.base.views[v] = view_desc(cams[c0 + v], width, height, work, (uint64_t)v * width * height);
            work += tile_padded_rays(width, height);
        }
        p.base.total_work = work;
        p.base.stats = t->stats_enabled ? t->stats : nullptr;
        const size_t off = (size_t)c0 * width * height;
        p.geom = t->geom;
        p.offsets = t->offsets;
        p.neighbors = t->neighbors;
        p.max_dt = ts->max_dt;
        p.loss_kind = ts->loss;
        p.inv_count = (float)(1.0 / (3.0 * total_rays));
        p.target = target + 3 * off;
        p.rgb_out = rgb_out ? rgb_out + 3 * off : nullptr;
        p.loss = loss;
        p.ray_state = t->ray_state;
        p.d_density = grads->d_density_dev;
        p.d_sh = grads->d_sh_dev;
        p.d_site = want_site ? t->site_grads : nullptr;
        if (rec_chunks) {
            const size_t words = tiles * rec_chunks;
            SP_CUDA(cudaMemsetAsync(t->rec_table, 0xff, words * sizeof(uint32_t), s), "record reset");
            SP_CUDA(cudaMemsetAsync(t->rec_table + words, 0, sizeof(uint32_t), s), "record reset");
            p.rec_pool = t->rec_pool;
            p.rec_table = t->rec_table;
            p.rec_next = t->rec_table + words;
            p.rec_chunks = rec_chunks;
            p.rec_limit = std::min<uint32_t>(t->rec_entries, ts->max_steps);
            p.pool_chunks = (uint32_t)std::min<size_t>(t->rec_pool_chunks, 0xfffffff0u);
        }
        // split orders: the forward takes the stable second order, the replay
        // the first (unstable) one
        p.base.tile_order = BV_SPLAT_SPLIT_ORDER ? t->train_order.second(order) : order;
        p.base.tile_cost = time_tiles ? t->train_order.cost : nullptr;
        SP_CUDA(launch_splat_train(p, false, s), "splat training forward launch");
        if (rec_chunks) {
            SP_CUDA(cudaMemcpyAsync(t->rec_demand, p.rec_next, sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, s), "record demand");
            SP_CUDA(cudaEventRecord(t->rec_event, s), "event");
        }
        p.base.stats = nullptr;
        p.base.tile_cost = nullptr;
        p.base.tile_order = order;
        SP_CUDA(launch_splat_train(p, true, s), "splat training backward launch");
        t->last_launches += 2;
        if (time_tiles) {
            SP_CUDA(t->train_order.end(tiles, n_cams, width, height, s), "tile order");
            t->last_launches += t->train_order.order_launches();
        }
    }
    if (want_site) {
        SP_CUDA(launch_fold_site_grads(t->site_grads, t->n, grads->d_positions_dev,
                                       grads->d_radii_dev, s), "site gradient fold");
        t->last_launches += 1;
    }
    if (t->stats_enabled) SP_CUDA(cudaEventRecord(t->ev[1], s), "event");
    return mark_call_end(t, s);
}

}  // extern "C"
