// Windowed front-to-back gather over a BVH of particle support boxes, shared
// by the Gaussian tracers (SH colour and relight) and the PowerFoam splat.
//
// The reference enumerates candidates with hardware ray queries over proxy
// meshes and keeps, per batch, the next K hits above a cursor in strict
// (depth, index) order (gaussian_trace.wgsl:66-135, relight.wgsl:626-690).
// Here one pass walks the BVH (bv_bvh.h) front to back and keeps the W
// smallest (t, index) keys strictly above the cursor, pruning boxes that end
// before the cursor or start after the window's current last key, so that a
// pass touches only a thin slab of the tree.  The next pass starts above the
// window's last key, which makes the sequence of composited hits independent
// of W (the reference's own cursor test, trace.rs:965-998).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bv_bvh.h"

namespace bv {

struct WinRay {
    float ox, oy, oz, dx, dy, dz;
    float ix, iy, iz;  // 1 / d
};

struct WinKey {
    float t;
    uint32_t idx;  // the particle's index in the filtered model order (tie-break)
    uint32_t pos;  // position in the BVH-ordered particle table
};

// A key with one more payload word (the splat's entry / exit plane indices).
struct WinKey2 {
    float t;
    uint32_t idx;
    uint32_t pos;
    uint32_t aux;
};

__device__ __forceinline__ bool win_less(float ta, uint32_t ia, float tb, uint32_t ib) {
    return ta < tb || (ta == tb && ia < ib);
}

// 1/d with |d| raised to at least 1e-30, so that a box face through the ray
// origin gives 0 * finite rather than 0 * inf = NaN in the slab test.
__device__ __forceinline__ float win_inverse(float d) {
    return 1.0f / (fabsf(d) < 1e-30f ? copysignf(1e-30f, d) : d);
}

// Slab test of a box against the ray over [0, t_end], widened by a relative
// margin so that rounding can only keep a box, never drop one.
__device__ __forceinline__ bool win_slab(const float4 &lo, const float4 &hi, const WinRay &r,
                                         float t_end, float &tn, float &tf) {
    const float ax = (lo.x - r.ox) * r.ix, bx = (hi.x - r.ox) * r.ix;
    const float ay = (lo.y - r.oy) * r.iy, by = (hi.y - r.oy) * r.iy;
    const float az = (lo.z - r.oz) * r.iz, bz = (hi.z - r.oz) * r.iz;
    tn = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), 0.0f));
    tf = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), t_end));
    tn = tn - (1e-5f * fabsf(tn) + 1e-6f);
    tf = tf + (1e-5f * fabsf(tf) + 1e-6f);
    return tn <= tf;
}

// A traversal stack shared by the 32 lanes of a warp, held across their
// registers: entry i lives in lane i % 32, slot i / 32.  Every lane calls
// push/pop with the same arguments (the stack pointer is warp-uniform).
template <int S>
struct WarpStack {
    static_assert(S <= 96, "at most three register slots per lane");
    uint32_t slot[(S + 31) / 32] = {};
    int sp = 0;

    __device__ __forceinline__ void push(uint32_t v, uint32_t lane) {
        if (sp >= S) return;
        if ((uint32_t)(sp & 31) == lane) {
#pragma unroll
            for (int k = 0; k < (S + 31) / 32; ++k)
                if (k == (sp >> 5)) slot[k] = v;
        }
        ++sp;
    }
    __device__ __forceinline__ uint32_t pop() {
        --sp;
        uint32_t mine = slot[0];
#pragma unroll
        for (int k = 1; k < (S + 31) / 32; ++k)
            if (k == (sp >> 5)) mine = slot[k];
        return __shfl_sync(0xffffffffu, mine, sp & 31);
    }
};

// One pass fills a lane's buf[0..count) with the W smallest keys above its
// cursor (all keys when !cursor_valid) in ascending order and returns count.
// Every hit's depth must lie inside its leaf box's slab interval.  S bounds
// the traversal stack (the BVH depth plus one).
//
// The pass is warp-cooperative: all 32 lanes of the warp call it together,
// each with its own ray, cursor and window; lanes that need no pass (no ray,
// or done) pass want = false.  The warp walks one BVH traversal: a child is
// entered when any wanting lane's ray overlaps it and is not pruned for that
// lane, and each lane tests the primitives of entered leaves against its own
// ray only where the leaf is live for it.  Camera rays of an 8x4 pixel tile
// are coherent, so the union of their traversals is close to each one, and
// node and primitive loads are warp-uniform (one broadcast transaction).
// The window a lane ends with is the W smallest keys above its cursor,
// whatever the traversal order, because pruning only drops boxes that cannot
// hold such a key.
// `hit(pos, mine, limit, key)` is called by every lane for every primitive
// of an entered leaf and must return false where mine is false (it may use
// warp collectives); on a hit it fills key.t and key.idx and may overwrite
// the payload (key.pos starts as the table position).  limit is the lane's
// current window end (+inf while the window has room): a key at or past it
// cannot enter.
template <int W, int S, class Key, class Hit>
__device__ __forceinline__ int win_gather_warp(const BvhNode *__restrict__ nodes,
                                               const WinRay &ray, float t_end, bool want,
                                               bool cursor_valid, float cur_t, uint32_t cur_idx,
                                               Key (&buf)[W], uint32_t &nodes_visited,
                                               Hit hit) {
    const uint32_t lane = threadIdx.x & 31u;
    int count = 0;
    WarpStack<S> stack;
    stack.push(0u, lane);
    while (stack.sp > 0) {
        const uint32_t ni = stack.pop();
        const BvhNode nd = nodes[ni];
        if (want) nodes_visited += 1;
        float tn[2], tf[2];
        bool ok[2];
        const float4 lo[2] = {nd.l_lo, nd.r_lo}, hi[2] = {nd.l_hi, nd.r_hi};
        const uint32_t cnts[2] = {__float_as_uint(nd.l_hi.w), __float_as_uint(nd.r_hi.w)};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            ok[c] = want && cnts[c] != kBvhNoChild &&
                    win_slab(lo[c], hi[c], ray, t_end, tn[c], tf[c]);
            if (ok[c] && cursor_valid && tf[c] < cur_t) ok[c] = false;
            if (ok[c] && count == W && tn[c] > buf[W - 1].t) ok[c] = false;
        }
        const uint32_t live0 = __ballot_sync(0xffffffffu, ok[0]);
        const uint32_t live1 = __ballot_sync(0xffffffffu, ok[1]);
        // nearer child (by the lanes that enter both) is handled last, so
        // that it is popped first / its hits fill the windows first
        const uint32_t near1 = __ballot_sync(0xffffffffu, ok[0] && ok[1] && tn[1] < tn[0]);
        const uint32_t near0 = __ballot_sync(0xffffffffu, ok[0] && ok[1] && !(tn[1] < tn[0]));
        const int first = __popc(near1) > __popc(near0) ? 1 : 0;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int c = k == 0 ? 1 - first : first;
            if ((c == 0 ? live0 : live1) == 0u) continue;
            const uint32_t ref = __float_as_uint(c == 0 ? nd.l_lo.w : nd.r_lo.w);
            const uint32_t cnt = cnts[c];
            if (cnt == 0u) {
                stack.push(ref, lane);
                continue;
            }
            const bool mine = ok[c];
            for (uint32_t p = ref; p < ref + cnt; ++p) {
                Key nk;
                nk.pos = p;
                const float limit = count == W ? buf[W - 1].t : __int_as_float(0x7f800000);
                if (!hit(p, mine, limit, nk)) continue;
                if (cursor_valid && !win_less(cur_t, cur_idx, nk.t, nk.idx)) continue;
                if (count == W && !win_less(nk.t, nk.idx, buf[W - 1].t, buf[W - 1].idx)) continue;
#pragma unroll
                for (int i = 0; i < W; ++i) {
                    if (i < count && win_less(nk.t, nk.idx, buf[i].t, buf[i].idx)) {
                        const Key tmp = buf[i];
                        buf[i] = nk;
                        nk = tmp;
                    }
                }
#pragma unroll
                for (int i = 0; i < W; ++i)
                    if (i == count) buf[i] = nk;
                if (count < W) count += 1;
            }
        }
    }
    return count;
}

// buf[i] with a runtime i, by a static scan (keeps buf in registers).
template <int W, class Key>
__device__ __forceinline__ Key win_at(const Key (&buf)[W], int i) {
    Key h = buf[0];
#pragma unroll
    for (int j = 0; j < W; ++j)
        if (j == i) h = buf[j];
    return h;
}

}  // namespace bv

namespace bv {

// The window of win_gather_warp held in shared memory instead of registers
// (the W keys are the bulk of a lane's registers; in shared memory they let
// more warps stay resident).  Key i of thread tid sits at [i][tid] of each
// field array, so the lanes of a warp touch consecutive words.
template <int W, class Key>
struct SmemWindow {
    float *t;
    uint32_t *idx, *pos, *aux;  // aux unused for WinKey
    int stride;

    __device__ __forceinline__ Key get(int i) const {
        Key k;
        k.t = t[i * stride];
        k.idx = idx[i * stride];
        k.pos = pos[i * stride];
        get_aux(k, i);
        return k;
    }
    __device__ __forceinline__ void set(int i, const Key &k) {
        t[i * stride] = k.t;
        idx[i * stride] = k.idx;
        pos[i * stride] = k.pos;
        set_aux(k, i);
    }
    __device__ __forceinline__ void get_aux(WinKey &, int) const {}
    __device__ __forceinline__ void get_aux(WinKey2 &k, int i) const { k.aux = aux[i * stride]; }
    __device__ __forceinline__ void set_aux(const WinKey &, int) {}
    __device__ __forceinline__ void set_aux(const WinKey2 &k, int i) { aux[i * stride] = k.aux; }
};

// win_gather_warp with the window in shared memory: the same traversal,
// pruning and key order, so a pass ends with the same window.  The
// window's last key is mirrored in registers for the pruning tests.
template <int W, int S, class Key, class Hit>
__device__ __forceinline__ int win_gather_warp_smem(const BvhNode *__restrict__ nodes,
                                                    const WinRay &ray, float t_end, bool want,
                                                    bool cursor_valid, float cur_t,
                                                    uint32_t cur_idx, SmemWindow<W, Key> &win,
                                                    uint32_t &nodes_visited, Hit hit) {
    const uint32_t lane = threadIdx.x & 31u;
    int count = 0;
    float last_t = __int_as_float(0x7f800000);
    uint32_t last_idx = 0xffffffffu;
    WarpStack<S> stack;
    stack.push(0u, lane);
    while (stack.sp > 0) {
        const uint32_t ni = stack.pop();
        const BvhNode nd = nodes[ni];
        if (want) nodes_visited += 1;
        float tn[2], tf[2];
        bool ok[2];
        const float4 lo[2] = {nd.l_lo, nd.r_lo}, hi[2] = {nd.l_hi, nd.r_hi};
        const uint32_t cnts[2] = {__float_as_uint(nd.l_hi.w), __float_as_uint(nd.r_hi.w)};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            ok[c] = want && cnts[c] != kBvhNoChild &&
                    win_slab(lo[c], hi[c], ray, t_end, tn[c], tf[c]);
            if (ok[c] && cursor_valid && tf[c] < cur_t) ok[c] = false;
            if (ok[c] && count == W && tn[c] > last_t) ok[c] = false;
        }
        const uint32_t live0 = __ballot_sync(0xffffffffu, ok[0]);
        const uint32_t live1 = __ballot_sync(0xffffffffu, ok[1]);
        const uint32_t near1 = __ballot_sync(0xffffffffu, ok[0] && ok[1] && tn[1] < tn[0]);
        const uint32_t near0 = __ballot_sync(0xffffffffu, ok[0] && ok[1] && !(tn[1] < tn[0]));
        const int first = __popc(near1) > __popc(near0) ? 1 : 0;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int c = k == 0 ? 1 - first : first;
            if ((c == 0 ? live0 : live1) == 0u) continue;
            const uint32_t ref = __float_as_uint(c == 0 ? nd.l_lo.w : nd.r_lo.w);
            const uint32_t cnt = cnts[c];
            if (cnt == 0u) {
                stack.push(ref, lane);
                continue;
            }
            const bool mine = ok[c];
            for (uint32_t p = ref; p < ref + cnt; ++p) {
                Key nk;
                nk.pos = p;
                const float limit = count == W ? last_t : __int_as_float(0x7f800000);
                if (!hit(p, mine, limit, nk)) continue;
                if (cursor_valid && !win_less(cur_t, cur_idx, nk.t, nk.idx)) continue;
                if (count == W && !win_less(nk.t, nk.idx, last_t, last_idx)) continue;
                // insertion: shift the larger keys up one slot (the last one
                // drops out of a full window)
                int i = count < W ? count : W - 1;
                while (i > 0) {
                    const float ti = win.t[(i - 1) * win.stride];
                    const uint32_t ii = win.idx[(i - 1) * win.stride];
                    if (!win_less(nk.t, nk.idx, ti, ii)) break;
                    win.set(i, win.get(i - 1));
                    --i;
                }
                win.set(i, nk);
                if (count < W) count += 1;
                last_t = win.t[(count - 1) * win.stride];
                last_idx = win.idx[(count - 1) * win.stride];
            }
        }
    }
    return count;
}

// A tracer's window of W 12-byte keys per thread of a BLOCK-thread block:
// in registers (SMEM 0) or in dynamic shared memory (SMEM 1, 12 W BLOCK
// bytes set at launch).  TRACE_WINDOW_DECL declares what lives across
// passes, TRACE_WINDOW_GATHER runs one pass, TRACE_WINDOW_KEY(i) reads key i.
#define TRACE_WINDOW_DECL_1(W, BLOCK)                                              \
    extern __shared__ uint32_t s_trace_win[];                                     \
    SmemWindow<W, WinKey> trace_win{reinterpret_cast<float *>(s_trace_win) + threadIdx.x, \
                                    s_trace_win + 1 * (W) * (BLOCK) + threadIdx.x,     \
                                    s_trace_win + 2 * (W) * (BLOCK) + threadIdx.x,     \
                                    s_trace_win, (BLOCK)}
#define TRACE_WINDOW_PASS_1(W, S, NODES, RAY, TEND, WANT, CV, CT, CI, NV, HIT) \
    win_gather_warp_smem<W, S>(NODES, RAY, TEND, WANT, CV, CT, CI, trace_win, NV, HIT)
#define TRACE_WINDOW_KEY_1(W, i) trace_win.get(i)
#define TRACE_WINDOW_DECL_0(W, BLOCK) WinKey trace_buf[W]
#define TRACE_WINDOW_PASS_0(W, S, NODES, RAY, TEND, WANT, CV, CT, CI, NV, HIT) \
    win_gather_warp<W, S>(NODES, RAY, TEND, WANT, CV, CT, CI, trace_buf, NV, HIT)
#define TRACE_WINDOW_KEY_0(W, i) win_at(trace_buf, i)
#define TRACE_CAT_(a, b) a##b
#define TRACE_CAT(a, b) TRACE_CAT_(a, b)
#define TRACE_WINDOW_DECL(SMEM, W, BLOCK) TRACE_CAT(TRACE_WINDOW_DECL_, SMEM)(W, BLOCK)
#define TRACE_WINDOW_PASS(SMEM, ...) TRACE_CAT(TRACE_WINDOW_PASS_, SMEM)(__VA_ARGS__)
#define TRACE_WINDOW_KEY(SMEM, W, i) TRACE_CAT(TRACE_WINDOW_KEY_, SMEM)(W, i)

}  // namespace bv
