// Windowed front-to-back gather over a BVH of particle support boxes, shared
// by the Gaussian tracers (SH colour and relight).
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

__device__ __forceinline__ bool win_less(float ta, uint32_t ia, float tb, uint32_t ib) {
    return ta < tb || (ta == tb && ia < ib);
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

// One pass: fills buf[0..count) with the W smallest keys above the cursor
// (all keys when !cursor_valid) in ascending order and returns count.
// `hit(pos, t, idx)` tests the particle at table position pos and returns
// its key when the ray hits it; every hit's depth must lie inside its leaf
// box's slab interval.  S bounds the traversal stack (the BVH depth plus
// one).
template <int W, int S, class Hit>
__device__ __forceinline__ int win_gather(const BvhNode *__restrict__ nodes, const WinRay &ray,
                                          float t_end, bool cursor_valid, float cur_t,
                                          uint32_t cur_idx, WinKey (&buf)[W],
                                          uint32_t &nodes_visited, Hit hit) {
    int count = 0;
    uint32_t stack[S];
    int sp = 0;
    stack[sp++] = 0u;
    while (sp > 0) {
        const uint32_t ni = stack[--sp];
        const BvhNode nd = nodes[ni];
        nodes_visited += 1;
        float tn[2], tf[2];
        bool ok[2];
        const float4 lo[2] = {nd.l_lo, nd.r_lo}, hi[2] = {nd.l_hi, nd.r_hi};
        const uint32_t cnts[2] = {__float_as_uint(nd.l_hi.w), __float_as_uint(nd.r_hi.w)};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            ok[c] = cnts[c] != kBvhNoChild && win_slab(lo[c], hi[c], ray, t_end, tn[c], tf[c]);
            if (ok[c] && cursor_valid && tf[c] < cur_t) ok[c] = false;
            if (ok[c] && count == W && tn[c] > buf[W - 1].t) ok[c] = false;
        }
        // push the farther child first so that the nearer one is visited next
        const int first = (ok[0] && ok[1] && tn[1] < tn[0]) ? 1 : 0;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int c = k == 0 ? 1 - first : first;
            if (!ok[c]) continue;
            const uint32_t ref = __float_as_uint(c == 0 ? nd.l_lo.w : nd.r_lo.w);
            const uint32_t cnt = cnts[c];
            if (cnt == 0u) {
                if (sp < S) stack[sp++] = ref;
                continue;
            }
            for (uint32_t p = ref; p < ref + cnt; ++p) {
                float t;
                uint32_t id;
                if (!hit(p, t, id)) continue;
                if (cursor_valid && !win_less(cur_t, cur_idx, t, id)) continue;
                if (count == W && !win_less(t, id, buf[W - 1].t, buf[W - 1].idx)) continue;
                // insertion into the sorted window (static indexing keeps buf
                // in registers)
                WinKey nk{t, id, p};
#pragma unroll
                for (int i = 0; i < W; ++i) {
                    if (i < count && win_less(nk.t, nk.idx, buf[i].t, buf[i].idx)) {
                        const WinKey tmp = buf[i];
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
template <int W>
__device__ __forceinline__ WinKey win_at(const WinKey (&buf)[W], int i) {
    WinKey h = buf[0];
#pragma unroll
    for (int j = 0; j < W; ++j)
        if (j == i) h = buf[j];
    return h;
}

}  // namespace bv
