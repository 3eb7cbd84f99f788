// Segment arithmetic shared by the walk kernels and the PowerFoam splat
// training kernels: the current cell, the support-sphere hit, the clipped
// interval of a recorded segment and the exact derivatives of its length
// (trace.rs:1077-1124, :1199-1325), the compensated colour accumulator and
// the site-gradient scatter.  Compiled with -fmad=false like its includers.
#pragma once

#include "bv_device.cuh"

namespace bv {
namespace {

// ---------------------------------------------------------------------------
// The walk's current cell: its site, CSR range and density.
// ---------------------------------------------------------------------------
struct Cell {
    uint32_t id, begin, end;
    float x, y, z, r, density;
};

__device__ __forceinline__ Cell load_cell(const DeviceModel &m, uint32_t id) {
    const float4 g = __ldg(m.geom + id);
    Cell c;
    c.id = id;
    c.begin = __ldg(m.offsets + id);
    c.end = __ldg(m.offsets + id + 1);
    c.x = g.x;
    c.y = g.y;
    c.z = g.z;
    c.r = g.w;
    c.density = __ldg(m.density + id);
    return c;
}

__device__ __forceinline__ Cell cell_from_face(const FaceEntry &f) {
    Cell c;
    c.id = f.link.x;
    c.begin = f.link.y;
    c.end = f.link.z;
    c.x = f.site.x;
    c.y = f.site.y;
    c.z = f.site.z;
    c.r = f.site.w;
    c.density = __uint_as_float(f.link.w);
    return c;
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

// The clipped interval of one recorded segment (path_interval_jacobian,
// trace.rs:1199-1325 without oriented surfaces) and which boundary is a
// sphere clip.
struct Interval {
    float start, end;
    bool start_sphere, end_sphere;
};

template <bool BOUNDED>
__device__ __forceinline__ bool record_interval(const Ray &ray, const Cell &c, float t0, float t1,
                                                Interval &iv) {
    iv.start = t0;
    iv.end = t1;
    iv.start_sphere = iv.end_sphere = false;
    if (BOUNDED) {
        float nt, ft, root, b;
        if (!sphere_hit(ray, c.x, c.y, c.z, c.r, nt, ft, root, b)) return false;
        if (nt > iv.start) {
            iv.start = nt;
            iv.start_sphere = true;
        }
        if (ft < iv.end) {
            iv.end = ft;
            iv.end_sphere = true;
        }
    }
    return !(iv.end <= iv.start || !isfinite(iv.start) || !isfinite(iv.end));
}

// d dt / d (x, y, z, r) of the previous, current and next site for a
// recorded segment; prev/next equal to the current cell mean a fixed
// boundary (t = 0 or the far plane).
struct Jacobians {
    float4 jp, jc, jn;
};

__device__ __forceinline__ Jacobians interval_jacobians(const Ray &ray, const Interval &iv,
                                                        uint32_t prev, float4 pp, const Cell &c,
                                                        bool has_next, float4 np, float t0,
                                                        float t1) {
    Jacobians J;
    float4 qprev = make_float4(0.f, 0.f, 0.f, 0.f), qcur = qprev;
    float4 nj = qprev, fj = qprev;
    if (iv.start_sphere || iv.end_sphere) {
        float nt, ft, root, b;
        sphere_hit(ray, c.x, c.y, c.z, c.r, nt, ft, root, b);
        const float ocx = ray.ox - c.x, ocy = ray.oy - c.y, ocz = ray.oz - c.z;
        const float px = ocx - b * ray.dx, py = ocy - b * ray.dy, pz = ocz - b * ray.dz;
        const float rx = px / root, ry = py / root, rz = pz / root;
        const float rr = c.r / root;
        nj = make_float4(ray.dx - rx, ray.dy - ry, ray.dz - rz, -rr);
        fj = make_float4(ray.dx + rx, ray.dy + ry, ray.dz + rz, rr);
    }
    if (iv.start_sphere) {
        qcur = nj;
    } else if (prev != c.id) {
        face_jacobian(ray, c.x, c.y, c.z, c.r, pp.x, pp.y, pp.z, pp.w, t0, qcur, qprev);
    }
    J.jp = make_float4(0.f, 0.f, 0.f, 0.f);
    J.jc = J.jp;
    J.jn = J.jp;
    J.jc = f4sub(J.jc, qcur);
    J.jp = f4sub(J.jp, qprev);
    if (iv.end_sphere) {
        J.jc = f4add(J.jc, fj);
    } else if (has_next) {
        float4 cj, aj;
        face_jacobian(ray, c.x, c.y, c.z, c.r, np.x, np.y, np.z, np.w, t1, cj, aj);
        J.jc = f4add(J.jc, cj);
        J.jn = f4add(J.jn, aj);
    }
    return J;
}

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

// Site gradients (x, y, z, radius) go to a float4-per-site table with one
// vector atomic; fold_site_grads_kernel adds it to the caller's tables.
__device__ __forceinline__ void scatter_site(float4 *d_site, uint32_t cell, float gdt, float4 j) {
    atomicAdd(d_site + cell, make_float4(gdt * j.x, gdt * j.y, gdt * j.z, gdt * j.w));
}

// Lanes of a warp that scatter into the same cell at the same replay step
// (coherent rays walk the same cells, and composite the same supports) are
// reduced first: __match_any_sync
// groups them, a binary tree over their ranks sums the values, and the
// rank-0 lane issues one vector atomic per float4.  At level l the lane of
// rank r (r a multiple of 2^(l+1)) adds the value of rank r + 2^l; that
// partner is found by pointer doubling: each lane knows the next member of
// its group, and the member 2^l ranks above is the 2^(l-1)-above member's
// own 2^(l-1)-above member (one shuffle per level).  All 32 lanes must call
// these together.
struct PeerTree {
    int levels;          // warp-uniform tree depth
    bool leader;         // rank 0 of its group
    int src[5];          // partner lane per level
    bool recv[5];        // adds the partner's value at that level
};

__device__ __forceinline__ PeerTree peer_tree(bool valid, uint32_t key) {
    PeerTree t;
    const unsigned lane = threadIdx.x & 31u;
    const unsigned peers = __match_any_sync(kFull, valid ? key : 0xffffffffu);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    const int n = __popc(peers);
    const unsigned maxn = __reduce_max_sync(kFull, valid ? (unsigned)n : 1u);
    t.levels = maxn <= 1 ? 0 : 32 - __clz(maxn - 1);
    t.leader = rank == 0;
    const unsigned above = peers & ~((2u << lane) - 1u);  // members after this lane
    int up = above ? __ffs(above) - 1 : 32;                 // 2^l ranks above; 32: none
#pragma unroll
    for (int l = 0; l < 5; ++l) {
        if (l > 0 && l < t.levels) {
            const int far = __shfl_sync(kFull, up, up < 32 ? up : (int)lane);
            up = up < 32 ? far : 32;
        }
        const bool r = (rank & ((2 << l) - 1)) == 0 && up < 32;
        t.recv[l] = r;
        t.src[l] = r ? up : (int)lane;
    }
    return t;
}

// Sums M values over each lane group: per tree level the M shuffles are
// issued together and the level test is taken once for all of them.
template <int M>
__device__ __forceinline__ void group_sum(const PeerTree &t, float (&v)[M]) {
#pragma unroll
    for (int l = 0; l < 5; ++l) {
        if (l >= t.levels) break;
        float o[M];
#pragma unroll
        for (int i = 0; i < M; ++i) o[i] = __shfl_sync(kFull, v[i], t.src[l]);
        if (t.recv[l]) {
#pragma unroll
            for (int i = 0; i < M; ++i) v[i] += o[i];
        }
    }
}

}  // namespace
}  // namespace bv
