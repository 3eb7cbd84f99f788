// Device helpers shared by the walk and splat kernels: exp, SH evaluation,
// ray generation and the persistent ray dispenser.  Every translation unit
// that includes this file is compiled with -fmad=false, so each expression
// is the written sequence of IEEE-rounded operations (the CPU restatement's).
#pragma once

#include <cuda_bf16.h>

#include "bv_internal.h"

#ifndef BV_REFILL_MIN
#define BV_REFILL_MIN 32
#endif

namespace bv {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kRefillMin = BV_REFILL_MIN;

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

// log(x): x = m 2^e, m in [sqrt(1/2), sqrt(2)), log(1+f) = 2 atanh(f/(2+f))
// arranged as f - (f^2/2 - s (f^2/2 + R)); same sequence as the oracle.
__device__ __forceinline__ float bv_logf(float x) {
    if (x != x || x < 0.0f) return __int_as_float(0x7fc00000);
    if (x == 0.0f) return __int_as_float(0xff800000);
    if (x == __int_as_float(0x7f800000)) return x;
    uint32_t u = __float_as_uint(x);
    int e = 0;
    if (u < 0x00800000u) {
        u = __float_as_uint(x * 16777216.0f);
        e = -24;
    }
    e += (int)((u >> 23) & 0xffu) - 127;
    float m = __uint_as_float((u & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421353816986083984375f) {
        m = m * 0.5f;
        e += 1;
    }
    const float f = m - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    float p = 0.1538461595773697f;
    p = __fmaf_rn(p, z, 0.1818181872367859f);
    p = __fmaf_rn(p, z, 0.2222222238779068f);
    p = __fmaf_rn(p, z, 0.2857142984867096f);
    p = __fmaf_rn(p, z, 0.4000000059604645f);
    p = __fmaf_rn(p, z, 0.6666666865348816f);
    const float R = z * p;
    const float hfsq = 0.5f * f * f;
    const float ef = (float)e;
    return ef * 0.693115234375f -
           ((hfsq - (s * (hfsq + R) + ef * 3.19461832987144589424133e-05f)) - f);
}

__device__ __forceinline__ float bv_powf(float x, float y) {
    if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : __int_as_float(0x7f800000));
    return bv_expf(y * bv_logf(x));
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

}  // namespace
}  // namespace bv
