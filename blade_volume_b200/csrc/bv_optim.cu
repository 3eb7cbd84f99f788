// Optimizer step over a tracer's device model: Adam on the density, SH,
// site-position and radius tables from the gradient tables of
// bv_forward_backward, followed by a refresh of the walk's face table.
//
// The reference trains through meganeura's Adam (not vendored), configured
// per parameter group by configure_optimizer / radfoam_v1_lrs
// (blade-volume-train/src/diff_render.rs:3215-3330): learning-rate
// multipliers for log_density, positions and SH (DC and higher order), with
// the density parameter passed through density_activation (:4649-4656,
// ReLU or softplus(beta x)/beta) before it reaches the tracer.  Here the
// update is Kingma & Ba's Adam with bias correction, in FP32, written as
//   m = b1 m + (1 - b1) g,   v = b2 v + (1 - b2) g^2,
//   p = p - lr (m / c1) / (sqrt(v / c2) + eps),   c_i = 1 - b_i^t,
// with c1, c2 formed on the host in FP64 and rounded once.  The density
// table is the activation of a raw parameter x kept here; its gradient is
// dL/dx = dL/dsigma * act'(x).
//
// Compiled with -fmad=false: every kernel is a sequence of rounded FP32
// operations in the written order, so the oracle's FP32 restatement matches
// bit for bit.  Every kernel streams its tables once (HBM-bound).

#include <cuda_bf16.h>

#include "bv_device.cuh"
#include "bv_internal.h"

namespace bv {
namespace {

constexpr int kOptBlock = 256;

__device__ __forceinline__ float adam_update(float p, float g, float &m, float &v,
                                             const AdamScalars &a, float lr) {
    m = a.beta1 * m + a.one_minus_beta1 * g;
    v = a.beta2 * v + a.one_minus_beta2 * (g * g);
    const float mhat = m / a.c1;
    const float vhat = v / a.c2;
    return p - (lr * mhat) / (sqrtf(vhat) + a.eps);
}

// density_activation (diff_render.rs:4649-4656) and its derivative.
__device__ __forceinline__ float act(float x, uint32_t kind, float beta) {
    if (kind == BV_DENSITY_RELU) return fmaxf(x, 0.0f);
    if (kind == BV_DENSITY_SOFTPLUS) {
        const float bx = beta * x;
        const float sp = bx > 20.0f ? bx : bv_logf(1.0f + bv_expf(bx));
        return sp / beta;
    }
    return x;
}

__device__ __forceinline__ float act_grad(float x, uint32_t kind, float beta) {
    if (kind == BV_DENSITY_RELU) return x > 0.0f ? 1.0f : 0.0f;
    if (kind == BV_DENSITY_SOFTPLUS) return 1.0f / (1.0f + bv_expf(-(beta * x)));
    return 1.0f;
}

// inv_density_activation (diff_render.rs:4658-4672): the raw parameter whose
// activation is the stored density.
__global__ void __launch_bounds__(kOptBlock) init_density_param_kernel(const float *density,
                                                                      float *param, uint32_t n,
                                                                      uint32_t kind, float beta) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float y = density[i];
    float x = y;
    if (kind == BV_DENSITY_SOFTPLUS) {
        const float by = beta * y;
        x = by > 20.0f ? by : bv_logf(fmaxf(bv_expf(by) - 1.0f, 1e-20f));
        x = x / beta;
    }
    param[i] = x;
}

__global__ void __launch_bounds__(kOptBlock) adam_density_kernel(AdamParams P) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    const float x = P.density_param[i];
    const float g = P.g_density[i] * act_grad(x, P.activation, P.softplus_beta);
    const float xn = adam_update(x, g, P.m_density[i], P.v_density[i], P.s, P.lr_density);
    P.density_param[i] = xn;
    P.density[i] = act(xn, P.activation, P.softplus_beta);
}

// SH coefficient c of site i (c < 3K): DC (c < 3) and higher-order rates.
template <bool BF16>
__global__ void __launch_bounds__(kOptBlock) adam_sh_kernel(AdamParams P) {
    // 32-bit index arithmetic: n * 3K < 2^31 is checked on the host
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= P.n * P.sh_row) return;
    const uint32_t i = k / P.sh_row, c = k - i * P.sh_row;
    const float lr = c < 3u ? P.lr_sh_dc : P.lr_sh_rest;
    if (lr == 0.0f) return;
    const size_t dev = (size_t)i * P.sh_stride + c;
    const float p = BF16 ? P.sh_master[k] : static_cast<float *>(P.sh)[dev];
    const float pn = adam_update(p, P.g_sh[k], P.m_sh[k], P.v_sh[k], P.s, lr);
    if (BF16) {
        P.sh_master[k] = pn;
        static_cast<__nv_bfloat16 *>(P.sh)[dev] = __float2bfloat16_rn(pn);
    } else {
        static_cast<float *>(P.sh)[dev] = pn;
    }
}

// Site positions (x, y, z) and, for PowerFoam, radii; a table whose rate is
// zero is left as it is (frozen, moments untouched).
__global__ void __launch_bounds__(kOptBlock) adam_geom_kernel(AdamParams P) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.n) return;
    float4 s = P.geom[i];
    if (P.g_pos && P.lr_position != 0.0f) {
        float *xyz[3] = {&s.x, &s.y, &s.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const size_t j = (size_t)i * 3 + a;
            *xyz[a] = adam_update(*xyz[a], P.g_pos[j], P.m_pos[j], P.v_pos[j], P.s, P.lr_position);
        }
    }
    if (P.g_radius && P.lr_radius != 0.0f)
        s.w = adam_update(s.w, P.g_radius[i], P.m_radius[i], P.v_radius[i], P.s, P.lr_radius);
    P.geom[i] = s;
}

// The walk reads neighbour sites and densities through the face table:
// re-gather them for every CSR entry.
__global__ void __launch_bounds__(kOptBlock) refresh_faces_kernel(FaceEntry *faces, uint32_t m,
                                                                 const float4 *geom,
                                                                 const float *density) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const uint32_t j = faces[k].link.x;
    faces[k].site = geom[j];
    faces[k].link.w = __float_as_uint(density[j]);
}

inline int blocks_for(uint64_t n) { return (int)((n + kOptBlock - 1) / kOptBlock); }

}  // namespace

cudaError_t launch_init_density_param(const float *density, float *param, uint32_t n,
                                      uint32_t kind, float beta, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    init_density_param_kernel<<<blocks_for(n), kOptBlock, 0, s>>>(density, param, n, kind, beta);
    return cudaGetLastError();
}

cudaError_t launch_adam_step(const AdamParams &p, FaceEntry *faces, uint32_t m_edges,
                             bool bf16, cudaStream_t s) {
    if (p.n == 0) return cudaSuccess;
    if (p.g_density && p.lr_density != 0.0f)
        adam_density_kernel<<<blocks_for(p.n), kOptBlock, 0, s>>>(p);
    if (p.g_sh && (p.lr_sh_dc != 0.0f || p.lr_sh_rest != 0.0f)) {
        const uint64_t total = (uint64_t)p.n * p.sh_row;
        if (bf16)
            adam_sh_kernel<true><<<blocks_for(total), kOptBlock, 0, s>>>(p);
        else
            adam_sh_kernel<false><<<blocks_for(total), kOptBlock, 0, s>>>(p);
    }
    if ((p.g_pos && p.lr_position != 0.0f) || (p.g_radius && p.lr_radius != 0.0f))
        adam_geom_kernel<<<blocks_for(p.n), kOptBlock, 0, s>>>(p);
    if (m_edges)
        refresh_faces_kernel<<<blocks_for(m_edges), kOptBlock, 0, s>>>(faces, m_edges, p.geom,
                                                                       p.density);
    return cudaGetLastError();
}

}  // namespace bv
