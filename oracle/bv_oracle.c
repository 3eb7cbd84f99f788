/*
 * CPU oracle for the blade-volume ray-tracing hot path.  TEST INFRASTRUCTURE:
 * the checker for the CUDA kernels, never part of the shipped library.
 *
 * Restates blade-volume/src/trace.rs (walk, recorder, Jacobians, splats),
 * blade-volume/src/lib.rs:526-541 (containing cell) and the training
 * gradient contract of blade-volume-train/src/diff_render.rs.  Build with
 * -ffp-contract=off: every FP32 expression below is evaluated in the order
 * the reference writes it (glam's Vec3::dot is ((x*x' + y*y') + z*z')).
 */
#include "bv_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* small vector helpers in glam's operation order                      */
/* ------------------------------------------------------------------ */
static inline float dot3f(const float a[3], const float b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline double dot3d(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

/*
 * exp(x) for FP32, written from Cody & Waite's argument reduction
 * (x = k*ln2 + r, ln2 split into a 12-bit-short high part and a low part)
 * followed by the degree-7 Taylor polynomial of e^r on |r| <= ln2/2 in
 * Horner form with fused multiply-adds, and an exact scaling by 2^k.
 * The CUDA kernels evaluate the identical operation sequence, so α and T
 * agree bit for bit between the oracle and the device.  The reference's
 * f32::exp is the platform libm; both are within 2 ulp of exp (checked in
 * tests/test_oracle_golden.py).
 */
float bvo_expf(float x) {
    if (x != x) return x;
    if (x > 88.72283935546875f) return INFINITY;
    if (x < -103.972084045410156f) return 0.0f;
    const float k = rintf(x * 1.44269502162933349609375f);
    float r = fmaf(k, -0.693115234375f, x);
    r = fmaf(k, -3.19461832987144589424133e-05f, r);
    float p = 1.98412701138295233249664e-04f;
    p = fmaf(p, r, 1.38888892251998186111450e-03f);
    p = fmaf(p, r, 8.33333376795053482055664e-03f);
    p = fmaf(p, r, 4.16666679084300994873047e-02f);
    p = fmaf(p, r, 1.66666671633720397949219e-01f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    if (ki > 127) {
        p = p * 2.0f;
        ki -= 1;
    }
    if (ki < -126) {
        /* subnormal result: scale by 2^(ki+64), then by 2^-64 */
        union { uint32_t u; float f; } s = {(uint32_t)(ki + 64 + 127) << 23};
        p = p * s.f;
        return p * 5.42101086242752217004e-20f;
    }
    union { uint32_t u; float f; } s = {(uint32_t)(ki + 127) << 23};
    return p * s.f;
}

/* tan(fov/2) for the ray mapping (radfoam.wgsl:268).  Computed once per
 * camera on the host in FP64 and rounded to FP32; the product library uses
 * the same expression and hands the result to the kernels. */
float bvo_tan_half(float fov) { return (float)tan((double)(0.5f * fov)); }

/* Pixel -> world ray, radfoam.wgsl:44-52 with qrot (common.wgsl:386-390)
 * and glam's normalize (v * (1/|v|)). */
void bvo_camera_ray(const bvo_camera *cam, uint32_t width, uint32_t height, uint32_t x,
                    uint32_t y, float origin[3], float dir[3]) {
    const float tx = bvo_tan_half(cam->fov[0]);
    const float ty = bvo_tan_half(cam->fov[1]);
    const float px = ((float)x + 0.5f) / (float)width;
    const float py = ((float)y + 0.5f) / (float)height;
    const float ndc_x = px * 2.0f - 1.0f;
    const float ndc_y = py * 2.0f - 1.0f;
    const float v[3] = {(ndc_x - cam->principal[0]) * tx, (ndc_y - cam->principal[1]) * ty, 1.0f};
    const float *q = cam->orientation;
    /* t = 2 * cross(q.xyz, v) */
    const float c0 = q[1] * v[2] - q[2] * v[1];
    const float c1 = q[2] * v[0] - q[0] * v[2];
    const float c2 = q[0] * v[1] - q[1] * v[0];
    const float t[3] = {2.0f * c0, 2.0f * c1, 2.0f * c2};
    /* v + q.w * t + cross(q.xyz, t) */
    const float e0 = q[1] * t[2] - q[2] * t[1];
    const float e1 = q[2] * t[0] - q[0] * t[2];
    const float e2 = q[0] * t[1] - q[1] * t[0];
    const float r[3] = {(v[0] + q[3] * t[0]) + e0, (v[1] + q[3] * t[1]) + e1,
                        (v[2] + q[3] * t[2]) + e2};
    const float len = sqrtf(dot3f(r, r));
    const float inv = 1.0f / len;
    dir[0] = r[0] * inv;
    dir[1] = r[1] * inv;
    dir[2] = r[2] * inv;
    origin[0] = cam->position[0];
    origin[1] = cam->position[1];
    origin[2] = cam->position[2];
}

/* ------------------------------------------------------------------ */
/* SH evaluation (trace.rs:242-402)                                    */
/* ------------------------------------------------------------------ */
static const float SH_C[16] = {
    0.2820948f,  -0.48860252f, 0.48860252f, -0.48860252f, 1.0925485f,  -1.0925485f,
    0.31539157f, -1.0925485f,  0.54627424f, -0.5900436f,  2.8906114f,  -0.4570458f,
    0.37317634f, -0.4570458f,  1.4453057f,  -0.5900436f,
};

static inline uint32_t sh_comps(uint32_t degree) {
    uint32_t d = (degree > 3 ? 3 : degree) + 1;
    return d * d;
}

/* SH basis values in the order and with the products that trace.rs uses;
 * y[m] multiplies the coefficient after the constant: color += (C_m*coef)*y[m]
 * for degree 1, ((C_m*coef)*a)*b for the two-factor degree-2 terms. */
void bvo_eval_rgb_sh(const bvo_model *m, uint32_t point, const float dir[3], float out[3],
                     float unclamped[3]) {
    const uint32_t deg = m->sh_degree > 3 ? 3 : m->sh_degree;
    const uint32_t comps = sh_comps(deg);
    const float *c = m->sh + (size_t)point * 3u * comps;
    const float x = dir[0], y = dir[1], z = dir[2];
    const float xx = x * x, yy = y * y, zz = z * z;
    float r = 0.0f, g = 0.0f, b = 0.0f;
    r += SH_C[0] * c[0];
    g += SH_C[0] * c[1];
    b += SH_C[0] * c[2];
    if (deg >= 1) {
        r += SH_C[1] * c[3] * y;  g += SH_C[1] * c[4] * y;  b += SH_C[1] * c[5] * y;
        r += SH_C[2] * c[6] * z;  g += SH_C[2] * c[7] * z;  b += SH_C[2] * c[8] * z;
        r += SH_C[3] * c[9] * x;  g += SH_C[3] * c[10] * x; b += SH_C[3] * c[11] * x;
    }
    if (deg >= 2) {
        r += SH_C[4] * c[12] * x * y; g += SH_C[4] * c[13] * x * y; b += SH_C[4] * c[14] * x * y;
        r += SH_C[5] * c[15] * y * z; g += SH_C[5] * c[16] * y * z; b += SH_C[5] * c[17] * y * z;
        const float t6 = 3.0f * zz - 1.0f;
        r += SH_C[6] * c[18] * t6; g += SH_C[6] * c[19] * t6; b += SH_C[6] * c[20] * t6;
        r += SH_C[7] * c[21] * x * z; g += SH_C[7] * c[22] * x * z; b += SH_C[7] * c[23] * x * z;
        const float t8 = xx - yy;
        r += SH_C[8] * c[24] * t8; g += SH_C[8] * c[25] * t8; b += SH_C[8] * c[26] * t8;
    }
    if (deg >= 3) {
        const float t9 = y * (3.0f * xx - yy);
        r += SH_C[9] * c[27] * t9; g += SH_C[9] * c[28] * t9; b += SH_C[9] * c[29] * t9;
        const float t10 = x * y * z;
        r += SH_C[10] * c[30] * t10; g += SH_C[10] * c[31] * t10; b += SH_C[10] * c[32] * t10;
        const float t11 = y * (5.0f * zz - 1.0f);
        r += SH_C[11] * c[33] * t11; g += SH_C[11] * c[34] * t11; b += SH_C[11] * c[35] * t11;
        const float t12 = z * (5.0f * zz - 3.0f);
        r += SH_C[12] * c[36] * t12; g += SH_C[12] * c[37] * t12; b += SH_C[12] * c[38] * t12;
        const float t13 = x * (5.0f * zz - 1.0f);
        r += SH_C[13] * c[39] * t13; g += SH_C[13] * c[40] * t13; b += SH_C[13] * c[41] * t13;
        const float t14 = z * (xx - yy);
        r += SH_C[14] * c[42] * t14; g += SH_C[14] * c[43] * t14; b += SH_C[14] * c[44] * t14;
        const float t15 = x * (xx - 3.0f * yy);
        r += SH_C[15] * c[45] * t15; g += SH_C[15] * c[46] * t15; b += SH_C[15] * c[47] * t15;
    }
    r = 0.5f + r;
    g = 0.5f + g;
    b = 0.5f + b;
    if (unclamped) {
        unclamped[0] = r;
        unclamped[1] = g;
        unclamped[2] = b;
    }
    out[0] = fmaxf(r, 0.0f);
    out[1] = fmaxf(g, 0.0f);
    out[2] = fmaxf(b, 0.0f);
}

/* SH basis Y_m(dir) in FP64 for the gradient oracle (same polynomials). */
static void sh_basis_d(uint32_t deg, const double d[3], double Y[16]) {
    const double x = d[0], y = d[1], z = d[2];
    const double xx = x * x, yy = y * y, zz = z * z;
    for (int i = 0; i < 16; ++i) Y[i] = 0.0;
    Y[0] = (double)SH_C[0];
    if (deg >= 1) {
        Y[1] = (double)SH_C[1] * y;
        Y[2] = (double)SH_C[2] * z;
        Y[3] = (double)SH_C[3] * x;
    }
    if (deg >= 2) {
        Y[4] = (double)SH_C[4] * x * y;
        Y[5] = (double)SH_C[5] * y * z;
        Y[6] = (double)SH_C[6] * (3.0 * zz - 1.0);
        Y[7] = (double)SH_C[7] * x * z;
        Y[8] = (double)SH_C[8] * (xx - yy);
    }
    if (deg >= 3) {
        Y[9] = (double)SH_C[9] * y * (3.0 * xx - yy);
        Y[10] = (double)SH_C[10] * x * y * z;
        Y[11] = (double)SH_C[11] * y * (5.0 * zz - 1.0);
        Y[12] = (double)SH_C[12] * z * (5.0 * zz - 3.0);
        Y[13] = (double)SH_C[13] * x * (5.0 * zz - 1.0);
        Y[14] = (double)SH_C[14] * z * (xx - yy);
        Y[15] = (double)SH_C[15] * x * (xx - 3.0 * yy);
    }
}

/* Magnitudes that an FP32 evaluation of each basis value rounds: the basis
 * with every difference turned into a sum (3 zz - 1 -> 3 zz + 1, ...), so
 * that a basis value near a zero of its polynomial carries the error of its
 * unreduced terms (error-budget use only). */
static void sh_basis_mag_d(uint32_t deg, const double d[3], double M[16]) {
    const double x = fabs(d[0]), y = fabs(d[1]), z = fabs(d[2]);
    const double xx = x * x, yy = y * y, zz = z * z;
    for (int i = 0; i < 16; ++i) M[i] = 0.0;
    M[0] = fabs((double)SH_C[0]);
    if (deg >= 1) {
        M[1] = fabs((double)SH_C[1]) * y;
        M[2] = fabs((double)SH_C[2]) * z;
        M[3] = fabs((double)SH_C[3]) * x;
    }
    if (deg >= 2) {
        M[4] = fabs((double)SH_C[4]) * x * y;
        M[5] = fabs((double)SH_C[5]) * y * z;
        M[6] = fabs((double)SH_C[6]) * (3.0 * zz + 1.0);
        M[7] = fabs((double)SH_C[7]) * x * z;
        M[8] = fabs((double)SH_C[8]) * (xx + yy);
    }
    if (deg >= 3) {
        M[9] = fabs((double)SH_C[9]) * y * (3.0 * xx + yy);
        M[10] = fabs((double)SH_C[10]) * x * y * z;
        M[11] = fabs((double)SH_C[11]) * y * (5.0 * zz + 1.0);
        M[12] = fabs((double)SH_C[12]) * z * (5.0 * zz + 3.0);
        M[13] = fabs((double)SH_C[13]) * x * (5.0 * zz + 1.0);
        M[14] = fabs((double)SH_C[14]) * z * (xx + yy);
        M[15] = fabs((double)SH_C[15]) * x * (xx + 3.0 * yy);
    }
}

/* ------------------------------------------------------------------ */
/* geometry kernels of the walk                                        */
/* ------------------------------------------------------------------ */
static inline float read_radius(const bvo_model *m, uint32_t i) {
    return m->radii ? m->radii[i] : 0.0f;
}

/* Exit distance through face k (neighbour j) of the cell at cp with power
 * radius cr, evaluated in double from the FP32 inputs: the re-evaluation of
 * the tie-break below. */
static double face_t_f64(const bvo_model *m, const float cp[3], float cr, uint32_t j,
                         const float o[3], const float d[3]) {
    const float *np = m->points + 4 * (size_t)j;
    const double off[3] = {(double)np[0] - cp[0], (double)np[1] - cp[1], (double)np[2] - cp[2]};
    double shift = 0.5;
    if (m->radii) {
        const double rj = m->radii[j], ri = cr;
        shift = 0.5 + 0.5 * (ri * ri - rj * rj) / fmax(dot3d(off, off), 1e-20);
    }
    const double rel[3] = {cp[0] + shift * off[0] - o[0], cp[1] + shift * off[1] - o[1],
                           cp[2] + shift * off[2] - o[2]};
    const double dd[3] = {d[0], d[1], d[2]};
    return dot3d(rel, off) / dot3d(off, dd);
}

/* Spacing of FP32 values at |x| (x finite). */
static inline float ulp_f(float x) {
    union { float f; uint32_t u; } a = {fabsf(x)}, b;
    b.u = a.u + 1u;
    return b.f - a.f;
}

/* find_exit_face (trace.rs:170-205). Returns face index or -1.
 * tie_break != 0: when the runner-up's FP32 distance is within
 * BVO_TIE_ULPS ulps of the winner's, both are re-evaluated in FP64 and the
 * smaller wins (equal: the earlier face in CSR order, the reference's rule). */
#define BVO_TIE_ULPS 4.0f
static int find_exit_face(const bvo_model *m, uint32_t cell, const float cp[3], float cr,
                          const float o[3], const float d[3], float t0, float depth,
                          float *best_out, int tie_break) {
    const uint32_t begin = m->offsets[cell], end = m->offsets[cell + 1];
    float best = depth, second = INFINITY;
    int face = -1, face2 = -1;
    const float ri2 = cr * cr;
    for (uint32_t k = begin; k < end; ++k) {
        const uint32_t j = m->neighbors[k];
        const float *np = m->points + 4 * (size_t)j;
        const float off[3] = {np[0] - cp[0], np[1] - cp[1], np[2] - cp[2]};
        float shift;
        if (m->radii) {
            const float rj = m->radii[j];
            const float dsq = fmaxf(dot3f(off, off), 1e-20f);
            shift = 0.5f + 0.5f * (ri2 - rj * rj) / dsq;
        } else {
            shift = 0.5f;
        }
        const float fo[3] = {cp[0] + shift * off[0], cp[1] + shift * off[1], cp[2] + shift * off[2]};
        const float dp = dot3f(off, d);
        if (dp > 0.0f) {
            const float rel[3] = {fo[0] - o[0], fo[1] - o[1], fo[2] - o[2]};
            const float t = dot3f(rel, off) / dp;
            if (isfinite(t) && t > t0 && t < best) {
                second = best;
                face2 = face;
                best = t;
                face = (int)(k - begin);
            } else if (isfinite(t) && t > t0 && t < second && t < depth) {
                second = t;
                face2 = (int)(k - begin);
            }
        }
    }
    if (tie_break && face >= 0 && face2 >= 0 && second - best <= BVO_TIE_ULPS * ulp_f(best)) {
        const double tb = face_t_f64(m, cp, cr, m->neighbors[begin + (uint32_t)face], o, d);
        const double t2 = face_t_f64(m, cp, cr, m->neighbors[begin + (uint32_t)face2], o, d);
        if (t2 < tb || (t2 == tb && face2 < face)) {
            face = face2;
            best = second;
        }
    }
    *best_out = best;
    return face;
}

/* support_interval (trace.rs:209-238). Returns 1 when non-empty. */
static int support_interval(int bounded, const float o[3], const float d[3], const float c[3],
                            float radius, float t0, float t1, float *s, float *e) {
    if (!bounded) {
        if (t1 > t0) {
            *s = t0;
            *e = t1;
            return 1;
        }
        return 0;
    }
    const float oc[3] = {o[0] - c[0], o[1] - c[1], o[2] - c[2]};
    const float a = dot3f(d, d);
    if (!isfinite(a) || a <= 0.0f) return 0;
    const float b = dot3f(oc, d);
    const float cc = dot3f(oc, oc) - radius * radius;
    const float disc = b * b - a * cc;
    if (disc <= 0.0f) return 0;
    const float root = sqrtf(disc);
    const float near_t = (-b - root) / a;
    const float far_t = (-b + root) / a;
    const float cs = fmaxf(t0, near_t);
    const float ce = fminf(t1, far_t);
    if (ce > cs) {
        *s = cs;
        *e = ce;
        return 1;
    }
    return 0;
}

int bvo_support_interval(int bounded, const float o[3], const float d[3], const float c[3],
                         float radius, float t0, float t1, float out[2]) {
    return support_interval(bounded, o, d, c, radius, t0, t1, &out[0], &out[1]);
}

/* sphere_intersection_jacobians (trace.rs:1101-1124); dir normalized. */
static int sphere_jac(const float o[3], const float d[3], const float c[3], float radius,
                      float *near_t, float *far_t, float nj[4], float fj[4]) {
    const float oc[3] = {o[0] - c[0], o[1] - c[1], o[2] - c[2]};
    const float b = dot3f(oc, d);
    const float disc = b * b - (dot3f(oc, oc) - radius * radius);
    if (disc <= 0.0f || !isfinite(disc)) return 0;
    const float root = sqrtf(disc);
    const float perp[3] = {oc[0] - b * d[0], oc[1] - b * d[1], oc[2] - b * d[2]};
    const float rdc[3] = {perp[0] / root, perp[1] / root, perp[2] / root};
    const float rdr = radius / root;
    *near_t = -b - root;
    *far_t = -b + root;
    if (nj) {
        nj[0] = d[0] - rdc[0]; nj[1] = d[1] - rdc[1]; nj[2] = d[2] - rdc[2]; nj[3] = -rdr;
        fj[0] = d[0] + rdc[0]; fj[1] = d[1] + rdc[1]; fj[2] = d[2] + rdc[2]; fj[3] = rdr;
    }
    return 1;
}

/* face_intersection_jacobians (trace.rs:1077-1097). */
static void face_jac(const float o[3], const float d[3], const float cp[3], float cr,
                     const float ap[3], float ar, float t, float cj[4], float aj[4]) {
    const float n[3] = {ap[0] - cp[0], ap[1] - cp[1], ap[2] - cp[2]};
    const float den = dot3f(d, n);
    if (!isfinite(den) || fabsf(den) <= 1e-20f) {
        memset(cj, 0, 16);
        memset(aj, 0, 16);
        return;
    }
    for (int i = 0; i < 3; ++i) {
        cj[i] = (o[i] - cp[i] + t * d[i]) / den;
        aj[i] = (ap[i] - o[i] - t * d[i]) / den;
    }
    cj[3] = cr / den;
    aj[3] = -ar / den;
}

/* path_interval_jacobian (trace.rs:1199-1325) without oriented surfaces.
 * Returns 1 and fills *e when the clipped interval is non-empty. */
static int path_interval_jacobian(const bvo_model *m, const float o[3], const float d[3],
                                  int bounded, uint32_t prev, uint32_t cell, uint32_t next,
                                  float t0, float t1, bvo_path_entry *e) {
    const float *cpp = m->points + 4 * (size_t)cell;
    const float cp[3] = {cpp[0], cpp[1], cpp[2]};
    const float cr = read_radius(m, cell);
    float start = t0, end = t1;
    int start_sphere = 0, end_sphere = 0;
    float nj[4] = {0}, fj[4] = {0};
    float qd_prev[4] = {0}, qd_cur[4] = {0};
    if (bounded) {
        float sn, sf;
        if (!sphere_jac(o, d, cp, cr, &sn, &sf, nj, fj)) return 0;
        if (sn > start) {
            start = sn;
            start_sphere = 1;
        }
        if (sf < end) {
            end = sf;
            end_sphere = 1;
        }
    }
    if (start_sphere) {
        memcpy(qd_cur, nj, 16);
    } else if (prev != cell) {
        const float *pp = m->points + 4 * (size_t)prev;
        const float ppos[3] = {pp[0], pp[1], pp[2]};
        face_jac(o, d, cp, cr, ppos, read_radius(m, prev), t0, qd_cur, qd_prev);
    }
    const float query_near = start;
    if (end <= start || !isfinite(start) || !isfinite(end)) return 0;
    float dprev[4] = {0}, dcur[4] = {0}, dnext[4] = {0};
    for (int i = 0; i < 4; ++i) {
        dcur[i] -= qd_cur[i];
        dprev[i] -= qd_prev[i];
    }
    if (end_sphere) {
        for (int i = 0; i < 4; ++i) dcur[i] += fj[i];
    } else if (next != cell) {
        const float *np = m->points + 4 * (size_t)next;
        const float npos[3] = {np[0], np[1], np[2]};
        float cj[4], aj[4];
        face_jac(o, d, cp, cr, npos, read_radius(m, next), t1, cj, aj);
        for (int i = 0; i < 4; ++i) {
            dcur[i] += cj[i];
            dnext[i] += aj[i];
        }
    }
    e->previous_cell = prev;
    e->cell = cell;
    e->next_cell = next;
    e->dt = end - start;
    memcpy(e->dt_d_previous, dprev, 16);
    memcpy(e->dt_d_current, dcur, 16);
    memcpy(e->dt_d_next, dnext, 16);
    e->surface_query_near = query_near;
    memcpy(e->surface_query_d_previous, qd_prev, 16);
    memcpy(e->surface_query_d_current, qd_cur, 16);
    e->t_start = start;
    return 1;
}

static int normalize_direction(const float in[3], float out[3]) {
    const float len = sqrtf(dot3f(in, in));
    if (len <= 0.0f || !isfinite(len)) return 0;
    out[0] = in[0] / len;
    out[1] = in[1] / len;
    out[2] = in[2] / len;
    return 1;
}

/* ------------------------------------------------------------------ */
/* trace_one_ray (trace.rs:1680-1820)                                  */
/* ------------------------------------------------------------------ */
static bvo_trace_result trace_one_ray_impl(const bvo_model *m, const float origin[3],
                                           const float direction[3],
                                           const bvo_trace_settings *s, uint32_t *cells,
                                           uint32_t cap, uint32_t *cell_count) {
    bvo_trace_result res;
    memset(&res, 0, sizeof(res));
    res.last_point = s->start_point;
    res.peak_point = -1;
    if (cell_count) *cell_count = 0;
    float d[3];
    if (!normalize_direction(direction, d)) return res;
    const float *o = origin;
    float t0 = 0.0f, T = 1.0f;
    float acc[3] = {0.0f, 0.0f, 0.0f};
    float depth_mode = 0.0f, peak_weight = 0.0f;
    int32_t peak_point = -1;
    uint32_t current = s->start_point;
    const float *p = m->points + 4 * (size_t)current;
    float cp[3] = {p[0], p[1], p[2]};
    float cr = read_radius(m, current);
    const int bounded = m->radii != NULL;
    uint32_t steps = 0, visited = 0;
    while (steps < s->max_steps) {
        steps += 1;
        if (T <= s->weight_threshold || t0 > s->depth) break;
        if (cells && visited < cap) cells[visited] = current;
        visited += 1;
        float best;
        const int face = find_exit_face(m, current, cp, cr, o, d, t0, s->depth, &best, s->tie_break);
        float ss, se;
        if (support_interval(bounded, o, d, cp, cr, t0, best, &ss, &se)) {
            const float dens = m->points[4 * (size_t)current + 3] * 1.0f;
            if (dens > 1e-6f) {
                const float dt = se - ss;
                const float alpha = 1.0f - bvo_expf(-dens * dt);
                const float w = T * alpha;
                if (s->eval_mode == BVO_EVAL_CONSTANT) {
                    acc[0] += w * s->constant_rgb[0];
                    acc[1] += w * s->constant_rgb[1];
                    acc[2] += w * s->constant_rgb[2];
                } else if (s->eval_mode == BVO_EVAL_SH) {
                    float c[3];
                    bvo_eval_rgb_sh(m, current, d, c, NULL);
                    acc[0] += w * c[0];
                    acc[1] += w * c[1];
                    acc[2] += w * c[2];
                }
                if (w > peak_weight) {
                    peak_weight = w;
                    depth_mode = 0.5f * (ss + se);
                    peak_point = (int32_t)current;
                }
                T *= 1.0f - alpha;
            }
        }
        if (face < 0) {
            t0 = best;
            break;
        }
        const uint32_t next = m->neighbors[m->offsets[current] + (uint32_t)face];
        const float *np = m->points + 4 * (size_t)next;
        t0 = fmaxf(t0, best);
        current = next;
        cp[0] = np[0];
        cp[1] = np[1];
        cp[2] = np[2];
        cr = read_radius(m, next);
    }
    res.rgba[0] = acc[0];
    res.rgba[1] = acc[1];
    res.rgba[2] = acc[2];
    res.rgba[3] = 1.0f - T;
    res.steps = steps;
    res.last_point = current;
    res.t_end = t0;
    res.depth_mode = depth_mode;
    res.peak_weight = peak_weight;
    res.peak_point = peak_point;
    if (cell_count) *cell_count = visited;
    return res;
}

bvo_trace_result bvo_trace_one_ray(const bvo_model *m, const float origin[3],
                                   const float direction[3], const bvo_trace_settings *s) {
    return trace_one_ray_impl(m, origin, direction, s, NULL, 0, NULL);
}

void bvo_render_walk_tb(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                        uint32_t height, uint32_t max_steps, float weight_threshold,
                        uint32_t start_point, int tie_break, float *out_rgba, uint32_t *out_steps,
                        uint32_t *cells, uint32_t cap, uint32_t *cell_count, int threads) {
    bvo_trace_settings s;
    memset(&s, 0, sizeof(s));
    s.weight_threshold = weight_threshold;
    s.max_steps = max_steps;
    s.start_point = start_point;
    s.depth = cam->depth;
    s.eval_mode = BVO_EVAL_SH;
    s.tie_break = tie_break;
    const long total = (long)width * (long)height;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
#endif
    for (long i = 0; i < total; ++i) {
        const uint32_t x = (uint32_t)(i % width), y = (uint32_t)(i / width);
        float o[3], d[3];
        bvo_camera_ray(cam, width, height, x, y, o, d);
        bvo_trace_result r = trace_one_ray_impl(m, o, d, &s, cells ? cells + (size_t)i * cap : NULL,
                                                cap, cell_count ? cell_count + i : NULL);
        memcpy(out_rgba + 4 * (size_t)i, r.rgba, 16);
        if (out_steps) out_steps[i] = r.steps;
    }
    (void)threads;
}

void bvo_render_walk(const bvo_model *m, const bvo_camera *cam, uint32_t width, uint32_t height,
                     uint32_t max_steps, float weight_threshold, uint32_t start_point,
                     float *out_rgba, uint32_t *out_steps, uint32_t *cells, uint32_t cap,
                     uint32_t *cell_count, int threads) {
    bvo_render_walk_tb(m, cam, width, height, max_steps, weight_threshold, start_point, 0,
                       out_rgba, out_steps, cells, cap, cell_count, threads);
}

/* ------------------------------------------------------------------ */
/* record_path_jacobians (trace.rs:1573-1676)                          */
/* ------------------------------------------------------------------ */
static int record_walk(const bvo_model *m, const float origin[3], const float direction[3],
                       const bvo_trace_settings *s, bvo_path_entry *out, int capacity,
                       int *truncated) {
    float d[3];
    *truncated = 0;
    if (!normalize_direction(direction, d)) return 0;
    float t0 = 0.0f;
    uint32_t current = s->start_point, previous = current;
    const float *p = m->points + 4 * (size_t)current;
    float cp[3] = {p[0], p[1], p[2]};
    float cr = read_radius(m, current);
    const int bounded = m->radii != NULL;
    int count = 0, finished = 0;
    uint32_t steps = 0;
    while (steps < s->max_steps) {
        steps += 1;
        if (t0 > s->depth) {
            finished = 1;
            break;
        }
        float best;
        const int face = find_exit_face(m, current, cp, cr, origin, d, t0, s->depth, &best, 0);
        const uint32_t next =
            face >= 0 ? m->neighbors[m->offsets[current] + (uint32_t)face] : current;
        bvo_path_entry e;
        if (path_interval_jacobian(m, origin, d, bounded, previous, current, next, t0, best, &e)) {
            if (count < capacity) out[count] = e;
            count += 1;
        }
        if (face < 0) {
            finished = 1;
            break;
        }
        t0 = fmaxf(t0, best);
        previous = current;
        current = next;
        const float *np = m->points + 4 * (size_t)next;
        cp[0] = np[0];
        cp[1] = np[1];
        cp[2] = np[2];
        cr = read_radius(m, next);
    }
    *truncated = !finished;
    return count;
}

int bvo_record_path_jacobians(const bvo_model *m, const float origin[3],
                              const float direction[3], const bvo_trace_settings *s,
                              bvo_path_entry *out, int capacity) {
    int truncated;
    return record_walk(m, origin, direction, s, out, capacity, &truncated);
}

/* Path recorder over whole images (PathRecorder::dispatch_batch,
 * path_record.rs:519-594): rows [pixel][max_steps]; status = count | bit 31
 * when the step cap stopped the walk (path_record.rs:41). */

void bvo_record_image(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                      uint32_t width, uint32_t height, uint32_t max_steps,
                      const uint32_t *start_points, uint32_t *prev, uint32_t *cell,
                      uint32_t *next, float *dt, float *jp, float *jc, float *jn,
                      uint32_t *status, int threads) {
    const long per_view = (long)width * (long)height;
    const long total = per_view * (long)n_cams;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
#endif
    {
        bvo_path_entry *buf = (bvo_path_entry *)malloc(sizeof(bvo_path_entry) * (max_steps + 1));
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (long i = 0; i < total; ++i) {
            const uint32_t v = (uint32_t)(i / per_view);
            const long pix = i % per_view;
            float o[3], d[3];
            bvo_camera_ray(&cams[v], width, height, (uint32_t)(pix % width),
                           (uint32_t)(pix / width), o, d);
            bvo_trace_settings s;
            memset(&s, 0, sizeof(s));
            s.max_steps = max_steps;
            s.start_point = start_points[v];
            s.depth = cams[v].depth;
            int truncated = 0;
            const int count = record_walk(m, o, d, &s, buf, (int)max_steps, &truncated);
            const size_t row = (size_t)i * max_steps;
            for (int k = 0; k < count && k < (int)max_steps; ++k) {
                prev[row + k] = buf[k].previous_cell;
                cell[row + k] = buf[k].cell;
                next[row + k] = buf[k].next_cell;
                dt[row + k] = buf[k].dt;
                memcpy(jp + 4 * (row + k), buf[k].dt_d_previous, 16);
                memcpy(jc + 4 * (row + k), buf[k].dt_d_current, 16);
                memcpy(jn + 4 * (row + k), buf[k].dt_d_next, 16);
            }
            status[i] = (uint32_t)(count < (int)max_steps ? count : (int)max_steps) |
                        (truncated ? 0x80000000u : 0u);
        }
        free(buf);
    }
    (void)threads;
}

/* ------------------------------------------------------------------ */
/* PowerFoam splats (trace.rs:1327-1546)                               */
/* ------------------------------------------------------------------ */
/* The Cech-row clip of one support (trace.rs:1331-1385) before the sphere
 * clip: the entry / exit plane depths and the neighbours that set them
 * (the cell itself when no plane bounds that side).  0 when the support is
 * excluded (camera within 4 r), missed, outside (0, depth) or emptied by a
 * parallel face. */
static int splat_planes(const bvo_model *m, const float o[3], const float d[3], float depth,
                        uint32_t cell, float *near_out, float *far_out, uint32_t *prev_out,
                        uint32_t *next_out) {
    const float *cpp = m->points + 4 * (size_t)cell;
    const float cur[3] = {cpp[0], cpp[1], cpp[2]};
    const float cr = read_radius(m, cell);
    const float cam[3] = {cur[0] - o[0], cur[1] - o[1], cur[2] - o[2]};
    const float excl = 4.0f * cr;
    if (dot3f(cam, cam) < excl * excl) return 0;
    float sn, sf;
    if (!sphere_jac(o, d, cur, cr, &sn, &sf, NULL, NULL)) return 0;
    if (sf <= 0.0f || sn >= depth) return 0;
    float face_near = 0.0f, face_far = depth;
    uint32_t previous = cell, next = cell;
    for (uint32_t k = m->offsets[cell]; k < m->offsets[cell + 1]; ++k) {
        const uint32_t a = m->neighbors[k];
        const float *ap = m->points + 4 * (size_t)a;
        const float ar = read_radius(m, a);
        const float n[3] = {ap[0] - cur[0], ap[1] - cur[1], ap[2] - cur[2]};
        const float dsq = fmaxf(dot3f(n, n), 1.0e-20f);
        const float shift = 0.5f + 0.5f * (cr * cr - ar * ar) / dsq;
        const float fo[3] = {cur[0] + shift * n[0], cur[1] + shift * n[1], cur[2] + shift * n[2]};
        const float rel[3] = {fo[0] - o[0], fo[1] - o[1], fo[2] - o[2]};
        const float num = dot3f(rel, n);
        const float den = dot3f(d, n);
        if (den > 1.0e-20f) {
            const float t = num / den;
            if (t < face_far) {
                face_far = t;
                next = a;
            }
        } else if (den < -1.0e-20f) {
            const float t = num / den;
            if (t > face_near) {
                face_near = t;
                previous = a;
            }
        } else if (num < 0.0f) {
            return 0;
        }
    }
    *near_out = face_near;
    *far_out = face_far;
    *prev_out = previous;
    *next_out = next;
    return 1;
}

/* powerfoam_splat_interval (trace.rs:1331-1389). */
static int powerfoam_splat_interval(const bvo_model *m, const float o[3], const float d[3],
                                    float depth, uint32_t cell, bvo_path_entry *e) {
    float face_near, face_far;
    uint32_t previous, next;
    if (!splat_planes(m, o, d, depth, cell, &face_near, &face_far, &previous, &next)) return 0;
    return path_interval_jacobian(m, o, d, 1, previous, cell, next, face_near, face_far, e);
}

static int cmp_entry(const void *a, const void *b) {
    const bvo_path_entry *x = (const bvo_path_entry *)a, *y = (const bvo_path_entry *)b;
    /* total_cmp on the entry depth, then cell index (trace.rs:1404-1408). */
    if (x->t_start < y->t_start) return -1;
    if (x->t_start > y->t_start) return 1;
    if (x->cell < y->cell) return -1;
    if (x->cell > y->cell) return 1;
    return 0;
}

static int sorted_splats(const bvo_model *m, const float o[3], const float d[3], float depth,
                         uint32_t max_steps, bvo_path_entry **out) {
    int cap = 64, count = 0;
    bvo_path_entry *buf = (bvo_path_entry *)malloc(sizeof(bvo_path_entry) * (size_t)cap);
    for (uint32_t cell = 0; cell < m->n; ++cell) {
        bvo_path_entry e;
        if (powerfoam_splat_interval(m, o, d, depth, cell, &e)) {
            if (count == cap) {
                cap *= 2;
                buf = (bvo_path_entry *)realloc(buf, sizeof(bvo_path_entry) * (size_t)cap);
            }
            buf[count++] = e;
        }
    }
    qsort(buf, (size_t)count, sizeof(bvo_path_entry), cmp_entry);
    if ((uint32_t)count > max_steps) count = (int)max_steps;
    *out = buf;
    return count;
}

int bvo_record_powerfoam_splats(const bvo_model *m, const float origin[3],
                                const float direction[3], const bvo_trace_settings *s,
                                bvo_path_entry *out, int capacity) {
    float d[3];
    if (!normalize_direction(direction, d)) return 0;
    bvo_path_entry *buf = NULL;
    const int count = sorted_splats(m, origin, d, s->depth, s->max_steps, &buf);
    for (int i = 0; i < count && i < capacity; ++i) out[i] = buf[i];
    free(buf);
    return count;
}

bvo_trace_result bvo_trace_powerfoam_splats(const bvo_model *m, const float origin[3],
                                            const float direction[3],
                                            const bvo_trace_settings *s) {
    bvo_trace_result res;
    memset(&res, 0, sizeof(res));
    res.last_point = s->start_point;
    res.peak_point = -1;
    float d[3];
    if (!normalize_direction(direction, d)) return res;
    bvo_path_entry *buf = NULL;
    const int count = sorted_splats(m, origin, d, s->depth, s->max_steps, &buf);
    float T = 1.0f, acc[3] = {0, 0, 0}, depth_mode = 0.0f, peak_weight = 0.0f, t_end = 0.0f;
    int32_t peak_point = -1;
    uint32_t steps = 0, last = s->start_point;
    for (int i = 0; i < count; ++i) {
        if (T <= s->weight_threshold) break;
        const bvo_path_entry *e = &buf[i];
        steps += 1;
        last = e->cell;
        t_end = e->t_start + e->dt;
        const float dens = m->points[4 * (size_t)e->cell + 3] * 1.0f;
        if (dens <= 1.0e-6f) continue;
        const float alpha = 1.0f - bvo_expf(-dens * e->dt);
        const float w = T * alpha;
        if (s->eval_mode == BVO_EVAL_CONSTANT) {
            acc[0] += w * s->constant_rgb[0];
            acc[1] += w * s->constant_rgb[1];
            acc[2] += w * s->constant_rgb[2];
        } else if (s->eval_mode == BVO_EVAL_SH) {
            float c[3];
            bvo_eval_rgb_sh(m, e->cell, d, c, NULL);
            acc[0] += w * c[0];
            acc[1] += w * c[1];
            acc[2] += w * c[2];
        }
        if (w > peak_weight) {
            peak_weight = w;
            depth_mode = e->t_start + 0.5f * e->dt;
            peak_point = (int32_t)e->cell;
        }
        T *= 1.0f - alpha;
    }
    free(buf);
    res.rgba[0] = acc[0];
    res.rgba[1] = acc[1];
    res.rgba[2] = acc[2];
    res.rgba[3] = 1.0f - T;
    res.steps = steps;
    res.last_point = last;
    res.t_end = t_end;
    res.depth_mode = depth_mode;
    res.peak_weight = peak_weight;
    res.peak_point = peak_point;
    return res;
}

void bvo_render_splats(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                       uint32_t height, uint32_t max_steps, float weight_threshold,
                       float *out_rgba, uint32_t *out_steps, int threads) {
    bvo_trace_settings s;
    memset(&s, 0, sizeof(s));
    s.weight_threshold = weight_threshold;
    s.max_steps = max_steps;
    s.depth = cam->depth;
    s.eval_mode = BVO_EVAL_SH;
    const long total = (long)width * (long)height;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (long i = 0; i < total; ++i) {
        const uint32_t x = (uint32_t)(i % width), y = (uint32_t)(i / width);
        float o[3], d[3];
        bvo_camera_ray(cam, width, height, x, y, o, d);
        bvo_trace_result r = bvo_trace_powerfoam_splats(m, o, d, &s);
        memcpy(out_rgba + 4 * (size_t)i, r.rgba, 16);
        if (out_steps) out_steps[i] = r.steps;
    }
    (void)threads;
}

/* bvo_render_splats over a list of pixel indices (y * width + x) only:
 * out_rgba [n_px * 4], out_steps [n_px]. */
void bvo_render_splats_px(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                          uint32_t height, uint32_t max_steps, float weight_threshold,
                          uint32_t n_px, const uint32_t *px, float *out_rgba,
                          uint32_t *out_steps, int threads) {
    bvo_trace_settings s;
    memset(&s, 0, sizeof(s));
    s.weight_threshold = weight_threshold;
    s.max_steps = max_steps;
    s.depth = cam->depth;
    s.eval_mode = BVO_EVAL_SH;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (long k = 0; k < (long)n_px; ++k) {
        const uint32_t x = px[k] % width, y = px[k] / width;
        float o[3], d[3];
        bvo_camera_ray(cam, width, height, x, y, o, d);
        bvo_trace_result r = bvo_trace_powerfoam_splats(m, o, d, &s);
        memcpy(out_rgba + 4 * (size_t)k, r.rgba, 16);
        if (out_steps) out_steps[k] = r.steps;
    }
    (void)threads;
}

/* ------------------------------------------------------------------ */
/* start cell                                                          */
/* ------------------------------------------------------------------ */
/* Exact power-nearest site in FP64, ties to the lowest index; the FP32
 * restatement of lib.rs:526-541 is bvo_containing_cell_f32 below. */
uint32_t bvo_containing_cell_f64(const bvo_model *m, const float position[3]) {
    uint32_t best = 0;
    double best_d = INFINITY;
    for (uint32_t i = 0; i < m->n; ++i) {
        const float *p = m->points + 4 * (size_t)i;
        const double dx = (double)position[0] - (double)p[0];
        const double dy = (double)position[1] - (double)p[1];
        const double dz = (double)position[2] - (double)p[2];
        const double r = m->radii ? (double)m->radii[i] : 0.0;
        const double dist = (dx * dx + dy * dy + dz * dz) - r * r;
        if (dist < best_d) {
            best_d = dist;
            best = i;
        }
    }
    return best;
}

uint32_t bvo_containing_cell_f32(const bvo_model *m, const float position[3]) {
    uint32_t best = 0;
    float best_d = INFINITY;
    for (uint32_t i = 0; i < m->n; ++i) {
        const float *p = m->points + 4 * (size_t)i;
        const float dv[3] = {position[0] - p[0], position[1] - p[1], position[2] - p[2]};
        const float r = read_radius(m, i);
        const float dist = dot3f(dv, dv) - r * r;
        if (dist < best_d) {
            best_d = dist;
            best = i;
        }
    }
    return best;
}

/* ------------------------------------------------------------------ */
/* gradient oracle                                                     */
/* ------------------------------------------------------------------ */
enum { ROLE_FIXED = 0, ROLE_FACE = 1, ROLE_SPHERE = 2 };

typedef struct {
    uint32_t prev, cell, next;
    uint8_t start_role, end_role;
    float start32, end32; /* the FP32 walk's interval */
    float jp32[4], jc32[4], jn32[4]; /* its FP32 dt Jacobians (the recorder's) */
} seg_t;

/* Recorded walk of the training contract: record_path_jacobians' loop
 * (trace.rs:1573-1676) with the FP32 transmittance cut of trace_one_ray
 * (trace.rs:1724) evaluated on dt clamped to max_dt (diff_render.rs:2484).
 * Identical, operation for operation, to the device fwd+bwd walk. */
static inline void two_sum_f(float a, float b, float *s, float *e) {
    *s = a + b;
    const float bb = *s - a;
    *e = (a - (*s - bb)) + (b - bb);
}

static int record_training_walk(const bvo_model *m, const float o[3], const float d[3],
                                uint32_t start, uint32_t max_steps, float depth, float thr,
                                float max_dt, seg_t *segs, float rgb32[3]) {
    float ch[3] = {0.0f, 0.0f, 0.0f}, cl[3] = {0.0f, 0.0f, 0.0f};
    float t0 = 0.0f, T = 1.0f;
    uint32_t current = start, previous = start;
    const float *p = m->points + 4 * (size_t)current;
    float cp[3] = {p[0], p[1], p[2]};
    float cr = read_radius(m, current);
    const int bounded = m->radii != NULL;
    int count = 0;
    uint32_t steps = 0;
    while (steps < max_steps) {
        steps += 1;
        if (T <= thr || t0 > depth) break;
        float best;
        const int face = find_exit_face(m, current, cp, cr, o, d, t0, depth, &best, 0);
        const uint32_t next =
            face >= 0 ? m->neighbors[m->offsets[current] + (uint32_t)face] : current;
        float start_t = t0, end_t = best;
        uint8_t srole = previous != current ? ROLE_FACE : ROLE_FIXED;
        uint8_t erole = next != current ? ROLE_FACE : ROLE_FIXED;
        int ok = 1;
        if (bounded) {
            float sn, sf;
            if (!sphere_jac(o, d, cp, cr, &sn, &sf, NULL, NULL)) {
                ok = 0;
            } else {
                if (sn > start_t) {
                    start_t = sn;
                    srole = ROLE_SPHERE;
                }
                if (sf < end_t) {
                    end_t = sf;
                    erole = ROLE_SPHERE;
                }
            }
        }
        if (ok && end_t > start_t && isfinite(start_t) && isfinite(end_t)) {
            seg_t sg = {previous, current, next, srole, erole, start_t, end_t,
                        {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
            bvo_path_entry e;
            if (path_interval_jacobian(m, o, d, bounded, previous, current, next, t0, best, &e)) {
                memcpy(sg.jp32, e.dt_d_previous, 16);
                memcpy(sg.jc32, e.dt_d_current, 16);
                memcpy(sg.jn32, e.dt_d_next, 16);
            }
            segs[count++] = sg;
            const float dens = m->points[4 * (size_t)current + 3];
            if (dens > 1e-6f) {
                const float dt = fminf(end_t - start_t, max_dt);
                const float alpha = 1.0f - bvo_expf(-dens * dt);
                const float w = T * alpha;
                float c[3];
                bvo_eval_rgb_sh(m, current, d, c, NULL);
                for (int ch_i = 0; ch_i < 3; ++ch_i) {
                    float sum, err;
                    two_sum_f(ch[ch_i], w * c[ch_i], &sum, &err);
                    ch[ch_i] = sum;
                    cl[ch_i] = cl[ch_i] + err;
                }
                T = T * (1.0f - alpha);
            }
        }
        if (face < 0) break;
        t0 = fmaxf(t0, best);
        previous = current;
        current = next;
        const float *np = m->points + 4 * (size_t)next;
        cp[0] = np[0];
        cp[1] = np[1];
        cp[2] = np[2];
        cr = read_radius(m, next);
    }
    for (int i = 0; i < 3; ++i) rgb32[i] = ch[i] + cl[i];
    return count;
}

/* Recorded PowerFoam splats of the training contract: the sorted intervals
 * of record_powerfoam_splats_jacobians (trace.rs:1421-1452), truncated to
 * max_steps, integrated like the walk (dt clamped to max_dt, the FP32
 * transmittance cut).  Each segment carries the entry / exit neighbours and
 * roles that path_interval_jacobian differentiates.  Identical, operation
 * for operation, to the device splat fwd+bwd. */
static int record_training_splats(const bvo_model *m, const float o[3], const float d[3],
                                  uint32_t max_steps, float depth, float thr, float max_dt,
                                  seg_t *segs, float rgb32[3]) {
    float ch[3] = {0.0f, 0.0f, 0.0f}, cl[3] = {0.0f, 0.0f, 0.0f};
    float T = 1.0f;
    bvo_path_entry *ents = NULL;
    const int n = sorted_splats(m, o, d, depth, max_steps, &ents);
    int count = 0;
    for (int k = 0; k < n; ++k) {
        if (T <= thr) break;
        const uint32_t cell = ents[k].cell;
        float face_near, face_far;
        uint32_t previous, next;
        splat_planes(m, o, d, depth, cell, &face_near, &face_far, &previous, &next);
        const float *cpp = m->points + 4 * (size_t)cell;
        const float cp[3] = {cpp[0], cpp[1], cpp[2]};
        float sn, sf;
        sphere_jac(o, d, cp, read_radius(m, cell), &sn, &sf, NULL, NULL);
        float start_t = face_near, end_t = face_far;
        uint8_t srole = previous != cell ? ROLE_FACE : ROLE_FIXED;
        uint8_t erole = next != cell ? ROLE_FACE : ROLE_FIXED;
        if (sn > start_t) {
            start_t = sn;
            srole = ROLE_SPHERE;
        }
        if (sf < end_t) {
            end_t = sf;
            erole = ROLE_SPHERE;
        }
        seg_t sg = {previous, cell, next, srole, erole, start_t, end_t,
                    {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
        memcpy(sg.jp32, ents[k].dt_d_previous, 16);
        memcpy(sg.jc32, ents[k].dt_d_current, 16);
        memcpy(sg.jn32, ents[k].dt_d_next, 16);
        segs[count++] = sg;
        const float dens = m->points[4 * (size_t)cell + 3];
        if (dens > 1e-6f) {
            const float dt = fminf(end_t - start_t, max_dt);
            const float alpha = 1.0f - bvo_expf(-dens * dt);
            const float w = T * alpha;
            float c[3];
            bvo_eval_rgb_sh(m, cell, d, c, NULL);
            for (int ch_i = 0; ch_i < 3; ++ch_i) {
                float sum, err;
                two_sum_f(ch[ch_i], w * c[ch_i], &sum, &err);
                ch[ch_i] = sum;
                cl[ch_i] = cl[ch_i] + err;
            }
            T = T * (1.0f - alpha);
        }
    }
    free(ents);
    for (int i = 0; i < 3; ++i) rgb32[i] = ch[i] + cl[i];
    return count;
}

typedef struct {
    const double *pts; /* [n*4] */
    const double *sh;  /* [n*3K] */
    const double *rad; /* [n] or NULL */
} dparams;

static inline double drad(const dparams *P, uint32_t i) { return P->rad ? P->rad[i] : 0.0; }

/* Radical-plane hit t of face (c -> a) and its Jacobian (trace.rs:1077). */
static double face_t_d(const dparams *P, const double o[3], const double d[3], uint32_t c,
                       uint32_t a, double jc[4], double ja[4]) {
    const double *cp = P->pts + 4 * (size_t)c, *ap = P->pts + 4 * (size_t)a;
    const double rc = drad(P, c), ra = drad(P, a);
    const double n[3] = {ap[0] - cp[0], ap[1] - cp[1], ap[2] - cp[2]};
    double dsq = dot3d(n, n);
    if (dsq < 1e-20) dsq = 1e-20;
    const double shift = 0.5 + 0.5 * (rc * rc - ra * ra) / dsq;
    const double rel[3] = {cp[0] + shift * n[0] - o[0], cp[1] + shift * n[1] - o[1],
                           cp[2] + shift * n[2] - o[2]};
    const double den = dot3d(n, d);
    const double t = dot3d(rel, n) / den;
    if (fabs(den) <= 1e-20) {
        memset(jc, 0, 32);
        memset(ja, 0, 32);
        return t;
    }
    for (int i = 0; i < 3; ++i) {
        jc[i] = (o[i] - cp[i] + t * d[i]) / den;
        ja[i] = (ap[i] - o[i] - t * d[i]) / den;
    }
    jc[3] = rc / den;
    ja[3] = -ra / den;
    return t;
}

static int sphere_t_d(const dparams *P, const double o[3], const double d[3], uint32_t c,
                      int far_side, double *t, double j[4]) {
    const double *cp = P->pts + 4 * (size_t)c;
    const double r = drad(P, c);
    const double oc[3] = {o[0] - cp[0], o[1] - cp[1], o[2] - cp[2]};
    const double b = dot3d(oc, d);
    const double disc = b * b - (dot3d(oc, oc) - r * r);
    if (disc <= 0.0) return 0;
    const double root = sqrt(disc);
    const double sgn = far_side ? 1.0 : -1.0;
    *t = -b + sgn * root;
    for (int i = 0; i < 3; ++i) j[i] = d[i] + sgn * (oc[i] - b * d[i]) / root;
    j[3] = sgn * r / root;
    return 1;
}

typedef struct {
    double dt_raw, dt, sigma, alpha, T, w;
    double c[3], cu[3];
    double csum[3]; /* 0.5 + sum_m |Y_m coef_m|: the magnitude the FP32 SH sum rounds */
    double Et;      /* error budget of T at this segment (units of 2^-24) */
    double j_prev[4], j_cur[4], j_next[4];
} seg_eval_t;

static void eval_segment(const dparams *P, uint32_t K, const double o[3], const double d[3],
                         const double Y[16], const double Ymag[16], const seg_t *sg, double depth,
                         int use_f32_interval, seg_eval_t *ev) {
    memset(ev, 0, sizeof(*ev));
    double t_start = 0.0, t_end = 0.0;
    double jc[4], ja[4];
    /* start boundary */
    if (sg->start_role == ROLE_FACE) {
        t_start = face_t_d(P, o, d, sg->cell, sg->prev, jc, ja);
        for (int i = 0; i < 4; ++i) {
            ev->j_cur[i] -= jc[i];
            ev->j_prev[i] -= ja[i];
        }
    } else if (sg->start_role == ROLE_SPHERE) {
        double j[4];
        sphere_t_d(P, o, d, sg->cell, 0, &t_start, j);
        for (int i = 0; i < 4; ++i) ev->j_cur[i] -= j[i];
    } else {
        t_start = 0.0;
    }
    /* end boundary */
    if (sg->end_role == ROLE_FACE) {
        t_end = face_t_d(P, o, d, sg->cell, sg->next, jc, ja);
        for (int i = 0; i < 4; ++i) {
            ev->j_cur[i] += jc[i];
            ev->j_next[i] += ja[i];
        }
    } else if (sg->end_role == ROLE_SPHERE) {
        double j[4];
        sphere_t_d(P, o, d, sg->cell, 1, &t_end, j);
        for (int i = 0; i < 4; ++i) ev->j_cur[i] += j[i];
    } else {
        t_end = depth; /* no exit face: the fixed far plane */
    }
    ev->dt_raw = t_end - t_start;
    /* Without perturbed parameters the segment length is the FP32 walk's own
     * (what the device integrates and differentiates); the Jacobians above
     * are evaluated in FP64 at the same geometry. */
    if (use_f32_interval) {
        ev->dt_raw = (double)sg->end32 - (double)sg->start32;
        for (int i = 0; i < 4; ++i) {
            ev->j_prev[i] = sg->jp32[i];
            ev->j_cur[i] = sg->jc32[i];
            ev->j_next[i] = sg->jn32[i];
        }
    }
    const double *c = P->sh + (size_t)sg->cell * 3u * K;
    for (int ch = 0; ch < 3; ++ch) {
        double acc = 0.0, mag = 0.5;
        for (uint32_t k = 0; k < K; ++k) {
            acc += Y[k] * c[3 * k + ch];
            mag += Ymag[k] * fabs(c[3 * k + ch]);
        }
        ev->cu[ch] = 0.5 + acc;
        ev->c[ch] = ev->cu[ch] > 0.0 ? ev->cu[ch] : 0.0;
        ev->csum[ch] = mag;
    }
    ev->sigma = P->pts[4 * (size_t)sg->cell + 3];
}

static inline void atomic_add_d(double *p, double v) {
#ifdef _OPENMP
#pragma omp atomic update
#endif
    *p += v;
}

/* Per-entry FP32 error budget of one segment's gradient contributions (the
 * magnitudes that the device's FP32 evaluation and FP32 scatter round), in
 * units of 2^-24, added to the mass tables; also advances the suffix budget
 * Se past this segment.  First-order bounds: each product and sum carries one
 * relative rounding of its operands' magnitudes, 1 - alpha carries one
 * rounding of 1, and an error budget propagates through every factor. */
static void add_mass(const bvo_grad_mass *mass, const seg_eval_t *ev, const seg_t *sg,
                     uint32_t cell, uint32_t K, const double Y[16], const double Ymag[16],
                     const double g[3],
                     const double ge[3], const double S[3], double Se[3], double gs, double Tn,
                     float max_dt, int want_pos, int want_radius, double u32) {
    const double Etn = ev->Et * (1.0 - ev->alpha) + ev->T + Tn; /* budget of T_{k+1} */
    double egs = 0.0;
    for (int ch = 0; ch < 3; ++ch) {
        const double D = Tn * ev->c[ch] - S[ch];
        const double eD = (Etn + Tn) * ev->c[ch] + Tn * ev->csum[ch] + Se[ch] + fabs(S[ch]);
        egs += ge[ch] * fabs(D) + fabs(g[ch]) * eD;
    }
    if (mass->density) atomic_add_d(&mass->density[cell], ev->dt * egs + fabs(ev->dt * gs));
    if (mass->count_density) atomic_add_d(&mass->count_density[cell], 1.0);
    const double ew = ev->Et * ev->alpha + ev->T + ev->w; /* budget of w = T alpha */
    if (mass->sh) {
        for (int ch = 0; ch < 3; ++ch) {
            /* a colour within its FP32 rounding of 0 may clamp either way:
             * then the whole term may be present on one side and absent on
             * the other, an error of the term itself (|term| / 2^-24 in these
             * units) */
            const int near0 = fabs(ev->cu[ch]) <= 64.0 * u32 * ev->csum[ch];
            if (!(ev->cu[ch] > 0.0 || near0)) continue;
            for (uint32_t mm = 0; mm < K; ++mm) {
                const double term = fabs(g[ch] * ev->w * Y[mm]);
                const double v = (ge[ch] * ev->w + fabs(g[ch]) * ew) * fabs(Y[mm]) +
                                 fabs(g[ch]) * ev->w * Ymag[mm] + (near0 ? term / u32 : term);
                atomic_add_d(&mass->sh[(size_t)cell * 3 * K + 3 * mm + ch], v);
                if (mass->count_sh) atomic_add_d(&mass->count_sh[(size_t)cell * 3 * K + 3 * mm + ch], 1.0);
            }
        }
    }
    const int dt_active = ev->dt_raw > 0.0 && ev->dt_raw < (double)max_dt;
    if (dt_active && (want_pos || want_radius)) {
        const uint32_t who[3] = {sg->prev, cell, sg->next};
        const double *js[3] = {ev->j_prev, ev->j_cur, ev->j_next};
        const double gdt = ev->sigma * gs, egdt = ev->sigma * egs + fabs(gdt);
        for (int r = 0; r < 3; ++r) {
            if (want_pos && mass->pos) {
                for (int a = 0; a < 3; ++a) {
                    if (js[r][a] == 0.0) continue;
                    atomic_add_d(&mass->pos[3 * (size_t)who[r] + a], egdt * fabs(js[r][a]));
                    if (mass->count_pos) atomic_add_d(&mass->count_pos[3 * (size_t)who[r] + a], 1.0);
                }
            }
            if (want_radius && mass->radius && js[r][3] != 0.0) {
                atomic_add_d(&mass->radius[who[r]], egdt * fabs(js[r][3]));
                if (mass->count_radius) atomic_add_d(&mass->count_radius[who[r]], 1.0);
            }
        }
    }
    for (int ch = 0; ch < 3; ++ch) Se[ch] += ew * ev->c[ch] + ev->w * ev->csum[ch];
}

double bvo_forward_backward(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                            uint32_t width, uint32_t height, uint32_t max_steps,
                            float weight_threshold, float max_dt, const float *target,
                            int loss_kind, const bvo_params_f64 *override_params,
                            double *out_rgb, float *out_rgb32, double *d_density, double *d_sh,
                            double *d_pos, double *d_radius, int threads) {
    return bvo_forward_backward_ex(m, cams, n_cams, width, height, max_steps, weight_threshold,
                                   max_dt, target, loss_kind, override_params, out_rgb,
                                   out_rgb32, d_density, d_sh, d_pos, d_radius, threads, 0);
}

double bvo_forward_backward_ex(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                               uint32_t width, uint32_t height, uint32_t max_steps,
                               float weight_threshold, float max_dt, const float *target,
                               int loss_kind, const bvo_params_f64 *override_params,
                               double *out_rgb, float *out_rgb32, double *d_density,
                               double *d_sh, double *d_pos, double *d_radius, int threads,
                               int splats) {
    return bvo_forward_backward_mx(m, cams, n_cams, width, height, max_steps, weight_threshold,
                                   max_dt, target, loss_kind, override_params, out_rgb,
                                   out_rgb32, d_density, d_sh, d_pos, d_radius, threads, splats,
                                   NULL, NULL);
}

double bvo_forward_backward_mx(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                               uint32_t width, uint32_t height, uint32_t max_steps,
                               float weight_threshold, float max_dt, const float *target,
                               int loss_kind, const bvo_params_f64 *override_params,
                               double *out_rgb, float *out_rgb32, double *d_density,
                               double *d_sh, double *d_pos, double *d_radius, int threads,
                               int splats, const uint8_t *ray_mask, const bvo_grad_mass *mass) {
    const double u32 = 5.9604644775390625e-08; /* 2^-24 */
    const uint32_t deg = m->sh_degree > 3 ? 3 : m->sh_degree;
    const uint32_t K = sh_comps(deg);
    /* FP64 parameter view */
    double *own_pts = NULL, *own_sh = NULL, *own_rad = NULL;
    dparams P;
    if (override_params) {
        P.pts = override_params->points;
        P.sh = override_params->sh;
        P.rad = override_params->radii;
    } else {
        own_pts = (double *)malloc(sizeof(double) * 4 * (size_t)m->n);
        own_sh = (double *)malloc(sizeof(double) * 3 * K * (size_t)m->n);
        for (size_t i = 0; i < 4 * (size_t)m->n; ++i) own_pts[i] = m->points[i];
        for (size_t i = 0; i < 3 * (size_t)K * m->n; ++i) own_sh[i] = m->sh[i];
        if (m->radii) {
            own_rad = (double *)malloc(sizeof(double) * (size_t)m->n);
            for (size_t i = 0; i < m->n; ++i) own_rad[i] = m->radii[i];
        }
        P.pts = own_pts;
        P.sh = own_sh;
        P.rad = own_rad;
    }
    const long per_view = (long)width * (long)height;
    const long total = per_view * (long)n_cams;
    const double M = 3.0 * (double)total;
    double loss = 0.0;
    uint32_t *starts = (uint32_t *)malloc(sizeof(uint32_t) * n_cams);
    for (uint32_t v = 0; v < n_cams; ++v) starts[v] = bvo_containing_cell_f64(m, cams[v].position);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
#endif
    {
        seg_t *segs = (seg_t *)malloc(sizeof(seg_t) * (max_steps + 1));
        seg_eval_t *evs = (seg_eval_t *)malloc(sizeof(seg_eval_t) * (max_steps + 1));
        double local_loss = 0.0;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 32)
#endif
        for (long i = 0; i < total; ++i) {
            if (ray_mask && !ray_mask[i]) continue;
            const uint32_t v = (uint32_t)(i / per_view);
            const long pix = i % per_view;
            const uint32_t x = (uint32_t)(pix % width), y = (uint32_t)(pix / width);
            float of[3], df[3], dn[3];
            bvo_camera_ray(&cams[v], width, height, x, y, of, df);
            double C[3] = {0, 0, 0};
            int nseg = 0;
            double o[3] = {of[0], of[1], of[2]}, d[3] = {0, 0, 0}, Y[16];
            float rgb32[3] = {0.0f, 0.0f, 0.0f};
            if (normalize_direction(df, dn)) {
                d[0] = dn[0];
                d[1] = dn[1];
                d[2] = dn[2];
                nseg = splats ? record_training_splats(m, of, dn, max_steps, cams[v].depth,
                                                       weight_threshold, max_dt, segs, rgb32)
                              : record_training_walk(m, of, dn, starts[v], max_steps,
                                                     cams[v].depth, weight_threshold, max_dt,
                                                     segs, rgb32);
            }
            if (out_rgb32)
                for (int ch = 0; ch < 3; ++ch) out_rgb32[3 * (size_t)i + ch] = rgb32[ch];
            sh_basis_d(deg, d, Y);
            double Ymag[16];
            sh_basis_mag_d(deg, d, Ymag);
            double T = 1.0;
            /* FP32 error budget of the device's forward, in units of 2^-24:
             * Et bounds |T32 - T| before segment k (each 1 - alpha carries
             * one rounding of 1, each product one relative rounding), Cerr
             * bounds the colour's error. */
            double Et = 0.0, Cerr[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < nseg; ++k) {
                seg_eval_t *ev = &evs[k];
                eval_segment(&P, K, o, d, Y, Ymag, &segs[k], (double)cams[v].depth,
                             override_params == NULL, ev);
                double dt = ev->dt_raw;
                if (dt < 0.0) dt = 0.0;
                if (dt > (double)max_dt) dt = (double)max_dt;
                ev->dt = dt;
                ev->T = T;
                if (ev->sigma > 1e-6) {
                    ev->alpha = 1.0 - exp(-ev->sigma * dt);
                    ev->w = T * ev->alpha;
                    for (int ch = 0; ch < 3; ++ch) C[ch] += ev->w * ev->c[ch];
                    if (mass) {
                        ev->Et = Et;
                        const double ew = Et * ev->alpha + T + ev->w;
                        for (int ch = 0; ch < 3; ++ch) Cerr[ch] += ew * ev->c[ch] + ev->w * ev->csum[ch];
                        Et = Et * (1.0 - ev->alpha) + T + T * (1.0 - ev->alpha);
                    }
                    T *= 1.0 - ev->alpha;
                } else {
                    ev->alpha = 0.0;
                    ev->w = 0.0;
                }
            }
            double g[3];
            const float *tg = target ? target + 3 * (size_t)i : NULL;
            for (int ch = 0; ch < 3; ++ch) {
                const double diff = C[ch] - (tg ? (double)tg[ch] : 0.0);
                if (loss_kind == 0) {
                    local_loss += diff * diff / M;
                    g[ch] = 2.0 * diff / M;
                } else {
                    local_loss += fabs(diff) / M;
                    g[ch] = (diff > 0.0 ? 1.0 : (diff < 0.0 ? -1.0 : 0.0)) / M;
                }
                if (out_rgb) out_rgb[3 * (size_t)i + ch] = C[ch];
            }
            if (!d_density) continue;
            double S[3] = {0, 0, 0};
            /* error budgets (units of 2^-24) of dL/dC and of the suffix S */
            double ge[3], Se[3] = {0.0, 0.0, 0.0};
            for (int ch = 0; ch < 3; ++ch) {
                if (loss_kind == 0) {
                    ge[ch] = fabs(g[ch]) + 2.0 * Cerr[ch] / M;
                } else {
                    /* L1: a residual within the colour's rounding may take either sign */
                    const double diff = C[ch] - (tg ? (double)tg[ch] : 0.0);
                    ge[ch] = fabs(g[ch]) + (fabs(diff) <= 64.0 * u32 * (Cerr[ch] + fabs(C[ch]))
                                                ? 2.0 / (M * u32) : 0.0);
                }
            }
            for (int k = nseg - 1; k >= 0; --k) {
                const seg_eval_t *ev = &evs[k];
                if (ev->sigma <= 1e-6) continue;
                const double Tn = ev->T * (1.0 - ev->alpha);
                double gs = 0.0;
                for (int ch = 0; ch < 3; ++ch) gs += g[ch] * (Tn * ev->c[ch] - S[ch]);
                const uint32_t cell = segs[k].cell;
                if (mass) {
                    add_mass(mass, ev, segs + k, cell, K, Y, Ymag, g, ge, S, Se, gs, Tn, max_dt,
                             d_pos != NULL, d_radius != NULL, u32);
                }
#ifdef _OPENMP
#pragma omp atomic update
#endif
                d_density[cell] += ev->dt * gs;
                for (int ch = 0; ch < 3; ++ch) {
                    if (ev->cu[ch] > 0.0) {
                        for (uint32_t mm = 0; mm < K; ++mm) {
                            const double val = g[ch] * ev->w * Y[mm];
#ifdef _OPENMP
#pragma omp atomic update
#endif
                            d_sh[(size_t)cell * 3 * K + 3 * mm + ch] += val;
                        }
                    }
                }
                const int dt_active = ev->dt_raw > 0.0 && ev->dt_raw < (double)max_dt;
                if (dt_active && d_pos) {
                    const double gdt = ev->sigma * gs;
                    const uint32_t who[3] = {segs[k].prev, cell, segs[k].next};
                    const double *js[3] = {ev->j_prev, ev->j_cur, ev->j_next};
                    for (int r = 0; r < 3; ++r) {
                        for (int a = 0; a < 3; ++a) {
                            const double val = gdt * js[r][a];
                            if (val != 0.0) {
#ifdef _OPENMP
#pragma omp atomic update
#endif
                                d_pos[3 * (size_t)who[r] + a] += val;
                            }
                        }
                        if (d_radius && js[r][3] != 0.0) {
                            const double val = gdt * js[r][3];
#ifdef _OPENMP
#pragma omp atomic update
#endif
                            d_radius[who[r]] += val;
                        }
                    }
                }
                for (int ch = 0; ch < 3; ++ch) S[ch] += ev->w * ev->c[ch];
            }
        }
#ifdef _OPENMP
#pragma omp atomic update
#endif
        loss += local_loss;
        free(segs);
        free(evs);
    }
    free(starts);
    free(own_pts);
    free(own_sh);
    free(own_rad);
    (void)threads;
    return loss;
}

/* ------------------------------------------------------------------ */
/* relightable Gaussians (relight.wgsl kernel 2, point light)          */
/* ------------------------------------------------------------------ */

/*
 * log(x) for FP32 from the mathematics: x = m 2^e with m in [sqrt(1/2),
 * sqrt(2)), f = m - 1, s = f / (2 + f), and log(1 + f) = 2 atanh(s) written
 * as f - (f^2/2 - s (f^2/2 + R)) with R = z (2/3 + z (2/5 + ... + z 2/13)),
 * z = s^2 (the atanh series; the exact leading term f carries the result so
 * the rounding of the small correction stays below an ulp), plus e ln2 in
 * the same hi/lo split as bvo_expf.  The device evaluates the identical
 * sequence.
 */
float bvo_logf(float x) {
    if (x != x || x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (x == INFINITY) return INFINITY;
    union { float f; uint32_t u; } v = {x};
    int e = 0;
    if (v.u < 0x00800000u) { /* subnormal: scale by 2^24 */
        v.f = x * 16777216.0f;
        e = -24;
    }
    e += (int)((v.u >> 23) & 0xffu) - 127;
    v.u = (v.u & 0x007fffffu) | 0x3f800000u; /* m in [1, 2) */
    float m = v.f;
    if (m > 1.41421353816986083984375f) {
        m = m * 0.5f;
        e += 1;
    }
    const float f = m - 1.0f;
    const float s = f / (2.0f + f);
    const float z = s * s;
    float p = 0.1538461595773697f;
    p = fmaf(p, z, 0.1818181872367859f);
    p = fmaf(p, z, 0.2222222238779068f);
    p = fmaf(p, z, 0.2857142984867096f);
    p = fmaf(p, z, 0.4000000059604645f);
    p = fmaf(p, z, 0.6666666865348816f);
    const float R = z * p;
    const float hfsq = 0.5f * f * f;
    const float ef = (float)e;
    return ef * 0.693115234375f -
           ((hfsq - (s * (hfsq + R) + ef * 3.19461832987144589424133e-05f)) - f);
}

/* x^y = exp(y log x) for x >= 0. */
float bvo_powf(float x, float y) {
    if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
    return bvo_expf(y * bvo_logf(x));
}

static inline void sub3f(const float a[3], const float b[3], float o[3]) {
    o[0] = a[0] - b[0];
    o[1] = a[1] - b[1];
    o[2] = a[2] - b[2];
}

/* qrot (common.wgsl:386-390): v + q.w * t + cross(q.xyz, t), t = 2 cross(q.xyz, v) */
static void qrot_f(const float q[4], const float v[3], float out[3]) {
    const float t0 = 2.0f * (q[1] * v[2] - q[2] * v[1]);
    const float t1 = 2.0f * (q[2] * v[0] - q[0] * v[2]);
    const float t2 = 2.0f * (q[0] * v[1] - q[1] * v[0]);
    out[0] = (v[0] + q[3] * t0) + (q[1] * t2 - q[2] * t1);
    out[1] = (v[1] + q[3] * t1) + (q[2] * t0 - q[0] * t2);
    out[2] = (v[2] + q[3] * t2) + (q[0] * t1 - q[1] * t0);
}

uint32_t bvo_relight_prepare(uint32_t n, const float *points, const float *rotations,
                             const float *scales, const float *normals,
                             const uint32_t *material_indices, uint32_t *kept_index,
                             float *center, float *rotation, float *scale, float *opacity,
                             float *normal, float *radius, float *support_sq,
                             uint32_t *material) {
    uint32_t k = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const float o = points[4 * (size_t)i + 3];
        if (o <= 0.03f) continue; /* GAUSSIAN_MIN_ALPHA, gpu/relight.rs:211-213 */
        const float *s = scales + 3 * (size_t)i;
        kept_index[k] = i;
        memcpy(center + 3 * (size_t)k, points + 4 * (size_t)i, 12);
        memcpy(rotation + 4 * (size_t)k, rotations + 4 * (size_t)i, 16);
        memcpy(scale + 3 * (size_t)k, s, 12);
        opacity[k] = o;
        memcpy(normal + 3 * (size_t)k, normals + 3 * (size_t)i, 12);
        radius[k] = 3.0f * cbrtf(s[0] * s[1] * s[2]);
        support_sq[k] = 2.0f * logf(o / 0.03f);
        material[k] = material_indices[i];
        k += 1;
    }
    return k;
}

/* point_light_shade (relight.wgsl:190-261), diffuse_samples = 0. */
void bvo_point_light_shade(const bvo_point_light *L, const float position[3],
                           const float normal[3], const float view[3], const bvo_material *m,
                           float out[3]) {
    out[0] = out[1] = out[2] = 0.0f;
    float fl[3];
    sub3f(position, L->position, fl);
    const float d2 = dot3f(fl, fl);
    if (d2 <= 1.1920929e-7f) return;
    const float inv = 1.0f / sqrtf(d2);
    const float away[3] = {fl[0] * inv, fl[1] * inv, fl[2] * inv};
    float angular = 1.0f;
    if (L->exponent != 0.0f) angular = bvo_powf(fmaxf(dot3f(L->direction, away), 0.0f), L->exponent);
    const float towards[3] = {-away[0], -away[1], -away[2]};
    const float ndl = fmaxf(dot3f(normal, towards), 0.0f);
    if (ndl == 0.0f) return;
    const float a_d2 = angular / d2;
    const float rad[3] = {L->intensity[0] * a_d2, L->intensity[1] * a_d2, L->intensity[2] * a_d2};
    for (int c = 0; c < 3; ++c) out[c] = m->albedo[c] * rad[c] * ndl;
    if (m->specular_f0[0] == 0.0f && m->specular_f0[1] == 0.0f && m->specular_f0[2] == 0.0f) return;
    const float ndv = fmaxf(dot3f(normal, view), 0.0f);
    const float hs[3] = {towards[0] + view[0], towards[1] + view[1], towards[2] + view[2]};
    const float hs2 = dot3f(hs, hs);
    if (ndv == 0.0f || hs2 <= 1.1920929e-7f) return;
    const float hinv = 1.0f / sqrtf(hs2);
    const float h[3] = {hs[0] * hinv, hs[1] * hinv, hs[2] * hinv};
    const float ndh = fmaxf(dot3f(normal, h), 0.0f);
    const float vdh = fminf(fmaxf(dot3f(view, h), 0.0f), 1.0f);
    const float rc = fminf(fmaxf(m->roughness, 0.045f), 1.0f);
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
    for (int c = 0; c < 3; ++c) {
        const float fres = m->specular_f0[c] + (1.0f - m->specular_f0[c]) * grazing;
        out[c] += rad[c] * scale * fres;
    }
}

/* relight.rs:204-323: PointLight::sample + point_light_specular +
 * shade_point_light (the reference's CPU shading twin). */
void bvo_shade_point_light_cpu(const bvo_point_light *L, const float point[3],
                               const float normal_in[3], const float view_in[3],
                               const bvo_material *m, float out[3]) {
    out[0] = out[1] = out[2] = 0.0f;
    float fl[3];
    sub3f(point, L->position, fl);
    const float d2 = dot3f(fl, fl);
    if (!isfinite(d2) || d2 <= 1.1920929e-7f || !isfinite(L->exponent) || L->exponent < 0.0f)
        return;
    const float dl = sqrtf(d2);
    const float away[3] = {fl[0] / dl, fl[1] / dl, fl[2] / dl};
    float angular = 1.0f;
    if (L->exponent != 0.0f) {
        const float ln = sqrtf(dot3f(L->direction, L->direction));
        const float r = 1.0f / ln;
        if (!isfinite(r) || r <= 0.0f) return;
        const float dn[3] = {L->direction[0] * r, L->direction[1] * r, L->direction[2] * r};
        angular = powf(fmaxf(dot3f(dn, away), 0.0f), L->exponent);
    }
    const float towards[3] = {-away[0], -away[1], -away[2]};
    float rad[3];
    for (int c = 0; c < 3; ++c) rad[c] = L->intensity[c] * angular / d2;
    float cosine = 0.0f, n[3] = {0, 0, 0};
    {
        const float r = 1.0f / sqrtf(dot3f(normal_in, normal_in));
        if (isfinite(r) && r > 0.0f) {
            n[0] = normal_in[0] * r;
            n[1] = normal_in[1] * r;
            n[2] = normal_in[2] * r;
            cosine = fmaxf(dot3f(n, towards), 0.0f);
        }
    }
    for (int c = 0; c < 3; ++c) out[c] = m->albedo[c] * rad[c] * cosine;
    if (m->specular_f0[0] == 0.0f && m->specular_f0[1] == 0.0f && m->specular_f0[2] == 0.0f) return;
    const float rn = 1.0f / sqrtf(dot3f(normal_in, normal_in));
    const float rv = 1.0f / sqrtf(dot3f(view_in, view_in));
    if (!isfinite(rn) || !(rn > 0.0f) || !isfinite(rv) || !(rv > 0.0f)) return;
    const float nn[3] = {normal_in[0] * rn, normal_in[1] * rn, normal_in[2] * rn};
    const float v[3] = {view_in[0] * rv, view_in[1] * rv, view_in[2] * rv};
    const float ndl = fmaxf(dot3f(nn, towards), 0.0f);
    const float ndv = fmaxf(dot3f(nn, v), 0.0f);
    const float hs[3] = {towards[0] + v[0], towards[1] + v[1], towards[2] + v[2]};
    const float rh = 1.0f / sqrtf(dot3f(hs, hs));
    if (!isfinite(rh) || !(rh > 0.0f)) return;
    const float h[3] = {hs[0] * rh, hs[1] * rh, hs[2] * rh};
    if (ndl == 0.0f || ndv == 0.0f) return;
    const float ndh = fmaxf(dot3f(nn, h), 0.0f);
    const float vdh = fminf(fmaxf(dot3f(v, h), 0.0f), 1.0f);
    const float rc = fminf(fmaxf(m->roughness, 0.045f), 1.0f);
    const float alpha = rc * rc;
    const float a2 = alpha * alpha;
    const float den = ndh * ndh * (a2 - 1.0f) + 1.0f;
    const float pi = 3.14159265358979f;
    const float dist = a2 / fmaxf(pi * den * den, 1.17549435e-38f);
    const float sl = 2.0f * ndl / (ndl + sqrtf(a2 + (1.0f - a2) * ndl * ndl));
    const float sv = 2.0f * ndv / (ndv + sqrtf(a2 + (1.0f - a2) * ndv * ndv));
    const float g1 = 1.0f - vdh;
    const float g2 = g1 * g1;
    const float grazing = (g2 * g2) * g1;
    const float scale = pi * dist * (sl * sv) / (4.0f * ndv);
    for (int c = 0; c < 3; ++c) {
        const float fres = m->specular_f0[c] + (1.0f - m->specular_f0[c]) * grazing;
        out[c] += rad[c] * scale * fres;
    }
}

/* intersect_surfel, kernel 2 (relight.wgsl:419-441). */
int bvo_intersect_gaussian(const bvo_relight_scene *s, uint32_t i, const float o[3],
                           const float d[3], float t_end, float *t_out, float *alpha_out) {
    const float *q = s->rotation + 4 * (size_t)i;
    const float qi[4] = {-q[0], -q[1], -q[2], q[3]};
    const float *c = s->center + 3 * (size_t)i;
    const float *sc = s->scale + 3 * (size_t)i;
    float oc[3], lo[3], ld[3];
    sub3f(o, c, oc);
    qrot_f(qi, oc, lo);
    qrot_f(qi, d, ld);
    for (int k = 0; k < 3; ++k) {
        lo[k] = lo[k] / sc[k];
        ld[k] = ld[k] / sc[k];
    }
    const float t = -dot3f(lo, ld) / dot3f(ld, ld);
    if (t <= 0.0f || t >= t_end) return 0;
    const float lp[3] = {lo[0] + t * ld[0], lo[1] + t * ld[1], lo[2] + t * ld[2]};
    const float sq = dot3f(lp, lp);
    if (sq > s->support_sq[i]) return 0;
    const float response = fminf(0.999f, s->opacity[i] * bvo_expf(-0.5f * sq));
    *t_out = t;
    *alpha_out = 1.0f - bvo_powf(1.0f - response, 1.1f);
    return 1;
}

typedef struct {
    float t;
    uint32_t index;
    float alpha;
} relight_hit;

static int cmp_hit(const void *a, const void *b) {
    const relight_hit *x = (const relight_hit *)a, *y = (const relight_hit *)b;
    if (x->t < y->t) return -1;
    if (x->t > y->t) return 1;
    return (x->index > y->index) - (x->index < y->index);
}

/* trace_blended (relight.wgsl:626-744) over every hit in (t, index) order:
 * the reference's windowed traversal gives the same result for any window
 * (groups carry across windows; tests/relight_gpu_vs_cpu.rs:543-915). */
void bvo_relight_ray(const bvo_relight_scene *s, const bvo_point_light *lights,
                     uint32_t n_lights, const float o[3], const float d[3], float depth,
                     const float background[3], float rgba[4], uint32_t *hits_out) {
    relight_hit *hits = NULL;
    size_t nh = 0, cap = 0;
    for (uint32_t i = 0; i < s->n; ++i) {
        float t, a;
        if (!bvo_intersect_gaussian(s, i, o, d, depth, &t, &a)) continue;
        if (!(a > 0.0f)) continue;
        if (nh == cap) {
            cap = cap ? cap * 2 : 64;
            hits = (relight_hit *)realloc(hits, cap * sizeof(relight_hit));
        }
        hits[nh].t = t;
        hits[nh].index = i;
        hits[nh].alpha = a;
        nh += 1;
    }
    qsort(hits, nh, sizeof(relight_hit), cmp_hit);
    float radiance[3] = {0, 0, 0}, T = 1.0f;
    int active = 0;
    float limit = 0.0f, sum_c[3] = {0, 0, 0}, sum_w = 0.0f, group_T = 1.0f;
    uint32_t used = 0;
    int stopped = 0;
    for (size_t k = 0; k < nh; ++k) {
        const relight_hit *h = &hits[k];
        if (!active || h->t > limit) {
            if (active) {
                const float a_sum = fminf(1.0f, sum_w);
                const float a_union = 1.0f - group_T;
                const float alpha = a_union * (1.0f - 0.75f) + a_sum * 0.75f;
                const float wmax = fmaxf(sum_w, 1.0e-6f);
                for (int c = 0; c < 3; ++c) radiance[c] += T * (alpha * sum_c[c] / wmax);
                T *= 1.0f - alpha;
                active = 0;
                if (T <= 0.003f) {
                    stopped = 1;
                    break;
                }
            }
            active = 1;
            limit = h->t + 0.5f * s->radius[h->index];
            sum_c[0] = sum_c[1] = sum_c[2] = 0.0f;
            sum_w = 0.0f;
            group_T = 1.0f;
        }
        used += 1;
        const float point[3] = {o[0] + h->t * d[0], o[1] + h->t * d[1], o[2] + h->t * d[2]};
        const float *nrm = s->normal + 3 * (size_t)h->index;
        float n[3] = {nrm[0], nrm[1], nrm[2]};
        if (dot3f(n, d) > 0.0f) {
            n[0] = -n[0];
            n[1] = -n[1];
            n[2] = -n[2];
        }
        const float view[3] = {-d[0], -d[1], -d[2]};
        const bvo_material *mat = &s->materials[s->material[h->index]];
        float shade[3] = {0, 0, 0};
        for (uint32_t l = 0; l < n_lights; ++l) {
            float one[3];
            bvo_point_light_shade(&lights[l], point, n, view, mat, one);
            shade[0] += one[0];
            shade[1] += one[1];
            shade[2] += one[2];
        }
        for (int c = 0; c < 3; ++c) sum_c[c] += h->alpha * shade[c];
        sum_w += h->alpha;
        group_T *= 1.0f - h->alpha;
    }
    if (active && !stopped) {
        const float a_sum = fminf(1.0f, sum_w);
        const float a_union = 1.0f - group_T;
        const float alpha = a_union * (1.0f - 0.75f) + a_sum * 0.75f;
        const float wmax = fmaxf(sum_w, 1.0e-6f);
        for (int c = 0; c < 3; ++c) radiance[c] += T * (alpha * sum_c[c] / wmax);
        T *= 1.0f - alpha;
    }
    free(hits);
    for (int c = 0; c < 3; ++c) rgba[c] = radiance[c] + T * background[c];
    rgba[3] = 1.0f - T;
    if (hits_out) *hits_out = used;
}

/* trace_main (relight.wgsl:747-780): single normalisation of the ray. */
static void relight_camera_ray(const bvo_camera *cam, uint32_t width, uint32_t height,
                               uint32_t x, uint32_t y, float o[3], float d[3]) {
    bvo_camera_ray(cam, width, height, x, y, o, d);
}

void bvo_relight_render(const bvo_relight_scene *s, const bvo_point_light *lights,
                        uint32_t n_lights, const bvo_camera *cam, uint32_t width,
                        uint32_t height, const float background[3], float *out_rgba,
                        uint32_t *out_hits, int threads) {
    const long total = (long)width * (long)height;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
#endif
    for (long i = 0; i < total; ++i) {
        float o[3], d[3];
        relight_camera_ray(cam, width, height, (uint32_t)(i % width), (uint32_t)(i / width), o, d);
        bvo_relight_ray(s, lights, n_lights, o, d, cam->depth, background,
                        out_rgba + 4 * (size_t)i, out_hits ? out_hits + i : NULL);
    }
    (void)threads;
}

/* bvo_relight_render over a list of pixel indices (y * width + x) only. */
void bvo_relight_render_px(const bvo_relight_scene *s, const bvo_point_light *lights,
                           uint32_t n_lights, const bvo_camera *cam, uint32_t width,
                           uint32_t height, const float background[3], uint32_t n_px,
                           const uint32_t *px, float *out_rgba, uint32_t *out_hits, int threads) {
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (long k = 0; k < (long)n_px; ++k) {
        float o[3], d[3];
        relight_camera_ray(cam, width, height, px[k] % width, px[k] / width, o, d);
        bvo_relight_ray(s, lights, n_lights, o, d, cam->depth, background,
                        out_rgba + 4 * (size_t)k, out_hits ? out_hits + k : NULL);
    }
    (void)height;
    (void)threads;
}

/* ------------------------------------------------------------------ */
/* Gaussian ray tracing with SH colour (trace.rs:695-773)              */
/* ------------------------------------------------------------------ */

/* Maximum-response depth and alpha of particle i (trace.rs:731-747), the
 * local ray formed with qrot of the inverse rotation and a per-axis
 * division by the scale (gaussian_trace.wgsl:147-151). */
int bvo_gaussian_response(const bvo_gaussian_scene *s, uint32_t i, const float o[3],
                          const float d[3], const bvo_gaussian_settings *st, float *t_out,
                          float *alpha_out) {
    const float *q = s->rotation + 4 * (size_t)i;
    const float qi[4] = {-q[0], -q[1], -q[2], q[3]};
    const float *c = s->center + 3 * (size_t)i;
    const float *sc = s->scale + 3 * (size_t)i;
    float oc[3], lo[3], ld[3];
    sub3f(o, c, oc);
    qrot_f(qi, oc, lo);
    qrot_f(qi, d, ld);
    for (int k = 0; k < 3; ++k) {
        lo[k] = lo[k] / sc[k];
        ld[k] = ld[k] / sc[k];
    }
    const float t = -dot3f(lo, ld) / dot3f(ld, ld);
    if (!(t > st->t_start && t < st->t_end)) return 0;
    const float p[3] = {lo[0] + t * ld[0], lo[1] + t * ld[1], lo[2] + t * ld[2]};
    const float alpha = s->opacity[i] * bvo_expf(-0.5f * dot3f(p, p));
    if (!(alpha >= st->min_opacity)) return 0;
    *t_out = t;
    *alpha_out = alpha;
    return 1;
}

void bvo_trace_gaussians(const bvo_gaussian_scene *s, const float o[3], const float d[3],
                         const bvo_gaussian_settings *st, const float background[3],
                         float rgba[4], uint32_t *hits_out) {
    relight_hit *hits = NULL;
    size_t nh = 0, cap = 0;
    for (uint32_t i = 0; i < s->n; ++i) {
        float t, a;
        if (!bvo_gaussian_response(s, i, o, d, st, &t, &a)) continue;
        if (nh == cap) {
            cap = cap ? cap * 2 : 64;
            hits = (relight_hit *)realloc(hits, cap * sizeof(relight_hit));
        }
        hits[nh].t = t;
        hits[nh].index = i;
        hits[nh].alpha = a;
        nh += 1;
    }
    /* hits.sort_by(t.total_cmp, then index) (trace.rs:750): t is finite here */
    qsort(hits, nh, sizeof(relight_hit), cmp_hit);
    const bvo_model m = {NULL, NULL, s->sh, s->sh_degree, NULL, NULL, s->n};
    float radiance[3] = {0.0f, 0.0f, 0.0f}, T = 1.0f;
    uint32_t used = 0;
    for (size_t k = 0; k < nh; ++k) {
        if (T <= st->min_transmittance) break;
        float color[3], unclamped[3];
        bvo_eval_rgb_sh(&m, hits[k].index, d, color, unclamped);
        const float w = hits[k].alpha * T;
        for (int c = 0; c < 3; ++c) radiance[c] += w * color[c];
        T *= 1.0f - hits[k].alpha;
        used += 1;
    }
    free(hits);
    for (int c = 0; c < 3; ++c) rgba[c] = radiance[c] + T * background[c];
    rgba[3] = 1.0f - T;
    if (hits_out) *hits_out = used;
}

void bvo_gaussian_render(const bvo_gaussian_scene *s, const bvo_camera *cam, uint32_t width,
                         uint32_t height, float min_opacity, float min_transmittance,
                         const float background[3], float *out_rgba, uint32_t *out_hits,
                         int threads) {
    const bvo_gaussian_settings st = {min_opacity, min_transmittance, 0.0f, cam->depth};
    const long total = (long)width * (long)height;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads)
#endif
    for (long i = 0; i < total; ++i) {
        float o[3], d[3];
        relight_camera_ray(cam, width, height, (uint32_t)(i % width), (uint32_t)(i / width), o, d);
        bvo_trace_gaussians(s, o, d, &st, background, out_rgba + 4 * (size_t)i,
                            out_hits ? out_hits + i : NULL);
    }
    (void)threads;
}

/* bvo_gaussian_render over a list of pixel indices (y * width + x) only. */
void bvo_gaussian_render_px(const bvo_gaussian_scene *s, const bvo_camera *cam, uint32_t width,
                            uint32_t height, float min_opacity, float min_transmittance,
                            const float background[3], uint32_t n_px, const uint32_t *px,
                            float *out_rgba, uint32_t *out_hits, int threads) {
    const bvo_gaussian_settings st = {min_opacity, min_transmittance, 0.0f, cam->depth};
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (long k = 0; k < (long)n_px; ++k) {
        float o[3], d[3];
        relight_camera_ray(cam, width, height, px[k] % width, px[k] / width, o, d);
        bvo_trace_gaussians(s, o, d, &st, background, out_rgba + 4 * (size_t)k,
                            out_hits ? out_hits + k : NULL);
    }
    (void)height;
    (void)threads;
}

/* ------------------------------------------------------------------ */
/* FP64 accuracy oracle of the walk                                    */
/* ------------------------------------------------------------------ */

/* trace_one_ray (trace.rs:1680-1820) with every quantity in double: the
 * pixel ray (radfoam.wgsl:44-52 mapping), the exit-face search
 * (find_exit_face :170-205), the support clip (:209-238), exp and SH.  The
 * model's FP32 values are the exact inputs.  Used to state the FP32 path's
 * image error, never as the thing measured. */
static void camera_ray_d(const bvo_camera *cam, uint32_t width, uint32_t height, uint32_t x,
                         uint32_t y, double o[3], double d[3]) {
    const double tx = tan(0.5 * (double)cam->fov[0]), ty = tan(0.5 * (double)cam->fov[1]);
    const double px = ((double)x + 0.5) / (double)width, py = ((double)y + 0.5) / (double)height;
    const double v[3] = {(px * 2.0 - 1.0 - (double)cam->principal[0]) * tx,
                         (py * 2.0 - 1.0 - (double)cam->principal[1]) * ty, 1.0};
    const double q[4] = {cam->orientation[0], cam->orientation[1], cam->orientation[2],
                         cam->orientation[3]};
    const double t[3] = {2.0 * (q[1] * v[2] - q[2] * v[1]), 2.0 * (q[2] * v[0] - q[0] * v[2]),
                         2.0 * (q[0] * v[1] - q[1] * v[0])};
    const double r[3] = {v[0] + q[3] * t[0] + (q[1] * t[2] - q[2] * t[1]),
                         v[1] + q[3] * t[1] + (q[2] * t[0] - q[0] * t[2]),
                         v[2] + q[3] * t[2] + (q[0] * t[1] - q[1] * t[0])};
    const double len = sqrt(dot3d(r, r));
    for (int k = 0; k < 3; ++k) {
        d[k] = r[k] / len;
        o[k] = cam->position[k];
    }
}

static int find_exit_face_d(const bvo_model *m, uint32_t cell, const double o[3],
                            const double d[3], double t0, double depth, double *best_out) {
    const float *cpf = m->points + 4 * (size_t)cell;
    const double cp[3] = {cpf[0], cpf[1], cpf[2]};
    const double cr = m->radii ? (double)m->radii[cell] : 0.0;
    double best = depth;
    int face = -1;
    for (uint32_t k = m->offsets[cell]; k < m->offsets[cell + 1]; ++k) {
        const uint32_t j = m->neighbors[k];
        const float *np = m->points + 4 * (size_t)j;
        const double off[3] = {np[0] - cp[0], np[1] - cp[1], np[2] - cp[2]};
        double shift = 0.5;
        if (m->radii) {
            const double rj = m->radii[j];
            shift = 0.5 + 0.5 * (cr * cr - rj * rj) / fmax(dot3d(off, off), 1e-20);
        }
        const double dp = dot3d(off, d);
        if (dp > 0.0) {
            const double rel[3] = {cp[0] + shift * off[0] - o[0], cp[1] + shift * off[1] - o[1],
                                   cp[2] + shift * off[2] - o[2]};
            const double t = dot3d(rel, off) / dp;
            if (isfinite(t) && t > t0 && t < best) {
                best = t;
                face = (int)(k - m->offsets[cell]);
            }
        }
    }
    *best_out = best;
    return face;
}

static void trace_one_ray_d(const bvo_model *m, const double o[3], const double d[3],
                            uint32_t max_steps, double weight_threshold, double depth,
                            uint32_t start, double rgba[4], uint32_t *cells, uint32_t cap,
                            uint32_t *cell_count) {
    double t0 = 0.0, T = 1.0, acc[3] = {0.0, 0.0, 0.0};
    uint32_t cur = start, steps = 0, visited = 0;
    const uint32_t deg = m->sh_degree > 3 ? 3 : m->sh_degree;
    const uint32_t comps = sh_comps(deg);
    double Y[16];
    sh_basis_d(deg, d, Y);
    while (steps < max_steps) {
        steps += 1;
        if (T <= weight_threshold || t0 > depth) break;
        if (cells && visited < cap) cells[visited] = cur;
        visited += 1;
        double best;
        const int face = find_exit_face_d(m, cur, o, d, t0, depth, &best);
        double s = t0, e = best;
        int nonempty = e > s;
        if (m->radii) {
            const float *cpf = m->points + 4 * (size_t)cur;
            const double oc[3] = {o[0] - cpf[0], o[1] - cpf[1], o[2] - cpf[2]};
            const double a = dot3d(d, d), b = dot3d(oc, d);
            const double r = m->radii[cur];
            const double disc = b * b - a * (dot3d(oc, oc) - r * r);
            nonempty = 0;
            if (disc > 0.0) {
                const double root = sqrt(disc);
                s = fmax(t0, (-b - root) / a);
                e = fmin(best, (-b + root) / a);
                nonempty = e > s;
            }
        }
        const double dens = m->points[4 * (size_t)cur + 3];
        if (nonempty && dens > 1e-6) {
            const double alpha = 1.0 - exp(-dens * (e - s));
            const double w = T * alpha;
            const float *c = m->sh + (size_t)cur * 3u * comps;
            for (int ch = 0; ch < 3; ++ch) {
                double v = 0.0;
                for (uint32_t k = 0; k < comps; ++k) v += Y[k] * (double)c[3 * k + ch];
                acc[ch] += w * fmax(0.5 + v, 0.0);
            }
            T *= 1.0 - alpha;
        }
        if (face < 0) {
            t0 = best;
            break;
        }
        t0 = fmax(t0, best);
        cur = m->neighbors[m->offsets[cur] + (uint32_t)face];
    }
    rgba[0] = acc[0];
    rgba[1] = acc[1];
    rgba[2] = acc[2];
    rgba[3] = 1.0 - T;
    if (cell_count) *cell_count = visited;
}

void bvo_render_walk_f64(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                         uint32_t height, uint32_t max_steps, double weight_threshold,
                         uint32_t start_point, double *out_rgba, uint32_t *cells, uint32_t cap,
                         uint32_t *cell_count, int threads) {
    const long total = (long)width * (long)height;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
#endif
    for (long i = 0; i < total; ++i) {
        double o[3], d[3];
        camera_ray_d(cam, width, height, (uint32_t)(i % width), (uint32_t)(i / width), o, d);
        trace_one_ray_d(m, o, d, max_steps, weight_threshold, (double)cam->depth, start_point,
                        out_rgba + 4 * (size_t)i, cells ? cells + (size_t)i * cap : NULL, cap,
                        cell_count ? cell_count + i : NULL);
    }
    (void)threads;
}

/* ------------------------------------------------------------------ */
/* optimizer step (Adam), FP32                                         */
/* ------------------------------------------------------------------ */
float bvo_density_activation(float x, int kind, float beta) {
    if (kind == 1) return fmaxf(x, 0.0f);
    if (kind == 2) {
        const float bx = beta * x;
        const float sp = bx > 20.0f ? bx : bvo_logf(1.0f + bvo_expf(bx));
        return sp / beta;
    }
    return x;
}

static float density_activation_grad(float x, int kind, float beta) {
    if (kind == 1) return x > 0.0f ? 1.0f : 0.0f;
    if (kind == 2) return 1.0f / (1.0f + bvo_expf(-(beta * x)));
    return 1.0f;
}

float bvo_density_activation_inverse(float y, int kind, float beta) {
    if (kind != 2) return y;
    const float by = beta * y;
    const float x = by > 20.0f ? by : bvo_logf(fmaxf(bvo_expf(by) - 1.0f, 1e-20f));
    return x / beta;
}

typedef struct {
    float beta1, beta2, omb1, omb2, c1, c2, eps;
} adam_scalars;

static inline float adam_update(float p, float g, float *m, float *v, const adam_scalars *a,
                                float lr) {
    *m = a->beta1 * *m + a->omb1 * g;
    *v = a->beta2 * *v + a->omb2 * (g * g);
    const float mhat = *m / a->c1;
    const float vhat = *v / a->c2;
    return p - (lr * mhat) / (sqrtf(vhat) + a->eps);
}

void bvo_adam_step(bvo_adam_state *s, const bvo_adam_settings *a, uint32_t t, const float *gd,
                   const float *gsh, const float *gpos, const float *gr) {
    const adam_scalars k = {a->beta1, a->beta2, 1.0f - a->beta1, 1.0f - a->beta2,
                            (float)(1.0 - pow((double)a->beta1, (double)t)),
                            (float)(1.0 - pow((double)a->beta2, (double)t)), a->eps};
    const float beta = a->activation == 2 ? a->softplus_beta : 0.0f;
    for (uint32_t i = 0; i < s->n; ++i) {
        if (gd && a->lr_density != 0.0f) {
            const float g = gd[i] * density_activation_grad(s->x[i], a->activation, beta);
            s->x[i] = adam_update(s->x[i], g, &s->m_d[i], &s->v_d[i], &k, a->lr_density);
            s->density[i] = bvo_density_activation(s->x[i], a->activation, beta);
        }
        if (gsh)
            for (uint32_t c = 0; c < s->nsh; ++c) {
                const float lr = c < 3 ? a->lr_sh_dc : a->lr_sh_rest;
                if (lr == 0.0f) continue;
                const size_t j = (size_t)i * s->nsh + c;
                s->sh[j] = adam_update(s->sh[j], gsh[j], &s->m_sh[j], &s->v_sh[j], &k, lr);
            }
        if (gpos && a->lr_position != 0.0f)
            for (int c = 0; c < 3; ++c) {
                const size_t j = (size_t)i * 3 + c;
                s->pos[j] = adam_update(s->pos[j], gpos[j], &s->m_pos[j], &s->v_pos[j], &k,
                                        a->lr_position);
            }
        if (gr && s->radii && a->lr_radius != 0.0f)
            s->radii[i] = adam_update(s->radii[i], gr[i], &s->m_r[i], &s->v_r[i], &k, a->lr_radius);
    }
}

/* ------------------------------------------------------------------ */
/* FP64 accuracy oracles of the PowerFoam splat and the relight        */
/* ------------------------------------------------------------------ */
/* The same functions as bvo_trace_powerfoam_splats (trace.rs:1331-1546) and
 * bvo_relight_ray (relight.wgsl:419-441, :606-744, :190-261) with every
 * quantity in double and libm's exp / log / pow / cbrt: the model's FP32
 * values are the exact inputs.  Used only to state the FP32 paths' image
 * error, never as the thing measured. */

typedef struct {
    double t_start, dt;
    uint32_t cell;
} splat_d;

static int cmp_splat_d(const void *a, const void *b) {
    const splat_d *x = (const splat_d *)a, *y = (const splat_d *)b;
    if (x->t_start < y->t_start) return -1;
    if (x->t_start > y->t_start) return 1;
    return (x->cell > y->cell) - (x->cell < y->cell);
}

static void trace_splats_d(const bvo_model *m, const double o[3], const double d[3],
                           uint32_t max_steps, double thr, double depth, double rgba[4]) {
    size_t cap = 64, count = 0;
    splat_d *buf = (splat_d *)malloc(sizeof(splat_d) * cap);
    for (uint32_t cell = 0; cell < m->n; ++cell) {
        const float *cpf = m->points + 4 * (size_t)cell;
        const double cur[3] = {cpf[0], cpf[1], cpf[2]};
        const double cr = m->radii ? (double)m->radii[cell] : 0.0;
        const double cam[3] = {cur[0] - o[0], cur[1] - o[1], cur[2] - o[2]};
        if (dot3d(cam, cam) < (4.0 * cr) * (4.0 * cr)) continue;
        const double oc[3] = {o[0] - cur[0], o[1] - cur[1], o[2] - cur[2]};
        const double b = dot3d(oc, d);
        const double disc = b * b - (dot3d(oc, oc) - cr * cr);
        if (!(disc > 0.0)) continue;
        const double root = sqrt(disc);
        const double sn = -b - root, sf = -b + root;
        if (sf <= 0.0 || sn >= depth) continue;
        double face_near = 0.0, face_far = depth;
        int empty = 0;
        for (uint32_t k = m->offsets[cell]; k < m->offsets[cell + 1]; ++k) {
            const uint32_t a = m->neighbors[k];
            const float *apf = m->points + 4 * (size_t)a;
            const double ar = m->radii ? (double)m->radii[a] : 0.0;
            const double n[3] = {apf[0] - cur[0], apf[1] - cur[1], apf[2] - cur[2]};
            const double dsq = fmax(dot3d(n, n), 1e-20);
            const double shift = 0.5 + 0.5 * (cr * cr - ar * ar) / dsq;
            const double rel[3] = {cur[0] + shift * n[0] - o[0], cur[1] + shift * n[1] - o[1],
                                   cur[2] + shift * n[2] - o[2]};
            const double num = dot3d(rel, n), den = dot3d(d, n);
            if (den > 1e-20) {
                face_far = fmin(face_far, num / den);
            } else if (den < -1e-20) {
                face_near = fmax(face_near, num / den);
            } else if (num < 0.0) {
                empty = 1;
                break;
            }
        }
        if (empty) continue;
        const double start = fmax(face_near, sn), end = fmin(face_far, sf);
        if (!(end > start)) continue;
        if (count == cap) {
            cap *= 2;
            buf = (splat_d *)realloc(buf, sizeof(splat_d) * cap);
        }
        buf[count].t_start = start;
        buf[count].dt = end - start;
        buf[count].cell = cell;
        count += 1;
    }
    qsort(buf, count, sizeof(splat_d), cmp_splat_d);
    if (count > max_steps) count = max_steps;
    const uint32_t deg = m->sh_degree > 3 ? 3 : m->sh_degree;
    const uint32_t comps = sh_comps(deg);
    double Y[16];
    sh_basis_d(deg, d, Y);
    double T = 1.0, acc[3] = {0.0, 0.0, 0.0};
    for (size_t i = 0; i < count; ++i) {
        if (T <= thr) break;
        const double dens = m->points[4 * (size_t)buf[i].cell + 3];
        if (dens <= 1e-6) continue;
        const double alpha = 1.0 - exp(-dens * buf[i].dt);
        const double w = T * alpha;
        const float *c = m->sh + (size_t)buf[i].cell * 3u * comps;
        for (int ch = 0; ch < 3; ++ch) {
            double v = 0.0;
            for (uint32_t k = 0; k < comps; ++k) v += Y[k] * (double)c[3 * k + ch];
            acc[ch] += w * fmax(0.5 + v, 0.0);
        }
        T *= 1.0 - alpha;
    }
    free(buf);
    rgba[0] = acc[0];
    rgba[1] = acc[1];
    rgba[2] = acc[2];
    rgba[3] = 1.0 - T;
}

void bvo_render_splats_f64_px(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                              uint32_t height, uint32_t max_steps, double weight_threshold,
                              uint32_t n_px, const uint32_t *px, double *out_rgba, int threads) {
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (long k = 0; k < (long)n_px; ++k) {
        double o[3], d[3];
        camera_ray_d(cam, width, height, px[k] % width, px[k] / width, o, d);
        trace_splats_d(m, o, d, max_steps, weight_threshold, (double)cam->depth,
                       out_rgba + 4 * (size_t)k);
    }
    (void)threads;
}

static void qrot_d(const double q[4], const double v[3], double out[3]) {
    const double t0 = 2.0 * (q[1] * v[2] - q[2] * v[1]);
    const double t1 = 2.0 * (q[2] * v[0] - q[0] * v[2]);
    const double t2 = 2.0 * (q[0] * v[1] - q[1] * v[0]);
    out[0] = (v[0] + q[3] * t0) + (q[1] * t2 - q[2] * t1);
    out[1] = (v[1] + q[3] * t1) + (q[2] * t0 - q[0] * t2);
    out[2] = (v[2] + q[3] * t2) + (q[0] * t1 - q[1] * t0);
}

static void point_light_shade_d(const bvo_point_light *L, const double p[3], const double n[3],
                                const double view[3], const bvo_material *mt, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    const double fl[3] = {p[0] - L->position[0], p[1] - L->position[1], p[2] - L->position[2]};
    const double d2 = dot3d(fl, fl);
    if (d2 <= 1.1920929e-7) return;
    const double inv = 1.0 / sqrt(d2);
    const double away[3] = {fl[0] * inv, fl[1] * inv, fl[2] * inv};
    double angular = 1.0;
    if (L->exponent != 0.0f) {
        const double ld[3] = {L->direction[0], L->direction[1], L->direction[2]};
        angular = pow(fmax(dot3d(ld, away), 0.0), (double)L->exponent);
    }
    const double towards[3] = {-away[0], -away[1], -away[2]};
    const double ndl = fmax(dot3d(n, towards), 0.0);
    if (ndl == 0.0) return;
    double rad[3];
    for (int c = 0; c < 3; ++c) {
        rad[c] = (double)L->intensity[c] * angular / d2;
        out[c] = (double)mt->albedo[c] * rad[c] * ndl;
    }
    if (mt->specular_f0[0] == 0.0f && mt->specular_f0[1] == 0.0f && mt->specular_f0[2] == 0.0f)
        return;
    const double ndv = fmax(dot3d(n, view), 0.0);
    const double hs[3] = {towards[0] + view[0], towards[1] + view[1], towards[2] + view[2]};
    const double hs2 = dot3d(hs, hs);
    if (ndv == 0.0 || hs2 <= 1.1920929e-7) return;
    const double hinv = 1.0 / sqrt(hs2);
    const double h[3] = {hs[0] * hinv, hs[1] * hinv, hs[2] * hinv};
    const double ndh = fmax(dot3d(n, h), 0.0);
    const double vdh = fmin(fmax(dot3d(view, h), 0.0), 1.0);
    const double rc = fmin(fmax((double)mt->roughness, 0.045), 1.0);
    const double alpha = rc * rc, a2 = alpha * alpha;
    const double den = ndh * ndh * (a2 - 1.0) + 1.0;
    const double pi = 3.14159265358979323846;
    const double dist = a2 / fmax(pi * den * den, 1.1754944e-38);
    const double sl = 2.0 * ndl / (ndl + sqrt(a2 + (1.0 - a2) * ndl * ndl));
    const double sv = 2.0 * ndv / (ndv + sqrt(a2 + (1.0 - a2) * ndv * ndv));
    const double g1 = 1.0 - vdh;
    const double grazing = (g1 * g1) * (g1 * g1) * g1;
    const double scale = pi * dist * sl * sv / (4.0 * ndv);
    for (int c = 0; c < 3; ++c) {
        const double f0 = mt->specular_f0[c];
        out[c] += rad[c] * scale * (f0 + (1.0 - f0) * grazing);
    }
}

typedef struct {
    double t, alpha;
    uint32_t index;
} relight_hit_d;

static int cmp_hit_d(const void *a, const void *b) {
    const relight_hit_d *x = (const relight_hit_d *)a, *y = (const relight_hit_d *)b;
    if (x->t < y->t) return -1;
    if (x->t > y->t) return 1;
    return (x->index > y->index) - (x->index < y->index);
}

static void relight_ray_d(const bvo_relight_scene *s, const bvo_point_light *lights,
                          uint32_t n_lights, const double o[3], const double d[3], double depth,
                          const float background[3], double rgba[4]) {
    relight_hit_d *hits = NULL;
    size_t nh = 0, cap = 0;
    for (uint32_t i = 0; i < s->n; ++i) {
        const float *q = s->rotation + 4 * (size_t)i;
        const double qi[4] = {-(double)q[0], -(double)q[1], -(double)q[2], q[3]};
        const float *c = s->center + 3 * (size_t)i;
        const float *sc = s->scale + 3 * (size_t)i;
        const double oc[3] = {o[0] - c[0], o[1] - c[1], o[2] - c[2]};
        double lo[3], ld[3];
        qrot_d(qi, oc, lo);
        qrot_d(qi, d, ld);
        for (int k = 0; k < 3; ++k) {
            lo[k] /= (double)sc[k];
            ld[k] /= (double)sc[k];
        }
        const double t = -dot3d(lo, ld) / dot3d(ld, ld);
        if (t <= 0.0 || t >= depth) continue;
        const double lp[3] = {lo[0] + t * ld[0], lo[1] + t * ld[1], lo[2] + t * ld[2]};
        const double sq = dot3d(lp, lp);
        const double op = s->opacity[i];
        if (sq > 2.0 * log(op / 0.03)) continue;
        const double response = fmin(0.999, op * exp(-0.5 * sq));
        const double a = 1.0 - pow(1.0 - response, 1.1);
        if (!(a > 0.0)) continue;
        if (nh == cap) {
            cap = cap ? cap * 2 : 64;
            hits = (relight_hit_d *)realloc(hits, cap * sizeof(relight_hit_d));
        }
        hits[nh].t = t;
        hits[nh].alpha = a;
        hits[nh].index = i;
        nh += 1;
    }
    qsort(hits, nh, sizeof(relight_hit_d), cmp_hit_d);
    double radiance[3] = {0, 0, 0}, T = 1.0, limit = 0.0, sum_c[3] = {0, 0, 0}, sum_w = 0.0,
           group_T = 1.0;
    int active = 0, stopped = 0;
    for (size_t k = 0; k < nh; ++k) {
        const relight_hit_d *h = &hits[k];
        if (!active || h->t > limit) {
            if (active) {
                const double alpha = (1.0 - group_T) * 0.25 + fmin(1.0, sum_w) * 0.75;
                for (int c = 0; c < 3; ++c) radiance[c] += T * (alpha * sum_c[c] / fmax(sum_w, 1e-6));
                T *= 1.0 - alpha;
                active = 0;
                if (T <= 0.003) {
                    stopped = 1;
                    break;
                }
            }
            active = 1;
            const float *sc = s->scale + 3 * (size_t)h->index;
            limit = h->t + 0.5 * 3.0 * cbrt((double)sc[0] * (double)sc[1] * (double)sc[2]);
            sum_c[0] = sum_c[1] = sum_c[2] = 0.0;
            sum_w = 0.0;
            group_T = 1.0;
        }
        const double point[3] = {o[0] + h->t * d[0], o[1] + h->t * d[1], o[2] + h->t * d[2]};
        const float *nrm = s->normal + 3 * (size_t)h->index;
        double n[3] = {nrm[0], nrm[1], nrm[2]};
        if (dot3d(n, d) > 0.0) {
            n[0] = -n[0];
            n[1] = -n[1];
            n[2] = -n[2];
        }
        const double view[3] = {-d[0], -d[1], -d[2]};
        const bvo_material *mat = &s->materials[s->material[h->index]];
        double shade[3] = {0, 0, 0};
        for (uint32_t l = 0; l < n_lights; ++l) {
            double one[3];
            point_light_shade_d(&lights[l], point, n, view, mat, one);
            for (int c = 0; c < 3; ++c) shade[c] += one[c];
        }
        for (int c = 0; c < 3; ++c) sum_c[c] += h->alpha * shade[c];
        sum_w += h->alpha;
        group_T *= 1.0 - h->alpha;
    }
    if (active && !stopped) {
        const double alpha = (1.0 - group_T) * 0.25 + fmin(1.0, sum_w) * 0.75;
        for (int c = 0; c < 3; ++c) radiance[c] += T * (alpha * sum_c[c] / fmax(sum_w, 1e-6));
        T *= 1.0 - alpha;
    }
    free(hits);
    for (int c = 0; c < 3; ++c) rgba[c] = radiance[c] + T * (double)background[c];
    rgba[3] = 1.0 - T;
}

void bvo_relight_render_f64_px(const bvo_relight_scene *s, const bvo_point_light *lights,
                               uint32_t n_lights, const bvo_camera *cam, uint32_t width,
                               uint32_t height, const float background[3], uint32_t n_px,
                               const uint32_t *px, double *out_rgba, int threads) {
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
#endif
    for (long k = 0; k < (long)n_px; ++k) {
        double o[3], d[3];
        camera_ray_d(cam, width, height, px[k] % width, px[k] / width, o, d);
        relight_ray_d(s, lights, n_lights, o, d, (double)cam->depth, background,
                      out_rgba + 4 * (size_t)k);
    }
    (void)threads;
}
