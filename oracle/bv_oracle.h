/*
 * CPU oracle for the blade-volume ray-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against; nothing in the shipped library links or calls it.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * It restates, in plain C, the reference crate's CPU tracer
 * (blade-volume/src/trace.rs) and shading code (blade-volume/src/relight.rs,
 * blade-volume/shaders/relight.wgsl).  Every function cites the reference
 * lines it follows.  FP32 arithmetic is kept in the reference's operation
 * order and compiled with -ffp-contract=off so that no multiply-add is fused
 * behind the code's back; the few fused operations that the product kernels
 * also use are written as explicit fmaf() calls.
 *
 * Parity is pinned against the reference's own known-answer tests
 * (trace.rs tests, gpu/radfoam.rs point-index tests, relight.rs tests);
 * tests/test_oracle_golden.py replays them.  The reference itself (Rust +
 * WGSL) cannot be compiled or run on this machine.
 */
#ifndef BV_ORACLE_H
#define BV_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* PointCloudModel (blade-volume/src/lib.rs:174-239), walk subset. */
typedef struct {
    const float *points;       /* [n*4] x, y, z, density (lib.rs:176) */
    const float *radii;        /* [n] or NULL for plain RadFoam (lib.rs:195) */
    const float *sh;           /* [n*3*K], [point][component][rgb] (lib.rs:178-185) */
    uint32_t sh_degree;        /* 0..3 */
    const uint32_t *offsets;   /* CSR [n+1] */
    const uint32_t *neighbors; /* CSR [offsets[n]] */
    uint32_t n;
} bvo_model;

/* CameraParams (blade-volume/src/camera.rs:9-18), 48 bytes. */
typedef struct {
    float position[3];
    float depth;
    float orientation[4]; /* quaternion x, y, z, w */
    float fov[2];
    float principal[2];
} bvo_camera;

enum { BVO_EVAL_OPACITY = 0, BVO_EVAL_CONSTANT = 1, BVO_EVAL_SH = 2 };

/* TraceSettings (trace.rs:50-69). */
typedef struct {
    float weight_threshold;
    uint32_t max_steps;
    uint32_t start_point;
    float depth;
    int eval_mode;
    float constant_rgb[3];
    int tie_break; /* 1: FP64 re-evaluation of near-tied exit faces (render walk) */
} bvo_trace_settings;

/* TraceResult (trace.rs:71-103). peak_point = -1 for None. */
typedef struct {
    float rgba[4];
    uint32_t steps;
    uint32_t last_point;
    float t_end;
    float depth_mode;
    float peak_weight;
    int32_t peak_point;
} bvo_trace_result;

/* PathJacobianEntry (trace.rs:1021-1041), geometry subset. */
typedef struct {
    uint32_t previous_cell, cell, next_cell;
    float dt;
    float dt_d_previous[4];
    float dt_d_current[4];
    float dt_d_next[4];
    float surface_query_near;
    float surface_query_d_previous[4];
    float surface_query_d_current[4];
    float t_start; /* entry depth of the interval (splat sort key) */
} bvo_path_entry;

/* ---- arithmetic shared bit-for-bit with the CUDA kernels ---- */
float bvo_expf(float x);
float bvo_tan_half(float fov);
void bvo_camera_ray(const bvo_camera *cam, uint32_t width, uint32_t height, uint32_t x,
                    uint32_t y, float origin[3], float dir[3]);
void bvo_eval_rgb_sh(const bvo_model *m, uint32_t point, const float dir[3], float out[3],
                     float unclamped[3]);

/* support_interval (trace.rs:209-238): returns 1 and out = (start, end). */
int bvo_support_interval(int bounded, const float o[3], const float d[3], const float c[3],
                         float radius, float t0, float t1, float out[2]);

/* ---- forward walk (trace.rs:1680-1820) ---- */
bvo_trace_result bvo_trace_one_ray(const bvo_model *m, const float origin[3],
                                   const float direction[3], const bvo_trace_settings *s);

/* Image loop (blade-volume-train/src/render.rs:113-160) with the GPU ray
 * mapping (radfoam.wgsl:44-52); start_point is used as given.
 * out_rgba [h*w*4]; out_steps [h*w] may be NULL; cells [h*w*cap] (may be NULL)
 * receives the visited cell of every loop iteration, cell_count [h*w] the
 * number written (not truncated by cap). */
void bvo_render_walk(const bvo_model *m, const bvo_camera *cam, uint32_t width, uint32_t height,
                     uint32_t max_steps, float weight_threshold, uint32_t start_point,
                     float *out_rgba, uint32_t *out_steps, uint32_t *cells, uint32_t cap,
                     uint32_t *cell_count, int threads);
/* The same with the exit-face tie-break selected (0: the reference's rule). */
void bvo_render_walk_tb(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                        uint32_t height, uint32_t max_steps, float weight_threshold,
                        uint32_t start_point, int tie_break, float *out_rgba, uint32_t *out_steps,
                        uint32_t *cells, uint32_t cap, uint32_t *cell_count, int threads);

/* ---- path recorder (trace.rs:1548-1676) ---- */
int bvo_record_path_jacobians(const bvo_model *m, const float origin[3],
                              const float direction[3], const bvo_trace_settings *s,
                              bvo_path_entry *out, int capacity);

/* Path recorder over images of n_cams cameras: rows [P][max_steps] of the
 * recorded entries; jp/jc/jn are [P*max_steps*4]; status [P] = count | bit 31
 * when truncated by the step cap.  Unwritten slots are left untouched. */
void bvo_record_image(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                      uint32_t width, uint32_t height, uint32_t max_steps,
                      const uint32_t *start_points, uint32_t *prev, uint32_t *cell,
                      uint32_t *next, float *dt, float *jp, float *jc, float *jn,
                      uint32_t *status, int threads);

/* ---- PowerFoam splats (trace.rs:1327-1546) ---- */
int bvo_record_powerfoam_splats(const bvo_model *m, const float origin[3],
                                const float direction[3], const bvo_trace_settings *s,
                                bvo_path_entry *out, int capacity);
bvo_trace_result bvo_trace_powerfoam_splats(const bvo_model *m, const float origin[3],
                                            const float direction[3],
                                            const bvo_trace_settings *s);
void bvo_render_splats(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                       uint32_t height, uint32_t max_steps, float weight_threshold,
                       float *out_rgba, uint32_t *out_steps, int threads);

/* ---- start cell (lib.rs:526-541; gpu/radfoam.rs:77-112) ---- */
/* bvo_render_splats restricted to a list of pixel indices (y * width + x):
 * out_rgba [n_px * 4], out_steps [n_px] (may be NULL). */
void bvo_render_splats_px(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                          uint32_t height, uint32_t max_steps, float weight_threshold,
                          uint32_t n_px, const uint32_t *px, float *out_rgba,
                          uint32_t *out_steps, int threads);
uint32_t bvo_containing_cell_f64(const bvo_model *m, const float position[3]);
uint32_t bvo_containing_cell_f32(const bvo_model *m, const float position[3]);

/* ---- gradient oracle (FP64 over the FP32 walk's fixed path) ----
 * The training contract of blade-volume-train/src/diff_render.rs:943-1923:
 * recorded walk, dt clamped to max_dt (MAX_PATH_DT, :2510), raw = sigma*dt,
 * T = exp(-exclusive_cumsum), alpha = 1-exp(-raw), per-cell ReLU colour
 * (:2301-2303), per-pixel sum, loss over all pixel channels of the batch.
 * loss_kind 0 = L2 (mean squared error, metrics.rs:7), 1 = L1 (mean abs).
 * Gradients are accumulated (+=) into caller-zeroed FP64 tables:
 * d_density [n], d_sh [n*3K], d_pos [n*3], d_radius [n] (may be NULL).
 * Without params_override the segment lengths and their dt Jacobians are
 * those of the FP32 walk and recorder (the quantities the device integrates
 * and differentiates, as the reference's recorder hands FP32 Jacobians to
 * its graph) and everything downstream is FP64.
 * params_override: if non-NULL, [n*4] FP64 positions+density and
 * [n*3K] FP64 SH and [n] FP64 radii replace the model values and every
 * segment length is re-derived in FP64 from them (cells and boundary roles
 * stay those of the FP32 walk), which is what central finite differences on
 * a fixed path need.  out_rgb32
 * ([P*3], may be NULL) receives the FP32 colour of the walk, accumulated with
 * the same compensated (two-sum) sum the device forward kernel uses. */
typedef struct {
    const double *points; /* [n*4] */
    const double *sh;     /* [n*3K] */
    const double *radii;  /* [n] or NULL */
} bvo_params_f64;

double bvo_forward_backward(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                            uint32_t width, uint32_t height, uint32_t max_steps,
                            float weight_threshold, float max_dt, const float *target,
                            int loss_kind, const bvo_params_f64 *override_params,
                            double *out_rgb, float *out_rgb32, double *d_density, double *d_sh,
                            double *d_pos, double *d_radius, int threads);
/* splats != 0: PowerFoam splat semantics (record_powerfoam_splats_jacobians,
 * trace.rs:1421-1452) instead of the walk: the sorted support intervals of
 * every ray, truncated to max_steps, with the same integration and
 * gradients (the model must carry radii). */
double bvo_forward_backward_ex(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                               uint32_t width, uint32_t height, uint32_t max_steps,
                               float weight_threshold, float max_dt, const float *target,
                               int loss_kind, const bvo_params_f64 *override_params,
                               double *out_rgb, float *out_rgb32, double *d_density,
                               double *d_sh, double *d_pos, double *d_radius, int threads,
                               int splats);

/* Per-entry FP32 error budget of the gradient tables (test infrastructure):
 * for every gradient entry the sum, over the contributions that form it, of
 * the magnitudes that an FP32 evaluation of the same contract rounds (the
 * transmittance product, 1 - alpha, the SH sum, dL/dC through the colour,
 * the suffix, the scatter), in units of 2^-24.  An FP32 implementation of
 * the contract then differs from the FP64 gradient by at most a small
 * multiple of 2^-24 times this mass, plus the error of summing the entry's
 * terms in FP32 in any order, at most (count - 1) 2^-24 times the sum of
 * their magnitudes (which the mass bounds); count_* holds each entry's
 * number of terms.  Any table may be NULL. */
typedef struct {
    double *density; /* [n] */
    double *sh;      /* [n*3K] */
    double *pos;     /* [n*3] */
    double *radius;  /* [n] */
    double *count_density, *count_sh, *count_pos, *count_radius; /* same shapes */
} bvo_grad_mass;

/* bvo_forward_backward_ex restricted to the rays whose ray_mask byte is
 * non-zero (NULL: every ray; the loss normalisation still counts every ray
 * of the batch), optionally accumulating the error-budget tables. */
double bvo_forward_backward_mx(const bvo_model *m, const bvo_camera *cams, uint32_t n_cams,
                               uint32_t width, uint32_t height, uint32_t max_steps,
                               float weight_threshold, float max_dt, const float *target,
                               int loss_kind, const bvo_params_f64 *override_params,
                               double *out_rgb, float *out_rgb32, double *d_density,
                               double *d_sh, double *d_pos, double *d_radius, int threads,
                               int splats, const uint8_t *ray_mask, const bvo_grad_mass *mass);

/* ---- relightable Gaussians with finite point lights ----
 * blade-volume/shaders/relight.wgsl (kernel 2 = learned volumetric
 * Gaussian, point light enabled, diffuse_samples = 0) and
 * blade-volume/src/relight.rs.  Material / PointLight are the reference's
 * #[repr(C)] layouts (relight.rs:77-86, :176-181). */
typedef struct {
    float albedo[3];
    float roughness;
    float specular_f0[3];
    float pad;
} bvo_material;

typedef struct {
    float position[3];
    float direction[3];
    float intensity[3];
    float exponent;
} bvo_point_light;

/* Prepared particles (gpu/relight.rs:178-253): opacity > 0.03 only,
 * index = position in this filtered list. */
typedef struct {
    uint32_t n;
    const float *center;     /* [n*3] */
    const float *rotation;   /* [n*4] x, y, z, w */
    const float *scale;      /* [n*3] */
    const float *opacity;    /* [n] */
    const float *normal;     /* [n*3] */
    const float *radius;     /* [n] 3 * cbrt(sx sy sz) */
    const float *support_sq; /* [n] 2 * ln(opacity / 0.03) */
    const uint32_t *material;
    const bvo_material *materials;
} bvo_relight_scene;

float bvo_logf(float x);
float bvo_powf(float x, float y);
/* Fills the prepared arrays from a Gaussian PointCloudModel; returns the
 * number kept.  Output arrays must hold n entries. */
uint32_t bvo_relight_prepare(uint32_t n, const float *points, const float *rotations,
                             const float *scales, const float *normals,
                             const uint32_t *material_indices, uint32_t *kept_index,
                             float *center, float *rotation, float *scale, float *opacity,
                             float *normal, float *radius, float *support_sq,
                             uint32_t *material);
void bvo_point_light_shade(const bvo_point_light *light, const float position[3],
                           const float normal[3], const float view[3], const bvo_material *m,
                           float out[3]);
/* relight.rs shade_point_light (:295-323), CPU twin of the shader's. */
void bvo_shade_point_light_cpu(const bvo_point_light *light, const float point[3],
                               const float normal[3], const float view[3],
                               const bvo_material *m, float out[3]);
int bvo_intersect_gaussian(const bvo_relight_scene *s, uint32_t i, const float o[3],
                           const float d[3], float t_end, float *t, float *alpha);
/* One camera ray of trace_main + trace_blended: rgba = (radiance +
 * T * background, 1 - T); lights are summed (alpha is light-independent). */
void bvo_relight_ray(const bvo_relight_scene *s, const bvo_point_light *lights,
                     uint32_t n_lights, const float o[3], const float d[3], float depth,
                     const float background[3], float rgba[4], uint32_t *hits);
void bvo_relight_render(const bvo_relight_scene *s, const bvo_point_light *lights,
                        uint32_t n_lights, const bvo_camera *cam, uint32_t width,
                        uint32_t height, const float background[3], float *out_rgba,
                        uint32_t *out_hits, int threads);
/* bvo_relight_render restricted to a list of pixel indices (y * width + x). */
void bvo_relight_render_px(const bvo_relight_scene *s, const bvo_point_light *lights,
                           uint32_t n_lights, const bvo_camera *cam, uint32_t width,
                           uint32_t height, const float background[3], uint32_t n_px,
                           const uint32_t *px, float *out_rgba, uint32_t *out_hits, int threads);

/* ---- Gaussian ray tracing with SH colour (trace.rs:695-773) ----
 * Particles with opacity > min_opacity only (GaussianGpuCloud::new,
 * gpu/gaussian.rs:19-27); index = position in this filtered list, which
 * keeps the model's order.  A hit is the point of maximum response along
 * the ray: local ray R^-1 (o - mean) / scale (qrot of the inverse rotation,
 * common.wgsl:386-390, as gaussian_trace.wgsl:147-148 evaluates it),
 * t = -<o', d'> / |d'|^2 in (t_start, t_end), alpha = opacity *
 * exp(-|o' + t d'|^2 / 2) >= min_opacity; hits are composited in strict
 * (t, index) order until transmittance <= min_transmittance. */
typedef struct {
    uint32_t n;
    const float *center;   /* [n*3] */
    const float *rotation; /* [n*4] x, y, z, w */
    const float *scale;    /* [n*3] */
    const float *opacity;  /* [n] */
    const float *sh;       /* [n*3K] */
    uint32_t sh_degree;
} bvo_gaussian_scene;

typedef struct { /* GaussianTraceSettings (trace.rs:106-126) */
    float min_opacity;
    float min_transmittance;
    float t_start;
    float t_end;
} bvo_gaussian_settings;

int bvo_gaussian_response(const bvo_gaussian_scene *s, uint32_t i, const float o[3],
                          const float d[3], const bvo_gaussian_settings *st, float *t,
                          float *alpha);
/* One ray: rgba = (radiance + T * background, 1 - T); hits = composited. */
void bvo_trace_gaussians(const bvo_gaussian_scene *s, const float o[3], const float d[3],
                         const bvo_gaussian_settings *st, const float background[3],
                         float rgba[4], uint32_t *hits);
/* Image of one camera with the relight/trace_main ray mapping, t in (0, depth). */
void bvo_gaussian_render(const bvo_gaussian_scene *s, const bvo_camera *cam, uint32_t width,
                         uint32_t height, float min_opacity, float min_transmittance,
                         const float background[3], float *out_rgba, uint32_t *out_hits,
                         int threads);
/* bvo_gaussian_render restricted to a list of pixel indices (y * width + x). */
void bvo_gaussian_render_px(const bvo_gaussian_scene *s, const bvo_camera *cam, uint32_t width,
                            uint32_t height, float min_opacity, float min_transmittance,
                            const float background[3], uint32_t n_px, const uint32_t *px,
                            float *out_rgba, uint32_t *out_hits, int threads);

/* ---- FP64 accuracy oracle of the walk ----
 * trace_one_ray with every quantity in double (ray mapping, exit faces,
 * support clip, exp, SH); the FP32 model values are its exact inputs.
 * out_rgba [h*w*4] double; cells/cell_count as in bvo_render_walk. */
void bvo_render_walk_f64(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                         uint32_t height, uint32_t max_steps, double weight_threshold,
                         uint32_t start_point, double *out_rgba, uint32_t *cells, uint32_t cap,
                         uint32_t *cell_count, int threads);

/* ---- optimizer step (Adam) ----
 * Kingma & Ba's Adam with bias correction in FP32, the restatement the
 * device optimizer follows operation for operation; the density table is
 * the activation of a raw parameter (density_activation,
 * blade-volume-train/src/diff_render.rs:4649-4672): 0 identity, 1 ReLU,
 * 2 softplus(beta x)/beta.  c_i = 1 - beta_i^t in FP64, rounded once. */
typedef struct {
    float lr_density, lr_sh_dc, lr_sh_rest, lr_position, lr_radius;
    float beta1, beta2, eps;
    int activation;
    float softplus_beta;
} bvo_adam_settings;

typedef struct {
    uint32_t n, nsh;
    float *x, *m_d, *v_d;      /* [n] raw density parameter and moments */
    float *density;            /* [n] out: activation of x */
    float *sh, *m_sh, *v_sh;   /* [n*nsh] */
    float *pos, *m_pos, *v_pos; /* [n*3] */
    float *radii, *m_r, *v_r;  /* [n] or NULL */
} bvo_adam_state;

float bvo_density_activation(float x, int kind, float beta);
float bvo_density_activation_inverse(float y, int kind, float beta);
/* One step t (1-based); a NULL gradient skips its table, a zero rate freezes it. */
void bvo_adam_step(bvo_adam_state *s, const bvo_adam_settings *a, uint32_t t, const float *g_density,
                   const float *g_sh, const float *g_pos, const float *g_radii);

/* ---- FP64 accuracy oracles of the splat and the relight ----
 * bvo_render_splats_px / bvo_relight_render_px with every quantity in
 * double (libm exp, log, pow, cbrt); the FP32 model values are the exact
 * inputs.  out_rgba [n_px * 4] double. */
void bvo_render_splats_f64_px(const bvo_model *m, const bvo_camera *cam, uint32_t width,
                              uint32_t height, uint32_t max_steps, double weight_threshold,
                              uint32_t n_px, const uint32_t *px, double *out_rgba, int threads);
void bvo_relight_render_f64_px(const bvo_relight_scene *s, const bvo_point_light *lights,
                               uint32_t n_lights, const bvo_camera *cam, uint32_t width,
                               uint32_t height, const float background[3], uint32_t n_px,
                               const uint32_t *px, double *out_rgba, int threads);

#ifdef __cplusplus
}
#endif
#endif
