/*
 * blade_volume_b200 — C ABI of the B200 (sm_100a) ray-tracing hot path of
 * blade-volume: the RadFoam/PowerFoam cell walk with volumetric compositing,
 * its path recorder, and its L2/L1 gradient.
 *
 * Every entry point returns a bv_status; nothing aborts across the ABI.  All
 * pointers named *_dev are CUDA device pointers owned by the caller; host
 * pointers are read before the call returns.  A handle is not thread-safe:
 * one owner, one stream at a time (the reference serialises its GPU work the
 * same way, tests/radfoam_gpu_vs_cpu.rs:41-47).
 *
 * Reference interfaces replaced (paths relative to the blade-volume repo):
 *   RadFoamGpuTracer        blade-volume/src/gpu/radfoam_trace.rs:56-177
 *   RadFoamGpuCloud         blade-volume/src/gpu/radfoam.rs:25-49, :676
 *   PathRecorder            blade-volume/src/gpu/path_record.rs:225-595
 *   PathRecordBuffers       blade-volume/src/gpu/path_record.rs:614-1364
 *   training gradient       blade-volume-train/src/diff_render.rs:943-1923, :7181-7226
 */
#ifndef BLADE_VOLUME_B200_H
#define BLADE_VOLUME_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BV_ABI_VERSION 1u

typedef enum bv_status {
    BV_OK = 0,
    /* bad argument (null handle, zero size, ...): radfoam_trace.rs:113 asserts */
    BV_ERR_INVALID_ARGUMENT = 1,
    /* model rejected by validation: PointCloudModel::validate, lib.rs:246-483 */
    BV_ERR_INVALID_MODEL = 2,
    /* a CUDA runtime call failed; bv_last_error() has the text */
    BV_ERR_CUDA = 3,
    /* device allocation failed */
    BV_ERR_OUT_OF_MEMORY = 4,
    /* a per-ray candidate list overflowed: powerfoam_splat.rs:321 */
    BV_ERR_CANDIDATE_OVERFLOW = 5,
    /* a feature the model carries that this path does not implement */
    BV_ERR_NOT_SUPPORTED = 6,
    /* no CUDA device is available */
    BV_ERR_NO_DEVICE = 7,
    /* bv_server_wait: the request has not finished within the timeout */
    BV_ERR_TIMEOUT = 8,
    /* a serving request withdrawn by bv_server_cancel */
    BV_ERR_CANCELLED = 9,
} bv_status;

/* cudaStream_t; NULL selects the legacy default stream. */
typedef void *bv_stream;

/* CameraParams (blade-volume/src/camera.rs:9-18): 48 bytes, same layout. */
typedef struct bv_camera {
    float cam_position[3];
    float depth;
    float cam_orientation[4]; /* unit quaternion x, y, z, w */
    float fov[2];             /* local_dir = ((ndc - principal) * tan(fov / 2), 1) */
    float principal[2];
} bv_camera;

/* Store SH coefficients as BF16 on the device (FP32 arithmetic). */
#define BV_MODEL_SH_BF16 0x1u

/* PointCloudModel (blade-volume/src/lib.rs:174-239), walk subset.  The
 * arrays are the reference's own layouts, so a Rust caller passes
 * model.points.as_ptr() etc. directly. */
typedef struct bv_model_desc {
    uint32_t num_points;
    uint32_t sh_degree;                  /* 0..3 */
    const float *points;                 /* [N*4] x, y, z, density (lib.rs:176) */
    const float *sh_coefficients;        /* [N*3*K] [point][component][rgb] (lib.rs:185) */
    const float *radii;                  /* [N] PowerFoam radii, or NULL (lib.rs:195) */
    const uint32_t *adjacency_offsets;   /* CSR [N+1] */
    const uint32_t *adjacency_neighbors; /* CSR [offsets[N]] sorted, symmetric, no self */
    uint32_t flags;                      /* BV_MODEL_* */
    uint32_t reserved;
} bv_model_desc;

/* RadFoamTraceSettings (blade-volume/src/gpu/radfoam_trace.rs:4-23). */
typedef struct bv_trace_settings {
    uint32_t max_steps;                    /* default 1024 */
    uint32_t powerfoam_candidate_capacity; /* 0 = automatic */
    float weight_threshold;                /* default 0.001 */
    uint32_t debug_cell_density;           /* 1: output cells_visited/100 heat map */
} bv_trace_settings;

typedef struct bv_tracer bv_tracer;

/* Last error message of the calling thread (valid until the next call). */
const char *bv_last_error(void);
uint32_t bv_abi_version(void);

/* Host-side model validation, PointCloudModel::validate (lib.rs:246-483)
 * and validate_csr (adjacency.rs:717-790).  Needs no GPU.  On failure the
 * message (if err != NULL) names the first problem. */
bv_status bv_model_validate(const bv_model_desc *model, char *err, size_t err_len);

/* RadFoamGpuTracer::new (radfoam_trace.rs:63-104) + RadFoamGpuCloud::new
 * (radfoam.rs:119-533): validates the model, packs it into the device layout
 * and uploads it.  The tracer owns its device copy. */
bv_status bv_radfoam_tracer_new(const bv_model_desc *model, const bv_trace_settings *settings,
                                bv_tracer **out);

/* RadFoamGpuTracer::deinit (radfoam_trace.rs:173-176). */
void bv_radfoam_tracer_destroy(bv_tracer *tracer);

/* RadFoamGpuTracer::dispatch (radfoam_trace.rs:106-135).  Renders one image
 * of width x height into out_rgba_dev ([height][width][4] float32, RGB plus
 * alpha = 1 - transmittance; the reference writes an rgba16f texture).  The
 * start cell is the power-nearest site of the camera position, found on the
 * device in FP64 (radfoam.rs:77-112 uses a host kd-tree in FP32). */
bv_status bv_radfoam_tracer_dispatch(bv_tracer *tracer, float *out_rgba_dev,
                                     const bv_camera *camera, uint32_t width, uint32_t height,
                                     bv_stream stream);

/* Several cameras of one size in one launch: out is [n][height][width][4]. */
bv_status bv_radfoam_tracer_dispatch_batch(bv_tracer *tracer, float *out_rgba_dev,
                                           const bv_camera *cameras, uint32_t n_cameras,
                                           uint32_t width, uint32_t height, bv_stream stream);

/* Settings accessors (radfoam_trace.rs:137-171). */
bv_status bv_radfoam_tracer_set_max_steps(bv_tracer *tracer, uint32_t max_steps);
bv_status bv_radfoam_tracer_set_weight_threshold(bv_tracer *tracer, float weight_threshold);
bv_status bv_radfoam_tracer_set_debug_cell_density(bv_tracer *tracer, uint32_t enabled);
/* Exit-face choice of the render walk (dispatch / dispatch_batch).
 * BV_TIE_BREAK_REFERENCE (default): the first face in CSR order with the
 * smallest FP32 distance, find_exit_face (trace.rs:170-205) exactly.
 * BV_TIE_BREAK_F64: when the runner-up's FP32 distance lies within 4 ulps of
 * the winner's, both are re-evaluated in FP64 and the smaller wins (equal:
 * the earlier face).  Cell sequences then differ from the reference's only at
 * such near-ties, and follow the FP64 walk there.  No reference counterpart;
 * recording and training keep the reference's rule. */
#define BV_TIE_BREAK_REFERENCE 0u
#define BV_TIE_BREAK_F64 1u
bv_status bv_radfoam_tracer_set_tie_break(bv_tracer *tracer, uint32_t mode);
/* Training (bv_forward_backward): the forward records the exit face and the
 * unclamped SH colour of each ray's first `steps` walk steps (16 bytes per
 * ray and step, at most 8 GiB per launch of 32 views) and the replay reads
 * those instead of searching the cell's faces and evaluating its SH row
 * again; later steps are recomputed.  Default 256; 0 disables the record.
 * Results are identical for every setting.  No reference counterpart (the
 * reference records whole paths, path_record.rs:519). */
bv_status bv_radfoam_tracer_set_exit_record(bv_tracer *tracer, uint32_t steps);
uint32_t bv_radfoam_tracer_max_steps(const bv_tracer *tracer);
float bv_radfoam_tracer_weight_threshold(const bv_tracer *tracer);
uint32_t bv_radfoam_tracer_sh_degree(const bv_tracer *tracer);
/* Start cell of the last dispatch (radfoam_trace.rs:169-171); synchronises
 * the tracer's last stream. */
uint32_t bv_radfoam_tracer_start_point(bv_tracer *tracer);
uint32_t bv_radfoam_tracer_num_points(const bv_tracer *tracer);

/* RadFoamGpuCloud::containing_point (radfoam.rs:676): power-nearest site of
 * a position, FP64 on the device, ties to the lowest index.  Synchronous. */
bv_status bv_containing_point(bv_tracer *tracer, const float position[3], uint32_t *out_index);

/* ---- path recorder -------------------------------------------------------
 * PathRecordBuffers (path_record.rs:614-1364), row-major [pixels, max_steps].
 * Any stream pointer may be NULL to skip it.  Rows are written for recorded
 * steps only; path_status[p] = steps | BV_PATH_TRUNCATED (bit 31) when the
 * step cap stopped the ray (path_record.rs:41, :1248-1267). */
#define BV_PATH_TRUNCATED 0x80000000u

typedef struct bv_path_buffers {
    uint32_t *previous_cells_dev; /* [P*L] */
    uint32_t *cells_dev;          /* [P*L] */
    uint32_t *next_cells_dev;     /* [P*L] */
    float *dts_dev;               /* [P*L] */
    float *dt_grad_previous_dev;  /* [P*L*4] d dt / d (x, y, z, r) of the entry site */
    float *dt_grad_current_dev;   /* [P*L*4] of the cell's own site */
    float *dt_grad_next_dev;      /* [P*L*4] of the exit site */
    uint32_t *path_status_dev;    /* [P] */
    uint32_t max_steps;           /* L */
    uint32_t reserved;
} bv_path_buffers;

/* PathRecorder::dispatch_batch (path_record.rs:519-594) for the walk:
 * record_path_jacobians (trace.rs:1573-1676) per pixel, cameras of one size,
 * pixel p = view * height * width + y * width + x. */
bv_status bv_record_paths(bv_tracer *tracer, const bv_camera *cameras, uint32_t n_cameras,
                          uint32_t width, uint32_t height, const bv_path_buffers *buffers,
                          bv_stream stream);

/* ---- training gradient ---------------------------------------------------
 * The differentiable forward of diff_render.rs:943-1923 on the recorded walk:
 * dt clamped to max_dt (MAX_PATH_DT = 50, diff_render.rs:2510), raw =
 * sigma * dt, T = exp(-exclusive cumsum), alpha = 1 - exp(-raw), per-cell
 * ReLU colour (:2301-2303), per-pixel sum, then the loss over every channel
 * of every pixel of the batch (metrics.rs:7): L2 = mean squared error,
 * L1 = mean absolute error.  Gradients w.r.t. density, SH coefficients and
 * site positions (and radii for PowerFoam) are ADDED to the caller's tables
 * (zero them first), like the reference's scatter-add backward. */
typedef enum bv_loss { BV_LOSS_L2 = 0, BV_LOSS_L1 = 1 } bv_loss;

typedef struct bv_train_settings {
    uint32_t max_steps;     /* rows per pixel (L) */
    float weight_threshold; /* transmittance cut; 0 walks every recorded step */
    float max_dt;           /* segment clamp, 50 in the reference */
    uint32_t loss;          /* bv_loss */
} bv_train_settings;

typedef struct bv_grads {
    float *d_density_dev;   /* [N] */
    float *d_sh_dev;        /* [N*3*K], model layout */
    float *d_positions_dev; /* [N*3], or NULL to skip position gradients */
    float *d_radii_dev;     /* [N], PowerFoam only, or NULL */
} bv_grads;

/* Forward + loss + backward for a batch of cameras of one size.
 * target_rgb_dev [n][height][width][3]; loss_dev receives the scalar loss
 * (float, overwritten); rgb_out_dev (may be NULL) the rendered colours
 * [n][height][width][3].  Two walk launches: the forward kernel walks
 * every ray, forms its loss gradient dL/dC and records each step's exit face
 * and colour (the tracer's step record, up to its set number of steps per
 * ray); the replay kernel walks the same path again from that record,
 * recomputing transmittance, and scatters the parameter gradients (steps
 * past the record search and evaluate again).  Per ray, the colour and
 * dL/dC (48 bytes) pass between them.  The forward also times its 8x4
 * tiles, and two small launches order them so that the replay of the next
 * call of the same shape takes them heaviest first; the order changes no
 * result. */
bv_status bv_forward_backward(bv_tracer *tracer, const bv_camera *cameras, uint32_t n_cameras,
                              uint32_t width, uint32_t height, const float *target_rgb_dev,
                              const bv_train_settings *settings, const bv_grads *grads,
                              float *loss_dev, float *rgb_out_dev, bv_stream stream);

/* ---- optimizer step ---------------------------------------------------------
 * The trainer's Adam (meganeura, configured per parameter group by
 * configure_optimizer / radfoam_v1_lrs, blade-volume-train/src/diff_render.rs:
 * 3215-3330) over the gradient tables of bv_forward_backward, applied to the
 * tracer's own device model, so that a training loop needs no other library:
 * forward_backward -> adam_step -> forward_backward ...  Kingma & Ba's Adam
 * with bias correction in FP32.  The density table is the activation of a
 * raw parameter x (density_activation, diff_render.rs:4649-4656): identity,
 * ReLU, or softplus(beta x) / beta; x starts at the inverse activation of the
 * model's density (:4658-4672).  A table whose rate is 0 is frozen; a NULL
 * gradient pointer skips its table.  BF16 SH models keep an FP32 master copy
 * (starting at the BF16 values) and store each update rounded to BF16.  The
 * optimizer state (moments, raw density, master SH; 4 to 8 floats per
 * parameter) is allocated by the first call; its activation and beta must
 * stay the same across calls.  Position updates move sites within the
 * model's fixed adjacency (the reference rebuilds adjacency in its densify
 * schedule, outside this path). */
#define BV_DENSITY_IDENTITY 0u
#define BV_DENSITY_RELU 1u
#define BV_DENSITY_SOFTPLUS 2u

typedef struct bv_adam_settings {
    float lr_density;           /* rate of the raw density parameter */
    float lr_sh_dc;             /* SH component 0 (three DC coefficients per site) */
    float lr_sh_rest;           /* SH components 1..K-1 */
    float lr_position;          /* site positions */
    float lr_radius;            /* PowerFoam radii */
    float beta1;                /* 0.9 */
    float beta2;                /* 0.999 */
    float eps;                  /* 1e-15 in radfoam_v1 (diff_render.rs:3307) */
    uint32_t density_activation; /* BV_DENSITY_* */
    float softplus_beta;        /* beta > 0 for BV_DENSITY_SOFTPLUS */
} bv_adam_settings;

bv_status bv_radfoam_tracer_adam_step(bv_tracer *tracer, const bv_grads *grads,
                                      const bv_adam_settings *settings, bv_stream stream);
/* Optimizer steps taken so far. */
uint32_t bv_radfoam_tracer_adam_steps(const bv_tracer *tracer);

/* Reads the tracer's current device model back into host arrays in the
 * model's layout (the trainer's parameter readback, diff_render.rs:4812-4851):
 * points [N*4] (x, y, z, density), sh [N*3K], radii [N] (PowerFoam; may be
 * NULL).  Any pointer may be NULL to skip it.  Synchronises the device. */
bv_status bv_radfoam_tracer_read_model(bv_tracer *tracer, float *points, float *sh,
                                       float *radii);

/* ---- instrumentation -----------------------------------------------------
 * Device time (ms, CUDA events on the launch stream) and work counters of
 * the last dispatch / record / forward_backward call on this tracer.
 * Synchronises that stream. */
typedef struct bv_launch_stats {
    float kernel_ms;        /* traversal kernels (training: forward + replay) */
    float start_cell_ms;    /* start-cell search */
    float forward_ms;       /* training: forward + loss kernel */
    float backward_ms;      /* training: replay backward kernel */
    uint64_t rays;
    uint64_t steps;         /* walk loop iterations over all rays */
    uint64_t faces;         /* neighbour faces tested */
    uint32_t launches;      /* kernels launched by the call */
    uint32_t reserved;
} bv_launch_stats;

bv_status bv_radfoam_tracer_enable_stats(bv_tracer *tracer, uint32_t enabled);
bv_status bv_radfoam_tracer_last_stats(bv_tracer *tracer, bv_launch_stats *out);

/* ---- relightable Gaussians with finite point lights ------------------------
 * RelightTracer for learned volumetric Gaussians (gpu/relight.rs:313
 * new_gaussian, :841 set_point_light, :893 set_background, :905 dispatch;
 * shaders/relight.wgsl kernel 2).  Environment lighting and visibility rays
 * are not part of this path. */
typedef struct bv_material {   /* Material (relight.rs:77-86), 32 bytes */
    float albedo[3];
    float roughness;           /* GGX, clamped to [0.045, 1] in shading */
    float specular_f0[3];      /* all zero: diffuse only */
    float pad;
} bv_material;

typedef struct bv_point_light { /* PointLight (relight.rs:176-181) */
    float position[3];
    float direction[3];         /* brightest axis, used when exponent != 0 */
    float intensity[3];         /* unit-albedo diffuse response at distance 1 */
    float exponent;             /* 0: isotropic */
} bv_point_light;

/* Gaussian PointCloudModel with Transforms + PbrAttributes (lib.rs:174-239). */
typedef struct bv_gaussian_desc {
    uint32_t num_points;
    uint32_t num_materials;
    const float *points;              /* [N*4] mean xyz, opacity */
    const float *rotations;           /* [N*4] unit quaternion x, y, z, w */
    const float *scales;              /* [N*3] */
    const float *normals;             /* [N*3] unit PBR normals */
    const uint32_t *material_indices; /* [N] */
    const bv_material *materials;     /* [num_materials] */
} bv_gaussian_desc;

typedef struct bv_relight_settings { /* RelightSettings (gpu/relight.rs) subset */
    float background[3];             /* radiance behind uncovered pixels */
    uint32_t diffuse_samples;        /* must be 0 (no visibility ray) */
} bv_relight_settings;

typedef struct bv_relight_tracer bv_relight_tracer;

/* Validates (lib.rs:246-340), keeps particles with opacity > 0.03
 * (gpu/relight.rs:211), builds the device particle table and a BVH over
 * the support ellipsoids (sqrt(2 ln(opacity/0.03)) standard deviations). */
bv_status bv_relight_tracer_new_gaussian(const bv_gaussian_desc *model,
                                         const bv_relight_settings *settings,
                                         bv_relight_tracer **out);
void bv_relight_tracer_destroy(bv_relight_tracer *tracer);
/* set_point_light for each light; the reference holds one light per
 * dispatch, several lights here shade every hit with their sum (alpha does
 * not depend on the light, so this equals the sum of single-light renders
 * with a zero background).  At most 64. */
bv_status bv_relight_tracer_set_point_lights(bv_relight_tracer *tracer,
                                             const bv_point_light *lights, uint32_t n_lights);
bv_status bv_relight_tracer_set_background(bv_relight_tracer *tracer, const float rgb[3]);
/* Renders width x height into out_rgba_dev ([h][w][4] float32): radiance +
 * transmittance * background, alpha = 1 - transmittance (relight.wgsl:747-780).
 * Five launches: each particle's camera-origin terms into the tracer's
 * per-view table, the trace (its 8x4 tiles heaviest first by the previous
 * dispatch's tile times when that had the same size; the order changes no
 * result), and three small ones that order the tiles for the next dispatch.
 * Because the tables are rewritten by each dispatch, a dispatch on a
 * different stream than the tracer's previous one is ordered after it (an
 * event wait), so dispatches never overlap. */
bv_status bv_relight_tracer_dispatch(bv_relight_tracer *tracer, float *out_rgba_dev,
                                     const bv_camera *camera, uint32_t width, uint32_t height,
                                     bv_stream stream);
uint32_t bv_relight_tracer_num_particles(const bv_relight_tracer *tracer);
/* rays, composited hits (steps) and BVH nodes visited (faces) of the last dispatch */
bv_status bv_relight_tracer_enable_stats(bv_relight_tracer *tracer, uint32_t enabled);
bv_status bv_relight_tracer_last_stats(bv_relight_tracer *tracer, bv_launch_stats *out);

/* ---- PowerFoam splat render ----------------------------------------------
 * PowerFoamGpuSplatTracer (blade-volume/src/gpu/powerfoam_splat.rs:38-370):
 * per ray every support sphere it crosses (spheres within 4 r of the camera
 * excluded), each clipped by its Cech row into [face_near, face_far] and the
 * sphere, taken in (entry depth, cell) order, truncated to max_steps and
 * composited (trace_powerfoam_splats, trace.rs:1456-1546).  Unlike the walk
 * it stays correct when the overlap graph is disconnected.  The model must
 * carry radii; its CSR is the Cech overlap graph.  There is no per-ray
 * candidate scratch on this path, so a render never overflows; the
 * reference's capacity check is kept: validate_candidate_counts recounts
 * the support hits of the last dispatch's rays and returns
 * BV_ERR_CANDIDATE_OVERFLOW when one ray has more than the capacity
 * max(4 max_steps, 1024, settings.powerfoam_candidate_capacity)
 * (path_record.rs:58-63). */
typedef struct bv_splat_tracer bv_splat_tracer;

bv_status bv_powerfoam_splat_tracer_new(const bv_model_desc *model, const bv_trace_settings *settings,
                                        bv_splat_tracer **out);
void bv_powerfoam_splat_tracer_destroy(bv_splat_tracer *tracer);
/* Renders [height][width][4] float32 (RGB, alpha = 1 - transmittance).
 * Dispatches and training calls time their 8x4-pixel tiles; a later call of
 * the same shape (views, width, height) starts its tiles heaviest first by
 * those times (three more small launches per call build the order).  The
 * order changes no result.  A call on a different stream than the tracer's
 * previous call is ordered after it (an event wait): the tile orders, ray
 * state and interval record belong to the tracer. */
bv_status bv_powerfoam_splat_tracer_dispatch(bv_splat_tracer *tracer, float *out_rgba_dev,
                                             const bv_camera *camera, uint32_t width, uint32_t height,
                                             bv_stream stream);
bv_status bv_powerfoam_splat_tracer_dispatch_batch(bv_splat_tracer *tracer, float *out_rgba_dev,
                                                   const bv_camera *cameras, uint32_t n_cameras,
                                                   uint32_t width, uint32_t height, bv_stream stream);
/* Synchronous; *observed = the largest support-hit count of one ray. */
bv_status bv_powerfoam_splat_tracer_validate_candidate_counts(bv_splat_tracer *tracer,
                                                              uint32_t *observed);
/* Synchronous recount of the last dispatch's rays: the largest support-hit
 * count of one ray, the total over all rays and the Cech row entries of
 * those supports (either total pointer may be NULL). */
bv_status bv_powerfoam_splat_tracer_candidate_stats(bv_splat_tracer *tracer, uint32_t *max_hits,
                                                    uint64_t *total_hits, uint64_t *row_entries);
uint32_t bv_powerfoam_splat_tracer_candidate_capacity(const bv_splat_tracer *tracer);
uint32_t bv_powerfoam_splat_tracer_max_steps(const bv_splat_tracer *tracer);
float bv_powerfoam_splat_tracer_weight_threshold(const bv_splat_tracer *tracer);
bv_status bv_powerfoam_splat_tracer_set_weight_threshold(bv_splat_tracer *tracer, float weight_threshold);
/* rays, composited intervals (steps) and Cech row entries clipped (faces,
 * counting re-clips in later windows) of the last dispatch */
bv_status bv_powerfoam_splat_tracer_enable_stats(bv_splat_tracer *tracer, uint32_t enabled);
bv_status bv_powerfoam_splat_tracer_last_stats(bv_splat_tracer *tracer, bv_launch_stats *out);
/* Training (bv_powerfoam_splat_tracer_forward_backward): the forward records
 * up to `entries` composited intervals per ray (cell, length, entry / exit
 * planes, unclamped colour: 24 bytes each, in 12 KiB chunks per 8x4 pixel
 * tile taken as the tile's rays need them, from a pool that starts at two
 * chunks per tile and grows after a call that ran it dry, up to 12 GiB)
 * and the replay walks that list instead of traversing the BVH and clipping
 * Cech rows again; rays past either limit are traversed again.  Default
 * 1024; 0 disables the record.  Results are identical for every setting.
 * No reference counterpart. */
bv_status bv_powerfoam_splat_tracer_set_interval_record(bv_splat_tracer *tracer, uint32_t entries);
/* Forward + loss + backward with splat semantics: the training recorder's
 * PowerFoam splats (record_powerfoam_splats_jacobians, trace.rs:1421-1452;
 * path_record.rs:1107-1218 on the GPU) integrated and differentiated under
 * the same contract as bv_forward_backward: the sorted support intervals of
 * every ray, truncated to settings->max_steps and cut at
 * settings->weight_threshold, dt clamped to max_dt, L2/L1 loss; density,
 * SH, site-position and radius gradients (through each interval's exact
 * Jacobians w.r.t. the entry / exit neighbours and the support sphere)
 * accumulate into the caller's tables.  Same arguments as
 * bv_forward_backward. */
bv_status bv_powerfoam_splat_tracer_forward_backward(
    bv_splat_tracer *tracer, const bv_camera *cameras, uint32_t n_cameras, uint32_t width,
    uint32_t height, const float *target_rgb_dev, const bv_train_settings *settings,
    const bv_grads *grads, float *loss_dev, float *rgb_out_dev, bv_stream stream);

/* ---- Gaussian ray tracing with SH colour ---------------------------------
 * GaussianGpuCloud (blade-volume/src/gpu/gaussian.rs:94-280) and its draw
 * pass (shaders/gaussian.wgsl, gaussian_trace.wgsl:66-177) with the hit rule
 * of the CPU oracle trace_gaussians (trace.rs:695-773): particles with
 * opacity > min_opacity; per ray every particle whose maximum response
 * alpha = opacity * exp(-|R^-1 (o + t d - mean) / scale|^2 / 2) at its
 * maximum-response depth t in (0, camera depth) reaches min_opacity,
 * composited in strict (t, model index) order, colour max(0, 0.5 + SH(d)),
 * until the transmittance is at most min_transmittance. */
typedef struct bv_gaussian_sh_desc { /* Gaussian PointCloudModel (lib.rs:174-239) */
    uint32_t num_points;
    uint32_t sh_degree;              /* 0..3 */
    const float *points;             /* [N*4] mean xyz, opacity */
    const float *rotations;          /* [N*4] unit quaternion x, y, z, w */
    const float *scales;             /* [N*3] */
    const float *sh_coefficients;    /* [N*3*K] [point][component][rgb] */
} bv_gaussian_sh_desc;

typedef struct bv_gaussian_trace_settings { /* GaussianTraceSettings (trace.rs:106-126) */
    float min_opacity;        /* default 0.01; also InitParameters::min_opacity */
    float min_transmittance;  /* default 0.01 */
    float background[3];      /* radiance behind the last hit (gaussian.wgsl BACKGROUND) */
} bv_gaussian_trace_settings;

typedef struct bv_gaussian_tracer bv_gaussian_tracer;

/* Validates the model, keeps particles above min_opacity, builds the device
 * particle table and a BVH over the support ellipsoids.  settings may be
 * NULL (defaults). */
bv_status bv_gaussian_tracer_new(const bv_gaussian_sh_desc *model,
                                 const bv_gaussian_trace_settings *settings,
                                 bv_gaussian_tracer **out);
void bv_gaussian_tracer_destroy(bv_gaussian_tracer *tracer);
bv_status bv_gaussian_tracer_set_min_transmittance(bv_gaussian_tracer *tracer, float value);
bv_status bv_gaussian_tracer_set_background(bv_gaussian_tracer *tracer, const float rgb[3]);
/* particles kept (GaussianGpuCloud::num_points) */
uint32_t bv_gaussian_tracer_num_points(const bv_gaussian_tracer *tracer);
/* Renders width x height into out_rgba_dev ([h][w][4] float32):
 * (radiance + T * background, 1 - T).  Five launches: each particle's
 * camera-origin terms into the tracer's per-view table, the trace (its 8x4
 * tiles heaviest first by the previous dispatch's tile times when that had
 * the same size; the order changes no result), and three small ones that
 * order the tiles for the next dispatch.  Because the tables are rewritten
 * by each dispatch, a dispatch on a different stream than the tracer's
 * previous one is ordered after it (an event wait), so dispatches never
 * overlap. */
bv_status bv_gaussian_tracer_dispatch(bv_gaussian_tracer *tracer, float *out_rgba_dev,
                                      const bv_camera *camera, uint32_t width, uint32_t height,
                                      bv_stream stream);
/* rays, composited hits (steps) and BVH nodes visited (faces) of the last dispatch */
bv_status bv_gaussian_tracer_enable_stats(bv_gaussian_tracer *tracer, uint32_t enabled);
bv_status bv_gaussian_tracer_last_stats(bv_gaussian_tracer *tracer, bv_launch_stats *out);

/* ---- RadFoam / PowerFoam PLY model files ----------------------------------
 * The walk subset of blade_volume::io::load_radfoam / try_load
 * (blade-volume/src/io/radfoam_ply.rs:1141-1213): PLY 1.0, binary
 * little-endian or ASCII, elements `vertex` (x, y, z, density,
 * adjacency_offset, blade_sh_dc_0..2 or red/green/blue preview DC,
 * color_sh_<k>, optional radius) then `adjacency` (one uint per CSR entry),
 * with the reference's ASCII row rules (comment and blank lines skipped,
 * extra columns ignored, trailing data an error) and its CSR validation
 * (:1111-1139).  Oriented-surface and detail properties are rejected
 * (BV_ERR_INVALID_MODEL; the walk has no such terms).  Two calls: _info for
 * the sizes, then _read into caller arrays points [n*4] (x, y, z, density),
 * sh [n*3K] (K = (sh_degree+1)^2, [component][rgb]), offsets [n+1],
 * neighbors [num_adjacency] and radii [n] (required when has_radii).  The
 * arrays are a bv_model_desc's inputs.  Host only; no device is touched. */
typedef struct bv_ply_info {
    uint32_t num_points;
    uint32_t num_adjacency;
    uint32_t sh_degree;
    uint32_t has_radii;
} bv_ply_info;
bv_status bv_radfoam_ply_info(const char *path, bv_ply_info *out);
bv_status bv_radfoam_ply_read(const char *path, float *points, float *sh, uint32_t *offsets,
                              uint32_t *neighbors, float *radii);

/* ---- allocation-free start-cell search -----------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * hosts whose device memory is owned by their own pool (a renderer's frame
 * arena, a framework's caching allocator, a hard memory budget), where an
 * allocation behind the pool's back breaks its accounting and cudaMalloc or
 * cudaFree may synchronise the device mid-frame.  Same FP64 power-nearest
 * search as bv_containing_point, without a tracer and without allocating:
 *   sites_dev      [num_sites] float4 (x, y, z, power radius; 0 for plain
 *                  RadFoam), 16-byte aligned, device memory
 *   positions      [n_queries * 3] host floats, n_queries <= 32
 *   out_index_dev  [n_queries] device uint32, receives the site indices
 * Its scratch (per-block partials and counters, 113,792 bytes) is a fixed
 * device array that every GPU loading the library holds until exit; every
 * call shares it, so calls that overlap on the GPU (other streams, other
 * threads) race.  More than 32 queries is rejected with
 * BV_ERR_INVALID_ARGUMENT (any site count is searched by at most 296 blocks,
 * which the array holds).  The first call on each device, and again after
 * the device's context has been replaced (cudaDeviceReset), looks up the
 * array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture. */
bv_status bv_containing_points_noalloc(const float *sites_dev, uint32_t num_sites,
                                       const float *positions, uint32_t n_queries,
                                       uint32_t *out_index_dev, bv_stream stream);

/* ---- serving loop ----------------------------------------------------------
 * No counterpart in the reference (its viewer renders one camera per frame,
 * blade-volume-view/src/render.rs:145-567).  A server keeps several scenes
 * resident on the device and serves render and forward+backward requests
 * of mixed resolution and view count from any host thread:
 *   - a request is admitted when its device buffers fit in the HBM budget
 *     left after the scenes and fixed scratch (first in, first admitted);
 *   - BV_SERVE_BATCHED: the frames (views) of all admitted render requests
 *     are packed into batches, earliest-due frame first, each ONE start-cell
 *     launch plus ONE persistent traversal launch over every frame in it (any
 *     scene, any size), replayed from a captured CUDA graph; up to `slots`
 *     batches run concurrently on their own high-priority streams, and each
 *     frame is copied to the host as soon as its batch finishes.
 *     Forward+backward requests run on a low-priority stream of their own
 *     beside the batches, in launch pairs of at most train_chunk_rays work
 *     items with the training step record, so that frames interleave;
 *   - BV_SERVE_PLAIN: one request at a time through the tracer calls, one
 *     bv_radfoam_tracer_dispatch per view (the reference's tracer takes one
 *     camera per dispatch), or bv_forward_backward, then a synchronize: the
 *     per-request baseline.  BV_SERVE_PLAIN_BATCH: the same with one
 *     bv_radfoam_tracer_dispatch_batch over the request's views.
 * Every scene of a server has the same SH degree, radii presence and SH
 * storage.  Frames render bit for bit as bv_radfoam_tracer_dispatch_batch
 * renders them, in any batch. */
typedef struct bv_server bv_server;

typedef enum bv_serve_mode {
    BV_SERVE_BATCHED = 0,
    BV_SERVE_PLAIN = 1,       /* per request, one dispatch per view */
    BV_SERVE_PLAIN_BATCH = 2, /* per request, one dispatch_batch over its views */
} bv_serve_mode;
typedef enum bv_request_kind { BV_REQUEST_RENDER = 0, BV_REQUEST_FORWARD_BACKWARD = 1 } bv_request_kind;

typedef struct bv_server_settings {
    uint64_t hbm_budget_bytes;  /* scenes + gradient tables + scratch + request buffers */
    uint32_t mode;              /* bv_serve_mode */
    uint32_t max_batch_rays;    /* rays per batch; 0 = 2,097,152; >= the largest frame */
    uint32_t max_batch_views;   /* frames per batch, 1..1024; 0 = 256 */
    uint32_t slots;             /* batches in flight, 1..4; 0 = 2 */
    uint32_t max_steps;         /* 0 = 1024 */
    float weight_threshold;     /* transmittance cut, e.g. 0.001 */
    uint64_t max_train_rays;    /* largest forward+backward chunk (<= 32 views); 0 = 16 x 1920 x 1080 */
    uint32_t use_graphs;        /* 1: replay captured graphs, 0: launch directly */
    uint32_t train_chunk_rays;  /* forward+backward work per launch pair (tile-padded rays);
                                   0 = 524,288: each pair lasts a few ms, so frames
                                   interleave between them */
    uint32_t frame_period_us;   /* frame k of a request is due (k + 1) periods after its
                                   arrival; batches take the earliest-due frames first;
                                   0 = 16,000 */
    uint32_t train_record_steps;/* steps per ray held by the training step record (chunk x
                                   steps x 16 B of HBM; a replay searches past them):
                                   1..256 as given, 0 = the most of 256 that fits an eighth
                                   of the budget, BV_SERVE_NO_RECORD = none */
} bv_server_settings;

#define BV_SERVE_NO_RECORD 0xffffffffu

/* Scene flag: the server keeps gradient tables for the scene, into which
 * forward+backward requests that name no tables of their own accumulate. */
#define BV_SCENE_GRADIENTS 0x1u

typedef struct bv_request {
    uint32_t scene;
    uint32_t kind;                /* bv_request_kind */
    uint32_t n_views;             /* 1..1024 */
    uint32_t width, height;
    uint32_t reserved;
    const bv_camera *cameras;     /* host [n_views], copied by bv_server_submit */
    float *out_host;              /* render: [views][h][w][4]; fwd+bwd: [views][h][w][3] or NULL */
    const float *target_host;     /* fwd+bwd: [views][h][w][3], read once admitted */
    float *loss_host;             /* fwd+bwd: receives the loss */
    bv_train_settings train;      /* fwd+bwd */
    bv_grads grads;               /* fwd+bwd device tables; all NULL: the scene's own */
    double *frame_done_host;      /* optional [n_views]: server-clock time each frame landed */
} bv_request;

typedef struct bv_request_result {
    uint64_t id;
    int32_t status;               /* bv_status of the request */
    uint32_t kind;
    double submit_s;              /* server clock (seconds since bv_server_new) */
    double admit_s;               /* device buffers granted */
    double start_s;               /* first work enqueued on the GPU */
    double done_s;                /* every output on the host */
    uint64_t rays;
    char message[128];
} bv_request_result;

typedef struct bv_server_stats {
    uint64_t requests_done, frames_done, rays_done;
    uint64_t batches, graph_launches, kernel_launches;
    uint64_t arena_bytes, arena_peak_bytes, resident_bytes;
    uint64_t admission_waits;     /* times the head request did not fit */
    double busy_s;                /* wall time with work on the device */
    uint64_t arena_used_bytes;    /* request buffers held right now */
    uint64_t requests_cancelled;
} bv_server_stats;

bv_status bv_server_new(const bv_server_settings *settings, bv_server **out);
/* Uploads a scene (tracer packing); only before bv_server_start. */
bv_status bv_server_add_scene(bv_server *server, const bv_model_desc *model, uint32_t flags,
                              uint32_t *scene_id);
/* Device gradient tables of a BV_SCENE_GRADIENTS scene. */
bv_status bv_server_scene_grads(bv_server *server, uint32_t scene, bv_grads *out);
/* Reserves the request arena (budget minus resident), captures the batch
 * graphs and starts the scheduler thread. */
bv_status bv_server_start(bv_server *server);
/* Validates and queues a request; host buffers stay valid until it is done.
 * A request whose buffers can never fit the arena is refused here. */
bv_status bv_server_submit(bv_server *server, const bv_request *request, uint64_t *id);
/* Waits up to timeout_s for request id.  BV_OK once it has finished: out
 * holds its result (out->status is the request's own status) and the id is
 * forgotten.  BV_ERR_TIMEOUT if it has not finished, BV_ERR_INVALID_ARGUMENT
 * for an unknown id. */
bv_status bv_server_wait(bv_server *server, uint64_t id, double timeout_s, bv_request_result *out);
/* Withdraws request id.  A request not yet admitted finishes at once; an
 * admitted render request drops its frames that have not been launched and
 * finishes when its launched frames have landed; a forward+backward request
 * already on the device finishes when its work ends.  Either way its device
 * buffers go back to the arena, bv_server_wait reports BV_ERR_CANCELLED as
 * the request's status, and its host outputs are incomplete.  BV_OK also
 * for a request that had already finished (its status is then its own). */
bv_status bv_server_cancel(bv_server *server, uint64_t id);
bv_status bv_server_stats_get(bv_server *server, bv_server_stats *out);
double bv_server_clock(const bv_server *server);
/* Finishes queued work, stops the scheduler, frees everything. */
void bv_server_destroy(bv_server *server);

#ifdef __cplusplus
}
#endif
#endif /* BLADE_VOLUME_B200_H */
