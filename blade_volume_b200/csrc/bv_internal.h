// Internal device layout and launch descriptors of the B200 walk path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "blade_volume_b200.h"

namespace bv {

// Rays are handed out in tiles of 8x4 pixels so that a warp's 32 lanes start
// on neighbouring pixels and walk mostly the same cells.
constexpr int kTileW = 8;
constexpr int kTileH = 4;
constexpr int kTileRays = kTileW * kTileH;
// Views (cameras) per launch carried in the kernel parameter block.
constexpr int kMaxViewsPerLaunch = 32;

struct ViewDesc {  // 80 bytes
    float origin[3];
    float depth;
    float q[4];
    float tan_half[2];
    float principal[2];
    uint32_t width, height;
    uint32_t tiles_x;
    uint32_t ray_begin;    // first tile-ordered work index of this view
    uint64_t pixel_begin;  // first output pixel of this view
    uint64_t pad;
};

// One CSR entry (face) of the walk, 32 bytes: the neighbour's site record
// and everything the walk needs once it steps into that neighbour, so that a
// walk step costs one dependent round trip to memory (the current cell's
// face entries) instead of three (offsets -> neighbour index -> site).
struct __align__(16) FaceEntry {
    float4 site;  // neighbour j: x, y, z, power radius (0 for plain RadFoam)
    uint4 link;   // j, offsets[j], offsets[j+1], density[j] (float bits)
};

// SoA device copy of a model.  Appearance (SH rows) lives in its own table
// read once per step; geometry the walk reads per face lives in the face
// table; geom/density/offsets serve the start cell and the Jacobians.
struct DeviceModel {
    const float4 *geom;        // [N] x, y, z, radius (0 for plain RadFoam)
    const float *density;      // [N]
    const void *sh;            // [N][sh_stride] float or bf16
    const uint32_t *offsets;   // [N+1]
    const FaceEntry *faces;    // [M] CSR order
    uint32_t n;
    uint32_t sh_degree;
    uint32_t sh_stride;        // elements per SH row (>= 3K, padded to 16 bytes)
    uint32_t sh_bf16;
    uint32_t bounded;          // radii present (PowerFoam)
};

struct WalkParams {
    DeviceModel m;
    uint32_t max_steps;
    float weight_threshold;
    uint32_t n_views;
    uint32_t total_work;          // tile-ordered work items over all views
    const uint32_t *start_cells;  // [n_views]
    uint32_t *work_counter;       // persistent-kernel ray dispenser
    unsigned long long *stats;    // [3] rays, steps, faces (or null)
    float4 *out_rgba;             // [n_views][H][W]
    uint32_t debug_cell_density;
    uint32_t tie_break;           // FP64 re-evaluation of near-tied exit faces
    ViewDesc views[kMaxViewsPerLaunch];
};

struct RecordParams {
    DeviceModel m;
    uint32_t max_steps;
    uint32_t n_views;
    uint32_t total_work;
    const uint32_t *start_cells;
    uint32_t *work_counter;
    bv_path_buffers buf;
    ViewDesc views[kMaxViewsPerLaunch];
};

// Per-ray state handed from the training forward kernel to the replay
// kernel: the compensated colour (hi, lo) and dL/dC.  48 bytes per ray; no
// per-sample state is stored.
struct RayState {
    float4 c_hi;  // colour hi, dL/dC.r
    float4 c_lo;  // colour lo, dL/dC.g
    float4 g;     // dL/dC.b, unused x3
};

struct TrainParams {
    DeviceModel m;
    uint32_t max_steps;
    float weight_threshold;
    float max_dt;
    uint32_t loss_kind;
    float inv_count;              // 1 / (3 * rays in the batch)
    uint32_t n_views;
    uint32_t total_work;
    const uint32_t *start_cells;
    uint32_t *work_counter;       // [2]: forward, replay dispensers
    const float *target;          // [views][H][W][3]
    float *rgb_out;               // [views][H][W][3] or null
    RayState *ray_state;          // [views][H][W] scratch
    float *d_density;
    float *d_sh;
    float4 *d_site;               // [N] x, y, z, radius gradients (scratch) or null
    float *loss;                  // device scalar accumulator
    unsigned long long *stats;
    uint32_t *step_rec;           // exit face + SH colour per (ray, step < rec_steps), or null
    uint32_t rec_steps;           // 0: the replay searches and evaluates every step
    uint32_t work_begin;          // this launch covers work items [work_begin, +total_work)
    const uint32_t *tile_order;   // [tiles] tile of dispensed tile i, or null (bv_tile_order.cuh)
    uint32_t *tile_cost;          // [tiles] forward: each tile's duration, or null
    ViewDesc views[kMaxViewsPerLaunch];
};

constexpr int kMaxStartQueries = 32;
struct StartCellQueries {
    float position[kMaxStartQueries][3];
    uint32_t count;
};

// ---- serving: one traversal launch over the frames (views) of many
// requests, any resident scene and any resolution.  The batch is described
// by a table in device memory, so one captured CUDA graph serves every batch.
constexpr int kMaxServeScenes = 8;
constexpr int kMaxServeViews = 1024;
constexpr int kServeStartBlocks = 16;  // start-cell blocks per frame
constexpr int kServeStartRows = 64;    // frames searched concurrently

struct ServeView {  // 96 bytes
    ViewDesc v;           // ray_begin: first work item in the batch; pixel_begin unused
    uint32_t scene;
    uint32_t start_cell;  // written by the start-cell kernel of the batch
    uint64_t out;         // float4 * [height][width] of this frame
};

struct ServeHeader {  // 16 bytes, followed by the ServeView rows
    uint32_t n_views;
    uint32_t total_work;
    uint32_t pad[2];
};

struct ServeParams {
    DeviceModel scenes[kMaxServeScenes];
    uint32_t n_scenes;
    uint32_t max_steps;
    float weight_threshold;
    uint32_t pad;
    const ServeHeader *header;
    ServeView *views;
    uint32_t *work_counter;
    double *partial_dist;     // [kMaxServeViews][kServeStartBlocks]
    uint32_t *partial_index;  // [kMaxServeViews][kServeStartBlocks]
    uint32_t *counters;       // [kMaxServeViews], zero between launches
};

cudaError_t launch_serve_start_cells(const ServeParams &p, cudaStream_t s);
cudaError_t launch_serve_walk(const ServeParams &p, int grid, cudaStream_t s);
int serve_grid_size(int device);

// Launchers (bv_walk.cu / bv_start_cell.cu).
cudaError_t launch_walk_forward(const WalkParams &p, int grid, cudaStream_t s);
cudaError_t launch_record_paths(const RecordParams &p, int grid, cudaStream_t s);
cudaError_t launch_train_forward(const TrainParams &p, int grid, cudaStream_t s);
cudaError_t launch_train_backward(const TrainParams &p, int grid, cudaStream_t s);
cudaError_t launch_fold_site_grads(float4 *site, uint32_t n, float *d_pos, float *d_radius,
                                   cudaStream_t s);
// kind: 0 render, 1 training forward, 2 replay backward
int walk_grid_size(int device, int kind);

// FP64 power-nearest search: out[v] = argmin_i |q_v - p_i|^2 - r_i^2, ties to
// the lowest index.  partial/counters are scratch owned by the caller:
// partial [n_queries * blocks_per_query] and counters [n_queries] (zeroed
// once; the kernel leaves them zero).
struct StartCellScratch {
    double *partial_dist;
    uint32_t *partial_index;
    uint32_t *counters;
    int blocks_per_query;
};
// Adam over a tracer's tables (bv_optim.cu).  Scalars are formed on the host:
// one_minus_beta_i = 1 - beta_i in FP32, c_i = 1 - beta_i^t in FP64 rounded.
struct AdamScalars {
    float beta1, beta2, one_minus_beta1, one_minus_beta2, c1, c2, eps;
};

struct AdamParams {
    uint32_t n;
    uint32_t sh_row;     // 3K coefficients per site (dense gradient / moment rows)
    uint32_t sh_stride;  // elements per device SH row
    AdamScalars s;
    float lr_density, lr_sh_dc, lr_sh_rest, lr_position, lr_radius;
    uint32_t activation;  // BV_DENSITY_*
    float softplus_beta;
    float *density_param;  // [N] raw parameter x, density = act(x)
    float *density;        // [N] device model density
    const float *g_density;
    float *m_density, *v_density;
    void *sh;              // device SH table (FP32 or BF16 rows)
    float *sh_master;      // [N*3K] FP32 master copy when the table is BF16
    const float *g_sh;
    float *m_sh, *v_sh;
    float4 *geom;          // [N] x, y, z, radius
    const float *g_pos;    // [N*3]
    float *m_pos, *v_pos;
    const float *g_radius;  // [N] or null
    float *m_radius, *v_radius;
};

cudaError_t launch_init_density_param(const float *density, float *param, uint32_t n,
                                      uint32_t kind, float beta, cudaStream_t s);
cudaError_t launch_adam_step(const AdamParams &p, FaceEntry *faces, uint32_t m_edges, bool bf16,
                             cudaStream_t s);

// Sets the calling thread's bv_last_error() message.
void set_last_error(const char *message);

cudaError_t launch_start_cells(const float4 *geom, uint32_t n, const StartCellQueries &queries,
                               const StartCellScratch &scratch, uint32_t *out, cudaStream_t s);
int start_cell_blocks(uint32_t n);

// Camera helpers shared by the tracer calls and the serving engine
// (bv_api.cu): the view record of a camera, work items of a tile-padded
// image, camera validation (sets bv_last_error on failure).
ViewDesc view_desc(const bv_camera &c, uint32_t width, uint32_t height, uint32_t ray_begin,
                   uint64_t pixel_begin);
uint32_t tile_padded_rays(uint32_t width, uint32_t height);
bv_status validate_camera(const bv_camera &c);

// Accessors the serving engine uses on tracers it owns (bv_api.cu).
DeviceModel tracer_device_model(const bv_tracer *t);
size_t tracer_device_bytes(const bv_tracer *t);
// Hand the tracer a caller-owned ray-state buffer for bv_forward_backward
// (chunks larger than capacity are refused instead of growing it).
void tracer_lend_ray_state(bv_tracer *t, RayState *buffer, size_t capacity);
// Hand the tracer a caller-owned step-record buffer (words) for
// bv_forward_backward; the tracer never grows a lent record.
void tracer_lend_step_record(bv_tracer *t, uint32_t *buffer, size_t words);
// bv_forward_backward issues its forward and replay kernels over at most this
// many work items (tile-padded rays) per launch pair, so that the launches
// of one call stay short and other work on the device interleaves between
// them (0: one launch pair per group of 32 views).  Results are the same.
void tracer_set_train_chunk(bv_tracer *t, uint32_t work_items);

}  // namespace bv
