// C ABI of the B200 walk path: model validation and packing, the tracer
// handle (RadFoamGpuTracer), the path recorder and the training gradient.
//
// Host code only; the kernels live in bv_walk.cu and bv_start_cell.cu.

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "bv_internal.h"
#include "bv_tile_order.cuh"

// Training takes its tiles heaviest first by the previous call's tile times
// in the forward and the replay (1), in the replay only (2), or in launch
// order (0).  Measured on the headline (262,144 sites, 8 x 512^2): the
// forward keeps launch order faster (8.21 vs 8.65 ms: neighbouring tiles
// share cells in L1/L2), the replay takes the order with classes in no
// particular screen order faster (8.05 vs 9.04 ms in launch order, 8.64
// with classes in launch order: concurrent tiles from all over the screen
// scatter their gradient atomics into different cells).
#ifndef BV_WALK_TILE_ORDER
#define BV_WALK_TILE_ORDER 2
#endif
// The forward's own order (mode 2): tiles heaviest first in classes of
// floor(log2(time)) >> shift, launch order inside a class; -1: launch order.
// Measured on the headline: the forward takes 8.24 ms in launch order and
// 8.54 / 8.51 / 8.37 ms with shifts 0 / 1 / 2 (coarser classes keep more
// tiles in launch order; neighbouring tiles sharing cells in L1/L2 is worth
// more than the heavy tiles starting first).
#ifndef BV_WALK_FWD_ORDER_SHIFT
#define BV_WALK_FWD_ORDER_SHIFT -1
#endif

using namespace bv;

namespace {

thread_local std::string g_error;

// Step record of the training forward (exit face and unclamped SH colour,
// 16 bytes per ray and step): by default this many steps per ray, and at
// most this many bytes per launch.  The replay reads one face entry and the
// colour per recorded step instead of searching the cell's row and
// evaluating its SH row.  0 steps disables the record.
#ifndef BV_EXIT_REC_STEPS
#define BV_EXIT_REC_STEPS 256
#endif
constexpr uint32_t kExitRecSteps = BV_EXIT_REC_STEPS;
constexpr size_t kExitRecBytes = size_t(8) << 30;
constexpr size_t kStepRecWords = 4;  // face, r, g, b

bv_status fail(bv_status code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

bv_status cuda_fail(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return fail(BV_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return fail(BV_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return fail(BV_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define BV_CUDA(call, what)                          \
    do {                                             \
        cudaError_t e_ = (call);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

uint32_t sh_components(uint32_t degree) {
    const uint32_t d = (degree > 3 ? 3 : degree) + 1;
    return d * d;
}

uint16_t f32_to_bf16_rne(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);  // NaN
    const uint32_t rounding = ((u >> 16) & 1u) + 0x7fffu;
    return (uint16_t)((u + rounding) >> 16);
}

}  // namespace

void bv::set_last_error(const char *message) { g_error = message; }

struct bv_tracer {
    int device = 0;
    uint32_t n = 0;
    uint32_t m_edges = 0;
    uint32_t sh_degree = 0;
    uint32_t sh_stride = 0;
    bool bf16 = false;
    bool bounded = false;
    bv_trace_settings settings{};
    uint32_t tie_break = 0;            // render walk: FP64 exit-face tie-break
    // optimizer state (allocated by the first bv_radfoam_tracer_adam_step)
    uint32_t adam_t = 0;               // steps taken
    uint32_t adam_activation = 0;
    float adam_beta = 0.f;
    float *adam_buf = nullptr;         // one allocation: the arrays below
    float *density_param = nullptr, *m_density = nullptr, *v_density = nullptr;
    float *sh_master = nullptr, *m_sh = nullptr, *v_sh = nullptr;
    float *m_pos = nullptr, *v_pos = nullptr, *m_radius = nullptr, *v_radius = nullptr;
    // device model
    float4 *geom = nullptr;
    float *density = nullptr;
    void *sh = nullptr;
    uint32_t *offsets = nullptr;
    FaceEntry *faces = nullptr;
    // scratch
    uint32_t *start_cells = nullptr;   // [kMaxViewsPerLaunch]
    uint32_t *work_counter = nullptr;  // [4]
    unsigned long long *stats = nullptr;  // [4]
    double *partial_dist = nullptr;
    uint32_t *partial_index = nullptr;
    uint32_t *start_counters = nullptr;
    int start_blocks = 1;
    RayState *ray_state = nullptr;     // per-ray training state
    size_t ray_state_capacity = 0;
    bool ray_state_owned = true;       // false: lent by a serving engine
    float4 *site_grads = nullptr;      // [N] site gradient accumulator (kept zero)
    uint32_t *step_rec = nullptr;      // training forward's step record, read by the replay
    size_t step_rec_capacity = 0;      // words
    uint32_t step_rec_steps = kExitRecSteps;  // recorded steps per ray
    bool step_rec_owned = true;        // false: lent by a serving engine
    uint32_t train_chunk = 0;          // work items per training launch pair (0: a whole group)
    TileScheduler train_order;         // heaviest-first tiles between training calls (unstable)
    int grid_forward = 0;
    int grid_train_fwd = 0;
    int grid_train_bwd = 0;
    // instrumentation
    bool stats_enabled = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t last_stream = nullptr;
    uint32_t last_launches = 0;
    bool last_train = false;
    bool last_has_stats = false;
    uint32_t last_start_point = 0;
    bool start_point_pending = false;

    DeviceModel model() const {
        DeviceModel m;
        m.geom = geom;
        m.density = density;
        m.sh = sh;
        m.offsets = offsets;
        m.faces = faces;
        m.n = n;
        m.sh_degree = sh_degree;
        m.sh_stride = sh_stride;
        m.sh_bf16 = bf16 ? 1u : 0u;
        m.bounded = bounded ? 1u : 0u;
        return m;
    }
};

namespace {

void free_tracer(bv_tracer *t) {
    if (!t) return;
    t->train_order.release();
    cudaFree(t->geom);
    cudaFree(t->density);
    cudaFree(t->sh);
    cudaFree(t->offsets);
    cudaFree(t->faces);
    if (t->ray_state_owned) cudaFree(t->ray_state);
    cudaFree(t->site_grads);
    if (t->step_rec_owned) cudaFree(t->step_rec);
    cudaFree(t->start_cells);
    cudaFree(t->work_counter);
    cudaFree(t->stats);
    cudaFree(t->partial_dist);
    cudaFree(t->partial_index);
    cudaFree(t->start_counters);
    cudaFree(t->adam_buf);
    for (auto &e : t->ev)
        if (e) cudaEventDestroy(e);
    delete t;
}

// ViewDesc for camera c of a width x height image (radfoam.wgsl:44-52).
ViewDesc make_view(const bv_camera &c, uint32_t width, uint32_t height, uint32_t ray_begin,
                   uint64_t pixel_begin) {
    ViewDesc v;
    std::memset(&v, 0, sizeof(v));
    for (int i = 0; i < 3; ++i) v.origin[i] = c.cam_position[i];
    v.depth = c.depth;
    for (int i = 0; i < 4; ++i) v.q[i] = c.cam_orientation[i];
    // tan(fov / 2): FP64 on the host, rounded to FP32 once per camera.
    v.tan_half[0] = (float)std::tan((double)(0.5f * c.fov[0]));
    v.tan_half[1] = (float)std::tan((double)(0.5f * c.fov[1]));
    v.principal[0] = c.principal[0];
    v.principal[1] = c.principal[1];
    v.width = width;
    v.height = height;
    v.tiles_x = (width + kTileW - 1) / kTileW;
    v.ray_begin = ray_begin;
    v.pixel_begin = pixel_begin;
    return v;
}

uint32_t padded_rays(uint32_t width, uint32_t height) {
    const uint32_t tx = (width + kTileW - 1) / kTileW, ty = (height + kTileH - 1) / kTileH;
    return tx * ty * kTileRays;
}

bv_status check_camera(const bv_camera &c) {
    for (float v : c.cam_position)
        if (!std::isfinite(v)) return fail(BV_ERR_INVALID_ARGUMENT, "camera position must be finite");
    if (!std::isfinite(c.depth) || !(c.depth > 0.0f))
        return fail(BV_ERR_INVALID_ARGUMENT, "camera depth must be finite and positive");
    for (float v : c.cam_orientation)
        if (!std::isfinite(v)) return fail(BV_ERR_INVALID_ARGUMENT, "camera orientation must be finite");
    for (float v : c.fov)
        if (!std::isfinite(v)) return fail(BV_ERR_INVALID_ARGUMENT, "camera fov must be finite");
    return BV_OK;
}

// Launch the FP64 start-cell search for a chunk of cameras into
// t->start_cells[0..count).
bv_status launch_starts(bv_tracer *t, const bv_camera *cams, uint32_t count, cudaStream_t s) {
    StartCellQueries q;
    std::memset(&q, 0, sizeof(q));
    q.count = count;
    for (uint32_t i = 0; i < count; ++i)
        for (int k = 0; k < 3; ++k) q.position[i][k] = cams[i].cam_position[k];
    StartCellScratch sc{t->partial_dist, t->partial_index, t->start_counters, t->start_blocks};
    BV_CUDA(launch_start_cells(t->geom, t->n, q, sc, t->start_cells, s), "start-cell launch");
    return BV_OK;
}

bv_status begin_timing(bv_tracer *t, cudaStream_t s) {
    t->last_stream = s;
    t->last_launches = 0;
    t->last_train = false;
    t->last_has_stats = t->stats_enabled;
    if (t->stats_enabled) {
        BV_CUDA(cudaMemsetAsync(t->stats, 0, 4 * sizeof(unsigned long long), s), "stats reset");
        BV_CUDA(cudaEventRecord(t->ev[0], s), "event");
    }
    return BV_OK;
}

}  // namespace

DeviceModel bv::tracer_device_model(const bv_tracer *t) { return t->model(); }

ViewDesc bv::view_desc(const bv_camera &c, uint32_t width, uint32_t height, uint32_t ray_begin,
                       uint64_t pixel_begin) {
    return make_view(c, width, height, ray_begin, pixel_begin);
}

uint32_t bv::tile_padded_rays(uint32_t width, uint32_t height) { return padded_rays(width, height); }

bv_status bv::validate_camera(const bv_camera &c) { return check_camera(c); }

size_t bv::tracer_device_bytes(const bv_tracer *t) {
    const size_t n = t->n;
    const size_t sh_bytes = n * t->sh_stride * (t->bf16 ? 2 : 4);
    return n * (sizeof(float4) + sizeof(float) + sizeof(float4)) + (n + 1) * sizeof(uint32_t) +
           (size_t)std::max<uint32_t>(t->m_edges, 1) * sizeof(FaceEntry) + sh_bytes +
           (size_t)kMaxStartQueries * t->start_blocks * (sizeof(double) + sizeof(uint32_t));
}

void bv::tracer_lend_ray_state(bv_tracer *t, RayState *buffer, size_t capacity) {
    if (t->ray_state_owned) cudaFree(t->ray_state);
    t->ray_state = buffer;
    t->ray_state_capacity = capacity;
    t->ray_state_owned = false;
}

void bv::tracer_lend_step_record(bv_tracer *t, uint32_t *buffer, size_t words) {
    if (t->step_rec_owned) cudaFree(t->step_rec);
    t->step_rec = buffer;
    t->step_rec_capacity = buffer ? words : 0;
    t->step_rec_owned = false;
}

void bv::tracer_set_train_chunk(bv_tracer *t, uint32_t work_items) {
    // whole 8x4 tiles, so that a chunk's rays keep their tile-major record lines
    t->train_chunk = (work_items + kTileRays - 1) / kTileRays * kTileRays;
}

extern "C" {

const char *bv_last_error(void) { return g_error.c_str(); }

uint32_t bv_abi_version(void) { return BV_ABI_VERSION; }

bv_status bv_model_validate(const bv_model_desc *md, char *err, size_t err_len) {
    auto bad = [&](const char *fmt, auto... args) {
        char buf[512];
        snprintf(buf, sizeof(buf), fmt, args...);
        g_error = buf;
        if (err && err_len) {
            strncpy(err, buf, err_len - 1);
            err[err_len - 1] = '\0';
        }
        return BV_ERR_INVALID_MODEL;
    };
    if (!md) return bad("%s", "model descriptor is null");
    const uint32_t n = md->num_points;
    if (n == 0) return bad("%s", "model has no points");
    if (!md->points || !md->sh_coefficients) return bad("%s", "points and SH coefficients are required");
    if (md->sh_degree > 3) return bad("SH degree %u exceeds supported degree 3", md->sh_degree);
    if (!md->adjacency_offsets || (!md->adjacency_neighbors && md->adjacency_offsets[n] != 0))
        return bad("%s", "the cell walk requires CSR adjacency");
    for (uint32_t i = 0; i < n; ++i) {
        const float *p = md->points + 4 * (size_t)i;
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) ||
            !std::isfinite(p[3]) || p[3] < 0.0f)
            return bad("point %u must have finite coordinates and non-negative density/opacity", i);
    }
    const size_t nsh = (size_t)n * 3 * sh_components(md->sh_degree);
    for (size_t i = 0; i < nsh; ++i)
        if (!std::isfinite(md->sh_coefficients[i])) return bad("%s", "SH coefficients must be finite");
    if (md->radii) {
        for (uint32_t i = 0; i < n; ++i)
            if (!std::isfinite(md->radii[i]) || md->radii[i] < 0.0f)
                return bad("%s", "radii must be finite and non-negative");
    }
    // validate_csr_result (adjacency.rs:724-790)
    const uint32_t *off = md->adjacency_offsets;
    const uint32_t *nb = md->adjacency_neighbors;
    if (off[0] != 0) return bad("Invalid adjacency_offsets[0]: expected 0, got %u", off[0]);
    const uint32_t total = off[n];
    for (uint32_t i = 0; i < n; ++i)
        if (off[i + 1] < off[i] || off[i + 1] > total)
            return bad("Invalid adjacency offset range for point %u: [%u, %u)", i, off[i], off[i + 1]);
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t k = off[i]; k < off[i + 1]; ++k) {
            if (k + 1 < off[i + 1] && nb[k] >= nb[k + 1])
                return bad("Adjacency list for point %u must be sorted and unique", i);
            if (nb[k] >= n)
                return bad("Adjacency index out of bounds at entry %u: %u (num_points=%u)", k, nb[k], n);
            if (nb[k] == i) return bad("Adjacency list for point %u contains a self-edge", i);
        }
    }
    for (uint32_t i = 0; i < n; ++i) {
        for (uint32_t k = off[i]; k < off[i + 1]; ++k) {
            const uint32_t j = nb[k];
            uint32_t lo = off[j], hi = off[j + 1];
            bool found = false;
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo) / 2;
                if (nb[mid] == i) {
                    found = true;
                    break;
                }
                if (nb[mid] < i)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            if (!found) return bad("Adjacency edge %u->%u has no reverse edge", i, j);
        }
    }
    g_error.clear();
    return BV_OK;
}

bv_status bv_radfoam_tracer_new(const bv_model_desc *md, const bv_trace_settings *settings,
                                bv_tracer **out) {
    if (!out) return fail(BV_ERR_INVALID_ARGUMENT, "out handle pointer is null");
    *out = nullptr;
    if (bv_model_validate(md, nullptr, 0) != BV_OK) return BV_ERR_INVALID_MODEL;
    int device = 0;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) return cuda_fail(e == cudaSuccess ? cudaErrorNoDevice : e, "cudaGetDeviceCount");
    BV_CUDA(cudaGetDevice(&device), "cudaGetDevice");

    bv_tracer *t = new bv_tracer();
    t->train_order.stable = false;
    t->train_order.second_shift = BV_WALK_FWD_ORDER_SHIFT;
    t->device = device;
    t->n = md->num_points;
    t->m_edges = md->adjacency_offsets[md->num_points];
    t->sh_degree = md->sh_degree;
    t->bf16 = (md->flags & BV_MODEL_SH_BF16) != 0;
    t->bounded = md->radii != nullptr;
    if (settings) {
        t->settings = *settings;
    } else {
        t->settings.max_steps = 1024;
        t->settings.weight_threshold = 0.001f;
    }
    const uint32_t n = t->n;
    const uint32_t nsh = 3 * sh_components(t->sh_degree);
    const uint32_t align = t->bf16 ? 8u : 4u;  // 16-byte rows
    t->sh_stride = (nsh + align - 1) / align * align;

    // host packing
    std::vector<float4> geom(n);
    std::vector<float> dens(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float *p = md->points + 4 * (size_t)i;
        geom[i] = make_float4(p[0], p[1], p[2], md->radii ? md->radii[i] : 0.0f);
        dens[i] = p[3];
    }
    auto cleanup = [&](bv_status s) {
        free_tracer(t);
        return s;
    };
#define BV_TRY(call, what)                                            \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return cleanup(cuda_fail(e_, what));   \
    } while (0)
    BV_TRY(cudaMalloc(&t->geom, sizeof(float4) * n), "cudaMalloc geom");
    BV_TRY(cudaMalloc(&t->density, sizeof(float) * n), "cudaMalloc density");
    BV_TRY(cudaMalloc(&t->offsets, sizeof(uint32_t) * (n + 1)), "cudaMalloc offsets");
    BV_TRY(cudaMalloc(&t->faces, sizeof(FaceEntry) * (t->m_edges ? t->m_edges : 1)), "cudaMalloc faces");
    BV_TRY(cudaMemcpy(t->geom, geom.data(), sizeof(float4) * n, cudaMemcpyHostToDevice), "upload geom");
    BV_TRY(cudaMemcpy(t->density, dens.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "upload density");
    BV_TRY(cudaMemcpy(t->offsets, md->adjacency_offsets, sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice), "upload offsets");
    if (t->m_edges) {
        // face table: per CSR entry the neighbour's site and its own CSR range
        // and density, in CSR order
        std::vector<FaceEntry> faces(t->m_edges);
        for (uint32_t k = 0; k < t->m_edges; ++k) {
            const uint32_t j = md->adjacency_neighbors[k];
            uint32_t dbits;
            std::memcpy(&dbits, &dens[j], 4);
            faces[k].site = geom[j];
            faces[k].link = make_uint4(j, md->adjacency_offsets[j], md->adjacency_offsets[j + 1], dbits);
        }
        BV_TRY(cudaMemcpy(t->faces, faces.data(), sizeof(FaceEntry) * t->m_edges, cudaMemcpyHostToDevice), "upload faces");
    }
    if (t->bf16) {
        std::vector<uint16_t> row((size_t)n * t->sh_stride, 0);
        for (uint32_t i = 0; i < n; ++i)
            for (uint32_t k = 0; k < nsh; ++k)
                row[(size_t)i * t->sh_stride + k] = f32_to_bf16_rne(md->sh_coefficients[(size_t)i * nsh + k]);
        BV_TRY(cudaMalloc(&t->sh, row.size() * 2), "cudaMalloc sh");
        BV_TRY(cudaMemcpy(t->sh, row.data(), row.size() * 2, cudaMemcpyHostToDevice), "upload sh");
    } else {
        std::vector<float> row((size_t)n * t->sh_stride, 0.0f);
        for (uint32_t i = 0; i < n; ++i)
            std::memcpy(&row[(size_t)i * t->sh_stride], md->sh_coefficients + (size_t)i * nsh, nsh * 4);
        BV_TRY(cudaMalloc(&t->sh, row.size() * 4), "cudaMalloc sh");
        BV_TRY(cudaMemcpy(t->sh, row.data(), row.size() * 4, cudaMemcpyHostToDevice), "upload sh");
    }
    // scratch
    t->start_blocks = start_cell_blocks(n);
    BV_TRY(cudaMalloc(&t->start_cells, sizeof(uint32_t) * kMaxViewsPerLaunch), "cudaMalloc start cells");
    BV_TRY(cudaMalloc(&t->work_counter, sizeof(uint32_t) * 4), "cudaMalloc counter");
    BV_TRY(cudaMalloc(&t->stats, sizeof(unsigned long long) * 4), "cudaMalloc stats");
    BV_TRY(cudaMalloc(&t->partial_dist, sizeof(double) * kMaxStartQueries * t->start_blocks), "cudaMalloc partials");
    BV_TRY(cudaMalloc(&t->partial_index, sizeof(uint32_t) * kMaxStartQueries * t->start_blocks), "cudaMalloc partials");
    BV_TRY(cudaMalloc(&t->start_counters, sizeof(uint32_t) * kMaxStartQueries), "cudaMalloc counters");
    BV_TRY(cudaMemset(t->start_counters, 0, sizeof(uint32_t) * kMaxStartQueries), "memset counters");
    BV_TRY(cudaMemset(t->start_cells, 0, sizeof(uint32_t) * kMaxViewsPerLaunch), "memset start cells");
    BV_TRY(cudaMalloc(&t->site_grads, sizeof(float4) * n), "cudaMalloc site grads");
    BV_TRY(cudaMemset(t->site_grads, 0, sizeof(float4) * n), "memset site grads");
    for (auto &ev : t->ev) BV_TRY(cudaEventCreate(&ev), "cudaEventCreate");
    t->grid_forward = walk_grid_size(device, 0);
    t->grid_train_fwd = walk_grid_size(device, 1);
    t->grid_train_bwd = walk_grid_size(device, 2);
    BV_TRY(cudaDeviceSynchronize(), "upload");
#undef BV_TRY
    *out = t;
    g_error.clear();
    return BV_OK;
}

void bv_radfoam_tracer_destroy(bv_tracer *t) {
    if (!t) return;
    cudaDeviceSynchronize();
    free_tracer(t);
}

bv_status bv_radfoam_tracer_dispatch_batch(bv_tracer *t, float *out_rgba_dev,
                                           const bv_camera *cams, uint32_t n_cams, uint32_t width,
                                           uint32_t height, bv_stream stream) {
    if (!t || !out_rgba_dev || !cams) return fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (width == 0 || height == 0) return fail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (n_cams == 0) return fail(BV_ERR_INVALID_ARGUMENT, "no cameras");
    if ((uint64_t)padded_rays(width, height) * kMaxViewsPerLaunch >= (1ull << 32))
        return fail(BV_ERR_INVALID_ARGUMENT, "image too large");
    for (uint32_t i = 0; i < n_cams; ++i) {
        bv_status s = check_camera(cams[i]);
        if (s != BV_OK) return s;
    }
    cudaStream_t s = (cudaStream_t)stream;
    bv_status st = begin_timing(t, s);
    if (st != BV_OK) return st;
    for (uint32_t c0 = 0; c0 < n_cams; c0 += kMaxViewsPerLaunch) {
        const uint32_t nc = std::min<uint32_t>(kMaxViewsPerLaunch, n_cams - c0);
        st = launch_starts(t, cams + c0, nc, s);
        if (st != BV_OK) return st;
        if (t->stats_enabled && c0 == 0) BV_CUDA(cudaEventRecord(t->ev[1], s), "event");
        WalkParams p;
        std::memset(&p, 0, sizeof(p));
        p.m = t->model();
        p.max_steps = t->settings.max_steps;
        p.weight_threshold = t->settings.weight_threshold;
        p.n_views = nc;
        uint32_t work = 0;
        for (uint32_t v = 0; v < nc; ++v) {
            p.views[v] = make_view(cams[c0 + v], width, height, work,
                                   (uint64_t)v * width * height);
            work += padded_rays(width, height);
        }
        p.total_work = work;
        p.start_cells = t->start_cells;
        p.work_counter = t->work_counter;
        p.stats = t->stats_enabled ? t->stats : nullptr;
        p.out_rgba = reinterpret_cast<float4 *>(out_rgba_dev) + (size_t)c0 * width * height;
        p.debug_cell_density = t->settings.debug_cell_density;
        p.tie_break = t->tie_break;
        BV_CUDA(cudaMemsetAsync(t->work_counter, 0, sizeof(uint32_t), s), "counter reset");
        const int blocks_needed = (int)((work + 255) / 256);
        const int grid = std::min(t->grid_forward, std::max(blocks_needed, 1));
        BV_CUDA(launch_walk_forward(p, grid, s), "walk launch");
        t->last_launches += 2;
    }
    if (t->stats_enabled) BV_CUDA(cudaEventRecord(t->ev[2], s), "event");
    t->start_point_pending = true;
    return BV_OK;
}

bv_status bv_radfoam_tracer_dispatch(bv_tracer *t, float *out_rgba_dev, const bv_camera *camera,
                                     uint32_t width, uint32_t height, bv_stream stream) {
    return bv_radfoam_tracer_dispatch_batch(t, out_rgba_dev, camera, 1, width, height, stream);
}

bv_status bv_radfoam_tracer_set_max_steps(bv_tracer *t, uint32_t max_steps) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->settings.max_steps = max_steps;
    return BV_OK;
}

bv_status bv_radfoam_tracer_set_weight_threshold(bv_tracer *t, float w) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->settings.weight_threshold = w;
    return BV_OK;
}

bv_status bv_radfoam_tracer_set_debug_cell_density(bv_tracer *t, uint32_t enabled) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->settings.debug_cell_density = enabled ? 1u : 0u;
    return BV_OK;
}

bv_status bv_radfoam_tracer_set_tie_break(bv_tracer *t, uint32_t mode) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    if (mode > BV_TIE_BREAK_F64) return fail(BV_ERR_INVALID_ARGUMENT, "unknown tie-break mode");
    t->tie_break = mode;
    return BV_OK;
}

bv_status bv_radfoam_tracer_set_exit_record(bv_tracer *t, uint32_t steps) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->step_rec_steps = steps;
    if (steps == 0 && t->step_rec_owned) {
        cudaFree(t->step_rec);
        t->step_rec = nullptr;
        t->step_rec_capacity = 0;
    }
    return BV_OK;
}

uint32_t bv_radfoam_tracer_max_steps(const bv_tracer *t) { return t ? t->settings.max_steps : 0; }
float bv_radfoam_tracer_weight_threshold(const bv_tracer *t) {
    return t ? t->settings.weight_threshold : 0.0f;
}
uint32_t bv_radfoam_tracer_sh_degree(const bv_tracer *t) { return t ? t->sh_degree : 0; }
uint32_t bv_radfoam_tracer_num_points(const bv_tracer *t) { return t ? t->n : 0; }

uint32_t bv_radfoam_tracer_start_point(bv_tracer *t) {
    if (!t) return 0;
    if (t->start_point_pending) {
        cudaStreamSynchronize(t->last_stream);
        cudaMemcpy(&t->last_start_point, t->start_cells, 4, cudaMemcpyDeviceToHost);
        t->start_point_pending = false;
    }
    return t->last_start_point;
}

bv_status bv_containing_point(bv_tracer *t, const float position[3], uint32_t *out_index) {
    if (!t || !position || !out_index) return fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (!std::isfinite(position[0]) || !std::isfinite(position[1]) || !std::isfinite(position[2]))
        return fail(BV_ERR_INVALID_ARGUMENT, "query position must be finite");
    bv_camera c;
    std::memset(&c, 0, sizeof(c));
    for (int i = 0; i < 3; ++i) c.cam_position[i] = position[i];
    cudaStream_t s = nullptr;
    bv_status st = launch_starts(t, &c, 1, s);
    if (st != BV_OK) return st;
    BV_CUDA(cudaMemcpy(out_index, t->start_cells, 4, cudaMemcpyDeviceToHost), "read start cell");
    t->start_point_pending = false;
    t->last_start_point = *out_index;
    return BV_OK;
}

bv_status bv_record_paths(bv_tracer *t, const bv_camera *cams, uint32_t n_cams, uint32_t width,
                          uint32_t height, const bv_path_buffers *buf, bv_stream stream) {
    if (!t || !cams || !buf) return fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (width == 0 || height == 0 || n_cams == 0)
        return fail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (buf->max_steps == 0 || buf->max_steps >= BV_PATH_TRUNCATED)
        return fail(BV_ERR_INVALID_ARGUMENT, "path-record max_steps exceeds status encoding");
    for (uint32_t i = 0; i < n_cams; ++i) {
        bv_status s = check_camera(cams[i]);
        if (s != BV_OK) return s;
    }
    cudaStream_t s = (cudaStream_t)stream;
    bv_status st = begin_timing(t, s);
    if (st != BV_OK) return st;
    for (uint32_t c0 = 0; c0 < n_cams; c0 += kMaxViewsPerLaunch) {
        const uint32_t nc = std::min<uint32_t>(kMaxViewsPerLaunch, n_cams - c0);
        st = launch_starts(t, cams + c0, nc, s);
        if (st != BV_OK) return st;
        RecordParams p;
        std::memset(&p, 0, sizeof(p));
        p.m = t->model();
        p.max_steps = buf->max_steps;
        p.n_views = nc;
        uint32_t work = 0;
        const uint64_t pix0 = (uint64_t)c0 * width * height;
        for (uint32_t v = 0; v < nc; ++v) {
            p.views[v] = make_view(cams[c0 + v], width, height, work, pix0 + (uint64_t)v * width * height);
            work += padded_rays(width, height);
        }
        p.total_work = work;
        p.start_cells = t->start_cells;
        p.work_counter = t->work_counter;
        p.buf = *buf;
        BV_CUDA(launch_record_paths(p, 0, s), "record launch");
        t->last_launches += 2;
    }
    if (t->stats_enabled) {
        BV_CUDA(cudaEventRecord(t->ev[1], s), "event");
        BV_CUDA(cudaEventRecord(t->ev[2], s), "event");
    }
    return BV_OK;
}

bv_status bv_forward_backward(bv_tracer *t, const bv_camera *cams, uint32_t n_cams,
                              uint32_t width, uint32_t height, const float *target,
                              const bv_train_settings *ts, const bv_grads *grads, float *loss,
                              float *rgb_out, bv_stream stream) {
    if (!t || !cams || !target || !ts || !grads || !loss)
        return fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    if (!grads->d_density_dev || !grads->d_sh_dev)
        return fail(BV_ERR_INVALID_ARGUMENT, "density and SH gradient tables are required");
    if (width == 0 || height == 0 || n_cams == 0)
        return fail(BV_ERR_INVALID_ARGUMENT, "render size must be non-zero");
    if (ts->loss != BV_LOSS_L2 && ts->loss != BV_LOSS_L1)
        return fail(BV_ERR_INVALID_ARGUMENT, "unknown loss %u", ts->loss);
    if (!(ts->max_dt > 0.0f)) return fail(BV_ERR_INVALID_ARGUMENT, "max_dt must be positive");
    if (grads->d_radii_dev && !t->bounded)
        return fail(BV_ERR_INVALID_ARGUMENT, "radius gradients need a PowerFoam model");
    const uint32_t nsh = 3 * sh_components(t->sh_degree);
    if ((size_t)std::min<uint32_t>(n_cams, kMaxViewsPerLaunch) * width * height >= (1ull << 31))
        return fail(BV_ERR_INVALID_ARGUMENT, "batch too large");
    if ((nsh % 4) == 0 && (reinterpret_cast<uintptr_t>(grads->d_sh_dev) & 15u) != 0)
        return fail(BV_ERR_INVALID_ARGUMENT, "d_sh table must be 16-byte aligned");
    for (uint32_t i = 0; i < n_cams; ++i) {
        bv_status s = check_camera(cams[i]);
        if (s != BV_OK) return s;
    }
    cudaStream_t s = (cudaStream_t)stream;
    // per-ray state scratch for the largest chunk of this call
    const size_t chunk_rays = (size_t)std::min<uint32_t>(n_cams, kMaxViewsPerLaunch) * width * height;
    if (chunk_rays > t->ray_state_capacity && !t->ray_state_owned)
        return fail(BV_ERR_INVALID_ARGUMENT, "batch exceeds the lent ray-state scratch (%zu rays)",
                    t->ray_state_capacity);
    if (chunk_rays > t->ray_state_capacity) {
        cudaFree(t->ray_state);
        t->ray_state = nullptr;
        t->ray_state_capacity = 0;
        BV_CUDA(cudaMalloc(&t->ray_state, sizeof(RayState) * chunk_rays), "cudaMalloc ray state");
        t->ray_state_capacity = chunk_rays;
    }
    // step record: the first rec_steps steps of every ray of a launch, within
    // kExitRecBytes (or the buffer a serving engine lends, which budgets its
    // device memory itself); steps past the record replay the exit-face
    // search and the SH evaluation instead
    const size_t group_work =
        (size_t)std::min<uint32_t>(n_cams, kMaxViewsPerLaunch) * padded_rays(width, height);
    const size_t chunk_work = t->train_chunk ? std::min<size_t>(t->train_chunk, group_work) : group_work;
    uint32_t rec_steps = 0;
    if (t->step_rec_owned) {
        const size_t fit = kExitRecBytes / (chunk_work * kStepRecWords * sizeof(uint32_t));
        rec_steps = (uint32_t)std::min<size_t>({(size_t)t->step_rec_steps, (size_t)ts->max_steps, fit});
        const size_t need = chunk_work * rec_steps * kStepRecWords;
        if (rec_steps > 0 && need > t->step_rec_capacity) {
            cudaFree(t->step_rec);
            t->step_rec = nullptr;
            t->step_rec_capacity = 0;
            if (cudaMalloc(&t->step_rec, need * sizeof(uint32_t)) == cudaSuccess) {
                t->step_rec_capacity = need;
            } else {
                (void)cudaGetLastError();  // out of memory: replay searches
                t->step_rec = nullptr;
                rec_steps = 0;
            }
        }
    }
    if (!t->step_rec_owned && t->step_rec) {
        const size_t fit = t->step_rec_capacity / (chunk_work * kStepRecWords);
        rec_steps = (uint32_t)std::min<size_t>({(size_t)t->step_rec_steps, (size_t)ts->max_steps, fit});
    }
    // heaviest-first tiles (calls of one launch pair): the forward times its
    // tiles, the order for the next call of the same shape is built after it
    const uint32_t *order = nullptr;
    const size_t order_tiles = group_work / 32u;
    const bool time_tiles = n_cams <= (uint32_t)kMaxViewsPerLaunch && chunk_work == group_work &&
                            t->train_order.begin(BV_WALK_TILE_ORDER, order_tiles, n_cams, width,
                                                 height, order);
    bv_status st = begin_timing(t, s);
    if (st != BV_OK) return st;
    BV_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), s), "loss reset");
    const double total_rays = (double)n_cams * width * height;
    for (uint32_t c0 = 0; c0 < n_cams; c0 += kMaxViewsPerLaunch) {
        const uint32_t nc = std::min<uint32_t>(kMaxViewsPerLaunch, n_cams - c0);
        st = launch_starts(t, cams + c0, nc, s);
        if (st != BV_OK) return st;
        if (t->stats_enabled && c0 == 0) BV_CUDA(cudaEventRecord(t->ev[1], s), "event");
        TrainParams p;
        std::memset(&p, 0, sizeof(p));
        p.m = t->model();
        p.max_steps = ts->max_steps;
        p.weight_threshold = ts->weight_threshold;
        p.max_dt = ts->max_dt;
        p.loss_kind = ts->loss;
        p.inv_count = (float)(1.0 / (3.0 * total_rays));
        p.n_views = nc;
        uint32_t work = 0;
        for (uint32_t v = 0; v < nc; ++v) {
            p.views[v] = make_view(cams[c0 + v], width, height, work, (uint64_t)v * width * height);
            work += padded_rays(width, height);
        }
        const size_t off = (size_t)c0 * width * height;
        p.start_cells = t->start_cells;
        p.work_counter = t->work_counter;
        p.target = target + 3 * off;
        p.rgb_out = rgb_out ? rgb_out + 3 * off : nullptr;
        p.ray_state = t->ray_state;
        p.d_density = grads->d_density_dev;
        p.d_sh = grads->d_sh_dev;
        p.d_site = (grads->d_positions_dev || grads->d_radii_dev) ? t->site_grads : nullptr;
        p.loss = loss;
        p.stats = t->stats_enabled ? t->stats : nullptr;
        p.step_rec = rec_steps ? t->step_rec : nullptr;
        p.rec_steps = rec_steps;
        // mode 2: the replay takes `order`, the forward its own second order
        p.tile_order = BV_WALK_TILE_ORDER == 1 ? order : t->train_order.second(order);
        p.tile_cost = time_tiles ? t->train_order.cost : nullptr;
        t->last_launches += 1;  // start cells
        for (uint32_t b = 0; b < work; b += (uint32_t)chunk_work) {
            p.work_begin = b;
            p.total_work = std::min<uint32_t>((uint32_t)chunk_work, work - b);
            BV_CUDA(cudaMemsetAsync(t->work_counter, 0, 2 * sizeof(uint32_t), s), "counter reset");
            const int blocks_needed = std::max((int)((p.total_work + 255) / 256), 1);
            BV_CUDA(launch_train_forward(p, std::min(t->grid_train_fwd, blocks_needed), s),
                    "training forward launch");
            if (t->stats_enabled && c0 == 0 && b == 0) BV_CUDA(cudaEventRecord(t->ev[3], s), "event");
            const uint32_t *fwd_order = p.tile_order;
            p.tile_order = order;
            BV_CUDA(launch_train_backward(p, std::min(t->grid_train_bwd, blocks_needed), s),
                    "training backward launch");
            p.tile_order = fwd_order;
            t->last_launches += 2;
        }
    }
    if (grads->d_positions_dev || grads->d_radii_dev) {
        BV_CUDA(launch_fold_site_grads(t->site_grads, t->n, grads->d_positions_dev,
                                       grads->d_radii_dev, s), "site gradient fold");
        t->last_launches += 1;
    }
    if (t->stats_enabled) BV_CUDA(cudaEventRecord(t->ev[2], s), "event");
    if (time_tiles) {
        BV_CUDA(t->train_order.end(order_tiles, n_cams, width, height, s), "tile order");
        t->last_launches += t->train_order.order_launches();
    }
    t->start_point_pending = true;
    t->last_train = true;
    return BV_OK;
}

bv_status bv_radfoam_tracer_enable_stats(bv_tracer *t, uint32_t enabled) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    t->stats_enabled = enabled != 0;
    return BV_OK;
}

bv_status bv_radfoam_tracer_last_stats(bv_tracer *t, bv_launch_stats *out) {
    if (!t || !out) return fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->launches = t->last_launches;
    if (!t->last_has_stats) return BV_OK;
    BV_CUDA(cudaEventSynchronize(t->ev[2]), "event sync");
    float a = 0.f, b = 0.f;
    BV_CUDA(cudaEventElapsedTime(&a, t->ev[0], t->ev[1]), "elapsed");
    BV_CUDA(cudaEventElapsedTime(&b, t->ev[1], t->ev[2]), "elapsed");
    out->start_cell_ms = a;
    out->kernel_ms = b;
    if (t->last_train) {
        float f = 0.f;
        BV_CUDA(cudaEventElapsedTime(&f, t->ev[1], t->ev[3]), "elapsed");
        out->forward_ms = f;
        out->backward_ms = b - f;
    }
    unsigned long long h[4] = {0, 0, 0, 0};
    BV_CUDA(cudaMemcpy(h, t->stats, sizeof(h), cudaMemcpyDeviceToHost), "stats read");
    out->rays = h[0];
    out->steps = h[1];
    out->faces = h[2];
    return BV_OK;
}

bv_status bv_radfoam_tracer_adam_step(bv_tracer *t, const bv_grads *g, const bv_adam_settings *a,
                                      bv_stream stream) {
    if (!t || !g || !a) return fail(BV_ERR_INVALID_ARGUMENT, "null argument");
    const float rates[5] = {a->lr_density, a->lr_sh_dc, a->lr_sh_rest, a->lr_position,
                            a->lr_radius};
    for (float r : rates)
        if (!std::isfinite(r) || r < 0.0f)
            return fail(BV_ERR_INVALID_ARGUMENT, "learning rates must be finite and >= 0");
    if (!(a->beta1 >= 0.0f && a->beta1 < 1.0f && a->beta2 >= 0.0f && a->beta2 < 1.0f))
        return fail(BV_ERR_INVALID_ARGUMENT, "Adam betas must lie in [0, 1)");
    if (!(std::isfinite(a->eps) && a->eps >= 0.0f))
        return fail(BV_ERR_INVALID_ARGUMENT, "Adam eps must be finite and >= 0");
    if (a->density_activation > BV_DENSITY_SOFTPLUS)
        return fail(BV_ERR_INVALID_ARGUMENT, "unknown density activation %u", a->density_activation);
    if (a->density_activation == BV_DENSITY_SOFTPLUS &&
        !(std::isfinite(a->softplus_beta) && a->softplus_beta > 0.0f))
        return fail(BV_ERR_INVALID_ARGUMENT, "softplus beta must be finite and positive");
    if (g->d_radii_dev && !t->bounded)
        return fail(BV_ERR_INVALID_ARGUMENT, "radius gradients need a PowerFoam model");
    const uint32_t nsh = 3 * sh_components(t->sh_degree);
    if ((uint64_t)t->n * nsh >= (1ull << 31))
        return fail(BV_ERR_NOT_SUPPORTED, "more than 2^31 SH coefficients for the optimizer");
    const float beta = a->density_activation == BV_DENSITY_SOFTPLUS ? a->softplus_beta : 0.0f;
    cudaStream_t s = (cudaStream_t)stream;
    if (!t->adam_buf) {
        // raw density + 2 moments, (master) SH + 2 moments, positions and radii moments
        const size_t n = t->n;
        const size_t total = 3 * n + 3 * n * nsh + 6 * n + 2 * n;
        BV_CUDA(cudaMalloc(&t->adam_buf, sizeof(float) * total), "cudaMalloc optimizer state");
        float *q = t->adam_buf;
        t->density_param = q; q += n;
        t->m_density = q; q += n;
        t->v_density = q; q += n;
        t->sh_master = q; q += n * nsh;
        t->m_sh = q; q += n * nsh;
        t->v_sh = q; q += n * nsh;
        t->m_pos = q; q += 3 * n;
        t->v_pos = q; q += 3 * n;
        t->m_radius = q; q += n;
        t->v_radius = q;
        BV_CUDA(cudaMemsetAsync(t->m_density, 0, sizeof(float) * 2 * n, s), "zero moments");
        BV_CUDA(cudaMemsetAsync(t->m_sh, 0, sizeof(float) * 2 * n * nsh, s), "zero moments");
        BV_CUDA(cudaMemsetAsync(t->m_pos, 0, sizeof(float) * 8 * n, s), "zero moments");
        if (t->bf16) {
            // the FP32 master copy starts at the stored BF16 values (exact widening)
            std::vector<uint16_t> rows(n * t->sh_stride);
            BV_CUDA(cudaMemcpy(rows.data(), t->sh, rows.size() * 2, cudaMemcpyDeviceToHost),
                    "read SH");
            std::vector<float> master(n * nsh);
            for (size_t i = 0; i < n; ++i)
                for (uint32_t k = 0; k < nsh; ++k) {
                    const uint32_t u = (uint32_t)rows[i * t->sh_stride + k] << 16;
                    std::memcpy(&master[i * nsh + k], &u, 4);
                }
            BV_CUDA(cudaMemcpyAsync(t->sh_master, master.data(), sizeof(float) * master.size(),
                                    cudaMemcpyHostToDevice, s), "upload SH master");
            BV_CUDA(cudaStreamSynchronize(s), "SH master upload");
        }
        BV_CUDA(launch_init_density_param(t->density, t->density_param, t->n,
                                          a->density_activation, beta, s),
                "density parameter init");
        t->adam_activation = a->density_activation;
        t->adam_beta = beta;
        t->adam_t = 0;
    } else if (a->density_activation != t->adam_activation || beta != t->adam_beta) {
        return fail(BV_ERR_INVALID_ARGUMENT,
                    "the density activation is fixed by the first optimizer step");
    }
    t->adam_t += 1;
    AdamParams p;
    std::memset(&p, 0, sizeof(p));
    p.n = t->n;
    p.sh_row = nsh;
    p.sh_stride = t->sh_stride;
    p.s.beta1 = a->beta1;
    p.s.beta2 = a->beta2;
    p.s.one_minus_beta1 = 1.0f - a->beta1;
    p.s.one_minus_beta2 = 1.0f - a->beta2;
    p.s.c1 = (float)(1.0 - std::pow((double)a->beta1, (double)t->adam_t));
    p.s.c2 = (float)(1.0 - std::pow((double)a->beta2, (double)t->adam_t));
    p.s.eps = a->eps;
    p.lr_density = a->lr_density;
    p.lr_sh_dc = a->lr_sh_dc;
    p.lr_sh_rest = a->lr_sh_rest;
    p.lr_position = a->lr_position;
    p.lr_radius = a->lr_radius;
    p.activation = a->density_activation;
    p.softplus_beta = beta;
    p.density_param = t->density_param;
    p.density = t->density;
    p.g_density = g->d_density_dev;
    p.m_density = t->m_density;
    p.v_density = t->v_density;
    p.sh = t->sh;
    p.sh_master = t->sh_master;
    p.g_sh = g->d_sh_dev;
    p.m_sh = t->m_sh;
    p.v_sh = t->v_sh;
    p.geom = t->geom;
    p.g_pos = g->d_positions_dev;
    p.m_pos = t->m_pos;
    p.v_pos = t->v_pos;
    p.g_radius = t->bounded ? g->d_radii_dev : nullptr;
    p.m_radius = t->m_radius;
    p.v_radius = t->v_radius;
    BV_CUDA(launch_adam_step(p, t->faces, t->m_edges, t->bf16, s), "optimizer launch");
    return BV_OK;
}

uint32_t bv_radfoam_tracer_adam_steps(const bv_tracer *t) { return t ? t->adam_t : 0; }

bv_status bv_radfoam_tracer_read_model(bv_tracer *t, float *points, float *sh, float *radii) {
    if (!t) return fail(BV_ERR_INVALID_ARGUMENT, "null tracer");
    if (radii && !t->bounded) return fail(BV_ERR_INVALID_ARGUMENT, "the model has no radii");
    BV_CUDA(cudaDeviceSynchronize(), "synchronize");
    const size_t n = t->n;
    if (points || radii) {
        std::vector<float4> geom(n);
        std::vector<float> dens(n);
        BV_CUDA(cudaMemcpy(geom.data(), t->geom, sizeof(float4) * n, cudaMemcpyDeviceToHost),
                "read sites");
        BV_CUDA(cudaMemcpy(dens.data(), t->density, sizeof(float) * n, cudaMemcpyDeviceToHost),
                "read densities");
        for (size_t i = 0; i < n; ++i) {
            if (points) {
                points[4 * i + 0] = geom[i].x;
                points[4 * i + 1] = geom[i].y;
                points[4 * i + 2] = geom[i].z;
                points[4 * i + 3] = dens[i];
            }
            if (radii) radii[i] = geom[i].w;
        }
    }
    if (sh) {
        const uint32_t nsh = 3 * sh_components(t->sh_degree);
        if (t->bf16) {
            std::vector<uint16_t> rows(n * t->sh_stride);
            BV_CUDA(cudaMemcpy(rows.data(), t->sh, rows.size() * 2, cudaMemcpyDeviceToHost),
                    "read SH");
            for (size_t i = 0; i < n; ++i)
                for (uint32_t k = 0; k < nsh; ++k) {
                    const uint32_t u = (uint32_t)rows[i * t->sh_stride + k] << 16;
                    std::memcpy(&sh[i * nsh + k], &u, 4);
                }
        } else {
            std::vector<float> rows(n * t->sh_stride);
            BV_CUDA(cudaMemcpy(rows.data(), t->sh, rows.size() * 4, cudaMemcpyDeviceToHost),
                    "read SH");
            for (size_t i = 0; i < n; ++i)
                std::memcpy(&sh[i * nsh], &rows[i * t->sh_stride], sizeof(float) * nsh);
        }
    }
    return BV_OK;
}

}  // extern "C"
