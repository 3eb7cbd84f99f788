"""blade_volume_b200: B200 (sm_100a) ray-tracing hot path of blade-volume.

Python mirror of the reference crate's tracer API over the C ABI of
libbv_b200.so (include/blade_volume_b200.h):

* :class:`RadFoamGpuTracer`   blade-volume/src/gpu/radfoam_trace.rs:56-177
* :meth:`RadFoamGpuTracer.record_paths`   gpu/path_record.rs:519-594
* :meth:`RadFoamGpuTracer.forward_backward`   the trainer's gradient
  (blade-volume-train/src/diff_render.rs:943-1923, :7181-7226)
* :class:`PowerFoamSplatTracer`   gpu/powerfoam_splat.rs:38-370
* :class:`GaussianTracer`   gpu/gaussian.rs:94-280 + shaders/gaussian.wgsl
* :class:`RelightTracer`   gpu/relight.rs:313-934
* :class:`Server`   the serving loop (no counterpart in the reference)

Device buffers are torch CUDA tensors (torch is only the allocator and the
stream provider here).  There is no CPU fallback: constructing a tracer
without the CUDA library or without a GPU raises.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from .scenes import Camera, PointCloudModel  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
# BV_B200_LIBRARY selects another build of the same library (tuning sweeps).
LIB_PATH = os.environ.get("BV_B200_LIBRARY", os.path.join(HERE, "libbv_b200.so"))

BV_OK = 0
STATUS_NAMES = {0: "BV_OK", 1: "BV_ERR_INVALID_ARGUMENT", 2: "BV_ERR_INVALID_MODEL",
                3: "BV_ERR_CUDA", 4: "BV_ERR_OUT_OF_MEMORY", 5: "BV_ERR_CANDIDATE_OVERFLOW",
                6: "BV_ERR_NOT_SUPPORTED", 7: "BV_ERR_NO_DEVICE", 8: "BV_ERR_TIMEOUT",
                9: "BV_ERR_CANCELLED"}
MODEL_SH_BF16 = 0x1
PATH_TRUNCATED = 0x80000000
LOSS_L2, LOSS_L1 = 0, 1

# Every symbol include/blade_volume_b200.h declares.
EXPORTED_SYMBOLS = [
    "bv_last_error", "bv_abi_version", "bv_model_validate", "bv_radfoam_tracer_new",
    "bv_radfoam_tracer_destroy", "bv_radfoam_tracer_dispatch", "bv_radfoam_tracer_dispatch_batch",
    "bv_radfoam_tracer_set_max_steps", "bv_radfoam_tracer_set_weight_threshold",
    "bv_radfoam_tracer_set_debug_cell_density", "bv_radfoam_tracer_set_tie_break",
    "bv_radfoam_tracer_set_exit_record",
    "bv_radfoam_tracer_max_steps",
    "bv_radfoam_tracer_weight_threshold", "bv_radfoam_tracer_sh_degree",
    "bv_radfoam_tracer_start_point", "bv_radfoam_tracer_num_points", "bv_containing_point",
    "bv_record_paths", "bv_forward_backward", "bv_radfoam_tracer_enable_stats",
    "bv_radfoam_tracer_last_stats", "bv_containing_points_noalloc",
    "bv_relight_tracer_new_gaussian", "bv_relight_tracer_destroy",
    "bv_relight_tracer_set_point_lights", "bv_relight_tracer_set_background",
    "bv_relight_tracer_dispatch", "bv_relight_tracer_num_particles",
    "bv_relight_tracer_enable_stats", "bv_relight_tracer_last_stats",
    "bv_server_new", "bv_server_add_scene", "bv_server_scene_grads", "bv_server_start",
    "bv_server_submit", "bv_server_wait", "bv_server_stats_get", "bv_server_clock",
    "bv_server_destroy", "bv_server_cancel",
    "bv_powerfoam_splat_tracer_new", "bv_powerfoam_splat_tracer_destroy",
    "bv_powerfoam_splat_tracer_dispatch", "bv_powerfoam_splat_tracer_dispatch_batch",
    "bv_powerfoam_splat_tracer_validate_candidate_counts",
    "bv_powerfoam_splat_tracer_candidate_stats",
    "bv_powerfoam_splat_tracer_candidate_capacity", "bv_powerfoam_splat_tracer_max_steps",
    "bv_powerfoam_splat_tracer_weight_threshold",
    "bv_powerfoam_splat_tracer_set_weight_threshold", "bv_powerfoam_splat_tracer_enable_stats",
    "bv_powerfoam_splat_tracer_set_interval_record",
    "bv_powerfoam_splat_tracer_last_stats",
    "bv_gaussian_tracer_new", "bv_gaussian_tracer_destroy",
    "bv_gaussian_tracer_set_min_transmittance", "bv_gaussian_tracer_set_background",
    "bv_gaussian_tracer_num_points", "bv_gaussian_tracer_dispatch",
    "bv_gaussian_tracer_enable_stats", "bv_gaussian_tracer_last_stats",
    "bv_radfoam_tracer_adam_step", "bv_radfoam_tracer_adam_steps", "bv_radfoam_tracer_read_model",
    "bv_powerfoam_splat_tracer_forward_backward",
    "bv_radfoam_ply_info", "bv_radfoam_ply_read",
]
DENSITY_IDENTITY, DENSITY_RELU, DENSITY_SOFTPLUS = 0, 1, 2
SERVE_BATCHED, SERVE_PLAIN, SERVE_PLAIN_BATCH = 0, 1, 2
REQUEST_RENDER, REQUEST_FORWARD_BACKWARD = 0, 1
SCENE_GRADIENTS = 0x1
SERVE_NO_RECORD = 0xFFFFFFFF
BV_ERR_TIMEOUT = 8
BV_ERR_CANCELLED = 9


class BvError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class ModelDesc(C.Structure):
    _fields_ = [("num_points", C.c_uint32), ("sh_degree", C.c_uint32),
                ("points", C.POINTER(C.c_float)), ("sh_coefficients", C.POINTER(C.c_float)),
                ("radii", C.POINTER(C.c_float)), ("adjacency_offsets", C.POINTER(C.c_uint32)),
                ("adjacency_neighbors", C.POINTER(C.c_uint32)), ("flags", C.c_uint32),
                ("reserved", C.c_uint32)]


class PlyInfo(C.Structure):
    _fields_ = [("num_points", C.c_uint32), ("num_adjacency", C.c_uint32),
                ("sh_degree", C.c_uint32), ("has_radii", C.c_uint32)]


class CameraC(C.Structure):
    _fields_ = [("cam_position", C.c_float * 3), ("depth", C.c_float),
                ("cam_orientation", C.c_float * 4), ("fov", C.c_float * 2),
                ("principal", C.c_float * 2)]


class TraceSettings(C.Structure):
    _fields_ = [("max_steps", C.c_uint32), ("powerfoam_candidate_capacity", C.c_uint32),
                ("weight_threshold", C.c_float), ("debug_cell_density", C.c_uint32)]


class PathBuffers(C.Structure):
    _fields_ = [("previous_cells_dev", C.c_void_p), ("cells_dev", C.c_void_p),
                ("next_cells_dev", C.c_void_p), ("dts_dev", C.c_void_p),
                ("dt_grad_previous_dev", C.c_void_p), ("dt_grad_current_dev", C.c_void_p),
                ("dt_grad_next_dev", C.c_void_p), ("path_status_dev", C.c_void_p),
                ("max_steps", C.c_uint32), ("reserved", C.c_uint32)]


class TrainSettings(C.Structure):
    _fields_ = [("max_steps", C.c_uint32), ("weight_threshold", C.c_float),
                ("max_dt", C.c_float), ("loss", C.c_uint32)]


class Grads(C.Structure):
    _fields_ = [("d_density_dev", C.c_void_p), ("d_sh_dev", C.c_void_p),
                ("d_positions_dev", C.c_void_p), ("d_radii_dev", C.c_void_p)]


class LaunchStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_float), ("start_cell_ms", C.c_float),
                ("forward_ms", C.c_float), ("backward_ms", C.c_float), ("rays", C.c_uint64),
                ("steps", C.c_uint64), ("faces", C.c_uint64), ("launches", C.c_uint32),
                ("reserved", C.c_uint32)]


class AdamSettingsC(C.Structure):
    _fields_ = [("lr_density", C.c_float), ("lr_sh_dc", C.c_float), ("lr_sh_rest", C.c_float),
                ("lr_position", C.c_float), ("lr_radius", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("density_activation", C.c_uint32),
                ("softplus_beta", C.c_float)]


class MaterialC(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("roughness", C.c_float),
                ("specular_f0", C.c_float * 3), ("pad", C.c_float)]


class PointLightC(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("direction", C.c_float * 3),
                ("intensity", C.c_float * 3), ("exponent", C.c_float)]


class GaussianDesc(C.Structure):
    _fields_ = [("num_points", C.c_uint32), ("num_materials", C.c_uint32),
                ("points", C.POINTER(C.c_float)), ("rotations", C.POINTER(C.c_float)),
                ("scales", C.POINTER(C.c_float)), ("normals", C.POINTER(C.c_float)),
                ("material_indices", C.POINTER(C.c_uint32)), ("materials", C.c_void_p)]


class GaussianShDesc(C.Structure):
    _fields_ = [("num_points", C.c_uint32), ("sh_degree", C.c_uint32),
                ("points", C.POINTER(C.c_float)), ("rotations", C.POINTER(C.c_float)),
                ("scales", C.POINTER(C.c_float)), ("sh_coefficients", C.POINTER(C.c_float))]


class GaussianTraceSettingsC(C.Structure):
    _fields_ = [("min_opacity", C.c_float), ("min_transmittance", C.c_float),
                ("background", C.c_float * 3)]


class RelightSettings(C.Structure):
    _fields_ = [("background", C.c_float * 3), ("diffuse_samples", C.c_uint32)]


class ServerSettings(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("mode", C.c_uint32),
                ("max_batch_rays", C.c_uint32), ("max_batch_views", C.c_uint32),
                ("slots", C.c_uint32), ("max_steps", C.c_uint32), ("weight_threshold", C.c_float),
                ("max_train_rays", C.c_uint64), ("use_graphs", C.c_uint32),
                ("train_chunk_rays", C.c_uint32), ("frame_period_us", C.c_uint32),
                ("train_record_steps", C.c_uint32)]


class RequestC(C.Structure):
    _fields_ = [("scene", C.c_uint32), ("kind", C.c_uint32), ("n_views", C.c_uint32),
                ("width", C.c_uint32), ("height", C.c_uint32), ("reserved", C.c_uint32),
                ("cameras", C.POINTER(CameraC)), ("out_host", C.c_void_p),
                ("target_host", C.c_void_p), ("loss_host", C.c_void_p),
                ("train", TrainSettings), ("grads", Grads), ("frame_done_host", C.c_void_p)]


class RequestResult(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int32), ("kind", C.c_uint32),
                ("submit_s", C.c_double), ("admit_s", C.c_double), ("start_s", C.c_double),
                ("done_s", C.c_double), ("rays", C.c_uint64), ("message", C.c_char * 128)]


class ServerStats(C.Structure):
    _fields_ = [("requests_done", C.c_uint64), ("frames_done", C.c_uint64),
                ("rays_done", C.c_uint64), ("batches", C.c_uint64),
                ("graph_launches", C.c_uint64), ("kernel_launches", C.c_uint64),
                ("arena_bytes", C.c_uint64), ("arena_peak_bytes", C.c_uint64),
                ("resident_bytes", C.c_uint64), ("admission_waits", C.c_uint64),
                ("busy_s", C.c_double), ("arena_used_bytes", C.c_uint64),
                ("requests_cancelled", C.c_uint64)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libbv_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build it with `python -m blade_volume_b200.build` (nvcc, sm_100a)")
    L = C.CDLL(path)
    L.bv_last_error.restype = C.c_char_p
    L.bv_abi_version.restype = C.c_uint32
    L.bv_model_validate.argtypes = [C.POINTER(ModelDesc), C.c_char_p, C.c_size_t]
    L.bv_radfoam_ply_info.argtypes = [C.c_char_p, C.POINTER(PlyInfo)]
    L.bv_radfoam_ply_read.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]
    L.bv_radfoam_tracer_new.argtypes = [C.POINTER(ModelDesc), C.POINTER(TraceSettings),
                                        C.POINTER(C.c_void_p)]
    L.bv_radfoam_tracer_destroy.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_destroy.restype = None
    L.bv_radfoam_tracer_dispatch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(CameraC),
                                             C.c_uint32, C.c_uint32, C.c_void_p]
    L.bv_radfoam_tracer_dispatch_batch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(CameraC),
                                                   C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p]
    L.bv_radfoam_tracer_set_max_steps.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_radfoam_tracer_set_weight_threshold.argtypes = [C.c_void_p, C.c_float]
    L.bv_radfoam_tracer_set_debug_cell_density.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_radfoam_tracer_set_tie_break.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_radfoam_tracer_set_exit_record.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_radfoam_tracer_max_steps.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_max_steps.restype = C.c_uint32
    L.bv_radfoam_tracer_weight_threshold.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_weight_threshold.restype = C.c_float
    L.bv_radfoam_tracer_sh_degree.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_sh_degree.restype = C.c_uint32
    L.bv_radfoam_tracer_start_point.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_start_point.restype = C.c_uint32
    L.bv_radfoam_tracer_num_points.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_num_points.restype = C.c_uint32
    L.bv_containing_point.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32)]
    L.bv_record_paths.argtypes = [C.c_void_p, C.POINTER(CameraC), C.c_uint32, C.c_uint32,
                                  C.c_uint32, C.POINTER(PathBuffers), C.c_void_p]
    L.bv_forward_backward.argtypes = [C.c_void_p, C.POINTER(CameraC), C.c_uint32, C.c_uint32,
                                      C.c_uint32, C.c_void_p, C.POINTER(TrainSettings),
                                      C.POINTER(Grads), C.c_void_p, C.c_void_p, C.c_void_p]
    L.bv_radfoam_tracer_enable_stats.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_radfoam_tracer_last_stats.argtypes = [C.c_void_p, C.POINTER(LaunchStats)]
    L.bv_containing_points_noalloc.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(C.c_float),
                                               C.c_uint32, C.c_void_p, C.c_void_p]
    L.bv_relight_tracer_new_gaussian.argtypes = [C.POINTER(GaussianDesc),
                                                 C.POINTER(RelightSettings), C.POINTER(C.c_void_p)]
    L.bv_relight_tracer_destroy.argtypes = [C.c_void_p]
    L.bv_relight_tracer_destroy.restype = None
    L.bv_relight_tracer_set_point_lights.argtypes = [C.c_void_p, C.POINTER(PointLightC),
                                                     C.c_uint32]
    L.bv_relight_tracer_set_background.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    L.bv_relight_tracer_dispatch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(CameraC),
                                             C.c_uint32, C.c_uint32, C.c_void_p]
    L.bv_relight_tracer_num_particles.argtypes = [C.c_void_p]
    L.bv_relight_tracer_num_particles.restype = C.c_uint32
    L.bv_relight_tracer_enable_stats.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_relight_tracer_last_stats.argtypes = [C.c_void_p, C.POINTER(LaunchStats)]
    L.bv_server_new.argtypes = [C.POINTER(ServerSettings), C.POINTER(C.c_void_p)]
    L.bv_server_add_scene.argtypes = [C.c_void_p, C.POINTER(ModelDesc), C.c_uint32,
                                      C.POINTER(C.c_uint32)]
    L.bv_server_scene_grads.argtypes = [C.c_void_p, C.c_uint32, C.POINTER(Grads)]
    L.bv_server_start.argtypes = [C.c_void_p]
    L.bv_server_submit.argtypes = [C.c_void_p, C.POINTER(RequestC), C.POINTER(C.c_uint64)]
    L.bv_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(RequestResult)]
    L.bv_server_stats_get.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
    L.bv_server_cancel.argtypes = [C.c_void_p, C.c_uint64]
    L.bv_server_clock.argtypes = [C.c_void_p]
    L.bv_server_clock.restype = C.c_double
    L.bv_server_destroy.argtypes = [C.c_void_p]
    L.bv_server_destroy.restype = None
    L.bv_powerfoam_splat_tracer_new.argtypes = [C.POINTER(ModelDesc), C.POINTER(TraceSettings),
                                                C.POINTER(C.c_void_p)]
    L.bv_powerfoam_splat_tracer_destroy.argtypes = [C.c_void_p]
    L.bv_powerfoam_splat_tracer_destroy.restype = None
    L.bv_powerfoam_splat_tracer_dispatch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(CameraC),
                                                     C.c_uint32, C.c_uint32, C.c_void_p]
    L.bv_powerfoam_splat_tracer_dispatch_batch.argtypes = [C.c_void_p, C.c_void_p,
                                                           C.POINTER(CameraC), C.c_uint32,
                                                           C.c_uint32, C.c_uint32, C.c_void_p]
    L.bv_powerfoam_splat_tracer_validate_candidate_counts.argtypes = [C.c_void_p,
                                                                      C.POINTER(C.c_uint32)]
    L.bv_powerfoam_splat_tracer_candidate_stats.argtypes = [
        C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
    for name in ("candidate_capacity", "max_steps"):
        f = getattr(L, "bv_powerfoam_splat_tracer_" + name)
        f.argtypes = [C.c_void_p]
        f.restype = C.c_uint32
    L.bv_powerfoam_splat_tracer_weight_threshold.argtypes = [C.c_void_p]
    L.bv_powerfoam_splat_tracer_weight_threshold.restype = C.c_float
    L.bv_powerfoam_splat_tracer_set_weight_threshold.argtypes = [C.c_void_p, C.c_float]
    L.bv_powerfoam_splat_tracer_enable_stats.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_powerfoam_splat_tracer_set_interval_record.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_powerfoam_splat_tracer_last_stats.argtypes = [C.c_void_p, C.POINTER(LaunchStats)]
    L.bv_powerfoam_splat_tracer_forward_backward.argtypes = [
        C.c_void_p, C.POINTER(CameraC), C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
        C.POINTER(TrainSettings), C.POINTER(Grads), C.c_void_p, C.c_void_p, C.c_void_p]
    L.bv_radfoam_tracer_adam_step.argtypes = [C.c_void_p, C.POINTER(Grads),
                                              C.POINTER(AdamSettingsC), C.c_void_p]
    L.bv_radfoam_tracer_adam_steps.argtypes = [C.c_void_p]
    L.bv_radfoam_tracer_adam_steps.restype = C.c_uint32
    L.bv_radfoam_tracer_read_model.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bv_gaussian_tracer_new.argtypes = [C.POINTER(GaussianShDesc),
                                         C.POINTER(GaussianTraceSettingsC), C.POINTER(C.c_void_p)]
    L.bv_gaussian_tracer_destroy.argtypes = [C.c_void_p]
    L.bv_gaussian_tracer_destroy.restype = None
    L.bv_gaussian_tracer_set_min_transmittance.argtypes = [C.c_void_p, C.c_float]
    L.bv_gaussian_tracer_set_background.argtypes = [C.c_void_p, C.POINTER(C.c_float)]
    L.bv_gaussian_tracer_num_points.argtypes = [C.c_void_p]
    L.bv_gaussian_tracer_num_points.restype = C.c_uint32
    L.bv_gaussian_tracer_dispatch.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(CameraC),
                                              C.c_uint32, C.c_uint32, C.c_void_p]
    L.bv_gaussian_tracer_enable_stats.argtypes = [C.c_void_p, C.c_uint32]
    L.bv_gaussian_tracer_last_stats.argtypes = [C.c_void_p, C.POINTER(LaunchStats)]
    _lib = L
    return L


def _check(status: int):
    if status != BV_OK:
        raise BvError(status, load_library().bv_last_error().decode(errors="replace"))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _uptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def camera_c(cam: Camera) -> CameraC:
    c = CameraC()
    c.cam_position[:] = [float(v) for v in cam.position]
    c.depth = float(cam.depth)
    c.cam_orientation[:] = [float(v) for v in cam.orientation]
    c.fov[:] = [float(v) for v in cam.fov]
    c.principal[:] = [float(v) for v in cam.principal]
    return c


class _DescHolder:
    """Keeps the numpy arrays a ModelDesc points at alive."""

    def __init__(self, model: PointCloudModel):
        self.points = np.ascontiguousarray(model.points, dtype=np.float32)
        self.sh = np.ascontiguousarray(model.sh, dtype=np.float32)
        self.offsets = np.ascontiguousarray(model.offsets, dtype=np.uint32)
        self.neighbors = np.ascontiguousarray(model.neighbors, dtype=np.uint32)
        if self.neighbors.size == 0:
            self.neighbors = np.zeros(1, dtype=np.uint32)
        self.radii = (None if model.radii is None
                      else np.ascontiguousarray(model.radii, dtype=np.float32))
        self.desc = ModelDesc()
        self.desc.num_points = self.points.shape[0]
        self.desc.sh_degree = model.sh_degree
        self.desc.points = _fptr(self.points)
        self.desc.sh_coefficients = _fptr(self.sh)
        self.desc.radii = _fptr(self.radii) if self.radii is not None else None
        self.desc.adjacency_offsets = _uptr(self.offsets)
        self.desc.adjacency_neighbors = _uptr(self.neighbors)
        self.desc.flags = MODEL_SH_BF16 if model.sh_bf16 else 0


def validate_model(model: PointCloudModel) -> Optional[str]:
    """PointCloudModel::validate (lib.rs:246-483) through the C ABI; returns
    the error message or None.  Needs no GPU."""
    h = _DescHolder(model)
    buf = C.create_string_buffer(512)
    st = load_library().bv_model_validate(C.byref(h.desc), buf, 512)
    return None if st == BV_OK else buf.value.decode()


def containing_points_noalloc(sites, positions, out, stream=None):
    """bv_containing_points_noalloc: power-nearest site of up to 32 query
    positions without any device allocation.  ``sites`` is a CUDA float32
    tensor [N, 4] (x, y, z, power radius), ``out`` a CUDA int32 tensor with
    room for the indices; ``positions`` host floats [Q, 3]."""
    import torch

    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    if sites.dtype != torch.float32 or sites.dim() != 2 or sites.shape[1] != 4:
        raise ValueError("sites must be a float32 tensor of shape [N, 4]")
    if not sites.is_contiguous():
        raise ValueError("sites must be contiguous")
    if out.dtype != torch.int32 or out.numel() < p.shape[0]:
        raise ValueError(f"out must be an int32 tensor with at least {p.shape[0]} elements")
    if not out.is_contiguous():
        raise ValueError("out must be contiguous")
    if not sites.is_cuda or not out.is_cuda:
        raise ValueError("sites and out must be CUDA tensors")
    _check(load_library().bv_containing_points_noalloc(
        C.c_void_p(sites.data_ptr()), sites.shape[0], _fptr(p), p.shape[0],
        C.c_void_p(out.data_ptr()), _stream_handle(stream)))


class GradTables(dict):
    """The gradient tables of a tracer (d_density [N], d_sh [N*3K], d_pos
    [N*3], d_radius [N]) as views into ONE flat device buffer, ``flat``, so
    that the data-parallel step sums them with one collective and no copies.
    d_sh comes first, at the buffer's start, which keeps it 16-byte aligned."""

    flat = None


def _grad_tables(n: int, k3: int, radii: bool, device="cuda") -> GradTables:
    import torch

    sizes = [("d_sh", n * k3), ("d_density", n), ("d_pos", n * 3)]
    if radii:
        sizes.append(("d_radius", n))
    flat = torch.zeros(sum(s for _, s in sizes), dtype=torch.float32, device=device)
    g = GradTables()
    off = 0
    for name, size in sizes:
        g[name] = flat[off:off + size]
        off += size
    g.flat = flat
    return g


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        import torch

        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


class RadFoamGpuTracer:
    """RadFoamGpuTracer (radfoam_trace.rs:56-177) over the C ABI."""

    def __init__(self, model: PointCloudModel, max_steps: int = 1024,
                 weight_threshold: float = 0.001, debug_cell_density: bool = False):
        L = load_library()
        self.model = model
        h = _DescHolder(model)
        s = TraceSettings(max_steps, 0, weight_threshold, int(debug_cell_density))
        handle = C.c_void_p()
        _check(L.bv_radfoam_tracer_new(C.byref(h.desc), C.byref(s), C.byref(handle)))
        self._h = handle
        self.sh_components = model.sh_components

    # --- lifecycle
    def deinit(self):
        if getattr(self, "_h", None):
            load_library().bv_radfoam_tracer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass

    # --- settings (radfoam_trace.rs:137-171)
    def set_max_steps(self, v: int):
        _check(load_library().bv_radfoam_tracer_set_max_steps(self._h, v))

    def set_weight_threshold(self, v: float):
        _check(load_library().bv_radfoam_tracer_set_weight_threshold(self._h, v))

    def set_debug_cell_density(self, enabled: bool):
        _check(load_library().bv_radfoam_tracer_set_debug_cell_density(self._h, int(enabled)))

    def set_tie_break(self, enabled: bool):
        """Render walk: FP64 re-evaluation of exit faces tied within 4 FP32 ulps
        (False: the reference's first-minimum rule)."""
        _check(load_library().bv_radfoam_tracer_set_tie_break(self._h, int(enabled)))

    def set_exit_record(self, steps: int):
        """Training: exit faces recorded per ray by the forward for the replay
        (default 256 steps; 0: the replay searches every step's faces)."""
        _check(load_library().bv_radfoam_tracer_set_exit_record(self._h, int(steps)))

    @property
    def max_steps(self) -> int:
        return load_library().bv_radfoam_tracer_max_steps(self._h)

    @property
    def weight_threshold(self) -> float:
        return load_library().bv_radfoam_tracer_weight_threshold(self._h)

    @property
    def sh_degree(self) -> int:
        return load_library().bv_radfoam_tracer_sh_degree(self._h)

    def start_point(self) -> int:
        return load_library().bv_radfoam_tracer_start_point(self._h)

    def containing_point(self, position) -> int:
        p = np.ascontiguousarray(position, dtype=np.float32)
        out = C.c_uint32()
        _check(load_library().bv_containing_point(self._h, _fptr(p), C.byref(out)))
        return int(out.value)

    # --- render
    def dispatch(self, output, camera: Camera, size, stream=None):
        """Render into ``output`` (torch float32 CUDA tensor [H, W, 4])."""
        w, h = size
        cam = camera_c(camera)
        _check(load_library().bv_radfoam_tracer_dispatch(
            self._h, C.c_void_p(output.data_ptr()), C.byref(cam), w, h, _stream_handle(stream)))

    def dispatch_batch(self, output, cameras: Sequence[Camera], size, stream=None):
        w, h = size
        arr = (CameraC * len(cameras))(*[camera_c(c) for c in cameras])
        _check(load_library().bv_radfoam_tracer_dispatch_batch(
            self._h, C.c_void_p(output.data_ptr()), arr, len(cameras), w, h,
            _stream_handle(stream)))

    def render(self, cameras: Sequence[Camera], width: int, height: int):
        """Convenience: returns a torch tensor [views, H, W, 4]."""
        import torch

        out = torch.empty((len(cameras), height, width, 4), dtype=torch.float32, device="cuda")
        self.dispatch_batch(out, cameras, (width, height))
        return out

    # --- path recorder
    def record_paths(self, cameras: Sequence[Camera], width: int, height: int, max_steps: int,
                     jacobians: bool = True, stream=None):
        import torch

        P = len(cameras) * width * height
        dev = "cuda"
        bufs = dict(
            previous_cells=torch.full((P, max_steps), -1, dtype=torch.int32, device=dev),
            cells=torch.full((P, max_steps), -1, dtype=torch.int32, device=dev),
            next_cells=torch.full((P, max_steps), -1, dtype=torch.int32, device=dev),
            dts=torch.full((P, max_steps), float("nan"), dtype=torch.float32, device=dev),
            path_status=torch.zeros(P, dtype=torch.int32, device=dev),
        )
        if jacobians:
            for k in ("dt_grad_previous", "dt_grad_current", "dt_grad_next"):
                bufs[k] = torch.full((P, max_steps, 4), float("nan"), dtype=torch.float32,
                                     device=dev)
        pb = PathBuffers()
        for k, v in bufs.items():
            setattr(pb, k + "_dev", v.data_ptr())
        pb.max_steps = max_steps
        arr = (CameraC * len(cameras))(*[camera_c(c) for c in cameras])
        _check(load_library().bv_record_paths(self._h, arr, len(cameras), width, height,
                                              C.byref(pb), _stream_handle(stream)))
        return bufs

    # --- training gradient
    def forward_backward(self, cameras: Sequence[Camera], width: int, height: int, target,
                         grads: dict, max_steps: int = 1024, weight_threshold: float = 0.0,
                         max_dt: float = 50.0, loss: int = LOSS_L2, loss_out=None, rgb_out=None,
                         stream=None):
        import torch

        if loss_out is None:
            loss_out = torch.zeros(1, dtype=torch.float32, device="cuda")
        ts = TrainSettings(max_steps, weight_threshold, max_dt, loss)
        g = Grads(grads["d_density"].data_ptr(), grads["d_sh"].data_ptr(),
                  grads["d_pos"].data_ptr() if grads.get("d_pos") is not None else None,
                  grads["d_radius"].data_ptr() if grads.get("d_radius") is not None else None)
        arr = (CameraC * len(cameras))(*[camera_c(c) for c in cameras])
        _check(load_library().bv_forward_backward(
            self._h, arr, len(cameras), width, height, C.c_void_p(target.data_ptr()),
            C.byref(ts), C.byref(g), C.c_void_p(loss_out.data_ptr()),
            C.c_void_p(rgb_out.data_ptr()) if rgb_out is not None else None,
            _stream_handle(stream)))
        return loss_out

    def new_grads(self):
        import torch

        return _grad_tables(self.model.n, 3 * self.sh_components, self.model.radii is not None)

    def adam_step(self, grads: dict, lr_density=0.0, lr_sh_dc=0.0, lr_sh_rest=0.0,
                  lr_position=0.0, lr_radius=0.0, beta1=0.9, beta2=0.999, eps=1e-15,
                  density_activation=DENSITY_IDENTITY, softplus_beta=10.0, stream=None):
        """One Adam step of the device model from gradient tables (a dict as
        from new_grads); see bv_radfoam_tracer_adam_step."""
        g = Grads()
        g.d_density_dev = grads["d_density"].data_ptr() if grads.get("d_density") is not None else None
        g.d_sh_dev = grads["d_sh"].data_ptr() if grads.get("d_sh") is not None else None
        g.d_positions_dev = grads["d_pos"].data_ptr() if grads.get("d_pos") is not None else None
        g.d_radii_dev = grads["d_radius"].data_ptr() if grads.get("d_radius") is not None else None
        a = AdamSettingsC(lr_density, lr_sh_dc, lr_sh_rest, lr_position, lr_radius, beta1, beta2,
                          eps, density_activation, softplus_beta)
        _check(load_library().bv_radfoam_tracer_adam_step(self._h, C.byref(g), C.byref(a),
                                                          _stream_handle(stream)))

    @property
    def adam_steps(self) -> int:
        return load_library().bv_radfoam_tracer_adam_steps(self._h)

    def read_model(self):
        """(points [N, 4], sh [N, 3K], radii [N] or None) of the device model."""
        n = self.model.n
        pts = np.zeros((n, 4), np.float32)
        sh = np.zeros((n, 3 * self.sh_components), np.float32)
        rad = np.zeros(n, np.float32) if self.model.radii is not None else None
        _check(load_library().bv_radfoam_tracer_read_model(
            self._h, pts.ctypes.data, sh.ctypes.data, None if rad is None else rad.ctypes.data))
        return pts, sh, rad

    # --- instrumentation
    def enable_stats(self, enabled: bool = True):
        _check(load_library().bv_radfoam_tracer_enable_stats(self._h, int(enabled)))

    def last_stats(self) -> LaunchStats:
        s = LaunchStats()
        _check(load_library().bv_radfoam_tracer_last_stats(self._h, C.byref(s)))
        return s


class RelightTracer:
    """RelightTracer::new_gaussian / set_point_light / dispatch
    (gpu/relight.rs:313, :841, :905) over the C ABI."""

    def __init__(self, model, background=(0.0, 0.0, 0.0)):
        L = load_library()
        self.points = np.ascontiguousarray(model.points, np.float32)
        self.rotations = np.ascontiguousarray(model.rotations, np.float32)
        self.scales = np.ascontiguousarray(model.scales, np.float32)
        self.normals = np.ascontiguousarray(model.normals, np.float32)
        self.material_indices = np.ascontiguousarray(model.material_indices, np.uint32)
        self.materials = np.ascontiguousarray(model.materials, np.float32).reshape(-1, 8)
        d = GaussianDesc(len(self.points), len(self.materials), _fptr(self.points),
                         _fptr(self.rotations), _fptr(self.scales), _fptr(self.normals),
                         _uptr(self.material_indices), self.materials.ctypes.data)
        st = RelightSettings()
        st.background[:] = [float(v) for v in background]
        st.diffuse_samples = 0
        h = C.c_void_p()
        _check(L.bv_relight_tracer_new_gaussian(C.byref(d), C.byref(st), C.byref(h)))
        self._h = h

    def deinit(self):
        if getattr(self, "_h", None):
            load_library().bv_relight_tracer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass

    @property
    def num_particles(self) -> int:
        return load_library().bv_relight_tracer_num_particles(self._h)

    def set_point_lights(self, lights):
        arr = (PointLightC * len(lights))()
        for i, (pos, direction, intensity, exponent) in enumerate(lights):
            arr[i].position[:] = [float(v) for v in pos]
            arr[i].direction[:] = [float(v) for v in direction]
            arr[i].intensity[:] = [float(v) for v in intensity]
            arr[i].exponent = float(exponent)
        _check(load_library().bv_relight_tracer_set_point_lights(self._h, arr, len(lights)))

    def set_point_light(self, light):
        self.set_point_lights([light])

    def set_background(self, rgb):
        a = np.ascontiguousarray(rgb, np.float32)
        _check(load_library().bv_relight_tracer_set_background(self._h, _fptr(a)))

    def dispatch(self, output, camera: Camera, size, stream=None):
        w, h = size
        cam = camera_c(camera)
        _check(load_library().bv_relight_tracer_dispatch(
            self._h, C.c_void_p(output.data_ptr()), C.byref(cam), w, h, _stream_handle(stream)))

    def render(self, camera: Camera, width: int, height: int):
        import torch

        out = torch.empty((height, width, 4), dtype=torch.float32, device="cuda")
        self.dispatch(out, camera, (width, height))
        return out

    def enable_stats(self, enabled: bool = True):
        _check(load_library().bv_relight_tracer_enable_stats(self._h, int(enabled)))

    def last_stats(self) -> LaunchStats:
        s = LaunchStats()
        _check(load_library().bv_relight_tracer_last_stats(self._h, C.byref(s)))
        return s


class GaussianTracer:
    """GaussianGpuCloud::new (gpu/gaussian.rs:94-280) plus its ray-traced
    draw pass (shaders/gaussian.wgsl) over the C ABI: SH-coloured Gaussians
    composited in maximum-response order (trace_gaussians, trace.rs:695-773).
    ``model`` carries points [N, 4] (mean, opacity), rotations [N, 4] (x, y,
    z, w), scales [N, 3], sh [N, 3K] and sh_degree."""

    def __init__(self, model, min_opacity: float = 0.01, min_transmittance: float = 0.01,
                 background=(0.0, 0.0, 0.0)):
        L = load_library()
        self.points = np.ascontiguousarray(model.points, np.float32)
        self.rotations = np.ascontiguousarray(model.rotations, np.float32)
        self.scales = np.ascontiguousarray(model.scales, np.float32)
        self.sh = np.ascontiguousarray(model.sh, np.float32)
        d = GaussianShDesc(len(self.points), int(model.sh_degree), _fptr(self.points),
                           _fptr(self.rotations), _fptr(self.scales), _fptr(self.sh))
        st = GaussianTraceSettingsC()
        st.min_opacity = float(min_opacity)
        st.min_transmittance = float(min_transmittance)
        st.background[:] = [float(v) for v in background]
        h = C.c_void_p()
        _check(L.bv_gaussian_tracer_new(C.byref(d), C.byref(st), C.byref(h)))
        self._h = h

    def deinit(self):
        if getattr(self, "_h", None):
            load_library().bv_gaussian_tracer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass

    @property
    def num_points(self) -> int:
        return load_library().bv_gaussian_tracer_num_points(self._h)

    def set_min_transmittance(self, v: float):
        _check(load_library().bv_gaussian_tracer_set_min_transmittance(self._h, float(v)))

    def set_background(self, rgb):
        a = np.ascontiguousarray(rgb, np.float32)
        _check(load_library().bv_gaussian_tracer_set_background(self._h, _fptr(a)))

    def dispatch(self, output, camera: Camera, size, stream=None):
        w, h = size
        cam = camera_c(camera)
        _check(load_library().bv_gaussian_tracer_dispatch(
            self._h, C.c_void_p(output.data_ptr()), C.byref(cam), w, h, _stream_handle(stream)))

    def render(self, camera: Camera, width: int, height: int):
        import torch

        out = torch.empty((height, width, 4), dtype=torch.float32, device="cuda")
        self.dispatch(out, camera, (width, height))
        return out

    def enable_stats(self, enabled: bool = True):
        _check(load_library().bv_gaussian_tracer_enable_stats(self._h, int(enabled)))

    def last_stats(self) -> LaunchStats:
        s = LaunchStats()
        _check(load_library().bv_gaussian_tracer_last_stats(self._h, C.byref(s)))
        return s


class PowerFoamSplatTracer:
    """PowerFoamGpuSplatTracer (gpu/powerfoam_splat.rs:38-370) over the C ABI:
    the order-exact splat render of a PowerFoam model (radii required; the
    CSR is the Cech overlap graph), and training with splat semantics."""

    def __init__(self, model: PointCloudModel, max_steps: int = 1024,
                 weight_threshold: float = 0.001, candidate_capacity: int = 0):
        L = load_library()
        self.model = model
        self.sh_components = model.sh_components
        d = _DescHolder(model)
        s = TraceSettings(max_steps, candidate_capacity, weight_threshold, 0)
        h = C.c_void_p()
        _check(L.bv_powerfoam_splat_tracer_new(C.byref(d.desc), C.byref(s), C.byref(h)))
        self._h = h

    def deinit(self):
        if self._h:
            load_library().bv_powerfoam_splat_tracer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.deinit()
        except Exception:
            pass

    @property
    def candidate_capacity(self) -> int:
        return load_library().bv_powerfoam_splat_tracer_candidate_capacity(self._h)

    @property
    def max_steps(self) -> int:
        return load_library().bv_powerfoam_splat_tracer_max_steps(self._h)

    @property
    def weight_threshold(self) -> float:
        return load_library().bv_powerfoam_splat_tracer_weight_threshold(self._h)

    def set_weight_threshold(self, v: float):
        _check(load_library().bv_powerfoam_splat_tracer_set_weight_threshold(self._h, v))

    def dispatch(self, output, camera: Camera, size, stream=None):
        w, h = size
        cam = camera_c(camera)
        _check(load_library().bv_powerfoam_splat_tracer_dispatch(
            self._h, C.c_void_p(output.data_ptr()), C.byref(cam), w, h, _stream_handle(stream)))

    def dispatch_batch(self, output, cameras: Sequence[Camera], size, stream=None):
        w, h = size
        arr = (CameraC * len(cameras))(*[camera_c(c) for c in cameras])
        _check(load_library().bv_powerfoam_splat_tracer_dispatch_batch(
            self._h, C.c_void_p(output.data_ptr()), arr, len(cameras), w, h,
            _stream_handle(stream)))

    def render(self, cameras: Sequence[Camera], width: int, height: int):
        import torch

        out = torch.empty((len(cameras), height, width, 4), dtype=torch.float32, device="cuda")
        self.dispatch_batch(out, cameras, (width, height))
        return out

    def validate_candidate_counts(self) -> int:
        """Largest support-hit count of one ray in the last dispatch; raises
        BvError (BV_ERR_CANDIDATE_OVERFLOW) above the capacity."""
        v = C.c_uint32()
        _check(load_library().bv_powerfoam_splat_tracer_validate_candidate_counts(self._h,
                                                                                 C.byref(v)))
        return v.value

    def forward_backward(self, cameras: Sequence[Camera], width: int, height: int, target,
                         grads: dict, max_steps: int = 1024, weight_threshold: float = 0.0,
                         max_dt: float = 50.0, loss: int = LOSS_L2, loss_out=None, rgb_out=None,
                         stream=None):
        """bv_powerfoam_splat_tracer_forward_backward: the training step's
        gradients with splat semantics (same arguments as
        RadFoamGpuTracer.forward_backward)."""
        import torch

        if loss_out is None:
            loss_out = torch.zeros(1, dtype=torch.float32, device="cuda")
        ts = TrainSettings(max_steps, weight_threshold, max_dt, loss)
        g = Grads(grads["d_density"].data_ptr(), grads["d_sh"].data_ptr(),
                  grads["d_pos"].data_ptr() if grads.get("d_pos") is not None else None,
                  grads["d_radius"].data_ptr() if grads.get("d_radius") is not None else None)
        arr = (CameraC * len(cameras))(*[camera_c(c) for c in cameras])
        _check(load_library().bv_powerfoam_splat_tracer_forward_backward(
            self._h, arr, len(cameras), width, height, C.c_void_p(target.data_ptr()),
            C.byref(ts), C.byref(g), C.c_void_p(loss_out.data_ptr()),
            C.c_void_p(rgb_out.data_ptr()) if rgb_out is not None else None,
            _stream_handle(stream)))
        return loss_out

    def new_grads(self):
        import torch

        return _grad_tables(self.model.n, 3 * self.sh_components, True)

    def candidate_stats(self):
        """(max support hits of one ray, total hits, Cech row entries of the
        hit supports) over the last dispatch's rays."""
        mx, tot, ent = C.c_uint32(), C.c_uint64(), C.c_uint64()
        _check(load_library().bv_powerfoam_splat_tracer_candidate_stats(
            self._h, C.byref(mx), C.byref(tot), C.byref(ent)))
        return mx.value, tot.value, ent.value

    def enable_stats(self, enabled: bool = True):
        _check(load_library().bv_powerfoam_splat_tracer_enable_stats(self._h, 1 if enabled else 0))

    def set_interval_record(self, entries: int):
        """Training: composited intervals recorded per ray by the forward for
        the replay (default 1024; 0: the replay traverses every ray again)."""
        _check(load_library().bv_powerfoam_splat_tracer_set_interval_record(self._h, int(entries)))

    def last_stats(self) -> LaunchStats:
        st = LaunchStats()
        _check(load_library().bv_powerfoam_splat_tracer_last_stats(self._h, C.byref(st)))
        return st


def _host_ptr(a) -> int:
    """Address of a C-contiguous float32/float64 host buffer (numpy array or
    torch CPU tensor, pinned for overlapped copies)."""
    if hasattr(a, "data_ptr"):
        if a.is_cuda or not a.is_contiguous():
            raise ValueError("host buffers must be contiguous CPU tensors")
        return a.data_ptr()
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host buffers must be C-contiguous")
    return a.ctypes.data


class Server:
    """Serving loop over the C ABI (bv_server_*): resident scenes, admission
    under an HBM budget, continuous batching of render frames into one
    persistent traversal launch per batch (replayed CUDA graphs), or the
    plain one-request-at-a-time modes ("plain": one dispatch per view,
    "plain_batch": one dispatch over the request's views).  Host buffers passed to :meth:`submit`
    are kept alive here until :meth:`wait` returns their request.
    ``train_record_steps``: steps per ray of the training step record (1..256,
    0 = the most that fits an eighth of the budget, None = no record)."""

    def __init__(self, hbm_budget_bytes: int, mode: str = "batched", max_batch_rays: int = 0,
                 max_batch_views: int = 0, slots: int = 0, max_steps: int = 1024,
                 weight_threshold: float = 0.001, max_train_rays: int = 0,
                 use_graphs: bool = True, train_chunk_rays: int = 0, frame_period_us: int = 0,
                 train_record_steps: int = 0):
        L = load_library()
        s = ServerSettings()
        s.hbm_budget_bytes = int(hbm_budget_bytes)
        s.mode = {"batched": SERVE_BATCHED, "plain": SERVE_PLAIN,
                  "plain_batch": SERVE_PLAIN_BATCH}[mode]
        s.max_batch_rays = max_batch_rays
        s.max_batch_views = max_batch_views
        s.slots = slots
        s.max_steps = max_steps
        s.weight_threshold = weight_threshold
        s.max_train_rays = max_train_rays
        s.use_graphs = 1 if use_graphs else 0
        s.train_chunk_rays = train_chunk_rays
        s.frame_period_us = frame_period_us
        s.train_record_steps = SERVE_NO_RECORD if train_record_steps is None else train_record_steps
        h = C.c_void_p()
        _check(L.bv_server_new(C.byref(s), C.byref(h)))
        self._h = h
        self._keep = {}
        self.scenes = []

    def add_scene(self, model: PointCloudModel, gradients: bool = False) -> int:
        d = _DescHolder(model)
        sid = C.c_uint32()
        _check(load_library().bv_server_add_scene(self._h, C.byref(d.desc),
                                                  SCENE_GRADIENTS if gradients else 0,
                                                  C.byref(sid)))
        self.scenes.append(model)
        return sid.value

    def scene_grads(self, scene: int) -> Grads:
        g = Grads()
        _check(load_library().bv_server_scene_grads(self._h, scene, C.byref(g)))
        return g

    def start(self):
        _check(load_library().bv_server_start(self._h))

    def submit(self, scene: int, cameras: Sequence[Camera], width: int, height: int,
               out=None, target=None, loss=None, grads: Optional[dict] = None,
               max_steps: int = 1024, weight_threshold: float = 0.0, max_dt: float = 50.0,
               loss_kind: int = LOSS_L2, frame_done=None) -> int:
        """Queue a render request (``out`` [views, H, W, 4] float32 host) or,
        with ``target`` ([views, H, W, 3] float32 host) and ``loss`` (float32
        host [1]), a forward+backward request (``out`` then [views, H, W, 3]
        or None; ``grads`` a dict of CUDA tables as from
        RadFoamGpuTracer.new_grads, or None for the scene's own tables)."""
        r = RequestC()
        r.scene = scene
        r.n_views = len(cameras)
        r.width, r.height = width, height
        cams = (CameraC * len(cameras))(*[camera_c(c) for c in cameras])
        r.cameras = cams
        keep = [cams, out, target, loss, grads, frame_done]
        if target is None:
            r.kind = REQUEST_RENDER
            r.out_host = _host_ptr(out) if out is not None else None
        else:
            r.kind = REQUEST_FORWARD_BACKWARD
            r.out_host = _host_ptr(out) if out is not None else None
            r.target_host = _host_ptr(target)
            r.loss_host = _host_ptr(loss) if loss is not None else None
            r.train.max_steps = max_steps
            r.train.weight_threshold = weight_threshold
            r.train.max_dt = max_dt
            r.train.loss = loss_kind
            if grads is not None:
                r.grads.d_density_dev = grads["d_density"].data_ptr()
                r.grads.d_sh_dev = grads["d_sh"].data_ptr()
                if "d_pos" in grads:
                    r.grads.d_positions_dev = grads["d_pos"].data_ptr()
                if "d_radius" in grads:
                    r.grads.d_radii_dev = grads["d_radius"].data_ptr()
        if frame_done is not None:
            r.frame_done_host = _host_ptr(frame_done)
        rid = C.c_uint64()
        _check(load_library().bv_server_submit(self._h, C.byref(r), C.byref(rid)))
        self._keep[rid.value] = keep
        return rid.value

    def wait(self, rid: int, timeout: float = 120.0) -> dict:
        res = RequestResult()
        _check(load_library().bv_server_wait(self._h, rid, timeout, C.byref(res)))
        self._keep.pop(rid, None)
        return dict(id=res.id, status=res.status, kind=res.kind, submit_s=res.submit_s,
                    admit_s=res.admit_s, start_s=res.start_s, done_s=res.done_s, rays=res.rays,
                    message=res.message.decode(errors="replace"))

    def cancel(self, rid: int):
        """bv_server_cancel: withdraw a request (wait() then reports status
        BV_ERR_CANCELLED unless it had finished already)."""
        _check(load_library().bv_server_cancel(self._h, rid))

    def stats(self) -> dict:
        st = ServerStats()
        _check(load_library().bv_server_stats_get(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def clock(self) -> float:
        return load_library().bv_server_clock(self._h)

    def close(self):
        if self._h:
            load_library().bv_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
