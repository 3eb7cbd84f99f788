"""blade_volume_b200: B200 (sm_100a) ray-tracing hot path of blade-volume.

Python mirror of the reference crate's tracer API over the C ABI of
libbv_b200.so (include/blade_volume_b200.h):

* :class:`RadFoamGpuTracer`   blade-volume/src/gpu/radfoam_trace.rs:56-177
* :meth:`RadFoamGpuTracer.record_paths`   gpu/path_record.rs:519-594
* :meth:`RadFoamGpuTracer.forward_backward`   the trainer's gradient
  (blade-volume-train/src/diff_render.rs:943-1923, :7181-7226)

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
                6: "BV_ERR_NOT_SUPPORTED", 7: "BV_ERR_NO_DEVICE"}
MODEL_SH_BF16 = 0x1
PATH_TRUNCATED = 0x80000000
LOSS_L2, LOSS_L1 = 0, 1

# Every symbol include/blade_volume_b200.h declares.
EXPORTED_SYMBOLS = [
    "bv_last_error", "bv_abi_version", "bv_model_validate", "bv_radfoam_tracer_new",
    "bv_radfoam_tracer_destroy", "bv_radfoam_tracer_dispatch", "bv_radfoam_tracer_dispatch_batch",
    "bv_radfoam_tracer_set_max_steps", "bv_radfoam_tracer_set_weight_threshold",
    "bv_radfoam_tracer_set_debug_cell_density", "bv_radfoam_tracer_max_steps",
    "bv_radfoam_tracer_weight_threshold", "bv_radfoam_tracer_sh_degree",
    "bv_radfoam_tracer_start_point", "bv_radfoam_tracer_num_points", "bv_containing_point",
    "bv_record_paths", "bv_forward_backward", "bv_radfoam_tracer_enable_stats",
    "bv_radfoam_tracer_last_stats", "bv_containing_points_noalloc",
    "bv_relight_tracer_new_gaussian", "bv_relight_tracer_destroy",
    "bv_relight_tracer_set_point_lights", "bv_relight_tracer_set_background",
    "bv_relight_tracer_dispatch", "bv_relight_tracer_num_particles",
    "bv_relight_tracer_enable_stats", "bv_relight_tracer_last_stats",
]


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


class RelightSettings(C.Structure):
    _fields_ = [("background", C.c_float * 3), ("diffuse_samples", C.c_uint32)]


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
    p = np.ascontiguousarray(positions, dtype=np.float32).reshape(-1, 3)
    _check(load_library().bv_containing_points_noalloc(
        C.c_void_p(sites.data_ptr()), sites.shape[0], _fptr(p), p.shape[0],
        C.c_void_p(out.data_ptr()), _stream_handle(stream)))


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

        n = self.model.n
        K3 = 3 * self.sh_components
        g = dict(d_density=torch.zeros(n, dtype=torch.float32, device="cuda"),
                 d_sh=torch.zeros(n * K3, dtype=torch.float32, device="cuda"),
                 d_pos=torch.zeros(n * 3, dtype=torch.float32, device="cuda"))
        if self.model.radii is not None:
            g["d_radius"] = torch.zeros(n, dtype=torch.float32, device="cuda")
        return g

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
