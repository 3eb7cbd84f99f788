"""ctypes front end of the CPU oracle (test infrastructure only).

Wraps oracle/_build/libbv_oracle.so (built by oracle/build.py) with numpy in
and out.  Every function here is a checker: tests compare the CUDA library's
results against these.
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

from . import build as _build

_lib = None

f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
u32p = C.POINTER(C.c_uint32)


class Model(C.Structure):
    _fields_ = [("points", f32p), ("radii", f32p), ("sh", f32p), ("sh_degree", C.c_uint32),
                ("offsets", u32p), ("neighbors", u32p), ("n", C.c_uint32)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("depth", C.c_float), ("orientation", C.c_float * 4),
                ("fov", C.c_float * 2), ("principal", C.c_float * 2)]


class Settings(C.Structure):
    _fields_ = [("weight_threshold", C.c_float), ("max_steps", C.c_uint32),
                ("start_point", C.c_uint32), ("depth", C.c_float), ("eval_mode", C.c_int),
                ("constant_rgb", C.c_float * 3), ("tie_break", C.c_int)]


class TraceResult(C.Structure):
    _fields_ = [("rgba", C.c_float * 4), ("steps", C.c_uint32), ("last_point", C.c_uint32),
                ("t_end", C.c_float), ("depth_mode", C.c_float), ("peak_weight", C.c_float),
                ("peak_point", C.c_int32)]


class PathEntry(C.Structure):
    _fields_ = [("previous_cell", C.c_uint32), ("cell", C.c_uint32), ("next_cell", C.c_uint32),
                ("dt", C.c_float), ("dt_d_previous", C.c_float * 4),
                ("dt_d_current", C.c_float * 4), ("dt_d_next", C.c_float * 4),
                ("surface_query_near", C.c_float), ("surface_query_d_previous", C.c_float * 4),
                ("surface_query_d_current", C.c_float * 4), ("t_start", C.c_float)]


class Material(C.Structure):
    _fields_ = [("albedo", C.c_float * 3), ("roughness", C.c_float),
                ("specular_f0", C.c_float * 3), ("pad", C.c_float)]


class PointLight(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("direction", C.c_float * 3),
                ("intensity", C.c_float * 3), ("exponent", C.c_float)]


class RelightScene(C.Structure):
    _fields_ = [("n", C.c_uint32), ("center", f32p), ("rotation", f32p), ("scale", f32p),
                ("opacity", f32p), ("normal", f32p), ("radius", f32p), ("support_sq", f32p),
                ("material", u32p), ("materials", C.POINTER(Material))]


class GaussianScene(C.Structure):
    _fields_ = [("n", C.c_uint32), ("center", f32p), ("rotation", f32p), ("scale", f32p),
                ("opacity", f32p), ("sh", f32p), ("sh_degree", C.c_uint32)]


class GaussianSettings(C.Structure):
    _fields_ = [("min_opacity", C.c_float), ("min_transmittance", C.c_float),
                ("t_start", C.c_float), ("t_end", C.c_float)]


class AdamSettings(C.Structure):
    _fields_ = [("lr_density", C.c_float), ("lr_sh_dc", C.c_float), ("lr_sh_rest", C.c_float),
                ("lr_position", C.c_float), ("lr_radius", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("activation", C.c_int),
                ("softplus_beta", C.c_float)]


class AdamState(C.Structure):
    _fields_ = [("n", C.c_uint32), ("nsh", C.c_uint32), ("x", f32p), ("m_d", f32p),
                ("v_d", f32p), ("density", f32p), ("sh", f32p), ("m_sh", f32p), ("v_sh", f32p),
                ("pos", f32p), ("m_pos", f32p), ("v_pos", f32p), ("radii", f32p), ("m_r", f32p),
                ("v_r", f32p)]


class ParamsF64(C.Structure):
    _fields_ = [("points", f64p), ("sh", f64p), ("radii", f64p)]


EVAL_OPACITY, EVAL_CONSTANT, EVAL_SH = 0, 1, 2


class GradMass(C.Structure):
    _fields_ = [("density", f64p), ("sh", f64p), ("pos", f64p), ("radius", f64p),
                ("count_density", f64p), ("count_sh", f64p), ("count_pos", f64p),
                ("count_radius", f64p)]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        L.bvo_expf.restype = C.c_float
        L.bvo_expf.argtypes = [C.c_float]
        L.bvo_tan_half.restype = C.c_float
        L.bvo_tan_half.argtypes = [C.c_float]
        L.bvo_camera_ray.argtypes = [C.POINTER(Camera), C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, f32p, f32p]
        L.bvo_eval_rgb_sh.argtypes = [C.POINTER(Model), C.c_uint32, f32p, f32p, f32p]
        L.bvo_trace_one_ray.restype = TraceResult
        L.bvo_trace_one_ray.argtypes = [C.POINTER(Model), f32p, f32p, C.POINTER(Settings)]
        L.bvo_render_walk.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32, C.c_uint32,
                                      C.c_uint32, C.c_float, C.c_uint32, f32p, u32p, u32p,
                                      C.c_uint32, u32p, C.c_int]
        L.bvo_record_path_jacobians.restype = C.c_int
        L.bvo_record_path_jacobians.argtypes = [C.POINTER(Model), f32p, f32p, C.POINTER(Settings),
                                                C.POINTER(PathEntry), C.c_int]
        L.bvo_record_powerfoam_splats.restype = C.c_int
        L.bvo_record_powerfoam_splats.argtypes = [C.POINTER(Model), f32p, f32p,
                                                  C.POINTER(Settings), C.POINTER(PathEntry),
                                                  C.c_int]
        L.bvo_trace_powerfoam_splats.restype = TraceResult
        L.bvo_trace_powerfoam_splats.argtypes = [C.POINTER(Model), f32p, f32p,
                                                 C.POINTER(Settings)]
        L.bvo_render_splats.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                        C.c_uint32, C.c_uint32, C.c_float, f32p, u32p, C.c_int]
        L.bvo_record_image.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                       C.c_uint32, C.c_uint32, C.c_uint32, u32p, u32p, u32p,
                                       u32p, f32p, f32p, f32p, f32p, u32p, C.c_int]
        L.bvo_support_interval.restype = C.c_int
        L.bvo_support_interval.argtypes = [C.c_int, f32p, f32p, f32p, C.c_float, C.c_float,
                                           C.c_float, f32p]
        L.bvo_containing_cell_f64.restype = C.c_uint32
        L.bvo_containing_cell_f64.argtypes = [C.POINTER(Model), f32p]
        L.bvo_containing_cell_f32.restype = C.c_uint32
        L.bvo_containing_cell_f32.argtypes = [C.POINTER(Model), f32p]
        L.bvo_forward_backward.restype = C.c_double
        L.bvo_forward_backward.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                           C.c_uint32, C.c_uint32, C.c_uint32, C.c_float,
                                           C.c_float, f32p, C.c_int, C.POINTER(ParamsF64), f64p,
                                           f32p, f64p, f64p, f64p, f64p, C.c_int]
        L.bvo_forward_backward_ex.restype = C.c_double
        L.bvo_forward_backward_ex.argtypes = L.bvo_forward_backward.argtypes + [C.c_int]
        L.bvo_forward_backward_mx.restype = C.c_double
        L.bvo_forward_backward_mx.argtypes = L.bvo_forward_backward_ex.argtypes + [
            C.POINTER(C.c_uint8), C.POINTER(GradMass)]
        L.bvo_render_splats_px.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                           C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, u32p,
                                           f32p, u32p, C.c_int]
        L.bvo_relight_render_px.argtypes = [C.POINTER(RelightScene), C.POINTER(PointLight),
                                            C.c_uint32, C.POINTER(Camera), C.c_uint32,
                                            C.c_uint32, f32p, C.c_uint32, u32p, f32p, u32p,
                                            C.c_int]
        L.bvo_gaussian_render_px.argtypes = [C.POINTER(GaussianScene), C.POINTER(Camera),
                                             C.c_uint32, C.c_uint32, C.c_float, C.c_float, f32p,
                                             C.c_uint32, u32p, f32p, u32p, C.c_int]
        L.bvo_render_splats_f64_px.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                               C.c_uint32, C.c_uint32, C.c_double, C.c_uint32,
                                               u32p, f64p, C.c_int]
        L.bvo_relight_render_f64_px.argtypes = [C.POINTER(RelightScene), C.POINTER(PointLight),
                                                C.c_uint32, C.POINTER(Camera), C.c_uint32,
                                                C.c_uint32, f32p, C.c_uint32, u32p, f64p,
                                                C.c_int]
        L.bvo_logf.restype = C.c_float
        L.bvo_logf.argtypes = [C.c_float]
        L.bvo_powf.restype = C.c_float
        L.bvo_powf.argtypes = [C.c_float, C.c_float]
        L.bvo_relight_prepare.restype = C.c_uint32
        L.bvo_relight_prepare.argtypes = [C.c_uint32, f32p, f32p, f32p, f32p, u32p, u32p, f32p,
                                          f32p, f32p, f32p, f32p, f32p, f32p, u32p]
        L.bvo_point_light_shade.argtypes = [C.POINTER(PointLight), f32p, f32p, f32p,
                                            C.POINTER(Material), f32p]
        L.bvo_shade_point_light_cpu.argtypes = [C.POINTER(PointLight), f32p, f32p, f32p,
                                                C.POINTER(Material), f32p]
        L.bvo_intersect_gaussian.restype = C.c_int
        L.bvo_intersect_gaussian.argtypes = [C.POINTER(RelightScene), C.c_uint32, f32p, f32p,
                                             C.c_float, f32p, f32p]
        L.bvo_relight_ray.argtypes = [C.POINTER(RelightScene), C.POINTER(PointLight), C.c_uint32,
                                      f32p, f32p, C.c_float, f32p, f32p, u32p]
        L.bvo_relight_render.argtypes = [C.POINTER(RelightScene), C.POINTER(PointLight),
                                         C.c_uint32, C.POINTER(Camera), C.c_uint32, C.c_uint32,
                                         f32p, f32p, u32p, C.c_int]
        L.bvo_render_walk_tb.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                         C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_int,
                                         f32p, u32p, u32p, C.c_uint32, u32p, C.c_int]
        L.bvo_render_walk_f64.argtypes = [C.POINTER(Model), C.POINTER(Camera), C.c_uint32,
                                          C.c_uint32, C.c_uint32, C.c_double, C.c_uint32, f64p,
                                          u32p, C.c_uint32, u32p, C.c_int]
        L.bvo_density_activation.restype = C.c_float
        L.bvo_density_activation.argtypes = [C.c_float, C.c_int, C.c_float]
        L.bvo_density_activation_inverse.restype = C.c_float
        L.bvo_density_activation_inverse.argtypes = [C.c_float, C.c_int, C.c_float]
        L.bvo_adam_step.argtypes = [C.POINTER(AdamState), C.POINTER(AdamSettings), C.c_uint32,
                                    f32p, f32p, f32p, f32p]
        L.bvo_gaussian_response.restype = C.c_int
        L.bvo_gaussian_response.argtypes = [C.POINTER(GaussianScene), C.c_uint32, f32p, f32p,
                                            C.POINTER(GaussianSettings), f32p, f32p]
        L.bvo_trace_gaussians.argtypes = [C.POINTER(GaussianScene), f32p, f32p,
                                          C.POINTER(GaussianSettings), f32p, f32p, u32p]
        L.bvo_gaussian_render.argtypes = [C.POINTER(GaussianScene), C.POINTER(Camera), C.c_uint32,
                                          C.c_uint32, C.c_float, C.c_float, f32p, f32p, u32p,
                                          C.c_int]
        _lib = L
    return _lib


def _ptr(a, t):
    if a is None:
        return C.cast(None, t)
    return a.ctypes.data_as(t)


class OracleModel:
    """Holds contiguous copies of a PointCloudModel's arrays for the C side."""

    def __init__(self, points, sh, sh_degree, offsets, neighbors, radii=None):
        self.points = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 4)
        self.sh = np.ascontiguousarray(sh, dtype=np.float32).reshape(-1)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.uint32)
        self.neighbors = np.ascontiguousarray(neighbors, dtype=np.uint32)
        if len(self.neighbors) == 0:
            self.neighbors = np.zeros(1, dtype=np.uint32)
        self.radii = None if radii is None else np.ascontiguousarray(radii, dtype=np.float32)
        self.sh_degree = int(sh_degree)
        self.c = Model(_ptr(self.points, f32p), _ptr(self.radii, f32p), _ptr(self.sh, f32p),
                       self.sh_degree, _ptr(self.offsets, u32p), _ptr(self.neighbors, u32p),
                       len(self.points))

    @classmethod
    def from_scene(cls, m):
        return cls(m.points, m.sh, m.sh_degree, m.offsets, m.neighbors, m.radii)

    @property
    def n(self):
        return len(self.points)


def camera_struct(cam) -> Camera:
    c = Camera()
    c.position[:] = [float(v) for v in cam.position]
    c.depth = float(cam.depth)
    c.orientation[:] = [float(v) for v in cam.orientation]
    c.fov[:] = [float(v) for v in cam.fov]
    c.principal[:] = [float(v) for v in cam.principal]
    return c


def settings(max_steps=1024, weight_threshold=1e-3, start_point=0, depth=1e4, eval_mode=EVAL_SH,
             constant_rgb=(1.0, 1.0, 1.0)) -> Settings:
    s = Settings()
    s.weight_threshold = weight_threshold
    s.max_steps = max_steps
    s.start_point = start_point
    s.depth = depth
    s.eval_mode = eval_mode
    s.constant_rgb[:] = list(constant_rgb)
    return s


def expf(x: float) -> float:
    return float(lib().bvo_expf(float(x)))


def tan_half(fov: float) -> float:
    return float(lib().bvo_tan_half(float(fov)))


def camera_ray(cam, width, height, x, y):
    o = np.zeros(3, dtype=np.float32)
    d = np.zeros(3, dtype=np.float32)
    cs = camera_struct(cam)
    lib().bvo_camera_ray(C.byref(cs), width, height, x, y, _ptr(o, f32p), _ptr(d, f32p))
    return o, d


def eval_rgb_sh(model: OracleModel, point: int, direction):
    d = np.ascontiguousarray(direction, dtype=np.float32)
    out = np.zeros(3, dtype=np.float32)
    unc = np.zeros(3, dtype=np.float32)
    lib().bvo_eval_rgb_sh(C.byref(model.c), point, _ptr(d, f32p), _ptr(out, f32p),
                          _ptr(unc, f32p))
    return out, unc


def trace_one_ray(model: OracleModel, origin, direction, s: Settings) -> TraceResult:
    o = np.ascontiguousarray(origin, dtype=np.float32)
    d = np.ascontiguousarray(direction, dtype=np.float32)
    return lib().bvo_trace_one_ray(C.byref(model.c), _ptr(o, f32p), _ptr(d, f32p), C.byref(s))


def trace_powerfoam_splats(model: OracleModel, origin, direction, s: Settings) -> TraceResult:
    o = np.ascontiguousarray(origin, dtype=np.float32)
    d = np.ascontiguousarray(direction, dtype=np.float32)
    return lib().bvo_trace_powerfoam_splats(C.byref(model.c), _ptr(o, f32p), _ptr(d, f32p),
                                            C.byref(s))


def _entries(fn, model, origin, direction, s, capacity):
    o = np.ascontiguousarray(origin, dtype=np.float32)
    d = np.ascontiguousarray(direction, dtype=np.float32)
    buf = (PathEntry * capacity)()
    n = fn(C.byref(model.c), _ptr(o, f32p), _ptr(d, f32p), C.byref(s), buf, capacity)
    return [buf[i] for i in range(min(n, capacity))]


def record_path_jacobians(model, origin, direction, s, capacity=4096):
    return _entries(lib().bvo_record_path_jacobians, model, origin, direction, s, capacity)


def record_powerfoam_splats(model, origin, direction, s, capacity=4096):
    return _entries(lib().bvo_record_powerfoam_splats, model, origin, direction, s, capacity)


def support_interval(bounded, origin, direction, center, radius, t0, t1):
    o = np.ascontiguousarray(origin, dtype=np.float32)
    d = np.ascontiguousarray(direction, dtype=np.float32)
    c = np.ascontiguousarray(center, dtype=np.float32)
    out = np.zeros(2, dtype=np.float32)
    ok = lib().bvo_support_interval(int(bounded), _ptr(o, f32p), _ptr(d, f32p), _ptr(c, f32p),
                                    float(radius), float(t0), float(t1), _ptr(out, f32p))
    return (float(out[0]), float(out[1])) if ok else None


def containing_cell_f64(model: OracleModel, position) -> int:
    p = np.ascontiguousarray(position, dtype=np.float32)
    return int(lib().bvo_containing_cell_f64(C.byref(model.c), _ptr(p, f32p)))


def containing_cell_f32(model: OracleModel, position) -> int:
    p = np.ascontiguousarray(position, dtype=np.float32)
    return int(lib().bvo_containing_cell_f32(C.byref(model.c), _ptr(p, f32p)))


def render_walk(model: OracleModel, cam, width, height, max_steps=1024, weight_threshold=1e-3,
                start_point=None, cell_capacity=0, threads=0, tie_break=False):
    """Image of the walk forward; returns rgba [H, W, 4], steps [H, W] and
    (if cell_capacity > 0) the visited cells [H, W, cap] and counts [H, W].
    tie_break: FP64 re-evaluation of near-tied exit faces."""
    if start_point is None:
        start_point = containing_cell_f64(model, cam.position)
    rgba = np.zeros((height, width, 4), dtype=np.float32)
    steps = np.zeros((height, width), dtype=np.uint32)
    cells = counts = None
    if cell_capacity > 0:
        cells = np.zeros((height, width, cell_capacity), dtype=np.uint32)
        counts = np.zeros((height, width), dtype=np.uint32)
    cs = camera_struct(cam)
    lib().bvo_render_walk_tb(C.byref(model.c), C.byref(cs), width, height, max_steps,
                             weight_threshold, start_point, int(tie_break), _ptr(rgba, f32p),
                             _ptr(steps, u32p), _ptr(cells, u32p), cell_capacity,
                             _ptr(counts, u32p), threads)
    return rgba, steps, cells, counts


def render_walk_f64(model: OracleModel, cam, width, height, max_steps=1024,
                    weight_threshold=1e-3, start_point=None, cell_capacity=0, threads=0):
    """FP64 accuracy oracle of the walk image: rgba [H, W, 4] float64 and (if
    cell_capacity > 0) visited cells [H, W, cap] and counts [H, W]."""
    if start_point is None:
        start_point = containing_cell_f64(model, cam.position)
    rgba = np.zeros((height, width, 4), dtype=np.float64)
    cells = counts = None
    if cell_capacity > 0:
        cells = np.zeros((height, width, cell_capacity), dtype=np.uint32)
        counts = np.zeros((height, width), dtype=np.uint32)
    cs = camera_struct(cam)
    lib().bvo_render_walk_f64(C.byref(model.c), C.byref(cs), width, height, max_steps,
                              float(weight_threshold), start_point, _ptr(rgba, f64p),
                              _ptr(cells, u32p), cell_capacity, _ptr(counts, u32p), threads)
    return rgba, cells, counts


def psnr(image, reference, peak=1.0) -> float:
    """PSNR (dB) of image against reference over every channel given."""
    mse = float(np.mean((np.asarray(image, np.float64) - np.asarray(reference, np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(peak * peak / mse)


def render_splats_pixels(model: OracleModel, cam, width, height, pixels, max_steps=1024,
                         weight_threshold=1e-3, threads=0):
    """render_splats at the listed pixel indices (y * width + x) only:
    rgba [n, 4], steps [n]."""
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    rgba = np.zeros((len(px), 4), dtype=np.float32)
    steps = np.zeros(len(px), dtype=np.uint32)
    cs = camera_struct(cam)
    lib().bvo_render_splats_px(C.byref(model.c), C.byref(cs), width, height, max_steps,
                               weight_threshold, len(px), _ptr(px, u32p), _ptr(rgba, f32p),
                               _ptr(steps, u32p), threads)
    return rgba, steps


def render_splats_f64_pixels(model: OracleModel, cam, width, height, pixels, max_steps=1024,
                             weight_threshold=1e-3, threads=0):
    """FP64 accuracy oracle of render_splats at the listed pixels: rgba [n, 4]
    float64 (every quantity in double from the model's FP32 values)."""
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    rgba = np.zeros((len(px), 4), dtype=np.float64)
    cs = camera_struct(cam)
    lib().bvo_render_splats_f64_px(C.byref(model.c), C.byref(cs), width, height, max_steps,
                                   float(weight_threshold), len(px), _ptr(px, u32p),
                                   _ptr(rgba, f64p), threads)
    return rgba


def record_image(model: OracleModel, cams: Sequence, width, height, max_steps, starts=None,
                 threads=0):
    """Path-recorder rows for every pixel of every camera (PathRecordBuffers
    layout [P, max_steps]); unwritten slots hold the fill values -1 / NaN."""
    if starts is None:
        starts = [containing_cell_f64(model, c.position) for c in cams]
    P = len(cams) * width * height
    L = max_steps
    out = dict(previous_cells=np.full((P, L), 0xFFFFFFFF, np.uint32),
               cells=np.full((P, L), 0xFFFFFFFF, np.uint32),
               next_cells=np.full((P, L), 0xFFFFFFFF, np.uint32),
               dts=np.full((P, L), np.nan, np.float32),
               dt_grad_previous=np.full((P, L, 4), np.nan, np.float32),
               dt_grad_current=np.full((P, L, 4), np.nan, np.float32),
               dt_grad_next=np.full((P, L, 4), np.nan, np.float32),
               path_status=np.zeros(P, np.uint32))
    cam_arr = (Camera * len(cams))(*[camera_struct(c) for c in cams])
    st = np.ascontiguousarray(starts, dtype=np.uint32)
    lib().bvo_record_image(C.byref(model.c), cam_arr, len(cams), width, height, L, _ptr(st, u32p),
                           _ptr(out["previous_cells"], u32p), _ptr(out["cells"], u32p),
                           _ptr(out["next_cells"], u32p), _ptr(out["dts"], f32p),
                           _ptr(out["dt_grad_previous"], f32p), _ptr(out["dt_grad_current"], f32p),
                           _ptr(out["dt_grad_next"], f32p), _ptr(out["path_status"], u32p),
                           threads)
    return out


def render_splats(model: OracleModel, cam, width, height, max_steps=1024, weight_threshold=1e-3,
                  threads=0):
    rgba = np.zeros((height, width, 4), dtype=np.float32)
    steps = np.zeros((height, width), dtype=np.uint32)
    cs = camera_struct(cam)
    lib().bvo_render_splats(C.byref(model.c), C.byref(cs), width, height, max_steps,
                            weight_threshold, _ptr(rgba, f32p), _ptr(steps, u32p), threads)
    return rgba, steps


def forward_backward(model: OracleModel, cams: Sequence, width, height, max_steps=1024,
                     weight_threshold=0.0, max_dt=50.0, target=None, loss_kind=0,
                     override=None, want_grads=True, threads=0, splats=False, mask=None,
                     want_mass=False):
    """FP64 training-contract oracle.  Returns dict(loss, rgb, d_density,
    d_sh, d_pos, d_radius).  splats: PowerFoam splat semantics instead of the
    walk.  mask ([views, H, W] bool): only those rays are traced and
    contribute (the loss is still normalised over every ray of the batch).
    want_mass: also return mass_density, mass_sh, mass_pos, mass_radius, the
    per-entry FP32 error budget (units of 2^-24) of each gradient table, and
    count_<table>, the number of terms summed into each entry."""
    n = model.n
    K3 = model.sh.size // max(n, 1)
    cam_arr = (Camera * len(cams))(*[camera_struct(c) for c in cams])
    rgb = np.zeros((len(cams), height, width, 3), dtype=np.float64)
    rgb32 = np.zeros((len(cams), height, width, 3), dtype=np.float32)
    tgt = None if target is None else np.ascontiguousarray(target, dtype=np.float32)
    dd = dsh = dpos = drad = None
    if want_grads:
        dd = np.zeros(n, dtype=np.float64)
        dsh = np.zeros(n * K3, dtype=np.float64)
        dpos = np.zeros(n * 3, dtype=np.float64)
        drad = np.zeros(n, dtype=np.float64) if model.radii is not None else None
    ov = None
    keep = []
    if override is not None:
        pts, sh, rad = override
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1)
        sh = np.ascontiguousarray(sh, dtype=np.float64).reshape(-1)
        rad = None if rad is None else np.ascontiguousarray(rad, dtype=np.float64)
        keep = [pts, sh, rad]
        ov = ParamsF64(_ptr(pts, f64p), _ptr(sh, f64p), _ptr(rad, f64p))
    mk = None
    if mask is not None:
        mk = np.ascontiguousarray(np.asarray(mask, dtype=bool).reshape(-1), dtype=np.uint8)
        assert mk.size == len(cams) * width * height
    mass = None
    tables = ("density", "sh", "pos", "radius")
    if want_mass and want_grads:
        sizes = dict(density=n, sh=n * K3, pos=n * 3, radius=n)
        mass = {}
        for k in tables:
            has = k != "radius" or model.radii is not None
            mass[k] = np.zeros(sizes[k]) if has else None
            mass["count_" + k] = np.zeros(sizes[k]) if has else None
    gm = None if mass is None else GradMass(*[_ptr(mass[k], f64p) for k in tables],
                                            *[_ptr(mass["count_" + k], f64p) for k in tables])
    loss = lib().bvo_forward_backward_mx(
        C.byref(model.c), cam_arr, len(cams), width, height, max_steps, weight_threshold,
        max_dt, _ptr(tgt, f32p), loss_kind, C.byref(ov) if ov is not None else None,
        _ptr(rgb, f64p), _ptr(rgb32, f32p), _ptr(dd, f64p), _ptr(dsh, f64p), _ptr(dpos, f64p),
        _ptr(drad, f64p), threads, int(splats), _ptr(mk, C.POINTER(C.c_uint8)),
        C.byref(gm) if gm is not None else None)
    del keep
    out = dict(loss=loss, rgb=rgb, rgb32=rgb32, d_density=dd, d_sh=dsh,
               d_pos=None if dpos is None else dpos.reshape(n, 3), d_radius=drad)
    if mass is not None:
        out.update(mass_density=mass["density"], mass_sh=mass["sh"],
                   mass_pos=mass["pos"].reshape(n, 3), mass_radius=mass["radius"],
                   count_density=mass["count_density"], count_sh=mass["count_sh"],
                   count_pos=mass["count_pos"].reshape(n, 3), count_radius=mass["count_radius"])
    return out


# --------------------------------------------------------------------------
# relight
# --------------------------------------------------------------------------
def logf(x: float) -> float:
    return float(lib().bvo_logf(float(x)))


def powf(x: float, y: float) -> float:
    return float(lib().bvo_powf(float(x), float(y)))


def material_struct(albedo, roughness, f0):
    m = Material()
    m.albedo[:] = [float(v) for v in albedo]
    m.roughness = float(roughness)
    m.specular_f0[:] = [float(v) for v in f0]
    m.pad = 0.0
    return m


def light_struct(position, direction, intensity, exponent):
    L = PointLight()
    L.position[:] = [float(v) for v in position]
    L.direction[:] = [float(v) for v in direction]
    L.intensity[:] = [float(v) for v in intensity]
    L.exponent = float(exponent)
    return L


def point_light_shade(light, position, normal, view, material, cpu=False):
    out = np.zeros(3, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (position, normal, view)]
    fn = lib().bvo_shade_point_light_cpu if cpu else lib().bvo_point_light_shade
    fn(C.byref(light), *[_ptr(a, f32p) for a in args], C.byref(material), _ptr(out, f32p))
    return out


class RelightOracleScene:
    """Prepared relightable Gaussians (gpu/relight.rs:178-253) for the C side."""

    def __init__(self, points, rotations, scales, normals, material_indices, materials):
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = len(points)
        self.kept = np.zeros(n, np.uint32)
        self.center = np.zeros((n, 3), np.float32)
        self.rotation = np.zeros((n, 4), np.float32)
        self.scale = np.zeros((n, 3), np.float32)
        self.opacity = np.zeros(n, np.float32)
        self.normal = np.zeros((n, 3), np.float32)
        self.radius = np.zeros(n, np.float32)
        self.support_sq = np.zeros(n, np.float32)
        self.material = np.zeros(n, np.uint32)
        rot = np.ascontiguousarray(rotations, np.float32).reshape(-1, 4)
        sc = np.ascontiguousarray(scales, np.float32).reshape(-1, 3)
        nr = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        mi = np.ascontiguousarray(material_indices, np.uint32)
        k = lib().bvo_relight_prepare(n, _ptr(points, f32p), _ptr(rot, f32p), _ptr(sc, f32p),
                                      _ptr(nr, f32p), _ptr(mi, u32p), _ptr(self.kept, u32p),
                                      _ptr(self.center, f32p), _ptr(self.rotation, f32p),
                                      _ptr(self.scale, f32p), _ptr(self.opacity, f32p),
                                      _ptr(self.normal, f32p), _ptr(self.radius, f32p),
                                      _ptr(self.support_sq, f32p), _ptr(self.material, u32p))
        self.n = int(k)
        mats = np.ascontiguousarray(materials, np.float32).reshape(-1, 8)
        self.materials = (Material * len(mats))()
        for i, row in enumerate(mats):
            self.materials[i] = material_struct(row[0:3], row[3], row[4:7])
        self.c = RelightScene(self.n, _ptr(self.center, f32p), _ptr(self.rotation, f32p),
                              _ptr(self.scale, f32p), _ptr(self.opacity, f32p),
                              _ptr(self.normal, f32p), _ptr(self.radius, f32p),
                              _ptr(self.support_sq, f32p), _ptr(self.material, u32p),
                              self.materials)

    @classmethod
    def from_scene(cls, g):
        return cls(g.points, g.rotations, g.scales, g.normals, g.material_indices, g.materials)


def _lights(lights):
    arr = (PointLight * len(lights))()
    for i, L in enumerate(lights):
        arr[i] = L if isinstance(L, PointLight) else light_struct(*L)
    return arr


def relight_ray(scene: RelightOracleScene, lights, origin, direction, depth,
                background=(0.0, 0.0, 0.0)):
    out = np.zeros(4, np.float32)
    hits = np.zeros(1, np.uint32)
    o = np.ascontiguousarray(origin, np.float32)
    d = np.ascontiguousarray(direction, np.float32)
    bg = np.ascontiguousarray(background, np.float32)
    arr = _lights(lights)
    lib().bvo_relight_ray(C.byref(scene.c), arr, len(arr), _ptr(o, f32p), _ptr(d, f32p),
                          float(depth), _ptr(bg, f32p), _ptr(out, f32p), _ptr(hits, u32p))
    return out, int(hits[0])


def relight_render(scene: RelightOracleScene, lights, cam, width, height,
                   background=(0.0, 0.0, 0.0), threads=0):
    out = np.zeros((height, width, 4), np.float32)
    hits = np.zeros((height, width), np.uint32)
    bg = np.ascontiguousarray(background, np.float32)
    arr = _lights(lights)
    cs = camera_struct(cam)
    lib().bvo_relight_render(C.byref(scene.c), arr, len(arr), C.byref(cs), width, height,
                             _ptr(bg, f32p), _ptr(out, f32p), _ptr(hits, u32p), threads)
    return out, hits


def relight_render_pixels(scene: RelightOracleScene, lights, cam, width, height, pixels,
                          background=(0.0, 0.0, 0.0), threads=0):
    """relight_render at the listed pixel indices (y * width + x) only."""
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    out = np.zeros((len(px), 4), np.float32)
    hits = np.zeros(len(px), np.uint32)
    bg = np.ascontiguousarray(background, np.float32)
    arr = _lights(lights)
    cs = camera_struct(cam)
    lib().bvo_relight_render_px(C.byref(scene.c), arr, len(arr), C.byref(cs), width, height,
                                _ptr(bg, f32p), len(px), _ptr(px, u32p), _ptr(out, f32p),
                                _ptr(hits, u32p), threads)
    return out, hits


def relight_render_f64_pixels(scene: RelightOracleScene, lights, cam, width, height, pixels,
                              background=(0.0, 0.0, 0.0), threads=0):
    """FP64 accuracy oracle of relight_render at the listed pixels: rgba
    [n, 4] float64."""
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    out = np.zeros((len(px), 4), np.float64)
    bg = np.ascontiguousarray(background, np.float32)
    arr = _lights(lights)
    cs = camera_struct(cam)
    lib().bvo_relight_render_f64_px(C.byref(scene.c), arr, len(arr), C.byref(cs), width, height,
                                    _ptr(bg, f32p), len(px), _ptr(px, u32p), _ptr(out, f64p),
                                    threads)
    return out


# --------------------------------------------------------------------------
# Gaussian ray tracing with SH colour (trace.rs:695-773)
# --------------------------------------------------------------------------
class GaussianOracleScene:
    """Particles with opacity > min_opacity (gpu/gaussian.rs:19-27), in model
    order, for the C side."""

    def __init__(self, points, rotations, scales, sh, sh_degree, min_opacity=0.01):
        points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        keep = points[:, 3] > np.float32(min_opacity)
        self.kept = np.nonzero(keep)[0].astype(np.uint32)
        self.center = np.ascontiguousarray(points[keep, :3])
        self.opacity = np.ascontiguousarray(points[keep, 3])
        self.rotation = np.ascontiguousarray(
            np.asarray(rotations, np.float32).reshape(-1, 4)[keep])
        self.scale = np.ascontiguousarray(np.asarray(scales, np.float32).reshape(-1, 3)[keep])
        k = (int(sh_degree) + 1) ** 2
        self.sh = np.ascontiguousarray(np.asarray(sh, np.float32).reshape(-1, 3 * k)[keep])
        self.n = int(keep.sum())
        self.min_opacity = float(min_opacity)
        self.c = GaussianScene(self.n, _ptr(self.center, f32p), _ptr(self.rotation, f32p),
                               _ptr(self.scale, f32p), _ptr(self.opacity, f32p),
                               _ptr(self.sh, f32p), int(sh_degree))

    @classmethod
    def from_scene(cls, g, min_opacity=0.01):
        return cls(g.points, g.rotations, g.scales, g.sh, g.sh_degree, min_opacity)


def trace_gaussians(scene: GaussianOracleScene, origin, direction, min_transmittance=0.01,
                    t_start=0.0, t_end=10000.0, background=(0.0, 0.0, 0.0)):
    """One ray; returns (rgba, composited hits).  ``direction`` is used as
    given (normalise it first, as trace_gaussians does)."""
    out = np.zeros(4, np.float32)
    hits = np.zeros(1, np.uint32)
    o = np.ascontiguousarray(origin, np.float32)
    d = np.ascontiguousarray(direction, np.float32)
    bg = np.ascontiguousarray(background, np.float32)
    st = GaussianSettings(scene.min_opacity, float(min_transmittance), float(t_start),
                          float(t_end))
    lib().bvo_trace_gaussians(C.byref(scene.c), _ptr(o, f32p), _ptr(d, f32p), C.byref(st),
                              _ptr(bg, f32p), _ptr(out, f32p), _ptr(hits, u32p))
    return out, int(hits[0])


def gaussian_render(scene: GaussianOracleScene, cam, width, height, min_transmittance=0.01,
                    background=(0.0, 0.0, 0.0), threads=0):
    out = np.zeros((height, width, 4), np.float32)
    hits = np.zeros((height, width), np.uint32)
    bg = np.ascontiguousarray(background, np.float32)
    cs = camera_struct(cam)
    lib().bvo_gaussian_render(C.byref(scene.c), C.byref(cs), width, height, scene.min_opacity,
                              float(min_transmittance), _ptr(bg, f32p), _ptr(out, f32p),
                              _ptr(hits, u32p), threads)
    return out, hits


def gaussian_render_pixels(scene: GaussianOracleScene, cam, width, height, pixels,
                           min_transmittance=0.01, background=(0.0, 0.0, 0.0), threads=0):
    """gaussian_render at the listed pixel indices (y * width + x) only."""
    px = np.ascontiguousarray(pixels, dtype=np.uint32)
    out = np.zeros((len(px), 4), np.float32)
    hits = np.zeros(len(px), np.uint32)
    bg = np.ascontiguousarray(background, np.float32)
    cs = camera_struct(cam)
    lib().bvo_gaussian_render_px(C.byref(scene.c), C.byref(cs), width, height,
                                 scene.min_opacity, float(min_transmittance), _ptr(bg, f32p),
                                 len(px), _ptr(px, u32p), _ptr(out, f32p), _ptr(hits, u32p),
                                 threads)
    return out, hits


# --------------------------------------------------------------------------
# optimizer step (Adam, FP32)
# --------------------------------------------------------------------------
class AdamOracle:
    """FP32 Adam over a model's tables (bvo_adam_step); starts from the
    model's values, the raw density parameter at the inverse activation."""

    def __init__(self, points, sh, radii, activation=0, softplus_beta=10.0):
        points = np.asarray(points, np.float32).reshape(-1, 4)
        n = len(points)
        self.activation = int(activation)
        self.beta = float(softplus_beta) if activation == 2 else 0.0
        self.density = np.ascontiguousarray(points[:, 3])
        self.x = np.array([lib().bvo_density_activation_inverse(float(y), self.activation,
                                                                  self.beta)
                           for y in self.density], np.float32)
        self.pos = np.ascontiguousarray(points[:, :3]).copy()
        self.sh = np.ascontiguousarray(sh, np.float32).reshape(n, -1).copy()
        self.radii = None if radii is None else np.ascontiguousarray(radii, np.float32).copy()
        z = lambda a: np.zeros_like(a)  # noqa: E731
        self.m_d, self.v_d = z(self.x), z(self.x)
        self.m_sh, self.v_sh = z(self.sh), z(self.sh)
        self.m_pos, self.v_pos = z(self.pos), z(self.pos)
        r = self.radii if self.radii is not None else np.zeros(n, np.float32)
        self.m_r, self.v_r = z(r), z(r)
        self.t = 0
        self.c = AdamState(n, self.sh.shape[1], _ptr(self.x, f32p), _ptr(self.m_d, f32p),
                           _ptr(self.v_d, f32p), _ptr(self.density, f32p), _ptr(self.sh, f32p),
                           _ptr(self.m_sh, f32p), _ptr(self.v_sh, f32p), _ptr(self.pos, f32p),
                           _ptr(self.m_pos, f32p), _ptr(self.v_pos, f32p),
                           _ptr(self.radii, f32p), _ptr(self.m_r, f32p), _ptr(self.v_r, f32p))

    def step(self, settings: dict, g_density=None, g_sh=None, g_pos=None, g_radii=None):
        a = AdamSettings(settings.get("lr_density", 0.0), settings.get("lr_sh_dc", 0.0),
                         settings.get("lr_sh_rest", 0.0), settings.get("lr_position", 0.0),
                         settings.get("lr_radius", 0.0), settings.get("beta1", 0.9),
                         settings.get("beta2", 0.999), settings.get("eps", 1e-15),
                         self.activation, self.beta)
        self.t += 1
        conv = lambda g: None if g is None else np.ascontiguousarray(g, np.float32).reshape(-1)  # noqa: E731
        gs = [conv(g) for g in (g_density, g_sh, g_pos, g_radii)]
        lib().bvo_adam_step(C.byref(self.c), C.byref(a), self.t, *[_ptr(g, f32p) for g in gs])

    def points(self):
        return np.concatenate([self.pos, self.density[:, None]], axis=1).astype(np.float32)
