"""Pins the relight oracle (relight.wgsl kernel 2 + point light, and the
CPU twin relight.rs) against the reference's own tests."""

import math

import numpy as np
import pytest

from blade_volume_b200 import scenes
from oracle import oracle as O

SIZE = (96, 72)  # tests/relight_gpu_vs_cpu.rs:17


def test_point_light_distance_and_angular_falloff():
    """relight.rs:1024-1048."""
    light = O.light_struct((0, 0, 0), (0, 0, 1), (4, 8, 12), 2.0)
    white = O.material_struct((1, 1, 1), 0.5, (0, 0, 0))
    on_axis = O.point_light_shade(light, (0, 0, 2), (0, 0, -1), (0, 0, -1), white, cpu=True)
    assert list(on_axis) == [1.0, 2.0, 3.0]
    assert list(O.point_light_shade(light, (0, 0, 2), (0, 0, 1), (0, 0, -1), white,
                                    cpu=True)) == [0.0, 0.0, 0.0]
    towards = -np.array([0, 2, 2], np.float32) / np.linalg.norm([0, 2, 2])
    diag = O.point_light_shade(light, (0, 2, 2), towards, towards, white, cpu=True)
    assert np.abs(diag - [0.25, 0.5, 0.75]).max() < 1e-6


def test_point_light_shading_keeps_diffuse_only_explicit():
    """relight.rs:1050-1082."""
    light = O.light_struct((0, 0, 2), (0, 0, -1), (4, 4, 4), 0.0)
    m = O.material_struct((0.5, 0.5, 0.5), 0.25, (0, 0, 0))
    for cpu in (True, False):
        diffuse = O.point_light_shade(light, (0, 0, 0), (0, 0, 1), (0, 0, 1), m, cpu=cpu)
        assert list(diffuse) == [0.5, 0.5, 0.5]
    m = O.material_struct((0.5, 0.5, 0.5), 0.25, (0.04, 0.04, 0.04))
    for cpu in (True, False):
        assert np.all(O.point_light_shade(light, (0, 0, 0), (0, 0, 1), (0, 0, 1), m,
                                          cpu=cpu) > 0.5)


def test_shader_and_cpu_point_light_agree():
    """The shader form (relight.wgsl:190-261) and relight.rs:295-323 within
    the reference's GPU-vs-CPU point-light tolerance 0.002
    (tests/relight_gpu_vs_cpu.rs:466)."""
    rng = np.random.default_rng(0)
    worst = 0.0
    for _ in range(2000):
        L = O.light_struct(rng.uniform(-3, 3, 3), (0, 0, 1), rng.uniform(0, 6, 3), 0.0)
        p = rng.uniform(-1, 1, 3).astype(np.float32)
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        m = O.material_struct(rng.random(3), rng.uniform(0.2, 0.9), (0.04, 0.04, 0.04))
        a = O.point_light_shade(L, p, n.astype(np.float32), v.astype(np.float32), m)
        b = O.point_light_shade(L, p, n.astype(np.float32), v.astype(np.float32), m, cpu=True)
        worst = max(worst, float(np.abs(a - b).max() / max(1.0, np.abs(b).max())))
    assert worst < 0.002, worst


def camera(distance):
    """tests/relight_gpu_vs_cpu.rs:160-170."""
    fov_y = 0.9
    aspect = SIZE[0] / SIZE[1]
    return scenes.Camera(position=np.array([0, 0, -distance], np.float32), depth=100.0,
                         orientation=np.array([0, 0, 0, 1], np.float32),
                         fov=np.array([2 * math.atan(math.tan(0.5 * fov_y) * aspect), fov_y],
                                      np.float32),
                         principal=np.zeros(2, np.float32))


def gaussians(points, scale, normal=(0, 0, -1), materials=None, material_indices=None):
    n = len(points)
    mats = materials if materials is not None else [scenes.make_material((0.8, 0.4, 0.2), 0.9)]
    return scenes.GaussianModel(
        np.asarray(points, np.float32), np.tile(np.float32([0, 0, 0, 1]), (n, 1)),
        np.tile(np.asarray(scale, np.float32), (n, 1)), np.tile(np.float32(normal), (n, 1)),
        np.asarray(material_indices if material_indices is not None else [0] * n, np.uint32),
        np.asarray(mats, np.float32))


LIGHT = [((0.0, 0.0, -4.0), (0.0, 0.0, 1.0), (6.0, 5.0, 4.0), 0.0)]


def test_groups_across_windows_closed_form():
    """volumetric_gaussian_pbr_groups_across_traversal_batches
    (relight_gpu_vs_cpu.rs:625-750): 13 coincident Gaussians form one group,
    alpha = union + 0.75 (saturated - union), colour = mean shading;
    lit by a point light instead of the environment."""
    count = 13
    mats = [scenes.make_material((0.8, 0.1, 0.05), 0.7), scenes.make_material((0.05, 0.1, 0.8), 0.7)]
    g = gaussians([[0, 0, 0, 0.8]] * count, (0.45, 0.7, 0.25), materials=mats,
                  material_indices=[int(i + 1 == count) for i in range(count)])
    sc = O.RelightOracleScene.from_scene(g)
    cam = camera(4.0)
    bg = (0.02, 0.03, 0.05)
    img, _ = O.relight_render(sc, LIGHT, cam, *SIZE, background=bg)
    covered, worst = 0, 0.0
    for y in range(SIZE[1]):
        for x in range(SIZE[0]):
            o, d = O.camera_ray(cam, SIZE[0], SIZE[1], x, y)
            lo = o / np.float32([0.45, 0.7, 0.25])
            ld = d / np.float32([0.45, 0.7, 0.25])
            t = -lo.dot(ld) / ld.dot(ld)
            lp = lo + t * ld
            a = 0.0
            if t > 0:
                sq = lp.dot(lp)
                if sq <= 2 * math.log(0.8 / 0.03):
                    resp = min(0.8 * math.exp(-0.5 * sq), 0.999)
                    a = 1 - (1 - resp) ** 1.1
            union = 1 - (1 - a) ** count
            sat = min(count * a, 1.0)
            alpha = union + 0.75 * (sat - union)
            covered += alpha > 0
            point = o + t * d
            view = -d
            lit = np.zeros(3)
            for k in range(count):
                m = O.material_struct(mats[int(k + 1 == count)][0:3], 0.7, (0.04,) * 3)
                lit += O.point_light_shade(O.light_struct(*LIGHT[0]), point, (0, 0, -1), view,
                                           m) / count
            exp_rgb = alpha * lit + (1 - alpha) * np.asarray(bg)
            worst = max(worst, float(np.abs(img[y, x, :3] - exp_rgb).max()),
                        abs(float(img[y, x, 3]) - alpha))
    assert covered > 1000
    assert worst < 0.02, worst  # TOLERANCE, relight_gpu_vs_cpu.rs:21


def test_traverses_past_many_windows():
    """volumetric_gaussian_pbr_traverses_past_eight_batches (:829-915):
    192 thin sheets, the complete hit list decides alpha."""
    pts = [[0, 0, 0.2 * i, 0.031] for i in range(192)]
    g = gaussians(pts, (4.0, 4.0, 0.00005))
    sc = O.RelightOracleScene.from_scene(g)
    cam = camera(4.0)
    x, y = SIZE[0] // 2, SIZE[1] // 2
    o, d = O.camera_ray(cam, SIZE[0], SIZE[1], x, y)
    out, _ = O.relight_ray(sc, LIGHT, o, d, cam.depth)
    T, hits = 1.0, 0
    for p in pts:
        if T <= 0.003:
            break
        lo = (o - np.float32(p[:3])) / np.float32([4, 4, 0.00005])
        ld = d / np.float32([4, 4, 0.00005])
        t = -lo.dot(ld) / ld.dot(ld)
        lp = lo + t * ld
        resp = 0.031 * math.exp(-0.5 * lp.dot(lp))
        if t > 0 and resp >= 0.03:
            T *= 1 - (1 - (1 - min(resp, 0.999)) ** 1.1)
            hits += 1
    assert hits > 96
    assert abs(out[3] - (1 - T)) < 0.005


def test_respects_the_camera_depth_interval():
    """volumetric_gaussian_pbr_respects_the_camera_depth_interval (:753-827)."""
    cam = camera(4.0)
    cam.depth = 1.0
    x, y = SIZE[0] // 2, SIZE[1] // 2
    o, d = O.camera_ray(cam, SIZE[0], SIZE[1], x, y)
    near = O.RelightOracleScene.from_scene(gaussians([[0, 0, -3.5, 0.8]], (4, 4, 4)))
    far = O.RelightOracleScene.from_scene(gaussians([[0, 0, 0, 0.8]], (1, 1, 1)))
    assert O.relight_ray(near, LIGHT, o, d, cam.depth)[0][3] > 0.5
    assert O.relight_ray(far, LIGHT, o, d, cam.depth)[0][3] < 0.001


def test_log_and_pow_accuracy():
    worst = 0.0
    for x in np.concatenate([np.logspace(-30, 30, 4001), np.linspace(0.5, 2.0, 4001)]).astype(
            np.float32):
        ref = math.log(float(x))
        got = O.logf(float(x))
        worst = max(worst, abs(got - ref) / float(np.spacing(np.float32(abs(ref)) or 1e-30)))
    assert worst <= 2.0, worst
    # pow = exp(y log x): the rounding of y log x is amplified by |y log x|
    # (up to 7.6 here), hence 8 ulp
    for x in np.linspace(0.001, 1.0, 2001).astype(np.float32):
        ref = float(x) ** 1.1
        assert abs(O.powf(float(x), 1.1) - ref) <= 8 * float(np.spacing(np.float32(ref)))
