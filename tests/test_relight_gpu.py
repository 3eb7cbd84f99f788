"""Relightable Gaussians on the GPU (bv_relight_tracer_*) against the oracle.

The oracle scans every particle per ray (no acceleration structure) and
sorts all hits; the device traverses its BVH in windows of 16.  Equal
images (bit for bit) show that the BVH misses no hit, that the windowed
order equals the full sort, and that shading and blending are the
reference's arithmetic.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.test_relight_oracle import LIGHT, SIZE, camera, gaussians  # noqa: E402

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def gpu_render(model, lights, cam, w, h, background=(0.0, 0.0, 0.0)):
    t = bv.RelightTracer(model, background=background)
    t.set_point_lights(lights)
    out = t.render(cam, w, h)
    torch.cuda.synchronize()
    img = out.cpu().numpy()
    t.deinit()
    return img


def assert_same(model, lights, cam, w, h, background=(0.0, 0.0, 0.0)):
    gpu = gpu_render(model, lights, cam, w, h, background)
    ref, hits = O.relight_render(O.RelightOracleScene.from_scene(model), lights, cam, w, h,
                                 background)
    bad = np.flatnonzero((bits(gpu) != bits(ref)).any(axis=-1))
    assert bad.size == 0, (bad[:8], gpu.reshape(-1, 4)[bad[:3]], ref.reshape(-1, 4)[bad[:3]])
    return gpu, hits


def test_reference_group_case_13_coincident_gaussians():
    count = 13
    mats = [scenes.make_material((0.8, 0.1, 0.05), 0.7), scenes.make_material((0.05, 0.1, 0.8), 0.7)]
    g = gaussians([[0, 0, 0, 0.8]] * count, (0.45, 0.7, 0.25), materials=mats,
                  material_indices=[int(i + 1 == count) for i in range(count)])
    img, _ = assert_same(g, LIGHT, camera(4.0), *SIZE, background=(0.02, 0.03, 0.05))
    assert (img[..., 3] > 0).sum() > 1000


def test_reference_deep_traversal_192_sheets():
    g = gaussians([[0, 0, 0.2 * i, 0.031] for i in range(192)], (4.0, 4.0, 0.00005))
    _, hits = assert_same(g, LIGHT, camera(4.0), *SIZE, background=(0.02, 0.03, 0.05))
    assert hits.max() > 96


def test_reference_camera_depth_interval():
    cam = camera(4.0)
    cam.depth = 1.0
    near = gaussians([[0, 0, -3.5, 0.8]], (4, 4, 4))
    far = gaussians([[0, 0, 0, 0.8]], (1, 1, 1))
    img_near, _ = assert_same(near, LIGHT, cam, *SIZE)
    img_far, _ = assert_same(far, LIGHT, cam, *SIZE)
    c = (SIZE[1] // 2, SIZE[0] // 2)
    assert img_near[c][3] > 0.5 and img_far[c][3] < 0.001


@pytest.mark.parametrize("n,seed", [(3000, 1), (20000, 2)])
def test_random_anisotropic_scene_bit_exact(n, seed):
    g = scenes.relight_gaussians(n, seed=seed)
    cam = scenes.sphere_cameras(1, 3.0, seed, math.radians(60.0), 4 / 3, 100.0)[0]
    lights = scenes.sphere_lights(4)
    img, hits = assert_same(g, lights, cam, 64, 48)
    assert (img[..., 3] > 0.5).mean() > 0.05
    assert hits.max() > 16  # several windows per ray


def test_sixteen_lights_sum_single_light_renders():
    """The configuration's 16 lights: alpha is light-independent, radiance is
    the sum of single-light renders (zero background)."""
    g = scenes.relight_gaussians(4000, seed=3)
    cam = scenes.sphere_cameras(1, 3.0, 3, math.radians(60.0), 4 / 3, 100.0)[0]
    lights = scenes.sphere_lights(16)
    all16 = gpu_render(g, lights, cam, 48, 36)
    acc = np.zeros_like(all16)
    for L in lights:
        one = gpu_render(g, [L], cam, 48, 36)
        assert np.array_equal(bits(one[..., 3]), bits(all16[..., 3]))
        acc[..., :3] += one[..., :3]
    scale = max(1.0, float(np.abs(all16[..., :3]).max()))
    assert np.abs(acc[..., :3] - all16[..., :3]).max() <= 1e-5 * scale


def test_rejects_bad_models_and_lights():
    g = gaussians([[0, 0, 0, 0.8]], (1, 1, 1))
    g.rotations[0] = [0, 0, 0, 2.0]
    with pytest.raises(bv.BvError):
        bv.RelightTracer(g)
    g = gaussians([[0, 0, 0, 0.8]], (1, 1, 1))
    t = bv.RelightTracer(g)
    with pytest.raises(bv.BvError):
        t.set_point_lights([((0, 0, 0), (0, 0, 0), (1, 1, 1), 2.0)])  # exponent needs a direction
    with pytest.raises(bv.BvError):
        t.render(camera(4.0), 8, 8)  # no light set


def test_one_tracer_several_cameras():
    """Each dispatch rewrites the tracer's per-view table of particle origin
    terms: one tracer rendering camera A, B, then A again matches the oracle
    bit for bit every time."""
    g = scenes.relight_gaussians(4000, seed=5)
    cams = scenes.sphere_cameras(2, 3.0, 6, math.radians(60.0), 4 / 3, 100.0)
    lights = scenes.sphere_lights(3)
    osc = O.RelightOracleScene.from_scene(g)
    t = bv.RelightTracer(g)
    t.set_point_lights(lights)
    for cam in (cams[0], cams[1], cams[0]):
        img = t.render(cam, 48, 36).cpu().numpy()
        ref, _ = O.relight_render(osc, lights, cam, 48, 36, (0.0, 0.0, 0.0))
        assert np.array_equal(bits(img), bits(ref))
    t.deinit()


def test_dispatches_on_two_streams_are_ordered():
    """Two dispatches of one tracer on different streams, with no host
    synchronisation between them: the second waits for the first (both
    rewrite the per-view table), so both images match the oracle."""
    g = scenes.relight_gaussians(4000, seed=7)
    cams = scenes.sphere_cameras(2, 3.0, 8, math.radians(60.0), 4 / 3, 100.0)
    lights = scenes.sphere_lights(2)
    osc = O.RelightOracleScene.from_scene(g)
    t = bv.RelightTracer(g)
    t.set_point_lights(lights)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    out = [torch.empty((36, 48, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    t.enable_stats(True)
    t.dispatch(out[0], cams[0], (48, 36), stream=s1)
    t.dispatch(out[1], cams[1], (48, 36), stream=s2)
    assert t.last_stats().launches == 5  # origin terms, trace, tile order x 3
    torch.cuda.synchronize()
    for k in range(2):
        ref, _ = O.relight_render(osc, lights, cams[k], 48, 36, (0.0, 0.0, 0.0))
        assert np.array_equal(bits(out[k].cpu().numpy()), bits(ref))
    t.deinit()
