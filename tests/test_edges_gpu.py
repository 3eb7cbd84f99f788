"""Edge cases across the tracers against the oracle: ragged image sizes (edge
tiles with inactive lanes), more than 32 views in one call (several
launches), a camera inside the scene, and axis-aligned rays (exact zero
direction components through the slab tests)."""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu

RAGGED = (37, 23)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def axis_camera(position, depth=100.0, fov=1.2):
    return scenes.Camera(position=np.asarray(position, np.float32), depth=depth,
                         orientation=np.array([0, 0, 0, 1], np.float32),
                         fov=np.array([fov, fov], np.float32), principal=np.zeros(2, np.float32))


@pytest.fixture(scope="module")
def ball():
    return scenes.radfoam_ball(3000, seed=21, sh_degree=1)


@pytest.fixture(scope="module")
def foam():
    return scenes.powerfoam_mixture(4000, seed=21, sh_degree=1, radius_max=0.1)


def walk_ref(model, cam, w, h):
    om = O.OracleModel.from_scene(model)
    ref, *_ = O.render_walk(om, cam, w, h, 1024, 1e-3)
    return ref


@pytest.mark.parametrize("where", ["outside", "inside", "axis"])
def test_walk_ragged_inside_and_axis_aligned(ball, where):
    cam = {"outside": scenes.sphere_cameras(1, 3.0, 21, math.radians(60.0), 37 / 23, 100.0)[0],
           "inside": axis_camera([0.05, -0.02, 0.1]),
           "axis": axis_camera([0.0, 0.0, -3.0])}[where]
    t = bv.RadFoamGpuTracer(ball)
    got = t.render([cam], *RAGGED)[0].cpu().numpy()
    t.deinit()
    assert np.array_equal(bits(got), bits(walk_ref(ball, cam, *RAGGED)))


@pytest.mark.parametrize("where", ["outside", "inside", "axis"])
def test_splat_ragged_inside_and_axis_aligned(foam, where):
    cam = {"outside": scenes.sphere_cameras(1, 3.0, 22, math.radians(60.0), 37 / 23, 100.0)[0],
           "inside": axis_camera([0.05, -0.02, 0.1]),
           "axis": axis_camera([0.0, 0.0, -3.0])}[where]
    t = bv.PowerFoamSplatTracer(foam)
    got = t.render([cam], *RAGGED)[0].cpu().numpy()
    t.deinit()
    ref, _ = O.render_splats(O.OracleModel.from_scene(foam), cam, *RAGGED, 1024, 1e-3)
    assert np.array_equal(bits(got), bits(ref))


def test_more_than_32_views_in_one_call(ball, foam):
    cams = scenes.sphere_cameras(35, 3.0, 23, math.radians(60.0), 1.0, 100.0)
    w = h = 8
    t = bv.RadFoamGpuTracer(ball)
    s = bv.PowerFoamSplatTracer(foam)
    walk = t.render(cams, w, h).cpu().numpy()
    splat = s.render(cams, w, h).cpu().numpy()
    om_b, om_f = O.OracleModel.from_scene(ball), O.OracleModel.from_scene(foam)
    for v in (0, 31, 32, 34):
        ref, *_ = O.render_walk(om_b, cams[v], w, h, 1024, 1e-3)
        assert np.array_equal(bits(walk[v]), bits(ref)), v
        ref, _ = O.render_splats(om_f, cams[v], w, h, 1024, 1e-3)
        assert np.array_equal(bits(splat[v]), bits(ref)), v
    # training over 35 views: one call equals the oracle's loss over all views
    target = np.random.default_rng(2).random((35, h, w, 3)).astype(np.float32)
    tg = torch.from_numpy(target).cuda()
    for tracer, model, splats in ((t, ball, False), (s, foam, True)):
        grads = tracer.new_grads()
        loss = float(tracer.forward_backward(cams, w, h, tg, grads).item())
        ref = O.forward_backward(O.OracleModel.from_scene(model), cams, w, h, target=target,
                                 splats=splats)
        assert abs(loss - ref["loss"]) <= 1e-5 * ref["loss"]
        g = grads["d_density"].cpu().numpy()
        assert np.abs(g - ref["d_density"]).max() <= 1e-4 * np.abs(ref["d_density"]).max()
    t.deinit()
    s.deinit()


def test_gaussian_and_relight_ragged_and_axis_aligned():
    g = scenes.gaussian_sh(5000, seed=24, sh_degree=1, log_scale_mean=-3.0)
    rg = scenes.relight_gaussians(5000, seed=24)
    lights = scenes.sphere_lights(2)
    for cam in (scenes.sphere_cameras(1, 3.0, 24, math.radians(60.0), 37 / 23, 100.0)[0],
                axis_camera([0.0, 0.0, -3.0])):
        gt = bv.GaussianTracer(g)
        got = gt.render(cam, *RAGGED).cpu().numpy()
        gt.deinit()
        ref, _ = O.gaussian_render(O.GaussianOracleScene.from_scene(g), cam, *RAGGED)
        assert np.array_equal(bits(got), bits(ref))
        rt = bv.RelightTracer(rg)
        rt.set_point_lights(lights)
        got = rt.render(cam, *RAGGED).cpu().numpy()
        rt.deinit()
        ref, _ = O.relight_render(O.RelightOracleScene.from_scene(rg), lights, cam, *RAGGED)
        assert np.array_equal(bits(got), bits(ref))
