"""SH-coloured Gaussians on the GPU (bv_gaussian_tracer_*) against the oracle.

The oracle (trace_gaussians, trace.rs:695-773) scans every particle per ray
and sorts all hits; the device traverses its BVH in windows of 16 keys.
Bit-equal images show that the BVH misses no hit, that the windowed order is
the full (depth, index) sort, and that the compositing is the reference's
arithmetic.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.test_gaussian_oracle import model, two_gaussians  # noqa: E402

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def axis_camera(depth=100.0):
    """1x1 image whose only ray is exactly +z from the origin."""
    return scenes.Camera(position=np.zeros(3, np.float32), depth=depth,
                         orientation=np.array([0, 0, 0, 1], np.float32),
                         fov=np.array([1.0, 1.0], np.float32), principal=np.zeros(2, np.float32))


def assert_same(g, cam, w, h, min_opacity=0.01, min_transmittance=0.01, background=(0, 0, 0)):
    t = bv.GaussianTracer(g, min_opacity=min_opacity, min_transmittance=min_transmittance,
                          background=background)
    t.enable_stats(True)
    out = t.render(cam, w, h)
    st = t.last_stats()
    img = out.cpu().numpy()
    s = O.GaussianOracleScene.from_scene(g, min_opacity)
    assert t.num_points == s.n
    ref, hits = O.gaussian_render(s, cam, w, h, min_transmittance, background)
    t.deinit()
    bad = np.flatnonzero((bits(img) != bits(ref)).any(axis=-1))
    assert bad.size == 0, (bad[:8], img.reshape(-1, 4)[bad[:3]], ref.reshape(-1, 4)[bad[:3]])
    assert st.rays == w * h and st.steps == int(hits.sum())
    return img, hits


def test_reference_two_gaussians():
    img, hits = assert_same(two_gaussians(), axis_camera(10.0), 1, 1, min_transmittance=0.0)
    assert np.abs(img[0, 0] - [0.5, 0.0, 0.25, 0.75]).max() < 1e-6 and hits[0, 0] == 2


def test_equal_depth_hits_across_many_windows():
    """45 hits in groups of three at equal depth (trace.rs:965-998 at a
    scale that needs three windows of 16): the cursor keeps every hit once,
    in (t, index) order."""
    idx = np.arange(45)[::-1]
    g = model([[0, 0, 1.0 + i // 3, 0.04 + 0.01 * (i % 5)] for i in idx], [[1, 1, 1]] * 45,
              [[(i % 3) / 2.0, (i % 5) / 4.0, (i % 7) / 6.0] for i in idx])
    img, hits = assert_same(g, axis_camera(), 1, 1, min_transmittance=0.0)
    assert hits[0, 0] == 45


@pytest.mark.parametrize("deg", [0, 1, 2, 3])
def test_random_scene_bit_exact(deg):
    g = scenes.gaussian_sh(12000, seed=deg + 1, sh_degree=deg, log_scale_mean=-3.0)
    cam = scenes.sphere_cameras(1, 3.0, deg + 1, math.radians(60.0), 4 / 3, 100.0)[0]
    img, hits = assert_same(g, cam, 64, 48, background=(0.1, 0.2, 0.3))
    assert (img[..., 3] > 0.5).mean() > 0.05
    assert hits.max() > 16  # several windows per ray


def test_transmittance_and_background_settings():
    g = scenes.gaussian_sh(6000, seed=9, sh_degree=2, log_scale_mean=-3.0)
    cam = scenes.sphere_cameras(1, 3.0, 9, math.radians(60.0), 1.0, 100.0)[0]
    assert_same(g, cam, 40, 40, min_opacity=0.05, min_transmittance=0.2, background=(1, 0, 0))
    t = bv.GaussianTracer(g)
    t.set_min_transmittance(0.2)
    t.set_background([1.0, 0.0, 0.0])
    a = t.render(cam, 40, 40).cpu().numpy()
    b, _ = O.gaussian_render(O.GaussianOracleScene.from_scene(g, 0.01), cam, 40, 40, 0.2,
                             (1.0, 0.0, 0.0))
    assert np.array_equal(bits(a), bits(b))
    with pytest.raises(bv.BvError):
        t.set_min_transmittance(-1.0)
    t.deinit()


def test_one_tracer_several_cameras():
    """Each dispatch rewrites the tracer's per-view table of particle origin
    terms: one tracer rendering camera A, B, then A again matches the oracle
    bit for bit every time."""
    g = scenes.gaussian_sh(8000, seed=11, sh_degree=2, log_scale_mean=-3.0)
    cams = scenes.sphere_cameras(2, 3.0, 12, math.radians(60.0), 4 / 3, 100.0)
    s = O.GaussianOracleScene.from_scene(g, 0.01)
    t = bv.GaussianTracer(g)
    for cam in (cams[0], cams[1], cams[0]):
        img = t.render(cam, 48, 36).cpu().numpy()
        ref, _ = O.gaussian_render(s, cam, 48, 36, 0.01, (0, 0, 0))
        assert np.array_equal(bits(img), bits(ref))
    t.deinit()


def test_dispatches_on_two_streams_are_ordered_and_counted():
    """Two dispatches of one tracer on different streams, with no host
    synchronisation between them: the second waits for the first (both
    rewrite the tracer's per-view table), so both images match the oracle.
    The launch count reports the five kernels enqueued."""
    import torch

    g = scenes.gaussian_sh(8000, seed=13, sh_degree=1, log_scale_mean=-3.0)
    cams = scenes.sphere_cameras(2, 3.0, 14, math.radians(60.0), 4 / 3, 100.0)
    s = O.GaussianOracleScene.from_scene(g, 0.01)
    t = bv.GaussianTracer(g)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    out = [torch.empty((36, 48, 4), dtype=torch.float32, device="cuda") for _ in range(2)]
    t.enable_stats(True)
    t.dispatch(out[0], cams[0], (48, 36), stream=s1)
    t.dispatch(out[1], cams[1], (48, 36), stream=s2)
    assert t.last_stats().launches == 5  # origin terms, trace, tile order x 3
    torch.cuda.synchronize()
    for k in range(2):
        ref, _ = O.gaussian_render(s, cams[k], 48, 36, 0.01, (0, 0, 0))
        assert np.array_equal(bits(out[k].cpu().numpy()), bits(ref))
    t.deinit()
