"""PowerFoam splat render on the GPU (bv_powerfoam_splat_tracer_*) against
the oracle's trace_powerfoam_splats restatement (trace.rs:1456-1546).

The oracle scans every site per ray and sorts all clipped intervals; the
device walks its BVH in windows of 16.  Bit-identical images show that no
support is missed, that the windowed order is the full (depth, cell) sort,
and that clipping and compositing are the reference's arithmetic.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def gpu_render(model, cams, w, h, max_steps=1024, thr=1e-3):
    t = bv.PowerFoamSplatTracer(model, max_steps=max_steps, weight_threshold=thr)
    img = t.render(cams, w, h)
    torch.cuda.synchronize()
    out = img.cpu().numpy()
    t.deinit()
    return out


def assert_same(model, cams, w, h, max_steps=1024, thr=1e-3):
    gpu = gpu_render(model, cams, w, h, max_steps, thr)
    om = O.OracleModel.from_scene(model)
    for v, cam in enumerate(cams):
        ref, steps = O.render_splats(om, cam, w, h, max_steps, thr)
        bad = np.flatnonzero((bits(gpu[v]) != bits(ref)).any(axis=-1))
        assert bad.size == 0, (v, bad[:8], gpu[v].reshape(-1, 4)[bad[:3]], ref.reshape(-1, 4)[bad[:3]])
    return gpu


def test_reference_disconnected_supports_in_depth_order():
    """trace.rs:2397-2442: two supports with no overlap edge; the splat path
    finds both (the walk only the first)."""
    pts = np.array([[0, 0, 3, 1], [0, 0, 6, 1]], np.float32)
    m = scenes.PointCloudModel(pts, np.zeros((2, 3), np.float32), 0, np.zeros(3, np.uint32),
                               np.zeros(0, np.uint32), np.array([0.5, 0.5], np.float32))
    cam = scenes.looking_at((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), math.radians(10.0), 1.0, 10.0)
    img = assert_same(m, [cam], 1, 1, 32, 0.0)
    assert abs(img[0, 0, 0, 3] - (1.0 - math.exp(-2.0))) < 1e-5


@pytest.mark.parametrize("n,rmax,bf16,deg,seed", [
    (3000, 0.15, False, 3, 1),   # connected overlap graph, FP32 SH
    (3000, 0.15, True, 3, 2),    # BF16 SH storage
    (6000, 0.04, True, 3, 3),    # sparse radii: disconnected Cech graph
    (2000, 0.20, False, 1, 4),
    (2000, 0.20, False, 0, 5),
])
def test_random_powerfoam_bit_exact(n, rmax, bf16, deg, seed):
    m = scenes.powerfoam_mixture(n, seed=seed, sh_degree=deg, radius_max=rmax, bf16=bf16)
    cams = scenes.sphere_cameras(2, 3.0, seed, math.radians(50.0), 4 / 3, 100.0)
    # a camera inside the cloud: supports within 4 r of it are excluded
    cams.append(scenes.looking_at((0.05, -0.1, 0.2), (0.3, 0.2, -1.0), math.radians(70.0), 1.0, 100.0))
    img = assert_same(m, cams, 40, 30)
    assert (img[..., 3] > 0.05).mean() > 0.05


def test_max_steps_and_weight_threshold():
    m = scenes.powerfoam_mixture(3000, seed=7, radius_max=0.15, bf16=False)
    cams = scenes.sphere_cameras(1, 3.0, 7, math.radians(50.0), 1.0, 100.0)
    for max_steps, thr in ((1, 0.0), (3, 0.0), (17, 0.0), (40, 0.5), (1024, 0.2)):
        assert_same(m, cams, 24, 24, max_steps, thr)


def test_batched_views_equal_single_dispatch():
    m = scenes.powerfoam_mixture(4000, seed=8, radius_max=0.1)
    cams = scenes.sphere_cameras(5, 3.0, 8, math.radians(50.0), 1.0, 100.0)
    t = bv.PowerFoamSplatTracer(m)
    batch = t.render(cams, 33, 17).cpu().numpy()
    for v, cam in enumerate(cams):
        out = torch.empty((17, 33, 4), dtype=torch.float32, device="cuda")
        t.dispatch(out, cam, (33, 17))
        assert np.array_equal(bits(out.cpu().numpy()), bits(batch[v]))
    t.deinit()


def test_candidate_count_validation():
    # 1500 supports strung along the optical axis: the centre ray hits them all
    k = 1500
    pts = np.zeros((k, 4), np.float32)
    pts[:, 2] = np.linspace(2.0, 9.0, k, dtype=np.float32)
    pts[:, 3] = 0.5
    m = scenes.PointCloudModel(pts, np.zeros((k, 3), np.float32), 0, np.zeros(k + 1, np.uint32),
                               np.zeros(0, np.uint32), np.full(k, 0.3, np.float32))
    cam = scenes.looking_at((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), math.radians(1.0), 1.0, 20.0)
    t = bv.PowerFoamSplatTracer(m, max_steps=64)
    assert t.candidate_capacity == 1024
    t.render([cam], 3, 3)
    with pytest.raises(bv.BvError) as e:
        t.validate_candidate_counts()
    assert e.value.status == 5  # BV_ERR_CANDIDATE_OVERFLOW
    t.deinit()
    t = bv.PowerFoamSplatTracer(m, max_steps=64, candidate_capacity=4096)
    img = t.render([cam], 3, 3).cpu().numpy()
    assert t.validate_candidate_counts() == k
    ref, _ = O.render_splats(O.OracleModel.from_scene(m), cam, 3, 3, 64, 1e-3)
    assert np.array_equal(bits(img[0]), bits(ref))
    t.deinit()


def test_rejects_models_without_radii_and_bad_settings():
    m = scenes.radfoam_ball(500, seed=1, sh_degree=0)
    with pytest.raises(bv.BvError):
        bv.PowerFoamSplatTracer(m)
    p = scenes.powerfoam_mixture(500, seed=1, radius_max=0.1)
    with pytest.raises(bv.BvError):
        bv.PowerFoamSplatTracer(p, max_steps=0)


def test_stats_count_rays_and_intervals():
    m = scenes.powerfoam_mixture(3000, seed=9, radius_max=0.12, bf16=False)
    cam = scenes.sphere_cameras(1, 3.0, 9, math.radians(50.0), 1.0, 100.0)
    t = bv.PowerFoamSplatTracer(m, weight_threshold=0.0)
    t.enable_stats(True)
    t.render(cam, 20, 20)
    st = t.last_stats()
    _, steps = O.render_splats(O.OracleModel.from_scene(m), cam[0], 20, 20, 1024, 0.0)
    assert st.rays == 400 and st.steps == int(steps.sum()) and st.kernel_ms > 0
    t.deinit()


def test_repeated_renders_take_tiles_heaviest_first_bit_exact():
    """A dispatch of the same shape as the one before takes its tiles in the
    order of the previous dispatch's tile durations (three more launches build
    it); the image does not depend on that order, for the same cameras or
    moved ones."""
    m = scenes.powerfoam_mixture(3000, seed=4, radius_max=0.15)
    cams = scenes.sphere_cameras(2, 3.0, 5, math.radians(55.0), 1.0, 100.0)
    moved = scenes.sphere_cameras(2, 3.0, 6, math.radians(55.0), 1.0, 100.0)
    om = O.OracleModel.from_scene(m)
    t = bv.PowerFoamSplatTracer(m)
    try:
        for views in (cams, cams, moved, cams):
            img = t.render(views, 48, 40)
            torch.cuda.synchronize()
            assert t.last_stats().launches == 4  # render, tile order x 3
            got = img.cpu().numpy()
            for v, cam in enumerate(views):
                ref, _ = O.render_splats(om, cam, 48, 40)
                assert np.array_equal(bits(got[v]), bits(ref)), v
    finally:
        t.deinit()


def test_dispatches_on_two_streams_are_ordered():
    """Three dispatches of one tracer of the same shape, on alternating
    streams with no host synchronisation: each later one reads the tile
    order the one before it writes, so it waits for it; every image matches
    the oracle."""
    m = scenes.powerfoam_mixture(3000, seed=7, radius_max=0.15)
    cams = scenes.sphere_cameras(3, 3.0, 8, math.radians(55.0), 1.0, 100.0)
    om = O.OracleModel.from_scene(m)
    t = bv.PowerFoamSplatTracer(m)
    try:
        streams = [torch.cuda.Stream(), torch.cuda.Stream()]
        outs = [torch.empty((1, 40, 48, 4), dtype=torch.float32, device="cuda") for _ in cams]
        for k, cam in enumerate(cams):
            t.dispatch_batch(outs[k], [cam], (48, 40), stream=streams[k % 2])
        torch.cuda.synchronize()
        for k, cam in enumerate(cams):
            ref, _ = O.render_splats(om, cam, 48, 40)
            assert np.array_equal(bits(outs[k].cpu().numpy()[0]), bits(ref)), k
    finally:
        t.deinit()
