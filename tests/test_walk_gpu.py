"""GPU parity of the walk through the C ABI against the CPU oracle.

Bar: bit-exact for cell sequences, t/dt values and the FP32 pixels (the
kernels evaluate the oracle's operation sequence; see bv_walk.cu), plus the
reference's own GPU-vs-CPU tolerance (5e-3, radfoam_gpu_vs_cpu.rs:368) on
its own fixture and pixels.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests.golden.fixtures import TEST_PIXELS, branching_model, gpu_vs_cpu_camera  # noqa: E402

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def render_gpu(tracer, cams, w, h):
    out = tracer.render(cams, w, h)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def tiny():
    return scenes.radfoam_tiny()


def test_reference_branching_fixture_plain_and_power():
    """radfoam_gpu_vs_cpu.rs:437-484 fixture, camera and parameters."""
    cam = gpu_vs_cpu_camera()
    for radii in (None, "power"):
        model = branching_model()
        if radii == "power":
            model.radii = np.where(np.arange(model.n) < 64, 0.015, 0.030).astype(np.float32)
        t = bv.RadFoamGpuTracer(model, max_steps=256, weight_threshold=1e-4)
        out = torch.empty((8, 8, 4), dtype=torch.float32, device="cuda")
        t.dispatch(out, cam, (8, 8))
        gpu = out.cpu().numpy()
        om = O.OracleModel.from_scene(model)
        start = t.start_point()
        assert start == O.containing_cell_f64(om, cam.position) == 0
        ref, _, _, _ = O.render_walk(om, cam, 8, 8, 256, 1e-4, start)
        assert np.array_equal(bits(gpu), bits(ref))
        for x, y in TEST_PIXELS:
            assert np.abs(gpu[y, x] - ref[y, x]).max() <= 5e-3
        assert np.all(np.isfinite(gpu)) and gpu[..., 3].max() > 0.0


def test_tiny_workload_image_bit_exact(tiny):
    """16,384-site Delaunay ball, 128x128, SH degree 0: every pixel."""
    m, cam = tiny.model, tiny.cameras[0]
    t = bv.RadFoamGpuTracer(m, max_steps=tiny.max_steps, weight_threshold=tiny.weight_threshold)
    gpu = render_gpu(t, [cam], tiny.width, tiny.height)[0]
    om = O.OracleModel.from_scene(m)
    start = O.containing_cell_f64(om, cam.position)
    assert t.start_point() == start
    ref, steps, _, _ = O.render_walk(om, cam, tiny.width, tiny.height, tiny.max_steps,
                                     tiny.weight_threshold, start)
    mismatch = np.flatnonzero((bits(gpu) != bits(ref)).any(axis=-1))
    assert mismatch.size == 0, (mismatch[:10], gpu.reshape(-1, 4)[mismatch[:3]],
                                ref.reshape(-1, 4)[mismatch[:3]])
    assert steps.mean() > 5
    assert gpu[..., 3].min() > 0.0


def test_record_paths_bit_exact_cells_dt_and_jacobians(tiny):
    """PathRecorder rows vs record_path_jacobians: cells, entry/exit sites
    exact, dt and Jacobians bit-exact, status count + truncation bit."""
    m, cam = tiny.model, tiny.cameras[0]
    w = h = 64
    L = 24
    t = bv.RadFoamGpuTracer(m)
    gpu = t.record_paths([cam], w, h, L)
    torch.cuda.synchronize()
    om = O.OracleModel.from_scene(m)
    ref = O.record_image(om, [cam], w, h, L)
    g = {k: v.cpu().numpy() for k, v in gpu.items()}
    assert np.array_equal(g["path_status"].view(np.uint32), ref["path_status"])
    counts = ref["path_status"] & 0x7FFFFFFF
    assert (ref["path_status"] >> 31).sum() > 0, "expected truncated rays at L=24"
    assert (ref["path_status"] >> 31).sum() < len(counts)
    for p in range(len(counts)):
        c = int(counts[p])
        for key in ("previous_cells", "cells", "next_cells"):
            assert np.array_equal(g[key][p, :c].view(np.uint32), ref[key][p, :c]), (key, p)
        assert np.array_equal(bits(g["dts"][p, :c]), bits(ref["dts"][p, :c])), p
        for key in ("dt_grad_previous", "dt_grad_current", "dt_grad_next"):
            assert np.array_equal(bits(g[key][p, :c]), bits(ref[key][p, :c])), (key, p)


def test_visited_cell_sequences_bit_exact(tiny):
    """The render walk's per-ray visited cells equal the recorder's cells
    (plain RadFoam emits one segment per visited cell).  The threshold -1
    disables the transmittance cut (T <= 0 happens once T underflows)."""
    m, cam = tiny.model, tiny.cameras[0]
    om = O.OracleModel.from_scene(m)
    start = O.containing_cell_f64(om, cam.position)
    _, _, cells, counts = O.render_walk(om, cam, 32, 32, 1024, -1.0, start, cell_capacity=512)
    t = bv.RadFoamGpuTracer(m)
    gpu = t.record_paths([cam], 32, 32, 512, jacobians=False)
    torch.cuda.synchronize()
    gc = gpu["cells"].cpu().numpy().view(np.uint32).reshape(32, 32, 512)
    gs = gpu["path_status"].cpu().numpy().view(np.uint32).reshape(32, 32) & 0x7FFFFFFF
    assert np.array_equal(gs, counts)
    for y in range(32):
        for x in range(32):
            c = counts[y, x]
            assert np.array_equal(gc[y, x, :c], cells[y, x, :c])


def test_batched_views_equal_single_dispatch(tiny):
    m = tiny.model
    cams = scenes.sphere_cameras(5, 3.0, 7, math.radians(60), 1.0, 100.0)
    t = bv.RadFoamGpuTracer(m)
    batch = render_gpu(t, cams, 48, 40)
    for i, c in enumerate(cams):
        single = render_gpu(t, [c], 48, 40)[0]
        assert np.array_equal(bits(batch[i]), bits(single))
    om = O.OracleModel.from_scene(m)
    ref, _, _, _ = O.render_walk(om, cams[3], 48, 40, 1024, 1e-3,
                                 O.containing_cell_f64(om, cams[3].position))
    assert np.array_equal(bits(batch[3]), bits(ref))


def test_start_cell_matches_fp64_oracle(tiny):
    m = tiny.model
    t = bv.RadFoamGpuTracer(m)
    om = O.OracleModel.from_scene(m)
    rng = np.random.default_rng(11)
    qs = np.concatenate([rng.uniform(-1.5, 1.5, (48, 3)), m.points[:16, :3] + 1e-4])
    for q in qs.astype(np.float32):
        assert t.containing_point(q) == O.containing_cell_f64(om, q)


def test_powerfoam_walk_bf16_bit_exact():
    """PowerFoam walk (support-sphere clipping) with BF16 SH storage: the
    oracle gets the same BF16-rounded coefficients."""
    m = scenes.powerfoam_mixture(4096, seed=5, radius_max=0.12)
    assert m.sh_bf16 and m.radii is not None
    cams = scenes.sphere_cameras(2, 3.0, 1, math.radians(60), 1.0, 100.0)
    t = bv.RadFoamGpuTracer(m)
    gpu = render_gpu(t, cams, 64, 64)
    om = O.OracleModel.from_scene(m)
    for i, c in enumerate(cams):
        ref, _, _, _ = O.render_walk(om, c, 64, 64, 1024, 1e-3,
                                     O.containing_cell_f64(om, c.position))
        assert np.array_equal(bits(gpu[i]), bits(ref))
    assert gpu[..., 3].max() > 0.05


def test_edge_cases_tiny_images_and_max_steps(tiny):
    m = tiny.model
    t = bv.RadFoamGpuTracer(m, max_steps=3)
    cam = tiny.cameras[0]
    om = O.OracleModel.from_scene(m)
    start = O.containing_cell_f64(om, cam.position)
    for (w, h) in [(1, 1), (3, 7), (9, 5)]:
        gpu = render_gpu(t, [cam], w, h)[0]
        ref, _, _, _ = O.render_walk(om, cam, w, h, 3, 1e-3, start)
        assert np.array_equal(bits(gpu), bits(ref))
    with pytest.raises(bv.BvError):
        out = torch.empty((1, 1, 4), device="cuda")
        t.dispatch(out, cam, (0, 4))


def test_debug_cell_density_heatmap(tiny):
    t = bv.RadFoamGpuTracer(tiny.model, debug_cell_density=True)
    out = render_gpu(t, tiny.cameras, 16, 16)[0]
    assert np.all(out[..., 3] == 1.0)
    assert np.all((out[..., :3] >= 0) & (out[..., :3] <= 1))
