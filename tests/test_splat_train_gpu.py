"""PowerFoam training with splat semantics
(bv_powerfoam_splat_tracer_forward_backward) against the FP64 oracle.

The oracle records each ray's sorted support intervals as
record_powerfoam_splats_jacobians does (trace.rs:1421-1452) and evaluates the
training contract on them in FP64 (its gradients are pinned by central
differences in tests/test_train_oracle.py).  Bar, as for the walk: forward
colours bit-exact against the oracle's FP32 restatement, the loss within
1e-5 relative, every gradient entry within the element-wise bar of
tests/gradcheck.py.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import gradcheck  # noqa: E402
from tests.test_train_gpu import assert_table  # noqa: E402

pytestmark = pytest.mark.gpu

W = H = 40


def case(seed=3, n=4096, bf16=False, radius_max=0.1):
    m = scenes.powerfoam_mixture(n, seed=seed, radius_max=radius_max, bf16=bf16)
    cams = scenes.sphere_cameras(3, 3.0, seed + 1, math.radians(55.0), 1.0, 100.0)
    target = np.random.default_rng(seed).random((3, H, W, 3)).astype(np.float32)
    return m, cams, target


def run_gpu(m, cams, target, repeat=1, interval_record=None, **kw):
    t = bv.PowerFoamSplatTracer(m)
    if interval_record is not None:
        t.set_interval_record(interval_record)
    grads = t.new_grads()
    tg = torch.from_numpy(target).cuda()
    rgb = torch.zeros((len(cams), H, W, 3), dtype=torch.float32, device="cuda")
    loss_out = None
    for _ in range(repeat):
        loss_out = t.forward_backward(cams, W, H, tg, grads, rgb_out=rgb, **kw)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy().astype(np.float64) for k, v in grads.items()}
    out["d_pos"] = out["d_pos"].reshape(-1, 3)
    out["loss"] = float(loss_out.item())
    out["rgb"] = rgb.cpu().numpy()
    t.deinit()
    return out


@pytest.mark.parametrize("bf16,radius_max", [(False, 0.1), (True, 0.1), (False, 0.03)])
def test_splat_gradients_match_fp64_oracle(bf16, radius_max):
    m, cams, target = case(bf16=bf16, radius_max=radius_max)
    g = run_gpu(m, cams, target)
    om = O.OracleModel.from_scene(m)
    ref = O.forward_backward(om, cams, W, H, target=target, splats=True, want_mass=True)
    assert abs(g["loss"] - ref["loss"]) <= 1e-5 * ref["loss"]
    assert np.array_equal(g["rgb"].view(np.uint32), ref["rgb32"].view(np.uint32))
    assert len(gradcheck.check_all(g, ref, where=f"splat bf16={bf16} r={radius_max}")) == 4


# The replay walks the forward's recorded intervals of a ray when they all
# fit and traverses the BVH again otherwise: no record, a record of two
# intervals (rays split between both paths within a warp), one of twenty
# (records spanning two 16-interval chunks) and the default all give the
# oracle's results.
@pytest.mark.parametrize("entries", [0, 2, 20])
def test_interval_record_lengths_match_oracle(entries):
    m, cams, target = case(seed=8, n=3000)
    g = run_gpu(m, cams, target, interval_record=entries)
    om = O.OracleModel.from_scene(m)
    ref = O.forward_backward(om, cams, W, H, target=target, splats=True, want_mass=True)
    assert abs(g["loss"] - ref["loss"]) <= 1e-5 * ref["loss"]
    assert np.array_equal(g["rgb"].view(np.uint32), ref["rgb32"].view(np.uint32))
    assert len(gradcheck.check_all(g, ref, where=f"splat record {entries}")) == 4


def test_splat_training_settings_and_accumulation():
    m, cams, target = case(seed=6, n=2048)
    om = O.OracleModel.from_scene(m)
    for loss, max_dt, thr, steps in [(bv.LOSS_L1, 50.0, 0.0, 1024), (bv.LOSS_L2, 0.01, 0.0, 1024),
                                     (bv.LOSS_L2, 50.0, 1e-2, 1024), (bv.LOSS_L2, 50.0, 0.0, 3)]:
        g = run_gpu(m, cams, target, loss=loss, max_dt=max_dt, weight_threshold=thr,
                    max_steps=steps)
        ref = O.forward_backward(om, cams, W, H, target=target, loss_kind=loss, max_dt=max_dt,
                                 weight_threshold=thr, max_steps=steps, splats=True,
                                 want_mass=True)
        assert abs(g["loss"] - ref["loss"]) <= 1e-5 * ref["loss"], (loss, max_dt, thr, steps)
        gradcheck.check_all(g, ref, where=f"splat loss {loss} max_dt {max_dt} thr {thr}")
    once = run_gpu(m, cams, target)
    twice = run_gpu(m, cams, target, repeat=2)
    for k in ("d_density", "d_sh", "d_pos", "d_radius"):
        assert_table(k, twice[k], 2.0 * once[k], tol=1e-5)


def test_repeated_calls_take_tiles_heaviest_first_with_the_same_results():
    """A call of the same shape (views, width, height) as the one before
    takes its tiles in the order of the previous forward's tile durations
    (three more launches per call build that order), whether its cameras are
    the same or not.  Every call is held to the oracle."""
    m, cams, target = case(seed=5, n=3000)
    other = scenes.sphere_cameras(3, 3.0, 11, math.radians(55.0), 1.0, 100.0)
    om = O.OracleModel.from_scene(m)
    refs = {}
    t = bv.PowerFoamSplatTracer(m)
    try:
        tg = torch.from_numpy(target).cuda()
        for i, views in enumerate([cams, cams, cams, other, cams]):
            key = id(views)
            if key not in refs:
                refs[key] = O.forward_backward(om, views, W, H, target=target, splats=True,
                                               want_mass=True)
            ref = refs[key]
            grads = t.new_grads()
            rgb = torch.zeros((len(views), H, W, 3), dtype=torch.float32, device="cuda")
            loss = t.forward_backward(views, W, H, tg, grads, rgb_out=rgb)
            torch.cuda.synchronize()
            assert t.last_stats().launches == 6  # forward, backward, tile order x 3, site fold
            g = {k: v.cpu().numpy().astype(np.float64) for k, v in grads.items()}
            g["d_pos"] = g["d_pos"].reshape(-1, 3)
            assert abs(float(loss.item()) - ref["loss"]) <= 1e-5 * ref["loss"], i
            assert np.array_equal(rgb.cpu().numpy().view(np.uint32), ref["rgb32"].view(np.uint32)), i
            gradcheck.check_all(g, ref, where=f"tile order call {i}")
    finally:
        t.deinit()


def test_planes_at_the_same_depth_bound_the_interval_in_csr_order():
    """Site 0's Cech row holds site 1 (offset 0) and site 2 (offset 1).  Both
    planes cross the ray z = -10 + t along the axis at t = 11 exactly (num /
    den = 22 / 2 and 11 / 1 in FP32), so the exit plane of site 0's interval
    is a tie, which the reference's scan in CSR order gives to site 1.  The
    device stores the row nearest plane first (site 2's plane, 0.71 from the
    site, before site 1's, at 1.0) and must still pick site 1: the gradient of
    the exit plane's Jacobian lands on site 1's position."""
    pts = np.array([[0, 0, 0, 2.0], [0, 0, 2, 1.5], [1, 0, 1, 1.0]], np.float32)
    offsets = np.array([0, 2, 4, 6], np.uint32)
    neighbors = np.array([1, 2, 0, 2, 0, 1], np.uint32)
    sh = np.zeros((3, 3), np.float32)
    sh[:, 0] = [1.0, 0.2, 0.6]
    sh[:, 1] = [0.3, 1.0, 0.4]
    sh[:, 2] = [0.5, 0.7, 1.0]
    m = scenes.PointCloudModel(pts, sh, 0, offsets, neighbors, np.full(3, 1.2, np.float32))
    # the tie, in the clip's own FP32 operations
    o = np.float32(-10.0)
    t1 = np.float32(np.float32(2.0) * (np.float32(1.0) - o)) / np.float32(2.0)
    f2 = (np.float32(0.5), np.float32(0.5))
    t2 = np.float32(f2[0] * np.float32(1.0) + (f2[1] - o) * np.float32(1.0)) / np.float32(1.0)
    assert t1 == t2 == np.float32(11.0)
    cam = scenes.looking_at((0.0, 0.0, -10.0), (0.0, 0.0, 1.0), math.radians(10.0), 1.0, 100.0)
    target = np.zeros((1, 1, 1, 3), np.float32)
    om = O.OracleModel.from_scene(m)
    ref = O.forward_backward(om, [cam], 1, 1, target=target, splats=True, want_mass=True)
    t = bv.PowerFoamSplatTracer(m)
    try:
        grads = t.new_grads()
        rgb = torch.zeros((1, 1, 1, 3), dtype=torch.float32, device="cuda")
        loss = t.forward_backward([cam], 1, 1, torch.from_numpy(target).cuda(), grads, rgb_out=rgb)
        torch.cuda.synchronize()
        g = {k: v.cpu().numpy().astype(np.float64) for k, v in grads.items()}
    finally:
        t.deinit()
    g["d_pos"] = g["d_pos"].reshape(-1, 3)
    assert np.array_equal(rgb.cpu().numpy().view(np.uint32), ref["rgb32"].view(np.uint32))
    assert abs(float(loss.item()) - ref["loss"]) <= 1e-5 * ref["loss"]
    # the exit plane is site 1's: site 2, across the tied plane, gets nothing
    # (with site 2 first in the CSR row it would take the Jacobian instead)
    ref_pos = ref["d_pos"].reshape(-1, 3)
    assert ref_pos[1, 2] != 0 and not ref_pos[2].any()
    gradcheck.check_all(g, ref, where="tied exit planes")
