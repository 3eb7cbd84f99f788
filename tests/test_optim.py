"""Optimizer step (bv_radfoam_tracer_adam_step) against the FP32 Adam oracle.

The device applies Adam to the tracer's own tables from the gradient tables
of bv_forward_backward; the oracle (bvo_adam_step) applies the same update
to host copies fed with the device's gradient tables, so the parameters
after every step must agree bit for bit.  After an update the walk must
render the updated model exactly as the oracle renders it (the face table
refresh), and a few steps must lower the loss.
"""

import math

import numpy as np
import pytest

from blade_volume_b200 import scenes
from oracle import oracle as O

SETTINGS = dict(lr_density=0.1, lr_sh_dc=5e-3, lr_sh_rest=5e-4, lr_position=2e-4,
                beta1=0.9, beta2=0.999, eps=1e-15)


def test_oracle_activation_round_trip_and_descent():
    for kind, beta in ((0, 0.0), (1, 0.0), (2, 10.0)):
        for y in (0.05, 0.7, 3.0, 25.0):
            x = O.lib().bvo_density_activation_inverse(y, kind, beta)
            back = O.lib().bvo_density_activation(x, kind, beta)
            assert abs(back - y) <= 2e-6 * max(1.0, y), (kind, y, back)
    pts = np.array([[0, 0, 0, 1.0], [1, 0, 0, 2.0]], np.float32)
    sh = np.zeros((2, 3), np.float32)
    opt = O.AdamOracle(pts, sh, None, activation=2, softplus_beta=10.0)
    before = opt.points().copy()
    g = np.array([1.0, -1.0], np.float32)
    opt.step(dict(SETTINGS, lr_position=0.0), g_density=g, g_sh=np.ones((2, 3), np.float32))
    after = opt.points()
    # the first Adam step moves each parameter by lr against its gradient's sign
    assert after[0, 3] < before[0, 3] and after[1, 3] > before[1, 3]
    assert np.allclose(opt.sh, -SETTINGS["lr_sh_dc"], atol=1e-7)
    assert np.array_equal(after[:, :3], before[:, :3])  # frozen positions


torch = pytest.importorskip("torch")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def host(t):
    return None if t is None else t.detach().cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["plain_softplus", "power_bf16_relu"])
def test_adam_steps_bit_exact_and_render_follows(kind):
    import blade_volume_b200 as bv

    if kind == "plain_softplus":
        model = scenes.radfoam_ball(3000, seed=4, sh_degree=2)
        act, extra = bv.DENSITY_SOFTPLUS, {}
    else:
        model = scenes.powerfoam_mixture(6000, seed=4, sh_degree=1, radius_max=0.1)
        act, extra = bv.DENSITY_RELU, dict(lr_radius=1e-4)
    settings = dict(SETTINGS, **extra)
    cams = scenes.sphere_cameras(2, 3.0, 4, math.radians(60.0), 1.0, 100.0)
    target = scenes.perturbed(model, seed=9)
    tt = bv.RadFoamGpuTracer(target)
    tgt = tt.render(cams, 40, 40)[..., :3].contiguous()
    tt.deinit()
    tracer = bv.RadFoamGpuTracer(model)
    start_pts, start_sh, start_rad = tracer.read_model()
    opt = O.AdamOracle(start_pts, start_sh, start_rad, activation=act, softplus_beta=10.0)
    losses = []
    for step in range(4):
        grads = tracer.new_grads()
        loss = tracer.forward_backward(cams, 40, 40, tgt, grads)
        losses.append(float(loss.item()))
        tracer.adam_step(grads, density_activation=act, softplus_beta=10.0, **settings)
        opt.step(settings, host(grads["d_density"]), host(grads["d_sh"]), host(grads["d_pos"]),
                 host(grads.get("d_radius")))
        pts, sh, rad = tracer.read_model()
        want_sh = opt.sh if not model.sh_bf16 else scenes.round_to_bf16(opt.sh)
        assert np.array_equal(bits(pts), bits(opt.points())), step
        assert np.array_equal(bits(sh), bits(want_sh.reshape(sh.shape))), step
        if rad is not None:
            assert np.array_equal(bits(rad), bits(opt.radii)), step
    assert tracer.adam_steps == 4
    if kind == "plain_softplus":
        # the reference's starting rates descend on the dense ball; the sparse
        # PowerFoam case (loss ~1e-5) is there for the bit-exact update only
        assert losses[-1] < losses[0]
    # the walk renders the updated model (face table refreshed)
    updated = model.copy()
    updated.points = pts
    updated.sh = sh
    if rad is not None:
        updated.radii = rad
    om = O.OracleModel.from_scene(updated)
    got = tracer.render(cams[:1], 40, 40)[0].cpu().numpy()
    want, _, _, _ = O.render_walk(om, cams[0], 40, 40, 1024, 1e-3)
    assert np.array_equal(bits(got), bits(want))
    with pytest.raises(bv.BvError):  # the activation is fixed by the first step
        tracer.adam_step(grads, density_activation=bv.DENSITY_IDENTITY, **settings)
    tracer.deinit()
