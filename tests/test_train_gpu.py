"""GPU training gradient (bv_forward_backward) against the FP64 oracle.

Bar (FP32 arithmetic, FP32 atomics): the forward colours bit-exact against
the oracle's FP32 restatement of the training walk; the loss within 1e-5
relative of the FP64 oracle; every gradient entry within the element-wise
bar of tests/gradcheck.py (1e-4 relative plus the entry's own FP32 error
budget); plus central finite differences of the FP64 fixed-path loss on 64
sampled parameters.
"""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests import gradcheck  # noqa: E402

pytestmark = pytest.mark.gpu

W = H = 40


def case(kind="plain", seed=3, n=4096):
    if kind == "plain":
        m = scenes.radfoam_ball(n, seed=seed, sh_degree=3)
    elif kind == "deg1":
        m = scenes.radfoam_ball(n, seed=seed, sh_degree=1)
    else:
        m = scenes.powerfoam_mixture(n, seed=seed, radius_max=0.15, bf16=(kind == "power_bf16"))
    cams = scenes.sphere_cameras(3, 3.0, seed + 1, math.radians(55.0), 1.0, 100.0)
    target = np.random.default_rng(seed).random((3, H, W, 3)).astype(np.float32)
    return m, cams, target


def run_gpu(m, cams, target, max_dt=50.0, loss=bv.LOSS_L2, weight_threshold=0.0, repeat=1,
            exit_record=None):
    t = bv.RadFoamGpuTracer(m)
    if exit_record is not None:
        t.set_exit_record(exit_record)
    grads = t.new_grads()
    tg = torch.from_numpy(target).cuda()
    rgb = torch.zeros((len(cams), H, W, 3), dtype=torch.float32, device="cuda")
    loss_out = None
    for _ in range(repeat):
        loss_out = t.forward_backward(cams, W, H, tg, grads, max_dt=max_dt, loss=loss,
                                      weight_threshold=weight_threshold, rgb_out=rgb)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy().astype(np.float64) for k, v in grads.items()}
    out["d_pos"] = out["d_pos"].reshape(-1, 3)
    out["loss"] = float(loss_out.item())
    out["rgb"] = rgb.cpu().numpy()
    t.deinit()
    return out


def assert_table(name, got, ref, tol=1e-4):
    """Table-level agreement of two device results (accumulation tests)."""
    scale = np.abs(ref).max()
    assert scale > 0, name
    err = np.abs(got - ref).max() / scale
    assert err <= tol, (name, err)


def scaled(ref, k):
    """The oracle result of k identical accumulated passes."""
    out = dict(ref)
    for key, v in ref.items():
        if (key.startswith("d_") or key.startswith("mass_") or key.startswith("count_")) \
                and v is not None:
            out[key] = k * v
    return out


@pytest.mark.parametrize("kind", ["plain", "deg1", "power", "power_bf16"])
def test_gradients_match_fp64_oracle(kind):
    m, cams, target = case(kind)
    g = run_gpu(m, cams, target)
    om = O.OracleModel.from_scene(m)
    ref = O.forward_backward(om, cams, W, H, target=target, want_mass=True)
    assert abs(g["loss"] - ref["loss"]) <= 1e-5 * ref["loss"]
    assert np.array_equal(g["rgb"].view(np.uint32), ref["rgb32"].view(np.uint32))
    tables = gradcheck.check_all(g, ref, where=kind)
    assert len(tables) == (4 if m.radii is not None else 3)


# The replay reads the forward's recorded exit faces for the first `rec`
# steps of each ray and searches the rest: no record, a record that ends a few
# steps into every ray, and the default all give the oracle's results.
@pytest.mark.parametrize("kind,rec", [("plain", 0), ("plain", 3), ("power", 0), ("power", 5)])
def test_exit_record_lengths_match_oracle(kind, rec):
    m, cams, target = case(kind, seed=7, n=3000)
    g = run_gpu(m, cams, target, exit_record=rec, repeat=2)
    om = O.OracleModel.from_scene(m)
    ref = O.forward_backward(om, cams, W, H, target=target, want_mass=True)
    assert np.array_equal(g["rgb"].view(np.uint32), ref["rgb32"].view(np.uint32))
    # repeat=2 accumulates two identical passes
    gradcheck.check_all(g, scaled(ref, 2), where=f"{kind} record {rec}")


def test_l1_loss_clamped_dt_and_threshold():
    m, cams, target = case("plain", seed=5, n=2048)
    om = O.OracleModel.from_scene(m)
    for loss, max_dt, thr in [(bv.LOSS_L1, 50.0, 0.0), (bv.LOSS_L2, 0.04, 0.0),
                              (bv.LOSS_L2, 50.0, 1e-3)]:
        g = run_gpu(m, cams, target, max_dt=max_dt, loss=loss, weight_threshold=thr)
        ref = O.forward_backward(om, cams, W, H, target=target, loss_kind=loss, max_dt=max_dt,
                                 weight_threshold=thr, want_mass=True)
        assert abs(g["loss"] - ref["loss"]) <= 1e-5 * ref["loss"]
        gradcheck.check_all(g, ref, where=f"loss {loss} max_dt {max_dt} thr {thr}")


def test_gradients_accumulate_like_scatter_add():
    m, cams, target = case("plain", seed=7, n=2048)
    once = run_gpu(m, cams, target)
    twice = run_gpu(m, cams, target, repeat=2)
    for k in ("d_density", "d_sh", "d_pos"):
        assert_table(k, twice[k], 2.0 * once[k], tol=1e-5)


def test_gradients_match_central_finite_differences():
    """64 sampled parameters (density, SH, site positions), FP64 central
    differences of the fixed-path loss; the reference's FD check holds the
    recorded cell sequence fixed the same way (diff_render.rs:19-23)."""
    m, cams, target = case("plain", seed=9, n=2048)
    g = run_gpu(m, cams, target)
    om = O.OracleModel.from_scene(m)
    pts = m.points.astype(np.float64)
    sh = m.sh.astype(np.float64).reshape(-1)
    rng = np.random.default_rng(1)
    tables = [("density", g["d_density"]), ("pos", g["d_pos"].reshape(-1)), ("sh", g["d_sh"])]
    picks = []
    want = {"density": 22, "pos": 20, "sh": 64}
    for name, tab in tables:
        nz = np.flatnonzero(np.abs(tab) > 1e-2 * np.abs(tab).max())
        k = min(want[name], len(nz), 64 - len(picks))
        picks += [(name, int(i), tab[i]) for i in rng.choice(nz, size=k, replace=False)]
    assert len(picks) == 64
    # FP64 stencil well inside the shortest segments of the path (sub-1e-5
    # segments exist, and a step that flips one's sign leaves the fixed path)
    eps = 1e-7
    for name, idx, gpu_val in picks:
        def loss(delta):
            p, s = pts.copy(), sh.copy()
            if name == "density":
                p[idx, 3] += delta
            elif name == "sh":
                s[idx] += delta
            else:
                p[idx // 3, idx % 3] += delta
            return O.forward_backward(om, cams, W, H, target=target, override=(p, s, None),
                                      want_grads=False)["loss"]
        lp, lm = loss(eps), loss(-eps)
        fd = (lp - lm) / (2 * eps)
        roundoff = 8 * np.finfo(np.float64).eps * abs(lp) / eps  # FP64 stencil noise floor
        assert abs(gpu_val - fd) <= 2e-3 * max(abs(fd), abs(gpu_val)) + roundoff, (
            name, idx, gpu_val, fd)


def slab_scene(n=160000, seed=3):
    """Sites uniform in a 0.8 x 0.8 x 8 slab, viewed end-on: every ray of a
    narrow camera on the long axis walks 348-400 cells, beyond the 256 steps
    the training forward records per ray, so the replay reads the record for
    the first 256 steps and searches the rest."""
    rng = np.random.default_rng(seed)
    xyz = np.stack([rng.uniform(-0.4, 0.4, n), rng.uniform(-0.4, 0.4, n),
                    rng.uniform(-4.0, 4.0, n)], 1).astype(np.float32)
    off, nb = scenes.delaunay_csr(xyz)
    dens = rng.lognormal(-1.0, 1.0, n).astype(np.float32)
    sh = np.zeros((n, 48), np.float32)
    sh[:, 0:3] = scenes._dc_from_color(rng.random((n, 3)))
    sh[:, 3:] = rng.normal(0.0, 0.2, (n, 45))
    m = scenes.PointCloudModel(np.concatenate([xyz, dens[:, None]], 1).astype(np.float32), sh,
                               3, off, nb, None, False)
    cams = [scenes.looking_at((0.0, 0.0, -6.0), (0.0, 0.0, 0.0), math.radians(4.0), 1.0, 100.0),
            scenes.looking_at((0.05, -0.05, 6.0), (0.0, 0.0, 0.0), math.radians(4.0), 1.0,
                              100.0)]
    return m, cams


def test_rays_longer_than_the_step_record():
    m, cams = slab_scene()
    side = 32
    om = O.OracleModel.from_scene(m)
    _, steps, _, _ = O.render_walk(om, cams[0], side, side, 1024, 0.0)
    assert steps.min() > 256
    target = np.random.default_rng(4).random((2, side, side, 3)).astype(np.float32)
    t = bv.RadFoamGpuTracer(m)
    grads = t.new_grads()
    rgb = torch.zeros((2, side, side, 3), dtype=torch.float32, device="cuda")
    loss = t.forward_backward(cams, side, side, torch.from_numpy(target).cuda(), grads,
                              rgb_out=rgb)
    torch.cuda.synchronize()
    g = {k: v.cpu().numpy().astype(np.float64) for k, v in grads.items()}
    g["d_pos"] = g["d_pos"].reshape(-1, 3)
    got_loss, got_rgb = float(loss.item()), rgb.cpu().numpy()
    t.deinit()
    ref = O.forward_backward(om, cams, side, side, target=target, want_mass=True)
    assert abs(got_loss - ref["loss"]) <= 1e-5 * ref["loss"]
    assert np.array_equal(got_rgb.view(np.uint32), ref["rgb32"].view(np.uint32))
    gradcheck.check_all(g, ref, where="slab, rays of 348-400 steps")


def test_repeated_calls_take_tiles_heaviest_first_with_the_same_results():
    """A call of the same shape as the one before takes its tiles in the
    order of the previous forward's tile times, in its replay (two more launches per call
    build the order), for the same cameras or others; each call's colours
    are the oracle's bit for bit and its gradients within the element-wise
    bar."""
    m, cams, target = case("plain", seed=9, n=3000)
    other = scenes.sphere_cameras(3, 3.0, 21, math.radians(55.0), 1.0, 100.0)
    om = O.OracleModel.from_scene(m)
    refs = {}
    t = bv.RadFoamGpuTracer(m)
    try:
        tg = torch.from_numpy(target).cuda()
        for i, views in enumerate([cams, cams, other, cams]):
            if id(views) not in refs:
                refs[id(views)] = O.forward_backward(om, views, W, H, target=target,
                                                     want_mass=True)
            ref = refs[id(views)]
            grads = t.new_grads()
            rgb = torch.zeros((len(views), H, W, 3), dtype=torch.float32, device="cuda")
            loss = t.forward_backward(views, W, H, tg, grads, max_dt=50.0, weight_threshold=0.0,
                                      rgb_out=rgb)
            torch.cuda.synchronize()
            g = {k: v.cpu().numpy().astype(np.float64) for k, v in grads.items()}
            g["d_pos"] = g["d_pos"].reshape(-1, 3)
            assert np.array_equal(rgb.cpu().numpy().view(np.uint32), ref["rgb32"].view(np.uint32)), i
            assert abs(float(loss.item()) - ref["loss"]) <= 1e-5 * ref["loss"], i
            gradcheck.check_all(g, ref, where=f"walk tile order call {i}")
    finally:
        t.deinit()
