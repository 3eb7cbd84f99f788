"""Precision of the FP32 walk against the FP64 accuracy oracle, and the FP64
exit-face tie-break.

The FP64 oracle evaluates the reference's walk (trace.rs:1680-1820) with
every quantity in double; the FP32 path (device = FP32 oracle, bit for bit)
is compared with it per configuration in PSNR over RGB.  The tie-break
re-evaluates near-tied exit faces in FP64, so its cell sequences follow the
FP64 walk at those ties and its images move towards the FP64 image.
"""

import math

import numpy as np
import pytest

from blade_volume_b200 import scenes
from oracle import oracle as O

CAP = 512


def same_sequences(c1, n1, c2, n2):
    live = np.arange(c1.shape[-1])[None, None, :] < n1[..., None]
    return (n1 == n2) & np.all((c1 == c2) | ~live, axis=-1)


@pytest.fixture(scope="module")
def tiny():
    return scenes.radfoam_tiny()


def test_fp32_walk_against_fp64_oracle_and_tie_break(tiny):
    """16,384-site ball, 128^2: the FP32 walk is within 60 dB of the FP64
    walk; the tie-break brings the image closer and changes only rays whose
    sequences differed from the FP64 walk."""
    om = O.OracleModel.from_scene(tiny.model)
    cam = tiny.cameras[0]
    ref, _, c32, n32 = O.render_walk(om, cam, 128, 128, 1024, 1e-3, cell_capacity=CAP)
    tb, _, ct, nt = O.render_walk(om, cam, 128, 128, 1024, 1e-3, cell_capacity=CAP,
                                  tie_break=True)
    f64, c64, n64 = O.render_walk_f64(om, cam, 128, 128, 1024, 1e-3, cell_capacity=CAP)
    p_ref = O.psnr(ref[..., :3], f64[..., :3])
    p_tb = O.psnr(tb[..., :3], f64[..., :3])
    assert p_ref > 60.0 and p_tb >= p_ref
    ref_ok = same_sequences(c32, n32, c64, n64)
    tb_ok = same_sequences(ct, nt, c64, n64)
    assert tb_ok.sum() >= ref_ok.sum() and ref_ok.mean() > 0.999
    # the tie-break changes some rays, and only rays where the reference rule
    # left the FP64 walk
    changed = ~same_sequences(c32, n32, ct, nt)
    assert changed.any() and not np.any(changed & ref_ok)


# ---------------------------------------------------------------------------
# device (GPU) side
# ---------------------------------------------------------------------------
torch = pytest.importorskip("torch")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def gpu_render(model, cams, w, h, tie_break=False):
    import blade_volume_b200 as bv

    t = bv.RadFoamGpuTracer(model, max_steps=1024, weight_threshold=1e-3)
    t.set_tie_break(tie_break)
    img = t.render(cams, w, h).cpu().numpy()
    t.deinit()
    return img


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["ball", "powerfoam"])
def test_gpu_tie_break_bit_exact(kind, tiny):
    if kind == "ball":
        model, cam, w, h = tiny.model, tiny.cameras[0], 128, 128
    else:
        model = scenes.powerfoam_mixture(20000, seed=5, radius_max=0.08)
        cam = scenes.sphere_cameras(1, 3.0, 5, math.radians(60.0), 1.0, 100.0)[0]
        w = h = 96
    om = O.OracleModel.from_scene(model)
    for tb in (False, True):
        got = gpu_render(model, [cam], w, h, tie_break=tb)[0]
        want, _, _, _ = O.render_walk(om, cam, w, h, 1024, 1e-3, tie_break=tb)
        assert np.array_equal(bits(got), bits(want)), tb


PRECISION_CASES = {
    # configuration: (scene builder, cameras, side); sizes reduced from the
    # benchmark configurations so that the FP64 oracle finishes in seconds
    "radfoam 16,384 sites, SH0, 128^2": (lambda: scenes.radfoam_tiny().model, 1, 128, 60.0),
    "radfoam 262,144 sites, SH3, 1 x 256^2": (
        lambda: scenes.radfoam_ball(262144, seed=0, sh_degree=3), 1, 256, 60.0),
    # radii U[0, 0.05]: the 1M-site configuration's overlap density at 65,536 sites
    "powerfoam mixture 65,536 sites, SH3 BF16, 1 x 256^2": (
        lambda: scenes.powerfoam_mixture(65536, seed=0, radius_max=0.05, bf16=False), 1, 256,
        40.0),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(PRECISION_CASES))
def test_gpu_image_error_against_fp64_oracle(name):
    """Stated per configuration: PSNR of the device image against the FP64
    walk; the PowerFoam case stores SH in BF16 on the device while the FP64
    oracle reads the unrounded FP32 coefficients."""
    build, views, side, floor = PRECISION_CASES[name]
    model = build()
    cams = scenes.sphere_cameras(views, 3.0, 1, math.radians(60.0), 1.0, 100.0)
    device_model = model
    if "BF16" in name:
        device_model = model.copy()
        device_model.sh_bf16 = True
    om = O.OracleModel.from_scene(model)
    for tb in (False, True):
        got = gpu_render(device_model, cams, side, side, tie_break=tb)
        for v, cam in enumerate(cams):
            f64, _, _ = O.render_walk_f64(om, cam, side, side, 1024, 1e-3)
            p = O.psnr(got[v][..., :3], f64[..., :3])
            print(f"{name} tie_break={tb}: PSNR {p:.2f} dB vs FP64")
            assert p > floor
