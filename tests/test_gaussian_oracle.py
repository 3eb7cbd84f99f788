"""Pins the Gaussian trace oracle (trace_gaussians, trace.rs:695-773) against
the reference's own tests, and checks the C ABI's validation of Gaussian
models (no GPU needed: validation runs before any device call)."""

import numpy as np
import pytest

import blade_volume_b200 as bv
from blade_volume_b200 import scenes
from oracle import oracle as O


def dc(color):
    """trace.rs:779-782."""
    return ((np.asarray(color, np.float32) - 0.5) / np.float32(0.2820948)).astype(np.float32)


def model(points, scales, colors, rotations=None):
    n = len(points)
    rot = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1)) if rotations is None else rotations
    return scenes.GaussianShModel(np.asarray(points, np.float32), np.asarray(rot, np.float32),
                                  np.asarray(scales, np.float32),
                                  np.stack([dc(c) for c in colors]), 0)


def two_gaussians():
    """trace.rs:872-904: index order far (blue), near (red); the far one is
    broad enough that its support begins before the near one's."""
    return model([[0, 0, 4, 0.5], [0, 0, 2, 0.5]], [[1, 1, 1], [1, 1, 0.1]],
                 [[0, 0, 1], [1, 0, 0]])


def test_orders_maximum_response_not_proxy_entry():
    """trace.rs:906-933: red at t=2, then blue at t=4: (0.5, 0, 0.25, 0.75)."""
    s = O.GaussianOracleScene.from_scene(two_gaussians(), min_opacity=0.01)
    support = np.sqrt(2.0 * np.log(0.5 / 0.01))
    assert 4.0 - support < 2.0 - 0.1 * support
    rgba, hits = O.trace_gaussians(s, [0, 0, 0], [0, 0, 1], min_transmittance=0.0,
                                   t_start=0.0, t_end=10.0)
    assert np.abs(rgba - [0.5, 0.0, 0.25, 0.75]).max() < 1e-6
    assert hits == 2


def test_equal_depth_hits_composite_in_index_order():
    """trace.rs:965-998 (batch cursor): 13 hits at t = 1 + index // 3 come
    out in (t, index) order.  Listed in reverse so that model order and
    depth order disagree; distinct colours make the order visible."""
    idx = np.arange(13)[::-1]
    pts = [[0, 0, 1.0 + i // 3, 0.1 + 0.05 * (i % 4)] for i in idx]
    cols = [[(i % 3) / 2.0, (i % 5) / 4.0, (i % 7) / 6.0] for i in idx]
    g = model(pts, [[1, 1, 1]] * 13, cols)
    s = O.GaussianOracleScene.from_scene(g, 0.01)
    rgba, hits = O.trace_gaussians(s, [0, 0, 0], [0, 0, 1], 0.0, 0.0, 100.0)
    assert hits == 13
    # float64 restatement over the expected (t, model index) order
    order = sorted(range(13), key=lambda k: (g.points[k, 2], k))
    T, rad = 1.0, np.zeros(3)
    for k in order:
        a = float(g.points[k, 3])  # the ray passes through the mean: alpha = opacity
        rad += a * T * np.clip(np.array(cols[k]), 0, None)
        T *= 1.0 - a
    assert np.abs(rgba[:3] - rad).max() < 1e-5 and abs(rgba[3] - (1 - T)) < 1e-6


def test_hit_rule_opacity_filter_depth_range_and_cutoff():
    g = model([[0, 0, 2, 0.5], [0, 0, -2, 0.9], [0, 0, 3, 0.005], [0.3, 0, 5, 0.5],
               [0, 0, 7, 0.4]], [[1, 1, 1], [1, 1, 1], [1, 1, 1], [0.1, 0.1, 0.1], [1, 1, 1]],
              [[1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1], [0, 0, 1]])
    s = O.GaussianOracleScene.from_scene(g, 0.01)
    assert s.n == 4  # opacity 0.005 <= min_opacity is not loaded (gpu/gaussian.rs:19-27)
    # behind the origin (t <= t_start) and response exp(-4.5) * 0.5 < 0.01 both miss
    rgba, hits = O.trace_gaussians(s, [0, 0, 0], [0, 0, 1], 0.0, 0.0, 6.0)
    assert hits == 1 and np.allclose(rgba, [0.5, 0, 0, 0.5], atol=1e-6)
    rgba, hits = O.trace_gaussians(s, [0, 0, 0], [0, 0, 1], 0.0, 0.0, 10.0)
    assert hits == 2
    # transmittance cutoff: stop once T <= min_transmittance (checked before a hit)
    rgba, hits = O.trace_gaussians(s, [0, 0, 0], [0, 0, 1], 0.5, 0.0, 10.0)
    assert hits == 1


def sh_model(n=4, **kw):
    g = scenes.gaussian_sh(n, seed=1, sh_degree=1)
    for k, v in kw.items():
        setattr(g, k, v)
    return g


@pytest.mark.parametrize("mutate,needle", [
    (lambda g: g.rotations.__setitem__((0, 3), 2.0), "unit length"),
    (lambda g: g.scales.__setitem__((1, 0), 0.0), "positive"),
    (lambda g: g.points.__setitem__((2, 3), -0.5), "non-negative"),
    (lambda g: g.sh.__setitem__((3, 4), np.nan), "finite"),
])
def test_abi_rejects_invalid_gaussian_models(mutate, needle):
    g = sh_model()
    mutate(g)
    with pytest.raises(bv.BvError) as e:
        bv.GaussianTracer(g)
    assert e.value.status == 2 and needle in str(e.value)


def test_abi_rejects_bad_settings_and_empty_models():
    with pytest.raises(bv.BvError) as e:
        bv.GaussianTracer(sh_model(), min_opacity=0.0)
    assert e.value.status == 1
    with pytest.raises(bv.BvError) as e:
        bv.GaussianTracer(sh_model(), min_transmittance=1.5)
    assert e.value.status == 1
    g = sh_model()
    g.points[:, 3] = 0.001
    with pytest.raises(bv.BvError) as e:
        bv.GaussianTracer(g)
    assert "above min_opacity" in str(e.value)
