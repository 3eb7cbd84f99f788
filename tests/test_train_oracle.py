"""Pins the FP64 gradient oracle: analytic gradients of the training
contract (diff_render.rs:943-1923 restated with an L2 loss) against central
finite differences on the fixed recorded path, the way the reference checks
its graph (position_gradient_matches_central_finite_difference_for_fixed_path,
diff_render.rs:11961; eps 5e-3 there, tolerance abs < 5e-3 or rel < 2e-2)."""

import math

import numpy as np
import pytest

from blade_volume_b200 import scenes
from oracle import oracle as O


def small_case(seed=3, n=1024, radii=False):
    if radii:
        m = scenes.powerfoam_mixture(n, seed=seed, radius_max=0.25, bf16=False)
    else:
        m = scenes.radfoam_ball(n, seed=seed, sh_degree=2)
    cams = scenes.sphere_cameras(2, 3.0, seed, math.radians(50.0), 1.0, 100.0)
    rng = np.random.default_rng(seed)
    target = rng.random((2, 20, 20, 3)).astype(np.float32)
    return m, cams, target


def loss_at(om, cams, target, pts, sh, rad, max_dt, loss_kind, splats=False):
    r = O.forward_backward(om, cams, 20, 20, max_dt=max_dt, target=target, loss_kind=loss_kind,
                           override=(pts, sh, rad), want_grads=False, threads=4, splats=splats)
    return r["loss"]


@pytest.mark.parametrize("radii,loss_kind,max_dt,splats", [
    (False, 0, 50.0, False), (True, 0, 50.0, False), (False, 1, 50.0, False),
    (False, 0, 0.05, False),
    # PowerFoam splat semantics (record_powerfoam_splats_jacobians, trace.rs:1421)
    (True, 0, 50.0, True)])
def test_oracle_gradient_matches_central_differences(radii, loss_kind, max_dt, splats):
    m, cams, target = small_case(radii=radii)
    om = O.OracleModel.from_scene(m)
    pts = m.points.astype(np.float64)
    sh = m.sh.astype(np.float64).reshape(-1)
    rad = None if m.radii is None else m.radii.astype(np.float64)
    # FP64 parameters given explicitly: every segment length and Jacobian is
    # then derived in FP64, the same function the differences perturb
    g = O.forward_backward(om, cams, 20, 20, max_dt=max_dt, target=target, loss_kind=loss_kind,
                           override=(pts, sh, rad), threads=4, splats=splats)
    rng = np.random.default_rng(0)
    checks = []
    tables = [("density", g["d_density"]), ("sh", g["d_sh"]), ("pos", g["d_pos"].reshape(-1))]
    if rad is not None:
        tables.append(("radius", g["d_radius"]))
    for name, tab in tables:
        nz = np.flatnonzero(np.abs(tab) > 1e-3 * np.abs(tab).max())
        if loss_kind == 1 and name == "pos":
            continue  # L1's kink makes position FD noisy; density/SH are checked
        for idx in rng.choice(nz, size=min(6, len(nz)), replace=False):
            checks.append((name, int(idx), float(tab[idx])))
    assert len(checks) >= 12
    eps = 1e-7
    for name, idx, analytic in checks:
        def perturbed(delta):
            p, s, r = pts.copy(), sh.copy(), None if rad is None else rad.copy()
            if name == "density":
                p[idx, 3] += delta
            elif name == "sh":
                s[idx] += delta
            elif name == "pos":
                p[idx // 3, idx % 3] += delta
            else:
                r[idx] += delta
            return loss_at(om, cams, target, p, s, r, max_dt, loss_kind, splats)
        lp, lm = perturbed(eps), perturbed(-eps)
        fd = (lp - lm) / (2 * eps)
        scale = max(abs(fd), abs(analytic))
        roundoff = 8 * np.finfo(np.float64).eps * abs(lp) / eps  # FP64 stencil noise floor
        assert abs(fd - analytic) <= 2e-4 * scale + roundoff, (name, idx, analytic, fd)
