"""bv_containing_points_noalloc: the start-cell search for callers that
cannot call cudaMalloc (hosts whose device memory belongs to their own pool
allocator or budget).  Its scratch is a fixed device array inside the
library; this checks, through the C ABI, that two calls in a row return the
same site indices as the tracer's bv_containing_point (integer indices:
exact), and that oversized requests are refused.  Collected last, and
independent of the other test files' state."""

import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import blade_volume_b200 as bv  # noqa: E402
from blade_volume_b200 import scenes  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("powerfoam", [False, True])
def test_noalloc_matches_tracer_start_cells_two_calls(powerfoam):
    if powerfoam:
        m = scenes.powerfoam_mixture(6000, seed=4, radius_max=0.1, bf16=False)
    else:
        m = scenes.radfoam_ball(6000, seed=4, sh_degree=0)
    tracer = bv.RadFoamGpuTracer(m)
    radii = m.radii if m.radii is not None else np.zeros(m.n, np.float32)
    sites = torch.from_numpy(np.concatenate([m.points[:, :3], radii[:, None]], axis=1)
                             .astype(np.float32)).cuda()
    rng = np.random.default_rng(21)
    out = torch.full((32,), -1, dtype=torch.int32, device="cuda")
    for call in range(2):
        q = rng.uniform(-1.2, 1.2, (32 if call == 0 else 17, 3)).astype(np.float32)
        if call == 1:
            q[:5] = m.points[:5, :3]
        bv.containing_points_noalloc(sites, q, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()[: len(q)]
        want = np.array([tracer.containing_point(p) for p in q], dtype=np.int32)
        assert np.array_equal(got, want), (call, got, want)
    tracer.deinit()


def test_noalloc_rejects_more_than_32_queries():
    sites = torch.zeros((8, 4), dtype=torch.float32, device="cuda")
    out = torch.zeros(64, dtype=torch.int32, device="cuda")
    with pytest.raises(bv.BvError) as e:
        bv.containing_points_noalloc(sites, np.zeros((33, 3), np.float32), out)
    assert e.value.status == 1 and "32" in str(e.value)


def test_noalloc_full_scratch_capacity_and_cross_block_ties():
    """700,000 sites: the search runs its full 296 blocks, so the per-block
    partials fill the whole fixed array.  Duplicated sites far apart in
    index (so in different blocks) tie exactly; the lowest index must win.
    Checked against the FP64 oracle's exhaustive search."""
    from oracle import oracle as O

    n = 700_000
    rng = np.random.default_rng(5)
    xyz = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    radii = rng.uniform(0.0, 0.01, n).astype(np.float32)
    for lo, hi in [(5, 650_001), (1_000, 420_000), (123_456, 699_999)]:
        xyz[hi] = xyz[lo]
        radii[hi] = radii[lo]
    sites = torch.from_numpy(np.concatenate([xyz, radii[:, None]], axis=1)).cuda()
    pts = np.concatenate([xyz, np.ones((n, 1), np.float32)], axis=1)
    om = O.OracleModel(pts, np.zeros((n, 3), np.float32), 0, np.zeros(n + 1, np.uint32),
                       np.zeros(0, np.uint32), radii)
    out = torch.full((32,), -1, dtype=torch.int32, device="cuda")
    for call in range(2):
        q = rng.uniform(-1.1, 1.1, (32, 3)).astype(np.float32)
        q[:3] = xyz[[5, 1_000, 123_456]]
        bv.containing_points_noalloc(sites, q, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = np.array([O.containing_cell_f64(om, p) for p in q], dtype=np.int32)
        assert np.array_equal(got, want), (call, got, want)
        assert list(got[:3]) == [5, 1_000, 123_456]
