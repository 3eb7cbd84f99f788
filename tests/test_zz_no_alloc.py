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
