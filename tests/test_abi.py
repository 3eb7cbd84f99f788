"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and validates models the way PointCloudModel::validate
(blade-volume/src/lib.rs:246-483, adjacency.rs:717-790) does."""

import os
import re

import numpy as np
import pytest

import blade_volume_b200 as bv
from blade_volume_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    with open(os.path.join(ROOT, "include", "blade_volume_b200.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(bv_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = bv.load_library()
    declared = header_symbols()
    assert declared, "no declarations parsed"
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert sorted(bv.EXPORTED_SYMBOLS) == declared
    assert lib.bv_abi_version() == 1


def two_points(**kw):
    """valid_two_point_model-like fixture (lib.rs:607-660)."""
    pts = np.array([[0, 0, 0, 1], [1, 0, 0, 1]], np.float32)
    m = scenes.PointCloudModel(pts, np.zeros((2, 3), np.float32), 0,
                               np.array([0, 1, 2], np.uint32), np.array([1, 0], np.uint32))
    for k, v in kw.items():
        setattr(m, k, v)
    return m


def test_valid_model_passes():
    assert bv.validate_model(two_points()) is None


@pytest.mark.parametrize("offsets,neighbors,needle", [
    ([0, 1, 2], [0, 0], "self-edge"),                 # lib.rs:817-822
    ([0, 2, 3], [1, 1, 0], "sorted and unique"),       # lib.rs:824-829
    ([0, 1, 1], [1], "no reverse edge"),               # lib.rs:831-836
    ([0, 1, 2], [1, 5], "out of bounds"),              # lib.rs:806-811
    ([1, 1, 2], [1, 0], "adjacency_offsets[0]"),
])
def test_invalid_adjacency_rejected(offsets, neighbors, needle):
    m = two_points(offsets=np.array(offsets, np.uint32), neighbors=np.array(neighbors, np.uint32))
    err = bv.validate_model(m)
    assert err is not None and needle in err, err


def test_negative_density_and_bad_radii_rejected():
    """lib.rs:851-864."""
    m = two_points()
    m.points[0, 3] = -1.0
    assert "non-negative" in bv.validate_model(m)
    m = two_points(radii=np.array([np.nan, 1.0], np.float32))
    assert "radii" in bv.validate_model(m)
    m = two_points()
    m.sh[0, 0] = np.inf
    assert "finite" in bv.validate_model(m)


def test_sh_degree_limit():
    m = two_points()
    m.sh_degree = 4
    assert "SH degree" in bv.validate_model(m)


def test_generated_scene_is_valid():
    m = scenes.radfoam_ball(512, seed=3, sh_degree=1)
    assert bv.validate_model(m) is None
    assert 10.0 < m.mean_degree() < 20.0


def test_noalloc_wrapper_rejects_bad_tensors():
    """The Python mirror checks shapes, dtypes and placement before handing
    device pointers to bv_containing_points_noalloc (no GPU needed)."""
    torch = pytest.importorskip("torch")
    q = np.zeros((4, 3), np.float32)
    good_sites = torch.zeros((8, 4), dtype=torch.float32)
    good_out = torch.zeros(4, dtype=torch.int32)
    cases = [
        (torch.zeros((8, 3), dtype=torch.float32), good_out, "shape"),
        (torch.zeros((8, 4), dtype=torch.float64), good_out, "float32"),
        (torch.zeros((4, 8), dtype=torch.float32).t(), good_out, "contiguous"),
        (good_sites, torch.zeros(3, dtype=torch.int32), "at least 4"),
        (good_sites, torch.zeros(4, dtype=torch.int64), "int32"),
        (good_sites, good_out, "CUDA"),
    ]
    for sites, out, what in cases:
        with pytest.raises(ValueError) as e:
            bv.containing_points_noalloc(sites, q, out)
        assert what in str(e.value), (what, str(e.value))
