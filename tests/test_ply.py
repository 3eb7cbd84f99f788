"""RadFoam PLY reader/writer (blade_volume_b200.ply), the walk subset of the
reference's loader (blade-volume/src/io/radfoam_ply.rs)."""

import json
import os

import numpy as np
import pytest

import blade_volume_b200 as bv
from blade_volume_b200 import ply, scenes
from oracle import oracle as O


def same_model(a, b):
    assert a.sh_degree == b.sh_degree
    for name in ("points", "sh", "offsets", "neighbors"):
        assert np.array_equal(np.asarray(getattr(a, name)), np.asarray(getattr(b, name))), name
    assert (a.radii is None) == (b.radii is None)
    if a.radii is not None:
        assert np.array_equal(a.radii, b.radii)


@pytest.mark.parametrize("binary", [True, False])
@pytest.mark.parametrize("kind", ["radfoam", "powerfoam"])
def test_round_trip(tmp_path, binary, kind):
    m = (scenes.radfoam_ball(300, seed=2, sh_degree=2) if kind == "radfoam"
         else scenes.powerfoam_mixture(400, seed=2, sh_degree=1, radius_max=0.2, bf16=False))
    path = str(tmp_path / "m.ply")
    ply.save_radfoam_ply(m, path, binary=binary, comment="round trip")
    got = ply.load_radfoam_ply(path)
    same_model(m, got)
    assert bv.validate_model(got) is None
    # the loaded model traces exactly as the original
    cam = scenes.sphere_cameras(1, 3.0, 2, 1.0, 1.0, 100.0)[0]
    a, *_ = O.render_walk(O.OracleModel.from_scene(m), cam, 16, 16)
    b, *_ = O.render_walk(O.OracleModel.from_scene(got), cam, 16, 16)
    assert np.array_equal(a, b)


ASCII_SQUARE = """ply
format ascii 1.0
comment four points on a square, preview colours, SH degree 1 rest terms
element vertex 4
property float x
property float y
property float z
property uchar red
property uchar green
property uchar blue
property float density
property uint adjacency_offset
""" + "".join(f"property float color_sh_{k}\n" for k in range(9)) + """element adjacency 8
property uint adjacency
end_header
comment rows: x y z r g b density adjacency_offset sh_rest
0 0 0 255 0 128 0.5 2 0.1 0 0 0 0 0 0 0 -0.1
1 0 0 0 255 128 0.5 4 0 0 0 0 0 0 0 0 0
0 1 0 128 128 128 0.5 6 0 0 0 0 0 0 0 0 0
1 1 0 64 32 16 0.5 8 0 0 0 0 0 0 0 0 0
1
2
0
3
0
3
1
2
"""


def test_ascii_preview_colours_and_body_comments(tmp_path):
    path = tmp_path / "square.ply"
    path.write_text(ASCII_SQUARE)
    m = ply.load_radfoam_ply(str(path))
    assert m.n == 4 and m.sh_degree == 1 and m.radii is None
    assert list(m.offsets) == [0, 2, 4, 6, 8]
    assert list(m.neighbors) == [1, 2, 0, 3, 0, 3, 1, 2]
    # preview DC (radfoam_ply.rs:722-726)
    want = (np.float32([255, 0, 128]) / np.float32(255.0) - np.float32(0.5)) / np.float32(0.2820948)
    assert np.array_equal(m.sh[0, :3], want.astype(np.float32))
    assert m.sh[0, 3] == np.float32(0.1) and m.sh[0, 11] == np.float32(-0.1)
    assert bv.validate_model(m) is None


@pytest.mark.parametrize("edit,needle", [
    (lambda t: t.replace("ply\n", "plx\n", 1), "magic"),
    (lambda t: t.replace("format ascii 1.0", "format ascii 2.0"), "version"),
    (lambda t: t.replace("property uint adjacency\n", "property list uchar uint adjacency\n"),
     "list"),
    (lambda t: t.replace("property float color_sh_4\n", "property float color_sh_40\n"),
     "contiguous"),
    (lambda t: t.replace("property float density\n", "property float density\nproperty float nx\n"
                         "property float ny\nproperty float nz\n").replace(" 0.5 ", " 0.5 0 0 1 "),
     "not supported"),
    (lambda t: t.replace("\n3\n1\n2\n", "\n3\n1\n9\n"), "missing point"),
    (lambda t: t.replace("end_header\n", ""), "header token"),
])
def test_malformed_files_are_rejected(tmp_path, edit, needle):
    path = tmp_path / "bad.ply"
    path.write_text(edit(ASCII_SQUARE))
    with pytest.raises(ply.PlyError) as e:
        ply.load_radfoam_ply(str(path))
    assert needle in str(e.value)


def test_truncated_binary_body(tmp_path):
    m = scenes.radfoam_ball(64, seed=1, sh_degree=0)
    path = str(tmp_path / "m.ply")
    ply.save_radfoam_ply(m, path)
    with open(path, "r+b") as f:
        f.seek(0, 2)
        f.truncate(f.tell() - 4)
    with pytest.raises(ply.PlyError, match="binary body"):
        ply.load_radfoam_ply(path)


def test_rebuild_adjacency_after_moving_sites():
    m = scenes.radfoam_ball(500, seed=3, sh_degree=0)
    moved = m.copy()
    rng = np.random.default_rng(0)
    moved.points[:, :3] += rng.normal(0, 0.02, (m.n, 3)).astype(np.float32)
    fresh = scenes.rebuild_adjacency(moved)
    assert bv.validate_model(fresh) is None
    assert np.array_equal(fresh.points, moved.points)
    want_off, want_nb = scenes.delaunay_csr(moved.points[:, :3])
    assert np.array_equal(fresh.offsets, want_off) and np.array_equal(fresh.neighbors, want_nb)
    p = scenes.powerfoam_mixture(300, seed=3, sh_degree=0, radius_max=0.2)
    fresh = scenes.rebuild_adjacency(p)
    assert np.array_equal(fresh.offsets, p.offsets) and np.array_equal(fresh.neighbors, p.neighbors)


REFERENCE_FIXTURE = "/root/reference/blade-volume/tests/data/radfoam_tiny_ascii.ply"


@pytest.mark.skipif(not os.path.exists(REFERENCE_FIXTURE),
                    reason="the reference checkout is not present on this machine")
def test_loads_the_reference_ascii_fixture():
    """The reference's own fixture file (tests/data/radfoam_tiny_ascii.ply,
    loaded by tests/radfoam_cpu_ref.rs:16-42): body comment lines, rows with
    more columns than declared, preview colours.  Parsed points and CSR equal
    the transcription in tests/golden/reference_cases.json, the SH rows are
    the preview DC of grey 128 with zero rest, and the reference test's ray
    traces to a finite colour with steps > 0."""
    m = ply.load_radfoam_ply(REFERENCE_FIXTURE)
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_cases.json")) as f:
        cases = {c["name"]: c for c in json.load(f)["cases"]}
    want = cases["cpu_ref_traces_without_nan_on_tiny_fixture"]["model"]
    assert np.array_equal(m.points, np.asarray(want["points"], np.float32))
    assert np.array_equal(m.offsets, np.asarray(want["offsets"], np.uint32))
    assert np.array_equal(m.neighbors, np.asarray(want["neighbors"], np.uint32))
    assert m.sh_degree == 1  # 9 color_sh_* rest coefficients declared
    # preview DC of (128, 128, 128) (radfoam_ply.rs:722-726), SH rest all 0
    dc = (np.float32(128) / np.float32(255.0) - np.float32(0.5)) / np.float32(0.2820948)
    assert np.all(m.sh[:, :3] == dc) and np.all(m.sh[:, 3:] == 0.0)
    assert bv.validate_model(m) is None
    om = O.OracleModel.from_scene(m)
    s = O.settings(max_steps=16, weight_threshold=1e-4, start_point=0, depth=100.0,
                   eval_mode=O.EVAL_CONSTANT, constant_rgb=(1.0, 1.0, 1.0))
    r = O.trace_one_ray(om, (0.5, 0.5, -1.0), (0.0, 0.0, 1.0), s)
    assert all(np.isfinite(r.rgba[i]) for i in range(4)) and 0.0 <= r.rgba[3] <= 1.0
    assert r.steps > 0


def test_binary_and_ascii_files_read_alike(tmp_path):
    """The C reader gives the same arrays for the binary and the ASCII form
    of one model (floats written with repr, so they round-trip exactly)."""
    m = scenes.powerfoam_mixture(400, seed=9, sh_degree=2, radius_max=0.2, bf16=False)
    a, b = str(tmp_path / "m.bin.ply"), str(tmp_path / "m.txt.ply")
    ply.save_radfoam_ply(m, a, binary=True)
    ply.save_radfoam_ply(m, b, binary=False)
    same_model(ply.load_radfoam_ply(a), ply.load_radfoam_ply(b))
    with open(b, "a") as f:
        f.write("7\n")
    with pytest.raises(ply.PlyError, match="trailing"):
        ply.load_radfoam_ply(b)
