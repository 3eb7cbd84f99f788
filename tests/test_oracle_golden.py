"""Pins the CPU oracle against the reference crate's own known-answer tests.

The cases in tests/golden/reference_cases.json are transcribed from the
reference's test sources (each case names its file:line).  The reference
itself cannot run here, so these closed-form answers are what tie the oracle
to it; the CUDA path is then compared against the oracle.
"""

import json
import math
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "reference_cases.json")) as f:
    CASES = {c["name"]: c for c in json.load(f)["cases"]}


def model_of(spec):
    pts = np.asarray(spec["points"], dtype=np.float32)
    n = len(pts)
    K = (spec.get("sh_degree", 0) + 1) ** 2
    sh = np.asarray(spec.get("sh", [0.0] * (n * 3 * K)), dtype=np.float32)
    radii = spec.get("radii")
    return O.OracleModel(pts, sh, spec.get("sh_degree", 0), spec["offsets"], spec["neighbors"],
                         None if radii is None else np.asarray(radii, dtype=np.float32))


def settings_of(spec):
    mode = {"constant": O.EVAL_CONSTANT, "opacity": O.EVAL_OPACITY, "sh": O.EVAL_SH}[
        spec["eval_mode"]]
    return O.settings(spec["max_steps"], spec["weight_threshold"], spec["start_point"],
                      spec["depth"], mode, spec.get("constant_rgb", (1, 1, 1)))


def test_sh_color_clamps_negative_channels():
    c = CASES["sh_color_clamps_negative_channels_before_compositing"]
    m = model_of(c["model"])
    out, _ = O.eval_rgb_sh(m, 0, c["direction"])
    assert out[0] == 0.0
    assert abs(out[1] - 0.25) < 1e-6
    assert abs(out[2] - 2.0) < 1e-6


@pytest.mark.parametrize("name", ["terminal_cell_integrates_to_depth_without_an_exit_face",
                                  "power_foam_clips_cell_integration_to_support_sphere"])
def test_walk_known_answers(name):
    c = CASES[name]
    m = model_of(c["model"])
    s = settings_of(c["settings"])
    e = c["expect"]
    path = O.record_path_jacobians(m, c["ray"]["origin"], c["ray"]["direction"], s)
    assert [p.cell for p in path] == e["record_cells"]
    if e.get("record_dt_exact"):
        assert [p.dt for p in path] == e["record_dt"]
    else:
        for p, dt in zip(path, e["record_dt"]):
            assert abs(p.dt - dt) < e["record_dt_tol"]
    r = O.trace_one_ray(m, c["ray"]["origin"], c["ray"]["direction"], s)
    assert abs(r.rgba[3] - e["alpha"]) < e["alpha_tol"]
    assert r.t_end == e["t_end"]


def test_splats_discover_disconnected_supports():
    c = CASES["powerfoam_splats_discover_disconnected_supports_in_depth_order"]
    m = model_of(c["model"])
    s = settings_of(c["settings"])
    e = c["expect"]
    walked = O.record_path_jacobians(m, c["ray"]["origin"], c["ray"]["direction"], s)
    assert len(walked) == e["walk_entries"]
    splat = O.record_powerfoam_splats(m, c["ray"]["origin"], c["ray"]["direction"], s)
    assert [p.cell for p in splat] == e["splat_cells"]
    assert all(abs(p.dt - 1.0) < e["tol"] for p in splat)


def test_support_interval_non_unit_direction():
    c = CASES["support_sphere_preserves_non_unit_ray_parameterization"]
    unit = O.support_interval(True, c["origin"], [0, 0, 1], c["center"], c["radius"], c["t0"],
                              c["t1"])
    scaled = O.support_interval(True, c["origin"], [0, 0, 2], c["center"], c["radius"], c["t0"],
                                c["t1"])
    assert unit == tuple(c["expect"]["unit"])
    assert scaled == tuple(c["expect"]["scaled"])


def test_power_walk_matches_brute_force():
    """Independent O(N^2) power-cell oracle, as trace.rs:2496-2548 builds it."""
    c = CASES["power_foam_walk_matches_brute_force_bounded_cells"]
    m = model_of(c["model"])
    s = settings_of(c["settings"])
    o = np.asarray(c["ray"]["origin"], np.float32)
    d = np.asarray(c["ray"]["direction"], np.float32)
    walked = O.record_path_jacobians(m, o, d, s)
    pts = np.asarray(c["model"]["points"], np.float32)[:, :3]
    radii = np.asarray(c["model"]["radii"], np.float32)
    brute = []
    for i in range(len(pts)):
        near, far = np.float32(0.0), np.float32(s.depth)
        for j in range(len(pts)):
            if i == j:
                continue
            off = pts[j] - pts[i]
            shift = np.float32(0.5) + np.float32(0.5) * (radii[i] ** 2 - radii[j] ** 2) / np.float32(
                off @ off)
            face = pts[i] + shift * off
            den = np.float32(off @ d)
            t = np.float32((face - o) @ off) / den
            if den > 0:
                far = min(far, t)
            elif den < 0:
                near = max(near, t)
        iv = O.support_interval(True, o, d, pts[i], radii[i], near, far)
        if iv is not None:
            brute.append((iv[0], i, iv[1] - iv[0]))
    brute.sort()
    assert len(walked) == len(brute)
    for w, (_, cell, dt) in zip(walked, brute):
        assert w.cell == cell
        assert abs(w.dt - dt) < c["expect"]["dt_tol"]


def _perturbed_dt(c, cell, param_cell, comp, delta, query=False):
    spec = json.loads(json.dumps(c["model"]))
    if comp < 3:
        spec["points"][param_cell][comp] += delta
    else:
        spec["radii"][param_cell] += delta
    m = model_of(spec)
    path = O.record_path_jacobians(m, c["ray"]["origin"], c["ray"]["direction"],
                                   settings_of(c["settings"]))
    for e in path:
        if e.cell == cell:
            return e.surface_query_near if query else e.dt
    raise AssertionError("perturbation removed the cell from the fixed path")


@pytest.mark.parametrize("name", ["power_foam_face_jacobians_match_central_finite_differences",
                                  "power_foam_sphere_jacobian_matches_central_finite_differences"])
def test_path_jacobians_match_central_differences(name):
    """trace.rs:2590-2644 tolerances: abs < 2e-3 or rel < 1e-2, eps 1e-3 (FP32)."""
    c = CASES[name]
    e = c["expect"]
    m = model_of(c["model"])
    path = O.record_path_jacobians(m, c["ray"]["origin"], c["ray"]["direction"],
                                   settings_of(c["settings"]))
    entry = [p for p in path if p.cell == e["cell"]][0]
    assert entry.previous_cell == e["previous_cell"]
    assert entry.next_cell == e["next_cell"]
    if e.get("zero_previous_next"):
        assert list(entry.dt_d_previous) == [0, 0, 0, 0]
        assert list(entry.dt_d_next) == [0, 0, 0, 0]
    if e.get("zero_previous_next"):
        # trace.rs:2754-2769 checks only the current site's derivatives here
        checks = [(entry.cell, entry.dt_d_current, False),
                  (entry.cell, entry.surface_query_d_current, True)]
    else:
        checks = [(entry.previous_cell, entry.dt_d_previous, False),
                  (entry.cell, entry.dt_d_current, False),
                  (entry.next_cell, entry.dt_d_next, False),
                  (entry.previous_cell, entry.surface_query_d_previous, True),
                  (entry.cell, entry.surface_query_d_current, True)]
    eps = e["epsilon"]
    for param_cell, analytic, query in checks:
        for comp in range(4):
            plus = _perturbed_dt(c, entry.cell, param_cell, comp, eps, query)
            minus = _perturbed_dt(c, entry.cell, param_cell, comp, -eps, query)
            numerical = (plus - minus) / (2 * eps)
            expected = analytic[comp]
            absolute = abs(expected - numerical)
            scale = max(abs(expected), abs(numerical), 1e-4)
            assert absolute < e["abs_tol"] or absolute / scale < e["rel_tol"], (
                param_cell, comp, expected, numerical)


def test_path_keeps_true_entry_neighbor_across_skipped_cells():
    c = CASES["path_jacobian_keeps_true_entry_neighbor_across_skipped_cells"]
    m = model_of(c["model"])
    path = O.record_path_jacobians(m, c["ray"]["origin"], c["ray"]["direction"],
                                   settings_of(c["settings"]))
    assert [p.cell for p in path] == c["expect"]["cells"]
    assert path[1].previous_cell == c["expect"]["previous_of_second"]
    assert path[1].previous_cell != path[0].cell


def test_tetra_record_path_properties():
    c = CASES["tetra_record_path_and_trace_agree"]
    m = model_of(c["model"])
    s = settings_of(c["settings"])
    o, d = c["ray"]["origin"], c["ray"]["direction"]
    path = O.record_path_jacobians(m, o, d, s)
    assert path, "path is empty"
    for e in path:
        assert math.isfinite(e.dt) and e.dt >= 0.0
        assert e.cell < m.n
    traced = O.trace_one_ray(m, o, d, s)
    T, acc = 1.0, 0.0
    for e in path:
        sig = float(m.points[e.cell, 3])
        if sig <= 1e-6:
            continue
        a = 1.0 - math.exp(-sig * e.dt)
        acc += T * a
        T *= 1.0 - a
    assert abs(acc - traced.rgba[3]) < c["expect"]["alpha_tol"]
    s2 = settings_of(c["settings"])
    s2.max_steps = 2
    assert len(O.record_path_jacobians(m, o, d, s2)) <= 2


def test_opacity_trace_preserves_non_colour_results():
    c = CASES["opacity_trace_preserves_every_non_colour_result"]
    m = model_of(c["model"])
    s = settings_of(c["settings"])
    o, d = c["ray"]["origin"], c["ray"]["direction"]
    colour = O.trace_one_ray(m, o, d, s)
    s.eval_mode = O.EVAL_OPACITY
    opacity = O.trace_one_ray(m, o, d, s)
    assert list(opacity.rgba)[:3] == [0.0, 0.0, 0.0]
    assert opacity.rgba[3] == colour.rgba[3]
    for f in ("steps", "last_point", "t_end", "depth_mode", "peak_weight", "peak_point"):
        assert getattr(opacity, f) == getattr(colour, f)
    assert colour.peak_point >= 0


def test_tiny_fixture_traces_finite():
    c = CASES["cpu_ref_traces_without_nan_on_tiny_fixture"]
    m = model_of(c["model"])
    r = O.trace_one_ray(m, c["ray"]["origin"], c["ray"]["direction"], settings_of(c["settings"]))
    assert all(math.isfinite(v) for v in r.rgba)
    assert 0.0 <= r.rgba[3] <= 1.0
    assert r.steps > 0


def test_containing_cell_power_distance():
    c = CASES["containing_cell_uses_power_distance_for_weighted_clouds"]
    for case in c["cases"]:
        spec = {"points": c["points"], "radii": case["radii"], "sh_degree": 0,
                "offsets": [0, 0, 0], "neighbors": []}
        m = model_of(spec)
        assert O.containing_cell_f64(m, case["query"]) == case["expect"]
        assert O.containing_cell_f32(m, case["query"]) == case["expect"]


def test_containing_cell_matches_exhaustive():
    c = CASES["weighted_index_matches_exhaustive_power_distance"]
    n = len(c["points"])
    m = model_of({"points": c["points"], "radii": c["radii"], "sh_degree": 0,
                  "offsets": [0] * (n + 1), "neighbors": []})
    pts = np.asarray(c["points"], np.float32)[:, :3]
    radii = np.asarray(c["radii"], np.float32)
    for q in c["queries"]:
        qv = np.asarray(q, np.float32)
        dist = ((qv - pts) ** 2).sum(axis=1, dtype=np.float32) - radii ** 2
        expected = int(np.flatnonzero(dist == dist.min())[0])
        assert O.containing_cell_f32(m, qv) == expected
        assert O.containing_cell_f64(m, qv) == expected


def test_expf_within_two_ulp():
    """The exp used by oracle and kernels (Cody-Waite + degree-7 Taylor)."""
    xs = np.concatenate([np.linspace(-103.0, 88.0, 20001), np.linspace(-1, 1, 4001),
                         -np.logspace(-8, 2, 2001)]).astype(np.float32)
    worst = 0.0
    for x in xs:
        got = np.float32(O.expf(float(x)))
        ref = math.exp(float(x))
        if ref < 1.2e-38:
            continue
        ulp = float(np.spacing(np.float32(ref)))
        worst = max(worst, abs(float(got) - ref) / ulp)
    assert worst <= 2.0, worst
    assert O.expf(0.0) == 1.0
    assert O.expf(-200.0) == 0.0
    assert math.isinf(O.expf(100.0))
