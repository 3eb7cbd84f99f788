"""Writes tests/golden/reference_cases.json: the reference crate's own
known-answer tests for the trace hot path, transcribed as data.

The reference (Rust + WGSL) cannot be built or run on this machine, so its
expected values are taken from its test sources, where they are closed-form
numbers (1 - e^-6, ...), exact integers, or a property the test states.  Each
case records the source location it transcribes.  Run from the repo root:

    python tests/golden/make_reference_cases.py
"""

import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))

EMPTY_CSR = {"offsets": [0, 0], "neighbors": []}


def settings_for(start_point=0, **kw):
    """trace.rs:1853-1861."""
    s = {"start_point": start_point, "max_steps": 32, "weight_threshold": 0.0, "depth": 100.0,
         "eval_mode": "constant", "constant_rgb": [1.0, 1.0, 1.0]}
    s.update(kw)
    return s


def tetra_points():
    """trace.rs:1828-1851 (Delaunay of 4 points: the full tetrahedron)."""
    return [[0.0, 0.0, 0.0, 5.0], [0.5, 0.0, 0.0, 5.0], [0.0, 0.5, 0.0, 5.0], [0.0, 0.0, 0.5, 5.0]]


TETRA_CSR = {"offsets": [0, 3, 6, 9, 12], "neighbors": [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2]}


def three_in_a_row_csr():
    return {"offsets": [0, 1, 3, 4], "neighbors": [1, 0, 2, 1]}


def sh_dc(color):
    """trace.rs:779-782."""
    return [(c - 0.5) / 0.2820948 for c in color]


def weighted_index_points():
    """gpu/radfoam.rs:701-712."""
    pts, radii = [], []
    for index in range(32):
        x = float((index * 17 % 23) - 11)
        y = float((index * 11 % 19) - 9)
        z = float((index * 7 % 13) - 6)
        pts.append([x, y, z, 1.0])
        radii.append(float(index * 5 % 9) * 0.75)
    queries = [[q * 0.37 - 7.0, q * -0.19 + 3.0, q * 0.11 - 2.0] for q in range(40)]
    return pts, radii, queries


def cases():
    out = []
    out.append({
        "name": "sh_color_clamps_negative_channels_before_compositing",
        "source": "blade-volume/src/trace.rs:784-806",
        "kind": "eval_rgb_sh",
        "model": {"points": [[0.0, 0.0, 1.0, 1.0]], "sh": sh_dc([-1.0, 0.25, 2.0]),
                  "sh_degree": 0, **EMPTY_CSR},
        "direction": [0.0, 0.0, 1.0],
        "expect": {"rgb": [0.0, 0.25, 2.0], "exact": [True, False, False], "tol": 1e-6},
    })
    out.append({
        "name": "terminal_cell_integrates_to_depth_without_an_exit_face",
        "source": "blade-volume/src/trace.rs:2209-2244",
        "kind": "walk",
        "model": {"points": [[0.0, 0.0, 0.0, 2.0]], "sh_degree": 0, **EMPTY_CSR},
        "ray": {"origin": [0.0, 0.0, 0.0], "direction": [0.0, 0.0, 1.0]},
        "settings": settings_for(depth=3.0),
        "expect": {"record_cells": [0], "record_dt": [3.0], "record_dt_exact": True,
                   "alpha": 1.0 - math.exp(-6.0), "alpha_tol": 1e-6, "t_end": 3.0},
    })
    out.append({
        "name": "power_foam_clips_cell_integration_to_support_sphere",
        "source": "blade-volume/src/trace.rs:2246-2280",
        "kind": "walk",
        "model": {"points": [[0.0, 0.0, 0.0, 2.0]], "radii": [1.0], "sh_degree": 0, **EMPTY_CSR},
        "ray": {"origin": [0.0, 0.0, -2.0], "direction": [0.0, 0.0, 1.0]},
        "settings": settings_for(depth=10.0),
        "expect": {"record_cells": [0], "record_dt": [2.0], "record_dt_tol": 1e-6,
                   "alpha": 1.0 - math.exp(-4.0), "alpha_tol": 1e-6, "t_end": 10.0},
    })
    out.append({
        "name": "powerfoam_splats_discover_disconnected_supports_in_depth_order",
        "source": "blade-volume/src/trace.rs:2397-2442",
        "kind": "splats",
        "model": {"points": [[0.0, 0.0, 3.0, 1.0], [0.0, 0.0, 6.0, 1.0]], "radii": [0.5, 0.5],
                  "sh_degree": 0, "offsets": [0, 0, 0], "neighbors": []},
        "ray": {"origin": [0.0, 0.0, 0.0], "direction": [0.0, 0.0, 1.0]},
        "settings": settings_for(depth=10.0),
        "expect": {"walk_entries": 1, "splat_cells": [0, 1], "splat_dt": [1.0, 1.0],
                   "tol": 1e-6},
    })
    out.append({
        "name": "support_sphere_preserves_non_unit_ray_parameterization",
        "source": "blade-volume/src/trace.rs:2444-2461",
        "kind": "support_interval",
        "origin": [0.0, 0.0, -2.0], "center": [0.0, 0.0, 0.0], "radius": 1.0,
        "t0": 0.0, "t1": 10.0,
        "expect": {"unit": [1.0, 3.0], "scaled": [0.5, 1.5]},
    })
    out.append({
        "name": "power_foam_walk_matches_brute_force_bounded_cells",
        "source": "blade-volume/src/trace.rs:2463-2549",
        "kind": "walk_vs_brute_force",
        "model": {"points": [[0.0, 0.0, 0.0, 1.0], [2.0, 0.0, 0.0, 1.0], [4.0, 0.0, 0.0, 1.0]],
                  "radii": [1.4, 0.9, 1.6], "sh_degree": 0,
                  "offsets": [0, 2, 4, 6], "neighbors": [1, 2, 0, 2, 0, 1]},
        "ray": {"origin": [-2.0, 0.0, 0.0], "direction": [1.0, 0.0, 0.0]},
        "settings": settings_for(depth=8.0),
        "expect": {"dt_tol": 1e-5},
    })
    out.append({
        "name": "power_foam_face_jacobians_match_central_finite_differences",
        "source": "blade-volume/src/trace.rs:2646-2721",
        "kind": "jacobian_fd",
        "model": {"points": [[0.0, 0.0, 0.0, 1.0], [1.0, 0.0, 0.0, 1.0], [2.0, 0.0, 0.0, 1.0]],
                  "radii": [2.0, 2.0, 2.0], "sh_degree": 0, **three_in_a_row_csr()},
        "ray": {"origin": [-3.0, 0.2, -0.1], "direction": [1.0, 0.05, 0.02]},
        "settings": settings_for(depth=10.0),
        "expect": {"cell": 1, "previous_cell": 0, "next_cell": 2, "epsilon": 1e-3,
                   "abs_tol": 2e-3, "rel_tol": 1e-2},
    })
    out.append({
        "name": "power_foam_sphere_jacobian_matches_central_finite_differences",
        "source": "blade-volume/src/trace.rs:2723-2770",
        "kind": "jacobian_fd",
        "model": {"points": [[0.0, 0.0, 0.0, 1.0]], "radii": [1.0], "sh_degree": 0, **EMPTY_CSR},
        "ray": {"origin": [0.2, 0.1, -2.0], "direction": [0.0, 0.0, 1.0]},
        "settings": settings_for(depth=10.0),
        "expect": {"cell": 0, "previous_cell": 0, "next_cell": 0, "epsilon": 1e-3,
                   "abs_tol": 2e-3, "rel_tol": 1e-2, "zero_previous_next": True},
    })
    out.append({
        "name": "path_jacobian_keeps_true_entry_neighbor_across_skipped_cells",
        "source": "blade-volume/src/trace.rs:2859-2898",
        "kind": "walk_cells",
        "model": {"points": [[0.0, 0.0, 0.0, 1.0], [1.0, 0.0, 0.0, 1.0], [2.0, 0.0, 0.0, 1.0]],
                  "radii": [0.95, 0.1, 0.95], "sh_degree": 0, **three_in_a_row_csr()},
        "ray": {"origin": [-2.0, 0.2, 0.0], "direction": [1.0, 0.0, 0.0]},
        "settings": settings_for(depth=6.0),
        "expect": {"cells": [0, 2], "previous_of_second": 1},
    })
    out.append({
        "name": "tetra_record_path_and_trace_agree",
        "source": "blade-volume/src/trace.rs:2143-2207",
        "kind": "tetra",
        "model": {"points": tetra_points(), "sh_degree": 0, **TETRA_CSR},
        "ray": {"origin": [0.1, 0.1, -1.0], "direction": [0.0, 0.0, 1.0]},
        "settings": settings_for(),
        "expect": {"alpha_tol": 1e-4, "max_steps_2_entries_at_most": 2},
    })
    out.append({
        "name": "opacity_trace_preserves_every_non_colour_result",
        "source": "blade-volume/src/trace.rs:2115-2141",
        "kind": "opacity",
        "model": {"points": tetra_points(), "sh_degree": 0, **TETRA_CSR},
        "ray": {"origin": [-1.0, 0.1, 0.1], "direction": [1.0, 0.0, 0.0]},
        "settings": settings_for(),
        "expect": {},
    })
    out.append({
        "name": "cpu_ref_traces_without_nan_on_tiny_fixture",
        "source": "blade-volume/tests/radfoam_cpu_ref.rs:16-42 (tests/data/radfoam_tiny_ascii.ply)",
        "kind": "finite",
        "model": {"points": [[0.0, 0.0, 0.0, 0.1], [1.0, 0.0, 0.0, 0.1], [0.0, 1.0, 0.0, 0.1],
                             [1.02, 1.0, 0.0, 0.1]],
                  "sh_degree": 0, "offsets": [0, 3, 6, 9, 12],
                  "neighbors": [1, 2, 3, 0, 2, 3, 0, 1, 3, 0, 1, 2]},
        "ray": {"origin": [0.5, 0.5, -1.0], "direction": [0.0, 0.0, 1.0]},
        "settings": settings_for(max_steps=16, weight_threshold=1e-4),
        "expect": {},
    })
    out.append({
        "name": "containing_cell_uses_power_distance_for_weighted_clouds",
        "source": "blade-volume/src/lib.rs:838-849; blade-volume/src/gpu/radfoam.rs:686-698",
        "kind": "containing_cell",
        "points": [[0.0, 0.0, 0.0, 1.0], [10.0, 0.0, 0.0, 1.0]],
        "cases": [{"radii": None, "query": [0.0, 0.0, 0.0], "expect": 0},
                  {"radii": [0.0, 20.0], "query": [0.0, 0.0, 0.0], "expect": 1}],
    })
    pts, radii, queries = weighted_index_points()
    out.append({
        "name": "weighted_index_matches_exhaustive_power_distance",
        "source": "blade-volume/src/gpu/radfoam.rs:700-735",
        "kind": "containing_cell_exhaustive",
        "points": pts, "radii": radii, "queries": queries,
    })
    return out


def main():
    path = os.path.join(HERE, "reference_cases.json")
    with open(path, "w") as f:
        json.dump({"generated_by": "tests/golden/make_reference_cases.py", "cases": cases()}, f,
                  indent=1)
    print(path)


if __name__ == "__main__":
    main()
