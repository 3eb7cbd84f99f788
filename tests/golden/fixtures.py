"""Synthetic fixtures of the reference's own GPU-vs-CPU tests, restated.

* branching_model: blade-volume/tests/radfoam_synth_branch.rs:106-277
  (a spine along +Z with a ring of branch sites at every spine node; CSR
  sorted per row), used by tests/radfoam_gpu_vs_cpu.rs:437-448 with
  spine_len 64, dz 0.05, branch_degree 6, branch_radius 0.10,
  branch_z_offset 0.02, density 0.1, SH degree 3, DC 0.1.
* gpu_vs_cpu_camera: the test camera of radfoam_gpu_vs_cpu.rs:266-275 and
  its trace parameters :279-305 (8x8, max_steps 256, threshold 1e-4).
"""

import math

import numpy as np

from blade_volume_b200.scenes import Camera, PointCloudModel

TEST_PIXELS = [(0, 0), (1, 1), (1, 6), (3, 3), (4, 4), (6, 6)]  # radfoam_gpu_vs_cpu.rs:435


def branching_model(spine_len=64, dz=0.05, branch_degree=6, branch_radius=0.10,
                    branch_z_offset=0.02, density=0.1, sh_degree=3, dc=(0.1, 0.1, 0.1)):
    f32 = np.float32
    K = (sh_degree + 1) ** 2
    n_spine = spine_len
    n_total = n_spine + spine_len * branch_degree
    angles = [f32(f32(j) / f32(branch_degree)) * f32(2.0 * math.pi) for j in range(branch_degree)]
    pts = []
    for i in range(n_spine):
        pts.append([0.0, 0.0, f32(i) * f32(dz), density])
    for i in range(n_spine):
        sx, sy, sz = pts[i][0], pts[i][1], pts[i][2]
        for a in angles:
            x = f32(branch_radius) * f32(math.cos(a))
            y = f32(branch_radius) * f32(math.sin(a))
            pts.append([f32(sx) + x, f32(sy) + y, f32(sz) + f32(branch_z_offset), density])
    neigh = [[] for _ in range(n_total)]
    for i in range(n_spine):
        if i > 0:
            neigh[i].append(i - 1)
        if i + 1 < n_spine:
            neigh[i].append(i + 1)
        for j in range(branch_degree):
            b = n_spine + i * branch_degree + j
            neigh[i].append(b)
            neigh[b].append(i)
    offsets = [0]
    nb = []
    for lst in neigh:
        lst = sorted(set(lst))
        nb.extend(lst)
        offsets.append(len(nb))
    sh = np.zeros((n_total, 3 * K), dtype=np.float32)
    sh[:, 0:3] = dc
    if sh_degree >= 1:
        sh[:, 3] = 0.05
    if sh_degree >= 2:
        sh[:, 12] = 0.03
    if sh_degree >= 3:
        sh[:, 27] = 0.02
    return PointCloudModel(np.asarray(pts, dtype=np.float32), sh, sh_degree,
                           np.asarray(offsets, dtype=np.uint32), np.asarray(nb, dtype=np.uint32))


def gpu_vs_cpu_camera():
    return Camera(position=np.array([0.0, 0.0, -1.0], np.float32), depth=100.0,
                  orientation=np.array([0.0, 0.0, 0.0, 1.0], np.float32),
                  fov=np.array([1.0, 1.0], np.float32),
                  principal=np.array([0.08, -0.04], np.float32))
