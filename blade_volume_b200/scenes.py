"""Seeded synthetic scenes for the walk/trace hot path.

A scene is a :class:`PointCloudModel` with the same fields and array layouts
as the reference crate's ``PointCloudModel`` (blade-volume/src/lib.rs:174-239):

* ``points``      float32 [N, 4]  x, y, z, density
* ``sh``          float32 [N, 3*K] packed ``[component][rgb]`` (lib.rs:178-185)
* ``sh_degree``   0..3, K = (degree + 1)^2
* ``radii``       float32 [N] or None (PowerFoam power radii, lib.rs:195)
* ``offsets``     uint32 [N+1], ``neighbors`` uint32 [M]: sorted, symmetric
  CSR without self edges, as ``validate_csr`` requires (adjacency.rs:717)

Adjacency is the Delaunay edge set (scipy's Qhull, the same Delaunay class as
the reference's adjacency.rs:142) for plain RadFoam and the Cech overlap
graph ``|p_i - p_j| <= r_i + r_j`` (adjacency.rs:418) for PowerFoam.

The workloads follow the seeded descriptions of the benchmark configurations:

* ``radfoam_tiny``      16,384 sites, SH degree 0, one 128x128 camera
* ``radfoam_train``     262,144 sites, SH degree 3, 8 cameras at 512x512
* ``powerfoam_mixture`` 1,048,576 sites, radii U[0, 0.02], SH degree 3 (BF16)

and smaller variants of each (``n_sites``/``width`` overrides) for parity
tests.  They are synthetic stand-ins generated here; no dataset is read.
"""

from __future__ import annotations

import dataclasses
import math
from typing import List, Optional

import numpy as np

SH_C0 = 0.2820948  # trace.rs:244


@dataclasses.dataclass
class PointCloudModel:
    points: np.ndarray  # float32 [N, 4]
    sh: np.ndarray  # float32 [N, 3K]
    sh_degree: int
    offsets: np.ndarray  # uint32 [N+1]
    neighbors: np.ndarray  # uint32 [M]
    radii: Optional[np.ndarray] = None  # float32 [N]
    sh_bf16: bool = False

    @property
    def n(self) -> int:
        return int(self.points.shape[0])

    @property
    def sh_components(self) -> int:
        d = min(self.sh_degree, 3) + 1
        return d * d

    def mean_degree(self) -> float:
        return float(len(self.neighbors)) / max(self.n, 1)

    def copy(self) -> "PointCloudModel":
        return PointCloudModel(
            self.points.copy(),
            self.sh.copy(),
            self.sh_degree,
            self.offsets.copy(),
            self.neighbors.copy(),
            None if self.radii is None else self.radii.copy(),
            self.sh_bf16,
        )


@dataclasses.dataclass
class Camera:
    """CameraParams (blade-volume/src/camera.rs:9-18): 48 bytes."""

    position: np.ndarray  # float32 [3]
    depth: float
    orientation: np.ndarray  # float32 [4] quaternion xyzw
    fov: np.ndarray  # float32 [2]
    principal: np.ndarray  # float32 [2]

    def packed(self) -> np.ndarray:
        out = np.zeros(12, dtype=np.float32)
        out[0:3] = self.position
        out[3] = self.depth
        out[4:8] = self.orientation
        out[8:10] = self.fov
        out[10:12] = self.principal
        return out


@dataclasses.dataclass
class Workload:
    name: str
    model: PointCloudModel
    cameras: List[Camera]
    width: int
    height: int
    max_steps: int = 1024
    weight_threshold: float = 1e-3
    targets: Optional[np.ndarray] = None  # float32 [views, H, W, 3]


# --------------------------------------------------------------------------
# cameras
# --------------------------------------------------------------------------
def _quat_from_matrix(m: np.ndarray) -> np.ndarray:
    """Unit quaternion (x, y, z, w) of a rotation matrix with columns = axes
    (Shepperd's method, branch on the largest diagonal term)."""
    m = np.asarray(m, dtype=np.float64)
    tr = m[0, 0] + m[1, 1] + m[2, 2]
    if tr > 0.0:
        s = math.sqrt(tr + 1.0) * 2.0
        w = 0.25 * s
        x = (m[2, 1] - m[1, 2]) / s
        y = (m[0, 2] - m[2, 0]) / s
        z = (m[1, 0] - m[0, 1]) / s
    elif m[0, 0] > m[1, 1] and m[0, 0] > m[2, 2]:
        s = math.sqrt(1.0 + m[0, 0] - m[1, 1] - m[2, 2]) * 2.0
        w = (m[2, 1] - m[1, 2]) / s
        x = 0.25 * s
        y = (m[0, 1] + m[1, 0]) / s
        z = (m[0, 2] + m[2, 0]) / s
    elif m[1, 1] > m[2, 2]:
        s = math.sqrt(1.0 + m[1, 1] - m[0, 0] - m[2, 2]) * 2.0
        w = (m[0, 2] - m[2, 0]) / s
        x = (m[0, 1] + m[1, 0]) / s
        y = 0.25 * s
        z = (m[1, 2] + m[2, 1]) / s
    else:
        s = math.sqrt(1.0 + m[2, 2] - m[0, 0] - m[1, 1]) * 2.0
        w = (m[1, 0] - m[0, 1]) / s
        x = (m[0, 2] + m[2, 0]) / s
        y = (m[1, 2] + m[2, 1]) / s
        z = 0.25 * s
    q = np.array([x, y, z, w], dtype=np.float64)
    return q / np.linalg.norm(q)


def orientation_looking(forward, world_up=(0.0, 1.0, 0.0)) -> np.ndarray:
    """camera.rs:27-45: local frame right, down, forward."""
    f = np.asarray(forward, dtype=np.float64)
    n = np.linalg.norm(f)
    if n == 0.0:
        return np.array([0.0, 0.0, 0.0, 1.0])
    f = f / n
    up = np.asarray(world_up, dtype=np.float64)
    if abs(float(f @ up)) > 0.999:
        ref = np.array([0.0, 0.0, 1.0]) if abs(up[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    else:
        ref = up
    down = f * float(f @ ref) - ref
    down /= np.linalg.norm(down)
    right = np.cross(down, f)
    right /= np.linalg.norm(right)
    return _quat_from_matrix(np.stack([right, down, f], axis=1))


def looking_at(position, target, fov_y: float, aspect: float, depth: float) -> Camera:
    """CameraParams::looking_at (camera.rs:53-68)."""
    position = np.asarray(position, dtype=np.float64)
    target = np.asarray(target, dtype=np.float64)
    q = orientation_looking(target - position)
    fov_x = 2.0 * math.atan(math.tan(0.5 * fov_y) * aspect)
    return Camera(
        position=position.astype(np.float32),
        depth=float(np.float32(depth)),
        orientation=q.astype(np.float32),
        fov=np.array([fov_x, fov_y], dtype=np.float32),
        principal=np.zeros(2, dtype=np.float32),
    )


def sphere_cameras(count: int, radius: float, seed: int, fov_y: float, aspect: float,
                   depth: float) -> List[Camera]:
    """Fibonacci directions on a sphere, randomly rotated by ``seed``, each
    camera looking at the origin."""
    rng = np.random.default_rng(seed)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    dirs = []
    for i in range(count):
        y = 1.0 - 2.0 * (i + 0.5) / count
        r = math.sqrt(max(0.0, 1.0 - y * y))
        phi = golden * i
        dirs.append([math.cos(phi) * r, y, math.sin(phi) * r])
    dirs = np.asarray(dirs)
    # random rotation (QR of a Gaussian matrix)
    a = rng.standard_normal((3, 3))
    qm, rm = np.linalg.qr(a)
    qm = qm * np.sign(np.diag(rm))
    if np.linalg.det(qm) < 0:
        qm[:, 0] = -qm[:, 0]
    dirs = dirs @ qm.T
    return [looking_at(radius * d, (0.0, 0.0, 0.0), fov_y, aspect, depth) for d in dirs]


# --------------------------------------------------------------------------
# adjacency
# --------------------------------------------------------------------------
def _csr_from_pairs(n: int, a: np.ndarray, b: np.ndarray):
    """Sorted symmetric CSR of the undirected pairs (a, b), duplicates and
    self-pairs dropped.  scipy's COO -> CSR conversion is a counting sort by
    row, so this stays linear in the number of pairs."""
    import scipy.sparse as sp

    a = np.asarray(a, dtype=np.int64)
    b = np.asarray(b, dtype=np.int64)
    keep = a != b
    a, b = a[keep], b[keep]
    rows = np.concatenate([a, b])
    cols = np.concatenate([b, a])
    m = sp.csr_matrix((np.ones(len(rows), dtype=np.int32), (rows, cols)), shape=(n, n))
    m.sum_duplicates()
    m.sort_indices()
    return m.indptr.astype(np.uint32), m.indices.astype(np.uint32)


def _cached_csr(kind: str, build, *arrays):
    """build() memoised on disk when BV_SCENE_CACHE names a directory, keyed
    by the bytes of the input arrays (the adjacency of the large scenes
    takes most of a minute to build, and several processes of one run build
    the same scenes)."""
    import hashlib
    import os

    root = os.environ.get("BV_SCENE_CACHE")
    if not root:
        return build()
    h = hashlib.sha1(kind.encode())
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    path = os.path.join(root, f"{kind}_{h.hexdigest()}.npz")
    if os.path.exists(path):
        with np.load(path) as z:
            return z["offsets"], z["neighbors"]
    offsets, neighbors = build()
    os.makedirs(root, exist_ok=True)
    tmp = path + f".{os.getpid()}.tmp.npz"
    np.savez(tmp, offsets=offsets, neighbors=neighbors)
    os.replace(tmp, path)
    return offsets, neighbors


def delaunay_csr(xyz: np.ndarray):
    """Delaunay edges -> sorted symmetric CSR (adjacency.rs:55-136, :142)."""
    return _cached_csr("delaunay", lambda: _delaunay_csr(xyz), np.asarray(xyz, np.float32))


def _delaunay_csr(xyz: np.ndarray):
    from scipy.spatial import Delaunay

    tri = Delaunay(np.asarray(xyz, dtype=np.float64))
    s = tri.simplices.astype(np.int64)
    idx = np.array([[0, 1], [0, 2], [0, 3], [1, 2], [1, 3], [2, 3]])
    pairs = s[:, idx].reshape(-1, 2)
    return _csr_from_pairs(len(xyz), pairs[:, 0], pairs[:, 1])


def cech_csr(xyz: np.ndarray, radii: np.ndarray):
    """Cech overlap graph |p_i - p_j| <= r_i + r_j (adjacency.rs:405-420)."""
    return _cached_csr("cech", lambda: _cech_csr(xyz, radii), np.asarray(xyz, np.float32),
                       np.asarray(radii, np.float32))


def _cech_csr(xyz: np.ndarray, radii: np.ndarray):
    from scipy.spatial import cKDTree

    xyz32 = np.asarray(xyz, dtype=np.float32)
    r = np.maximum(np.asarray(radii, dtype=np.float32), 0.0)
    tree = cKDTree(xyz32.astype(np.float64))
    rmax = float(r.max()) if len(r) else 0.0
    pairs = tree.query_pairs(2.0 * rmax, output_type="ndarray")
    if len(pairs) == 0:
        return _csr_from_pairs(len(xyz), np.zeros(0), np.zeros(0))
    keep_a, keep_b = [], []
    for c0 in range(0, len(pairs), 1 << 22):  # chunks stay cache-sized
        a, b = pairs[c0:c0 + (1 << 22), 0], pairs[c0:c0 + (1 << 22), 1]
        d = xyz32[a] - xyz32[b]
        dist = np.sqrt((d.astype(np.float32) ** 2).sum(axis=1, dtype=np.float32))
        keep = dist <= (r[a] + r[b])
        keep_a.append(a[keep])
        keep_b.append(b[keep])
    return _csr_from_pairs(len(xyz), np.concatenate(keep_a), np.concatenate(keep_b))


def rebuild_adjacency(model: "PointCloudModel") -> "PointCloudModel":
    """A copy of the model with its CSR rebuilt from the current sites:
    Delaunay edges for RadFoam, the Cech overlap graph for PowerFoam
    (try_compute_adjacency / compute_cech, adjacency.rs:142-200, :418).  Use
    it after optimizer steps have moved sites, then build a new tracer."""
    out = model.copy()
    xyz = np.ascontiguousarray(out.points[:, :3], np.float32)
    if out.radii is None:
        out.offsets, out.neighbors = delaunay_csr(xyz)
    else:
        out.offsets, out.neighbors = cech_csr(xyz, out.radii)
    return out


# --------------------------------------------------------------------------
# generators
# --------------------------------------------------------------------------
def _uniform_ball(rng, n: int) -> np.ndarray:
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = rng.random(n) ** (1.0 / 3.0)
    return d * r[:, None]


def _dc_from_color(c: np.ndarray) -> np.ndarray:
    """DC coefficient giving colour c (trace.rs:779-782)."""
    return ((c - 0.5) / SH_C0).astype(np.float32)


def radfoam_ball(n_sites: int, seed: int, sh_degree: int, jitter: float = 0.0,
                 density_sigma: float = 1.0, higher_sigma: float = 0.2) -> PointCloudModel:
    rng = np.random.default_rng(seed)
    xyz = _uniform_ball(rng, n_sites)
    if jitter > 0.0:
        xyz = xyz + rng.normal(0.0, jitter, xyz.shape)
    xyz = xyz.astype(np.float32)
    density = rng.lognormal(0.0, density_sigma, n_sites).astype(np.float32)
    K = (sh_degree + 1) ** 2
    sh = np.zeros((n_sites, 3 * K), dtype=np.float32)
    sh[:, 0:3] = _dc_from_color(rng.random((n_sites, 3)))
    if K > 1:
        sh[:, 3:] = rng.normal(0.0, higher_sigma, (n_sites, 3 * (K - 1)))
    offsets, neighbors = delaunay_csr(xyz)
    points = np.concatenate([xyz, density[:, None]], axis=1).astype(np.float32)
    return PointCloudModel(points, sh, sh_degree, offsets, neighbors)


def mixture_points(rng, n: int, half_extent: float = 1.0) -> np.ndarray:
    """3-component Gaussian mixture (sigma in [0.15, 0.4]), samples outside
    the cube [-half_extent, half_extent]^3 are redrawn."""
    means = rng.uniform(-0.4, 0.4, (3, 3))
    sigmas = rng.uniform(0.15, 0.4, 3)
    weights = rng.dirichlet(np.ones(3))
    out = np.empty((0, 3))
    while len(out) < n:
        need = n - len(out)
        comp = rng.choice(3, size=int(need * 1.3) + 16, p=weights)
        pts = means[comp] + rng.standard_normal((len(comp), 3)) * sigmas[comp, None]
        inside = np.all(np.abs(pts) <= half_extent, axis=1)
        out = np.concatenate([out, pts[inside]])
    return out[:n]


def powerfoam_mixture(n_sites: int, seed: int, sh_degree: int = 3, radius_max: float = 0.02,
                      bf16: bool = True) -> PointCloudModel:
    rng = np.random.default_rng(seed)
    xyz = mixture_points(rng, n_sites).astype(np.float32)
    radii = rng.uniform(0.0, radius_max, n_sites).astype(np.float32)
    density = rng.lognormal(0.5, 1.2, n_sites).astype(np.float32)
    K = (sh_degree + 1) ** 2
    sh = np.zeros((n_sites, 3 * K), dtype=np.float32)
    sh[:, 0:3] = _dc_from_color(rng.random((n_sites, 3)))
    if K > 1:
        sh[:, 3:] = rng.normal(0.0, 0.2, (n_sites, 3 * (K - 1)))
    if bf16:
        sh = round_to_bf16(sh)
    offsets, neighbors = cech_csr(xyz, radii)
    points = np.concatenate([xyz, density[:, None]], axis=1).astype(np.float32)
    return PointCloudModel(points, sh, sh_degree, offsets, neighbors, radii, bf16)


def round_to_bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 to the nearest BF16 (ties to even) and widen back."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    rounding = ((u >> 16) & 1) + np.uint32(0x7FFF)
    r = ((u + rounding) & np.uint32(0xFFFF0000)).astype(np.uint32)
    return r.view(np.float32)


def perturbed(model: PointCloudModel, seed: int, density_sigma: float = 0.1,
              sh_sigma: float = 0.05) -> PointCloudModel:
    """Target scene: densities x exp(N(0, 0.1)), SH + N(0, 0.05)."""
    rng = np.random.default_rng(seed)
    out = model.copy()
    out.points[:, 3] *= np.exp(rng.normal(0.0, density_sigma, model.n)).astype(np.float32)
    out.sh = (out.sh + rng.normal(0.0, sh_sigma, out.sh.shape)).astype(np.float32)
    if out.sh_bf16:
        out.sh = round_to_bf16(out.sh)
    return out


# --------------------------------------------------------------------------
# named workloads
# --------------------------------------------------------------------------
def radfoam_tiny(n_sites: int = 16384, width: int = 128, height: int = 128) -> Workload:
    """Plain RadFoam forward: unit ball + N(0, 0.01) jitter, density
    lognormal(0, 1), SH degree 0 colour U[0, 1], camera at (0, 0, 3) looking
    at the origin, fov_y 60 deg, depth 100; seed 0."""
    model = radfoam_ball(n_sites, seed=0, sh_degree=0, jitter=0.01)
    cam = looking_at((0.0, 0.0, 3.0), (0.0, 0.0, 0.0), math.radians(60.0), width / height, 100.0)
    return Workload("radfoam_tiny", model, [cam], width, height, 1024, 1e-3)


def radfoam_train(n_sites: int = 262144, views: int = 8, width: int = 512, height: int = 512,
                  seed: int = 0, with_targets: bool = True, target_renderer=None) -> Workload:
    """RadFoam forward+backward: 262,144 sites in the unit ball, density
    lognormal(0, 1), SH degree 3 (DC from U[0, 1], higher terms N(0, 0.2)),
    8 cameras on the radius-3 sphere (Fibonacci directions, seed 1) at
    512x512.  Targets are renders of the perturbed scene (seed 2)."""
    model = radfoam_ball(n_sites, seed=seed, sh_degree=3)
    cams = sphere_cameras(views, 3.0, 1, math.radians(60.0), width / height, 100.0)
    w = Workload("radfoam_train", model, cams, width, height, 1024, 0.0)
    if with_targets and target_renderer is not None:
        w.targets = target_renderer(perturbed(model, seed=2), cams, width, height)
    return w


def powerfoam_mix(n_sites: int = 1048576, views: int = 4, width: int = 1024, height: int = 1024,
                  seed: int = 0) -> Workload:
    """PowerFoam with BF16 SH: 3-component mixture, radii U[0, 0.02], density
    lognormal(0.5, 1.2), Cech adjacency, 4 cameras at 1024x1024."""
    model = powerfoam_mixture(n_sites, seed=seed)
    cams = sphere_cameras(views, 3.0, 1, math.radians(60.0), width / height, 100.0)
    return Workload("powerfoam_mixture", model, cams, width, height, 1024, 1e-3)


# --------------------------------------------------------------------------
# relightable Gaussians
# --------------------------------------------------------------------------
@dataclasses.dataclass
class GaussianModel:
    """Gaussian PointCloudModel with explicit PBR attributes (lib.rs:174-239,
    Transforms + PbrAttributes): mean + opacity, rotation (xyzw), scale,
    unit normal, material index, and the material table (relight.rs:77-86:
    albedo[3], roughness, specular_f0[3], pad)."""

    points: np.ndarray  # float32 [N, 4]
    rotations: np.ndarray  # float32 [N, 4]
    scales: np.ndarray  # float32 [N, 3]
    normals: np.ndarray  # float32 [N, 3]
    material_indices: np.ndarray  # uint32 [N]
    materials: np.ndarray  # float32 [M, 8]

    @property
    def n(self) -> int:
        return int(self.points.shape[0])


def quat_to_matrix(q: np.ndarray) -> np.ndarray:
    """Rotation matrices [N, 3, 3] of unit quaternions (x, y, z, w)."""
    x, y, z, w = (q[:, i].astype(np.float64) for i in range(4))
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


def make_material(albedo, roughness, f0=(0.04, 0.04, 0.04)) -> np.ndarray:
    return np.array([*albedo, roughness, *f0, 0.0], dtype=np.float32)


def relight_gaussians(n: int = 1_000_000, seed: int = 0) -> GaussianModel:
    """1M anisotropic Gaussians: means from the 3-component mixture,
    log-scales N(-4, 0.5), rotations normalised N(0, 1)^4, opacity
    sigmoid(N(0, 1)), albedo U[0, 1], GGX roughness U[0.2, 0.9], F0 0.04,
    normal = the rotation's column of the smallest scale."""
    rng = np.random.default_rng(seed)
    means = mixture_points(rng, n).astype(np.float32)
    scales = np.exp(rng.normal(-4.0, 0.5, (n, 3))).astype(np.float32)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    q = q.astype(np.float32)
    opacity = (1.0 / (1.0 + np.exp(-rng.standard_normal(n)))).astype(np.float32)
    albedo = rng.random((n, 3)).astype(np.float32)
    roughness = rng.uniform(0.2, 0.9, n).astype(np.float32)
    R = quat_to_matrix(q)
    smallest = np.argmin(scales, axis=1)
    normals = R[np.arange(n), :, smallest]
    normals /= np.linalg.norm(normals, axis=1, keepdims=True)
    materials = np.zeros((n, 8), np.float32)
    materials[:, 0:3] = albedo
    materials[:, 3] = roughness
    materials[:, 4:7] = 0.04
    points = np.concatenate([means, opacity[:, None]], axis=1).astype(np.float32)
    return GaussianModel(points, q, scales, normals.astype(np.float32),
                         np.arange(n, dtype=np.uint32), materials)


def sphere_lights(count: int = 16, radius: float = 2.0, intensity: float = 5.0, seed: int = 3):
    """Isotropic point lights on a sphere (Fibonacci directions), as
    PointLight fields (position, direction, intensity, exponent)."""
    rng = np.random.default_rng(seed)
    golden = math.pi * (3.0 - math.sqrt(5.0))
    a = rng.standard_normal((3, 3))
    qm, rm = np.linalg.qr(a)
    qm = qm * np.sign(np.diag(rm))
    out = []
    for i in range(count):
        y = 1.0 - 2.0 * (i + 0.5) / count
        r = math.sqrt(max(0.0, 1.0 - y * y))
        d = np.array([math.cos(golden * i) * r, y, math.sin(golden * i) * r]) @ qm.T
        out.append((tuple((radius * d).astype(np.float32)), (0.0, 0.0, 1.0),
                    (intensity, intensity, intensity), 0.0))
    return out


def relight_workload(n: int = 1_000_000, width: int = 1024, height: int = 768, seed: int = 0):
    g = relight_gaussians(n, seed)
    cam = sphere_cameras(1, 3.0, 1, math.radians(60.0), width / height, 100.0)[0]
    return g, cam, sphere_lights()


# --------------------------------------------------------------------------
# SH-coloured Gaussians (GaussianGpuCloud input)
# --------------------------------------------------------------------------
@dataclasses.dataclass
class GaussianShModel:
    """Gaussian PointCloudModel with Transforms and SH colour (lib.rs:174-239):
    mean + opacity, rotation (x, y, z, w), scale, SH rows [N, 3K]."""

    points: np.ndarray  # float32 [N, 4]
    rotations: np.ndarray  # float32 [N, 4]
    scales: np.ndarray  # float32 [N, 3]
    sh: np.ndarray  # float32 [N, 3K]
    sh_degree: int

    @property
    def n(self) -> int:
        return int(self.points.shape[0])


def gaussian_sh(n: int = 1_000_000, seed: int = 0, sh_degree: int = 3,
                log_scale_mean: float = -4.0) -> GaussianShModel:
    """Anisotropic Gaussians with the relight scene's geometry distribution
    (means from the 3-component mixture, log-scales N(log_scale_mean, 0.5),
    rotations normalised N(0, 1)^4, opacity sigmoid(N(0, 1))) and SH colour:
    DC from a uniform [0, 1] colour, higher coefficients N(0, 0.2)."""
    rng = np.random.default_rng(seed)
    means = mixture_points(rng, n).astype(np.float32)
    scales = np.exp(rng.normal(log_scale_mean, 0.5, (n, 3))).astype(np.float32)
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    opacity = (1.0 / (1.0 + np.exp(-rng.standard_normal(n)))).astype(np.float32)
    k = (sh_degree + 1) ** 2
    sh = rng.normal(0.0, 0.2, (n, 3 * k)).astype(np.float32)
    sh[:, 0:3] = _dc_from_color(rng.random((n, 3)))
    points = np.concatenate([means, opacity[:, None]], axis=1).astype(np.float32)
    return GaussianShModel(points, q.astype(np.float32), scales, sh, sh_degree)
