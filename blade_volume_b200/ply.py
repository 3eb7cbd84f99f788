"""RadFoam / PowerFoam PLY reader and writer (the walk subset of the
reference's loader, blade-volume/src/io/radfoam_ply.rs).

File layout (radfoam_ply.rs:1-7, :122-260): PLY 1.0, binary little-endian
or ASCII, exactly two elements, `vertex` then `adjacency`.  A vertex row
carries x, y, z and density (float), `adjacency_offset` (uint, the CSR end
offset of that point), the DC colour either exactly as `blade_sh_dc_0..2`
(float) or as a preview `red/green/blue` (uchar, DC = (c/255 - 0.5) /
0.2820948, :722-726), the higher SH coefficients `color_sh_<k>` (float,
contiguous k, coefficient 3 + k of the model's [component][rgb] row; their
count fixes the SH degree, :435-450), and optionally `radius` (float,
PowerFoam).  The adjacency element holds one uint `adjacency` per CSR entry.

The reference also reads oriented-surface, surface-detail, surface-colour
and spherical-Voronoi properties; the hot path here has no such terms, so a
file carrying them is rejected with PlyError rather than rendered without
them.  Validation follows the reference's order: header, schema, body size,
CSR ranges (:1111-1139); PointCloudModel::validate's stricter checks run when
a tracer is built from the model.

Reading goes through the library's C ABI (bv_radfoam_ply_info /
bv_radfoam_ply_read, csrc/bv_ply.cu), so Python and a host in the
reference's language share one reader; writing stays here.
"""

from __future__ import annotations

import io
import os
from typing import Optional

import numpy as np

from .scenes import PointCloudModel


class PlyError(ValueError):
    pass


def load_radfoam_ply(path: str) -> PointCloudModel:
    """try_load (radfoam_ply.rs:1141-1213), walk subset, through the C ABI's
    bv_radfoam_ply_info / bv_radfoam_ply_read (the same reader a host in the
    reference's language binds); raises PlyError with the reader's message."""
    import ctypes as C

    from . import BV_OK, PlyInfo, load_library

    L = load_library()
    p = os.fsencode(path)
    info = PlyInfo()
    if L.bv_radfoam_ply_info(p, C.byref(info)) != BV_OK:
        raise PlyError(L.bv_last_error().decode())
    n, m = info.num_points, info.num_adjacency
    K = (info.sh_degree + 1) ** 2
    points = np.zeros((n, 4), np.float32)
    sh = np.zeros((n, 3 * K), np.float32)
    offsets = np.zeros(n + 1, np.uint32)
    neighbors = np.zeros(m, np.uint32)
    radii = np.zeros(n, np.float32) if info.has_radii else None
    ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    if L.bv_radfoam_ply_read(p, ptr(points), ptr(sh), ptr(offsets), ptr(neighbors),
                             ptr(radii)) != BV_OK:
        raise PlyError(L.bv_last_error().decode())
    return PointCloudModel(points, sh, info.sh_degree, offsets, neighbors, radii)


def save_radfoam_ply(model: PointCloudModel, path: str, binary: bool = True,
                     comment: Optional[str] = None) -> None:
    """Writes a model in the layout load_radfoam_ply (and the reference's
    try_load) reads, with exact DC coefficients."""
    n = model.n
    K = model.sh_components
    names = ["x", "y", "z", "density", "adjacency_offset", "blade_sh_dc_0", "blade_sh_dc_1",
             "blade_sh_dc_2"] + [f"color_sh_{k}" for k in range(3 * (K - 1))]
    types = ["<f4"] * 4 + ["<u4"] + ["<f4"] * (3 + 3 * (K - 1))
    if model.radii is not None:
        names.append("radius")
        types.append("<f4")
    vdt = np.dtype(list(zip(names, types)))
    verts = np.zeros(n, dtype=vdt)
    for c, name in enumerate(("x", "y", "z", "density")):
        verts[name] = model.points[:, c]
    verts["adjacency_offset"] = np.asarray(model.offsets[1:], np.uint32)
    sh = np.asarray(model.sh, np.float32).reshape(n, 3 * K)
    for c in range(3):
        verts[f"blade_sh_dc_{c}"] = sh[:, c]
    for k in range(3 * (K - 1)):
        verts[f"color_sh_{k}"] = sh[:, 3 + k]
    if model.radii is not None:
        verts["radius"] = model.radii
    adj = np.asarray(model.neighbors, np.uint32)
    ply_types = {"<f4": "float", "<u4": "uint"}
    hdr = io.StringIO()
    hdr.write("ply\n")
    hdr.write(f"format {'binary_little_endian' if binary else 'ascii'} 1.0\n")
    if comment:
        hdr.write(f"comment {comment}\n")
    hdr.write(f"element vertex {n}\n")
    for name, ty in zip(names, types):
        hdr.write(f"property {ply_types[ty]} {name}\n")
    hdr.write(f"element adjacency {len(adj)}\n")
    hdr.write("property uint adjacency\nend_header\n")
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(hdr.getvalue().encode("ascii"))
        if binary:
            f.write(verts.tobytes())
            f.write(adj.astype("<u4").tobytes())
        else:
            for row in verts:
                f.write((" ".join(repr(float(v)) if t == "<f4" else str(int(v))
                                  for v, t in zip(row, types)) + "\n").encode("ascii"))
            for a in adj:
                f.write(f"{int(a)}\n".encode("ascii"))
    os.replace(tmp, path)
