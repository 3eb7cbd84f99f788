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
"""

from __future__ import annotations

import io
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from .scenes import SH_C0, PointCloudModel

MAX_HEADER_BYTES = 1024 * 1024
_TYPES = {"float": "<f4", "float32": "<f4", "uint": "<u4", "uint32": "<u4", "uchar": "u1",
          "uint8": "u1"}
# properties of the reference format that this path does not render
_UNSUPPORTED_PREFIXES = ("nx", "ny", "nz", "surface_offset", "blade_surface_detail_",
                         "blade_surface_color_", "blade_spherical_voronoi_")


class PlyError(ValueError):
    pass


def _read_header(f) -> Tuple[str, List[Tuple[str, int, List[Tuple[str, str]]]]]:
    """(format, [(element, count, [(property, dtype)])]) (radfoam_ply.rs:452-596)."""
    fmt = None
    elements: List[Tuple[str, int, List[Tuple[str, str]]]] = []
    nbytes = 0
    first = True
    saw_end = False
    while True:
        line = f.readline()
        if not line:
            break
        nbytes += len(line)
        if nbytes > MAX_HEADER_BYTES:
            raise PlyError(f"RadFoam PLY header exceeds {MAX_HEADER_BYTES} bytes")
        words = line.decode("ascii", errors="replace").split()
        if first:
            if words != ["ply"]:
                raise PlyError("RadFoam PLY is missing the 'ply' magic")
            first = False
            continue
        if not words:
            continue
        head = words[0]
        if head == "format":
            if fmt is not None:
                raise PlyError("duplicate RadFoam PLY format line")
            if len(words) < 3 or words[2] != "1.0":
                raise PlyError(f"unsupported RadFoam PLY version '{' '.join(words[2:])}'")
            if words[1] not in ("binary_little_endian", "ascii"):
                raise PlyError(f"unsupported RadFoam PLY format '{words[1]}'")
            fmt = words[1]
        elif head in ("comment", "obj_info"):
            continue
        elif head == "element":
            if len(words) < 3:
                raise PlyError("RadFoam PLY element needs a name and a count")
            if any(e[0] == words[1] for e in elements):
                raise PlyError(f"duplicate RadFoam PLY element '{words[1]}'")
            try:
                count = int(words[2])
            except ValueError:
                raise PlyError(f"invalid count for element '{words[1]}'") from None
            elements.append((words[1], count, []))
        elif head == "property":
            if not elements:
                raise PlyError("RadFoam PLY property appears before an element")
            if len(words) > 1 and words[1] == "list":
                raise PlyError(f"RadFoam PLY list properties are unsupported in element "
                               f"'{elements[-1][0]}'")
            if len(words) < 3 or words[1] not in _TYPES:
                raise PlyError(f"unsupported RadFoam PLY scalar type "
                               f"'{words[1] if len(words) > 1 else ''}'")
            props = elements[-1][2]
            if any(p[0] == words[2] for p in props):
                raise PlyError(f"duplicate RadFoam PLY property '{elements[-1][0]}.{words[2]}'")
            props.append((words[2], _TYPES[words[1]]))
        elif head == "end_header":
            saw_end = True
            break
        else:
            raise PlyError(f"unexpected RadFoam PLY header token '{head}'")
    if first:
        raise PlyError("RadFoam PLY is missing the 'ply' magic")
    if not saw_end:
        raise PlyError("RadFoam PLY header has no end_header")
    if fmt is None:
        raise PlyError("RadFoam PLY has no format line")
    return fmt, elements


def _schema(elements) -> Dict[str, object]:
    """Property roles of the walk subset (radfoam_ply.rs:122-372)."""
    if len(elements) != 2 or elements[0][0] != "vertex" or elements[1][0] != "adjacency":
        raise PlyError("RadFoam PLY elements must be exactly 'vertex' followed by 'adjacency'")
    vprops = dict(elements[0][2])
    aprops = dict(elements[1][2])
    for name, want in (("x", "<f4"), ("y", "<f4"), ("z", "<f4"), ("density", "<f4"),
                       ("adjacency_offset", "<u4")):
        if name not in vprops:
            raise PlyError(f"RadFoam PLY element 'vertex' is missing property '{name}'")
        if vprops[name] != want:
            raise PlyError(f"RadFoam PLY property 'vertex.{name}' has the wrong type")
    if aprops.get("adjacency") != "<u4" or len(aprops) != 1:
        raise PlyError("RadFoam PLY adjacency element must hold one uint 'adjacency'")
    for name in vprops:
        if name.startswith(_UNSUPPORTED_PREFIXES):
            raise PlyError(f"RadFoam PLY property '{name}' (oriented-surface / detail terms) is "
                           "not supported on this path")
    exact = [f"blade_sh_dc_{i}" for i in range(3)]
    preview = ["red", "green", "blue"]
    has_exact = all(n in vprops for n in exact)
    has_preview = all(n in vprops for n in preview)
    if any(n in vprops for n in exact) and not has_exact:
        raise PlyError("RadFoam PLY needs all of blade_sh_dc_0..2")
    if not has_exact and not has_preview:
        raise PlyError("RadFoam PLY vertex needs exact blade_sh_dc_0..2 or red/green/blue "
                       "preview DC")
    if has_exact and any(vprops[n] != "<f4" for n in exact):
        raise PlyError("RadFoam PLY blade_sh_dc_* must be float32")
    if not has_exact and any(vprops[n] != "u1" for n in preview):
        raise PlyError("RadFoam PLY preview colours must be uchar")
    rest = []
    for name, ty in vprops.items():
        if name.startswith("color_sh_"):
            if ty != "<f4":
                raise PlyError(f"RadFoam PLY property '{name}' must be float32")
            try:
                rest.append(int(name[len("color_sh_"):]))
            except ValueError:
                raise PlyError(f"invalid RadFoam PLY property '{name}'") from None
    rest.sort()
    if rest != list(range(len(rest))):
        raise PlyError("RadFoam PLY color_sh indices must be contiguous")
    if len(rest) % 3:
        raise PlyError(f"RadFoam PLY color_sh property count {len(rest)} is not divisible by three")
    comps = len(rest) // 3 + 1
    degree = {1: 0, 4: 1, 9: 2, 16: 3}.get(comps)
    if degree is None:
        raise PlyError(f"RadFoam PLY has {comps} SH components, expected a complete degree up "
                       "to 3")
    if "radius" in vprops and vprops["radius"] != "<f4":
        raise PlyError("RadFoam PLY vertex radius must be float32")
    return dict(exact=has_exact, rest=len(rest), degree=degree, radius="radius" in vprops)


def load_radfoam_ply(path: str) -> PointCloudModel:
    """try_load (radfoam_ply.rs:1141-1213), walk subset."""
    with open(path, "rb") as f:
        fmt, elements = _read_header(f)
        sch = _schema(elements)
        body_start = f.tell()
        body = f.read()
    (_, n, vlist), (_, m, alist) = elements
    vdt = np.dtype([(name, ty) for name, ty in vlist])
    if fmt == "binary_little_endian":
        expected = n * vdt.itemsize + m * 4
        if len(body) != expected:
            raise PlyError(f"RadFoam PLY binary body is {len(body)} bytes, expected {expected}")
        verts = np.frombuffer(body, dtype=vdt, count=n)
        adj = np.frombuffer(body, dtype="<u4", count=m, offset=n * vdt.itemsize).astype(np.uint32)
    else:
        rows = [ln for ln in body.decode("ascii", errors="replace").splitlines()
                if ln.strip() and not ln.strip().startswith("comment")]
        if len(rows) < n + m:
            raise PlyError("RadFoam PLY ASCII body is truncated")
        verts = np.zeros(n, dtype=vdt)
        for i in range(n):
            tok = rows[i].split()
            if len(tok) != len(vlist):
                raise PlyError(f"RadFoam PLY vertex row {i} has {len(tok)} values, expected "
                               f"{len(vlist)}")
            for (name, ty), t in zip(vlist, tok):
                try:
                    verts[i][name] = float(t) if ty == "<f4" else int(t)
                except (ValueError, OverflowError):
                    raise PlyError(f"invalid RadFoam PLY value for '{name}'") from None
        try:
            adj = np.array([int(rows[n + k].split()[0]) for k in range(m)], dtype=np.uint32)
        except (ValueError, OverflowError, IndexError):
            raise PlyError("invalid RadFoam PLY adjacency row") from None
    offsets = np.zeros(n + 1, np.uint32)
    offsets[1:] = verts["adjacency_offset"]
    # validate_csr (radfoam_ply.rs:1111-1139)
    if n and (offsets[n] != m or np.any(offsets[1:] < offsets[:-1])):
        raise PlyError("invalid RadFoam PLY CSR offsets")
    if m and int(adj.max()) >= n:
        raise PlyError("RadFoam PLY adjacency references a missing point")
    K = (sch["degree"] + 1) ** 2
    sh = np.zeros((n, 3 * K), np.float32)
    if sch["exact"]:
        for c in range(3):
            sh[:, c] = verts[f"blade_sh_dc_{c}"]
    else:
        for c, name in enumerate(("red", "green", "blue")):
            sh[:, c] = ((verts[name].astype(np.float32) / np.float32(255.0) - np.float32(0.5))
                        / np.float32(SH_C0))
    for k in range(sch["rest"]):
        sh[:, 3 + k] = verts[f"color_sh_{k}"]
    points = np.stack([verts["x"], verts["y"], verts["z"], verts["density"]],
                      axis=1).astype(np.float32)
    radii = np.ascontiguousarray(verts["radius"], np.float32) if sch["radius"] else None
    return PointCloudModel(points, sh, sch["degree"], offsets, adj.astype(np.uint32), radii)


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
