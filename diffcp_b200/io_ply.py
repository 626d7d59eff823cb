"""Minimal binary/ASCII PLY triangle-mesh reader and binary writer (NumPy only),
replacing the Open3D mesh IO of initialization.py:104 and
simulation_without_grad.py:512-520."""
from __future__ import annotations

import numpy as np

_TYPES = {"char": "i1", "uchar": "u1", "short": "i2", "ushort": "u2", "int": "i4", "uint": "u4", "float": "f4",
          "double": "f8", "int8": "i1", "uint8": "u1", "int16": "i2", "uint16": "u2", "int32": "i4",
          "uint32": "u4", "float32": "f4", "float64": "f8"}


def read_ply(path):
    """Returns (vertices (N,3) float64, triangles (M,3) int64)."""
    with open(path, "rb") as fh:
        header = []
        while True:
            line = fh.readline()
            if not line:
                raise ValueError("truncated PLY header")
            line = line.decode("ascii").strip()
            header.append(line)
            if line == "end_header":
                break
        body = fh.read()
    fmt = None
    elements = []
    for line in header:
        t = line.split()
        if not t:
            continue
        if t[0] == "format":
            fmt = t[1]
        elif t[0] == "element":
            elements.append([t[1], int(t[2]), []])
        elif t[0] == "property":
            elements[-1][2].append(t[1:])
    if fmt == "ascii":
        return _read_ascii(body.decode("ascii").split(), elements)
    end = "<" if fmt == "binary_little_endian" else ">"
    off = 0
    verts = tris = None
    for name, count, props in elements:
        if name == "vertex":
            dt = np.dtype([(p[1], end + _TYPES[p[0]]) for p in props])
            arr = np.frombuffer(body, dtype=dt, count=count, offset=off)
            off += dt.itemsize * count
            verts = np.stack([arr["x"], arr["y"], arr["z"]], 1).astype(np.float64)
        elif name == "face":
            lst = props[0]
            cnt_t, idx_t = end + _TYPES[lst[1]], end + _TYPES[lst[2]]
            dt = np.dtype([("n", cnt_t), ("idx", idx_t, (3,))])
            arr = np.frombuffer(body, dtype=dt, count=count, offset=off)
            if np.any(arr["n"] != 3):
                raise ValueError("only triangle faces are supported")
            off += dt.itemsize * count
            tris = arr["idx"].astype(np.int64)
        else:
            raise ValueError("unsupported PLY element %s" % name)
    return verts, tris


def _read_ascii(tok, elements):
    pos = 0
    verts = tris = None
    for name, count, props in elements:
        if name == "vertex":
            n = len(props)
            vals = np.array(tok[pos:pos + n * count], dtype=np.float64).reshape(count, n)
            pos += n * count
            names = [p[1] for p in props]
            verts = vals[:, [names.index("x"), names.index("y"), names.index("z")]]
        elif name == "face":
            out = np.zeros((count, 3), dtype=np.int64)
            for i in range(count):
                k = int(tok[pos])
                out[i] = [int(x) for x in tok[pos + 1:pos + 1 + k]]
                pos += 1 + k
            tris = out
    return verts, tris


def vertex_normals(vertices, triangles):
    """Unit vertex normals: the sum of the adjacent triangles' cross-product
    (area-weighted) normals, normalised."""
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(triangles, dtype=np.int64)
    fn = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    n = np.zeros_like(v)
    for k in range(3):
        np.add.at(n, t[:, k], fn)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    return np.divide(n, ln, out=np.zeros_like(n), where=ln > 0)


def write_ply(path, vertices, triangles, normals=None, colors=None):
    """Binary little-endian PLY: double x, y, z [+ double nx, ny, nz]
    [+ uchar red, green, blue] per vertex, ``list uchar uint`` faces -- the
    layout Open3D's write_triangle_mesh produces for the reference's pose
    meshes (simulation_without_grad.py:512-520).  ``colors``: (3,) or (N, 3)
    in [0, 1]."""
    v = np.asarray(vertices, dtype="<f8")
    t = np.asarray(triangles, dtype="<u4")
    fields = [("x", "<f8"), ("y", "<f8"), ("z", "<f8")]
    props = "property double x\nproperty double y\nproperty double z\n"
    if normals is not None:
        fields += [("nx", "<f8"), ("ny", "<f8"), ("nz", "<f8")]
        props += "property double nx\nproperty double ny\nproperty double nz\n"
    if colors is not None:
        fields += [("red", "u1"), ("green", "u1"), ("blue", "u1")]
        props += "property uchar red\nproperty uchar green\nproperty uchar blue\n"
    rows = np.zeros(len(v), dtype=fields)
    rows["x"], rows["y"], rows["z"] = v[:, 0], v[:, 1], v[:, 2]
    if normals is not None:
        nrm = np.asarray(normals, dtype=np.float64)
        rows["nx"], rows["ny"], rows["nz"] = nrm[:, 0], nrm[:, 1], nrm[:, 2]
    if colors is not None:
        col = np.broadcast_to(np.clip(np.rint(np.asarray(colors, dtype=np.float64) * 255.0), 0, 255), (len(v), 3))
        rows["red"], rows["green"], rows["blue"] = col[:, 0], col[:, 1], col[:, 2]
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\n%selement face %d\n"
            "property list uchar uint vertex_indices\nend_header\n" % (len(v), props, len(t)))
    rec = np.zeros(len(t), dtype=[("n", "u1"), ("idx", "<u4", (3,))])
    rec["n"] = 3
    rec["idx"] = t
    with open(path, "wb") as fh:
        fh.write(head.encode("ascii"))
        fh.write(rows.tobytes())
        fh.write(rec.tobytes())
