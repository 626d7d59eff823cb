"""Minimal stand-in for the parts of ``open3d`` that the reference's
``src/initialization.py`` touches (mesh IO, surface area, debug geometry
objects).  Test infrastructure only: it lets the reference source be imported
unmodified by ``make_golden.py``.
"""
from __future__ import annotations

import types

import numpy as np


def read_ply_mesh(path):
    """Binary little-endian PLY with double/float xyz vertices and
    ``list uchar uint`` (or int) faces, as written by Open3D."""
    with open(path, "rb") as fh:
        header = []
        while True:
            line = fh.readline().decode("ascii").strip()
            header.append(line)
            if line == "end_header":
                break
        body = fh.read()
    n_v = n_f = 0
    vprops, fidx = [], None
    section = None
    for line in header:
        t = line.split()
        if t[:2] == ["element", "vertex"]:
            n_v, section = int(t[2]), "v"
        elif t[:2] == ["element", "face"]:
            n_f, section = int(t[2]), "f"
        elif t and t[0] == "property" and section == "v":
            vprops.append(({"double": "<f8", "float": "<f4"}[t[1]], t[2]))
        elif t and t[0] == "property" and section == "f":
            fidx = {"uint": "<u4", "int": "<i4"}[t[3]]
    vdt = np.dtype([(name, typ) for typ, name in vprops])
    verts = np.frombuffer(body, dtype=vdt, count=n_v)
    xyz = np.stack([verts["x"], verts["y"], verts["z"]], axis=1).astype(np.float64)
    off = vdt.itemsize * n_v
    fdt = np.dtype([("n", "u1"), ("idx", fidx, (3,))])
    faces = np.frombuffer(body, dtype=fdt, count=n_f, offset=off)
    return xyz, faces["idx"].astype(np.int64)


class TriangleMesh:
    def __init__(self, vertices=None, triangles=None):
        self.vertices = np.zeros((0, 3)) if vertices is None else vertices
        self.triangles = np.zeros((0, 3), dtype=np.int64) if triangles is None else triangles

    def get_surface_area(self):
        v = np.asarray(self.vertices, dtype=np.float64)
        t = np.asarray(self.triangles)
        a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
        return float(0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum())

    def compute_vertex_normals(self):
        return self

    def paint_uniform_color(self, _c):
        return self


class _Geom:
    def __init__(self, **kw):
        self.__dict__.update(kw)

    def paint_uniform_color(self, _c):
        return self


def _read_triangle_mesh(path):
    v, t = read_ply_mesh(path)
    return TriangleMesh(v, t)


io = types.SimpleNamespace(read_triangle_mesh=_read_triangle_mesh,
                           write_triangle_mesh=lambda *a, **k: True)
utility = types.SimpleNamespace(
    Vector3dVector=lambda a: np.asarray(a, dtype=np.float64),
    Vector2iVector=lambda a: np.asarray(a, dtype=np.int64),
    Vector3iVector=lambda a: np.asarray(a, dtype=np.int64),
)
geometry = types.SimpleNamespace(
    TriangleMesh=TriangleMesh,
    LineSet=lambda **kw: _Geom(**kw),
    PointCloud=lambda: _Geom(points=None),
)
