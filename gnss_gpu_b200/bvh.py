"""Building meshes and their bounding-volume hierarchy on the device.

`BuildingModel` holds a triangle mesh (ECEF, m); `BVHAccelerator` builds its
hierarchy in the library (pf_mesh_build: median splits, leaves of at most 4
triangles, stored in FP32 in an East/North/Up frame about the mesh's mean
vertex, each node holding the boxes of its two children) and keeps nodes
and triangles in device memory.  They mirror
python/gnss_gpu/raytrace.py BuildingModel and python/gnss_gpu/bvh.py
BVHAccelerator of the reference for the parts the 3D particle filters use:
construction from triangles or a Wavefront OBJ file and line-of-sight
queries (check_los, check_los_batch).  First-order multipath
(compute_multipath) belongs to the reference's ray-tracing subsystem and is
not built here.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class BuildingModel:
    """A triangle mesh: triangles (N, 3, 3) ECEF vertices in metres."""

    def __init__(self, triangles):
        tri = np.asarray(triangles, dtype=np.float64)
        if tri.ndim != 3 or tri.shape[1:] != (3, 3):
            raise ValueError("triangles must have shape [N, 3, 3]")
        self.triangles = np.ascontiguousarray(tri)

    @classmethod
    def create_box(cls, center, width, depth, height):
        """A closed axis-aligned box (12 triangles): width along x, depth
        along y, height along z, centred at `center`."""
        c = np.asarray(center, dtype=np.float64).reshape(3)
        h = np.array([width, depth, height], dtype=np.float64) / 2.0
        corner = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                           [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64) * h + c
        faces = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4),
                 (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6), (3, 0, 4), (3, 4, 7)]
        return cls(corner[np.asarray(faces)])

    @classmethod
    def from_obj(cls, filepath):
        """Vertices (v) and faces (f, fan-triangulated) of a Wavefront OBJ file."""
        verts, faces = [], []
        with open(filepath) as fh:
            for line in fh:
                parts = line.split()
                if not parts:
                    continue
                if parts[0] == "v":
                    verts.append([float(v) for v in parts[1:4]])
                elif parts[0] == "f":
                    idx = [int(p.split("/")[0]) for p in parts[1:]]
                    idx = [i - 1 if i > 0 else len(verts) + i for i in idx]
                    for k in range(1, len(idx) - 1):
                        faces.append((idx[0], idx[k], idx[k + 1]))
        v = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
        return cls(v[np.asarray(faces, dtype=np.int64).reshape(-1, 3)] if faces else np.zeros((0, 3, 3)))


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("CUDA is not available: the B200 ray tracer has no CPU path")
    return torch


class BVHAccelerator:
    """The hierarchy of a triangle mesh in device memory."""

    def __init__(self, triangles, device=None):
        tri = np.ascontiguousarray(np.asarray(triangles, dtype=np.float64))
        if tri.ndim != 3 or tri.shape[1:] != (3, 3):
            raise ValueError("triangles must have shape [N, 3, 3]")
        lib = N.load()
        torch = _torch()
        n = len(tri)
        nodes = np.zeros((max(1, n), 16), np.float32)
        tris = np.zeros((max(1, n), 12), np.float32)
        n_nodes = C.c_int(0)
        origin = np.zeros(3)
        rot = np.zeros(9)
        N.check(lib.pf_mesh_build(N.dptr(tri.reshape(-1)), n, N.vptr(nodes), N.vptr(tris), C.byref(n_nodes),
                                  N.dptr(origin), N.dptr(rot)))
        self.triangles = tri
        self.origin = origin
        self.rot = rot.reshape(3, 3)
        self._n_nodes = int(n_nodes.value)
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        self._nodes = torch.from_numpy(nodes[: max(1, self._n_nodes)].copy()).to(dev)
        self._tris = torch.from_numpy(tris.copy()).to(dev)
        torch.cuda.synchronize(dev)
        m = N.Mesh()
        m.nodes = C.c_void_p(self._nodes.data_ptr())
        m.tris = C.c_void_p(self._tris.data_ptr())
        m.n_nodes = self._n_nodes
        m.n_tris = n
        for i in range(3):
            m.origin[i] = origin[i]
        for i in range(9):
            m.rot[i] = rot[i]
        self.mesh = m
        self.device = dev

    @property
    def n_nodes(self):
        return self._n_nodes

    @property
    def n_triangles(self):
        return len(self.triangles)

    @classmethod
    def from_building_model(cls, building_model):
        return cls(building_model.triangles)

    @classmethod
    def from_obj(cls, filepath):
        return cls(BuildingModel.from_obj(filepath).triangles)

    def check_los_batch(self, rx_ecef, sat_ecef):
        """(N, n_sat) bool: True where receiver N sees satellite (N, s).
        Non-finite entries give False."""
        torch = _torch()
        rx = np.ascontiguousarray(np.asarray(rx_ecef, dtype=np.float64))
        sat = np.ascontiguousarray(np.asarray(sat_ecef, dtype=np.float64))
        if rx.ndim != 2 or rx.shape[1] != 3:
            raise ValueError("rx_ecef must have shape (N, 3)")
        if sat.ndim != 3 or sat.shape[2] != 3:
            raise ValueError("sat_ecef must have shape (N, n_sat, 3)")
        if rx.shape[0] != sat.shape[0]:
            raise ValueError("rx_ecef and sat_ecef must share the leading N")
        d_rx = torch.from_numpy(rx.reshape(-1)).to(self.device)
        d_sat = torch.from_numpy(sat.reshape(-1)).to(self.device)
        out = torch.zeros(rx.shape[0] * sat.shape[1], dtype=torch.uint8, device=self.device)
        stream = torch.cuda.current_stream(self.device)
        N.check(N.load().pf_mesh_los(C.byref(self.mesh), C.c_void_p(d_rx.data_ptr()), C.c_void_p(d_sat.data_ptr()),
                                     rx.shape[0], sat.shape[1], C.c_void_p(out.data_ptr()),
                                     C.c_void_p(stream.cuda_stream)))
        return out.cpu().numpy().reshape(rx.shape[0], sat.shape[1]).astype(bool)

    def check_los(self, rx_ecef, sat_ecef):
        """(n_sat,) bool: True where the receiver sees the satellite."""
        rx = np.asarray(rx_ecef, dtype=np.float64).reshape(1, 3)
        sat = np.asarray(sat_ecef, dtype=np.float64).reshape(1, -1, 3)
        return self.check_los_batch(rx, sat)[0]

    def compute_multipath(self, *a, **k):
        raise NotImplementedError("first-order multipath reflections are not built")

    compute_multipath_batch = compute_multipath
