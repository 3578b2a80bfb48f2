"""CPU tests of the mesh hierarchy builder (pf_mesh_build, host code of
the library): a valid tree over every triangle, boxes that hold their
contents, bounded depth; and the brute-force line-of-sight oracle."""
import ctypes as C

import numpy as np

from gnss_gpu_b200 import _native as N
from gnss_gpu_b200 import citysim as CS
from gnss_gpu_b200 import scenario as S
from gnss_gpu_b200.bvh import BuildingModel
from oracle import oracle as O


def _build(tri):
    L = N.load()
    n = len(tri)
    nodes = np.zeros((max(1, n), 16), np.float32)
    tris = np.zeros((max(1, n), 12), np.float32)
    nn = C.c_int(0)
    origin, rot = np.zeros(3), np.zeros(9)
    N.check(L.pf_mesh_build(N.dptr(np.ascontiguousarray(tri, np.float64).reshape(-1)), n, N.vptr(nodes), N.vptr(tris),
                            C.byref(nn), N.dptr(origin), N.dptr(rot)))
    return nodes[: nn.value], tris[:n], origin, rot.reshape(3, 3)


def city_mesh(seed=1, size=600.0):
    city = CS.make_city(seed, size=size)
    rot = S.enu_rotation_lla(35.63, 139.78)
    anchor = S.lla_to_ecef(35.63, 139.78, 40.0)
    return CS.city_triangles(city, anchor, rot), anchor, rot, city


def test_hierarchy_is_valid():
    """Every triangle in exactly one leaf; every child box holds the child's
    contents; a tree rooted at node 0 reaching every node; bounded depth."""
    tri, _, _, _ = city_mesh()
    nodes, tris, origin, rot = _build(tri)
    n = len(tri)
    assert 0 < len(nodes) <= n
    covered = np.zeros(n, int)
    seen = np.zeros(len(nodes), int)
    depth_max = 0
    stack = [(0, 0)]
    while stack:
        k, dep = stack.pop()
        seen[k] += 1
        depth_max = max(depth_max, dep)
        for off in (0, 8):
            lo, hi = nodes[k, off:off + 3], nodes[k, off + 4:off + 7]
            ref = nodes[k, 3 if off == 0 else 7].view(np.int32)
            if ref >= 0:
                for o2 in (0, 8):
                    assert np.all(nodes[ref, o2:o2 + 3] >= lo) and np.all(nodes[ref, o2 + 4:o2 + 7] <= hi)
                stack.append((int(ref), dep + 1))
            else:
                code = ~int(ref)
                s, c = code >> 3, (code & 7) + 1
                assert 1 <= c <= 4
                covered[s:s + c] += 1
                v0 = tris[s:s + c, 0:3]
                for v in (v0, v0 + tris[s:s + c, 4:7], v0 + tris[s:s + c, 8:11]):
                    assert np.all(v >= lo - 1e-3) and np.all(v <= hi + 1e-3)
    assert np.all(covered == 1)
    assert np.all(seen == 1)
    assert depth_max < 64  # the traversal stack: surface-area splits to depth 32, median splits below
    # the stored triangles are the input, in the mesh frame
    back = origin + (tris[:, 0:3].astype(np.float64)) @ rot
    assert np.allclose(np.sort(back[:, 0]), np.sort(tri[:, 0, 0]), atol=1e-2)


def test_empty_and_single_triangle_meshes():
    nodes, tris, _, _ = _build(np.zeros((0, 3, 3)))
    assert len(nodes) == 0
    nodes, tris, _, _ = _build(BuildingModel.create_box([0, 0, 0], 2, 2, 2).triangles[:1])
    # one leaf: a root with the leaf (triangle 0, count 1) on the left and a far point box on the right
    assert len(nodes) == 1 and ~int(nodes[0, 3].view(np.int32)) == 0
    assert np.all(nodes[0, 8:11] == 1e30) and np.all(nodes[0, 12:15] == 1e30)


def test_box_and_los_oracle():
    box = BuildingModel.create_box(center=[100.0, 0.0, 25.0], width=20.0, depth=20.0, height=50.0)
    assert box.triangles.shape == (12, 3, 3)
    los = O.los([[0.0, 0.0, 0.0]], [[[0.0, 0.0, 20000.0], [200.0, 0.0, 25.0], [150.0, 0.0, 10.0],
                                     [-200.0, 0.0, 5000.0], [105.0, 0.0, 25.0]]], box.triangles)
    assert los.tolist() == [[True, False, False, True, False]]
