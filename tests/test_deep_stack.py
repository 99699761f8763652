"""The traversal stack beyond its shared-memory part and at Photon's 64-entry limit.

A hand-made BVH: a spine of 79 interior nodes, each with the next spine node (nearer) and a side
node R_k (farther) as children, so the walk descends the spine pushing R_0, R_1, ... ; pushes past
64 entries are dropped, as Photon's traversal does (traverse.h). Each R_k holds two triangles at
depth 300 - 2k; at most levels both are tiny corner triangles the rays miss, at levels 5, 30 and 50
one covers the view, and at level 70 too — but R_70 was dropped, so the nearest hit the walk can
find is level 50's (stack entry 50, past the 24 entries kept in shared memory). Photon's own
traversal (oracle/_ref) on the same tree must give the same hits bit for bit, and they must be
level 50's triangle."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from photon_b200 import abi, native, workloads
import scenes

LEVELS = 80
HIT_LEVELS = (5, 30, 50, 70)


def _tri(v0, v1, v2, material=0):
    t = abi.TriGeom()
    t.v0 = abi.Vec3(*v0)
    t.e1 = abi.Vec3(*(np.subtract(v1, v0)))
    t.e2 = abi.Vec3(*(np.subtract(v2, v0)))
    t.material = material
    t.flags = 0
    return t, np.minimum(np.minimum(v0, v1), v2), np.maximum(np.maximum(v0, v1), v2)


def _deep_scene():
    box_desc, _, keep = scenes.scene("box")
    tris, boxes = [], []
    for k in range(LEVELS):
        z = 300.0 - 2.0 * k
        if k in HIT_LEVELS:
            a = _tri((-100.0, -100.0, z), (300.0, -100.0, z), (-100.0, 300.0, z))
        else:
            a = _tri((-100.0, -100.0, z), (-99.0, -100.0, z), (-100.0, -99.0, z))
        b = _tri((100.0, 100.0, z + 1.0), (99.0, 100.0, z + 1.0), (100.0, 99.0, z + 1.0))
        tris += [a[0], b[0]]
        boxes.append(((a[1], a[2]), (b[1], b[2])))
    # Node order: spine S_0..S_{L-2} (indices 0..L-2), then R_{L-1}..R_0 (children after parents).
    n_spine = LEVELS - 1
    r_index = {k: n_spine + (LEVELS - 1 - k) for k in range(LEVELS)}
    nodes = (abi.BvhNode * (n_spine + LEVELS))()

    def union(p, q):
        return np.minimum(p[0], q[0]), np.maximum(p[1], q[1])

    r_box = {}
    for k in range(LEVELS):
        (la, lb) = boxes[k]
        n = nodes[r_index[k]]
        n.lmin, n.lmax, n.left, n.lcount = abi.Vec3(*la[0]), abi.Vec3(*la[1]), 2 * k, 1
        n.rmin, n.rmax, n.right, n.rcount = abi.Vec3(*lb[0]), abi.Vec3(*lb[1]), 2 * k + 1, 1
        r_box[k] = union(la, lb)
    below = r_box[LEVELS - 1]  # what S_{L-2}'s near child holds
    for k in range(n_spine - 1, -1, -1):
        near_idx = k + 1 if k + 1 < n_spine else r_index[LEVELS - 1]
        n = nodes[k]
        n.lmin, n.lmax, n.left, n.lcount = abi.Vec3(*below[0]), abi.Vec3(*below[1]), near_idx, 0
        n.rmin, n.rmax, n.right, n.rcount = abi.Vec3(*r_box[k][0]), abi.Vec3(*r_box[k][1]), r_index[k], 0
        below = union(below, r_box[k])
    tri_arr = (abi.TriGeom * len(tris))(*tris)
    idx = np.zeros(3 * len(tris), np.int32)
    d = abi.SceneDesc.from_buffer_copy(box_desc)
    d.nodes, d.num_nodes = nodes, len(nodes)
    d.tris, d.num_tris = tri_arr, len(tris)
    d.indices = idx.ctypes.data_as(C.POINTER(C.c_int32))
    d.emissive, d.num_emissive, d.tri_emissive, d.emissive_alias = None, 0, None, None
    d.bounds_min, d.bounds_max = abi.Vec3(*below[0]), abi.Vec3(*below[1])
    return d, (keep, nodes, tri_arr, idx)


def test_deep_stack_restatement_equals_photons():
    """CPU: the oracle's restatement of the walk and Photon's own traversal agree on this tree."""
    if not O.reference_available():
        pytest.skip("Photon's CPU build (oracle/_ref) is missing")
    desc, keep = _deep_scene()
    cam = workloads.look_at((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 20.0, 64 / 48)
    a = O.orc_trace_primary(desc, cam, 64, 48, 0, 3)
    b = O.RefScene.from_desc(desc).trace_primary(cam, 64, 48, 0, 3)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    assert (O.hits_tri(a) == 2 * 50).all()


@pytest.mark.gpu
def test_deep_stack_walk_equals_photons_and_drops_past_64():
    if not O.reference_available():
        pytest.skip("Photon's CPU build (oracle/_ref) is missing")
    desc, keep = _deep_scene()
    w, h = 64, 48
    cam = workloads.look_at((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), 20.0, w / h)
    r = native.Renderer()
    r.upload(desc)
    ours = r.trace_primary(cam, w, h, 0, 3)
    r.close()
    theirs = O.RefScene.from_desc(desc).trace_primary(cam, w, h, 0, 3)
    assert np.array_equal(ours.view(np.uint32), theirs.view(np.uint32))
    tri = O.hits_tri(ours)
    assert (tri == 2 * 50).all(), np.unique(tri)
