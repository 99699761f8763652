"""The device BVH build (pt_bvh_build_options.gpu = 1) against the host build (gpu): the same tree and
the same triangle order, hence identical scene arrays, byte for byte."""
import ctypes as C
import time

import numpy as np
import pytest

from photon_b200 import native

pytestmark = pytest.mark.gpu


def _bytes(ptr, count, item_size):
    if count == 0 or not ptr:
        return b""
    return C.string_at(C.cast(ptr, C.c_void_p), count * item_size)


def _arrays(desc):
    return {
        "nodes": _bytes(desc.nodes, desc.num_nodes, 64),
        "tris": _bytes(desc.tris, desc.num_tris, 48),
        "indices": _bytes(desc.indices, 3 * desc.num_tris, 4),
        "tri_emissive": _bytes(desc.tri_emissive, desc.num_tris, 4),
        "emissive": _bytes(desc.emissive, desc.num_emissive, 8),
        "alias": _bytes(desc.emissive_alias, desc.num_emissive, 16),
        "scalars": (desc.num_nodes, desc.emissive_power, desc.p_env, desc.p_emissive, desc.p_punctual),
    }


@pytest.mark.parametrize("kind,triangles,opts", [
    ("box", 36, {}),
    ("terrain", 262144, {}),
    ("terrain", 262144, dict(bins=8, max_leaf=2)),
    ("terrain", 1048576, {}),
])
def test_device_build_equals_host_build(kind, triangles, opts):
    g = native.box_scene() if kind == "box" else native.terrain_scene(triangles, 3)
    t0 = time.perf_counter()
    host = g.build(**opts)
    t1 = time.perf_counter()
    dev = g.build(gpu=True, **opts)
    t2 = time.perf_counter()
    print(f"{kind} {triangles} {opts}: host build {1e3 * (t1 - t0):.0f} ms, device build {1e3 * (t2 - t1):.0f} ms")
    a, b = _arrays(host.desc), _arrays(dev.desc)
    for k in a:
        assert a[k] == b[k], k
