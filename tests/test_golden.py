"""The oracle against golden fixtures produced by Photon's own CPU code (tests/golden/make_golden.py):
the restatement must reproduce them bit-for-bit. Runs on the CPU, without Photon's build for the
library-built scenes."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O
from photon_b200 import abi, native

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    z = np.load(os.path.join(HERE, f"{name}.npz"))
    cam = abi.Camera.from_buffer_copy(z["camera"].tobytes())
    w, h, spp, depth, seed = (int(v) for v in z["meta"])
    return z, cam, abi.render_settings(w, h, max_depth=depth, seed=seed), spp


@pytest.mark.parametrize("name", ["box", "terrain", "cornell"])
def test_restatement_reproduces_golden(name):
    z, cam, rs, spp = load(name)
    if name == "cornell":
        if not O.reference_available():
            pytest.skip("Photon's built-in scene needs the reference build")
        keep = O.RefScene.builtin("cornell")
        desc = keep.desc
    else:
        g = native.box_scene() if name == "box" else native.terrain_scene()
        keep = g.build()
        desc = keep.desc
    img = O.orc_render(desc, cam, rs, spp, threads=4)
    assert np.array_equal(img.view(np.uint32), z["image"].view(np.uint32))
    hits = O.orc_trace_primary(desc, cam, rs.width, rs.height, 0, rs.seed)
    assert np.array_equal(hits.view(np.uint32), z["hits"].view(np.uint32))
    assert np.array_equal(O.orc_light_picks(desc, cam, rs, 0), z["picks"])
