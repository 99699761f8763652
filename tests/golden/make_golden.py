"""Generates the golden fixtures of tests/golden/ from Photon's own CPU code (oracle/_ref, built from
Photon's sources by oracle/Makefile) — run in a checkout where the reference build exists:

    python tests/golden/make_golden.py

For each scene: the radiance image of CpuRenderer::render (4 spp), the primary closest hits
(t, tri, u, v) of sample 0, and the first vertex's light picks. Scenes: Photon's built-in Cornell box
(built by Photon's Scene::build) and the library's procedural box and terrain (built by the library's
builder, rendered by Photon's renderer)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402
from photon_b200 import abi, native  # noqa: E402

CASES = {
    "cornell": dict(w=32, h=24, spp=4, depth=8, seed=1),
    "box": dict(w=32, h=32, spp=4, depth=8, seed=1),
    "terrain": dict(w=48, h=27, spp=4, depth=12, seed=1),
}


def scene(name):
    if name == "cornell":
        s = O.RefScene.builtin("cornell")
        return s, s.camera
    g = native.box_scene() if name == "box" else native.terrain_scene()
    b = g.build()
    return O.RefScene.from_desc(b.desc), g.camera


def main():
    for name, c in CASES.items():
        ref, camf = scene(name)
        cam = camf(c["w"] / c["h"])
        rs = abi.render_settings(c["w"], c["h"], max_depth=c["depth"], seed=c["seed"])
        img, _ = ref.render(cam, rs, c["spp"], threads=4)
        hits = ref.trace_primary(cam, c["w"], c["h"], 0, c["seed"])
        picks = ref.light_picks(cam, rs, 0)
        cam_arr = np.frombuffer(bytes(cam), np.float32).copy()
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), image=img, hits=hits, picks=picks, camera=cam_arr,
                            meta=np.array([c["w"], c["h"], c["spp"], c["depth"], c["seed"]], np.int64))
        print(name, img.mean(), (O.hits_tri(hits) >= 0).mean())


if __name__ == "__main__":
    main()
