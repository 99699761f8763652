"""Scenes the tests compare on: Photon's built-in scenes built by Photon's own Scene::build
(through the reference build in oracle/_ref) and the procedural benchmark scenes built by the
library's builder. Each entry yields (scene description, camera factory, keep-alive object)."""
from oracle import oracle as O
from photon_b200 import native


def photon_builtin(name, flat_normals=False):
    s = O.RefScene.builtin(name, flat_normals=flat_normals)
    return s.desc, s.camera, s


def generated(kind, triangles=262144, seed=1):
    g = native.box_scene() if kind == "box" else native.terrain_scene(triangles, seed)
    b = g.build()
    return b.desc, g.camera, (g, b)


def scene(name):
    if name in ("cornell", "materials", "glass", "furnace"):
        return photon_builtin(name)
    return generated(name)
