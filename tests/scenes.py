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


def random_rays(desc, n, seed=0):
    """(n, 8) float32 rays for any-hit walks: origins uniform in the scene box, directions uniform on
    the sphere, tmax infinite for half of them and uniform in (0, the box's diagonal) for the rest."""
    import numpy as np
    rng = np.random.default_rng(seed)
    lo = np.array([desc.bounds_min.x, desc.bounds_min.y, desc.bounds_min.z], np.float64)
    hi = np.array([desc.bounds_max.x, desc.bounds_max.y, desc.bounds_max.z], np.float64)
    o = lo + (hi - lo) * rng.random((n, 3))
    d = rng.standard_normal((n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = np.where(rng.random(n) < 0.5, np.inf, rng.random(n) * np.linalg.norm(hi - lo))
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3], rays[:, 3], rays[:, 4:7] = o, tmax, d
    return rays
