"""Seeded workloads of the batched and served configurations.

- `batch_views`: views of one scene for the batched form — resolutions drawn log-uniformly by seed
  between 320x180 and 1920x1080 (16:9), spp uniform from {1, 4, 16, 64}, cameras on a sphere of
  radius 1.5x the scene's extent, looking at its centre.
- `request_stream`: a Poisson request stream for the server — resolution from {256^2, 640x360,
  1280x720, 1920x1080} with probabilities {0.4, 0.3, 0.2, 0.1}, spp from {1, 8, 64}, max depth from
  {4, 8, 12}, scenes uniformly.
- `orbit_cameras`: the real-time sessions' camera paths — an orbit around the scene's centre,
  0.5 degrees per frame.
"""
import math

import numpy as np

from . import abi

RESOLUTIONS = [(256, 256), (640, 360), (1280, 720), (1920, 1080)]
RES_P = [0.4, 0.3, 0.2, 0.1]


def look_at(position, target, vfov_deg, aspect, up=(0.0, 1.0, 0.0)):
    """A pinhole camera (the look-at convention of Camera::view, scene.cpp:13-25)."""
    p = np.asarray(position, np.float64)
    t = np.asarray(target, np.float64)
    f = t - p
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    if np.linalg.norm(r) < 1e-9:
        r = np.array([1.0, 0.0, 0.0])
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return abi.Camera(abi.Vec3(*p), math.tan(math.radians(vfov_deg) / 2), abi.Vec3(*f), aspect, abi.Vec3(*r), 0.0,
                      abi.Vec3(*u), float(np.linalg.norm(t - p)))


def scene_sphere(desc):
    lo = np.array([desc.bounds_min.x, desc.bounds_min.y, desc.bounds_min.z])
    hi = np.array([desc.bounds_max.x, desc.bounds_max.y, desc.bounds_max.z])
    return (lo + hi) / 2, float(np.linalg.norm(hi - lo))


def sphere_camera(rng, center, extent, aspect, vfov=45.0):
    # Upper hemisphere positions (an orbit over the scene), radius 1.5x the extent.
    z = rng.uniform(0.15, 0.95)
    phi = rng.uniform(0, 2 * math.pi)
    s = math.sqrt(1 - z * z)
    d = np.array([s * math.cos(phi), z, s * math.sin(phi)])
    return look_at(center + 1.5 * extent * d, center, vfov, aspect)


def batch_views(desc, n=64, seed=2, max_depth=12):
    rng = np.random.default_rng(seed)
    center, extent = scene_sphere(desc)
    views = []
    for k in range(n):
        w = int(round(math.exp(rng.uniform(math.log(320), math.log(1920)))))
        w = max(320, min(1920, w))
        h = max(180, min(1080, int(round(w * 9 / 16))))
        spp = int(rng.choice([1, 4, 16, 64]))
        cam = sphere_camera(rng, center, extent, w / h)
        views.append(abi.View(cam, w, h, spp, 1000 + k, abi.path_options(max_depth=max_depth)))
    return views


def request_stream(scenes, n, rate, seed=7):
    """scenes: list of (scene_id, desc). Returns a list of dicts with arrival time (s) and request."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    spheres = {sid: scene_sphere(d) for sid, d in scenes}
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        sid, _ = scenes[int(rng.integers(len(scenes)))]
        w, h = RESOLUTIONS[int(rng.choice(4, p=RES_P))]
        spp = int(rng.choice([1, 8, 64]))
        depth = int(rng.choice([4, 8, 12]))
        center, extent = spheres[sid]
        cam = sphere_camera(rng, center, extent, w / h)
        out.append(dict(t=t, scene=sid, cam=cam, w=w, h=h, spp=spp, seed=7000 + k, path=abi.path_options(max_depth=depth)))
    return out


def orbit_cameras(desc, frames, aspect, start_deg=0.0, step_deg=0.5, radius=0.9, elevation=0.45, vfov=45.0):
    """`frames` cameras on a circle of `radius` x the scene extent around its centre, `elevation` x the
    extent above it, looking at the centre; consecutive cameras `step_deg` degrees apart."""
    center, extent = scene_sphere(desc)
    cams = []
    for k in range(frames):
        a = math.radians(start_deg + step_deg * k)
        pos = center + extent * np.array([radius * math.cos(a), elevation, radius * math.sin(a)])
        cams.append(look_at(pos, center, vfov, aspect))
    return cams
