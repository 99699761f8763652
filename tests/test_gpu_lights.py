"""Light tables rebuilt on the device (pt_rebuild_lights) against a scene rebuilt on the host
(pt_scene_build) with the same new materials, lights and environment: the renders are the same
bit for bit, which needs the emissive list, the alias table, the group probabilities and the
environment's distribution to be equal (light picks and MIS densities read them)."""
import ctypes as C

import numpy as np
import pytest

from photon_b200 import abi, native

pytestmark = pytest.mark.gpu


def _modified_raw(g, seed):
    """A copy of the generated raw scene with new emission, punctual intensities and environment."""
    raw = g.raw
    rng = np.random.default_rng(seed)
    mats = (abi.Material * raw.num_materials)()
    C.memmove(mats, raw.materials, C.sizeof(abi.Material) * raw.num_materials)
    for k in range(raw.num_materials):
        m = mats[k]
        if m.emission.x + m.emission.y + m.emission.z > 0:
            f = float(rng.uniform(0.2, 5.0))
            m.emission = abi.Vec3(m.emission.x * f, m.emission.y * f, m.emission.z * f)
        elif rng.random() < 0.05:
            m.emission = abi.Vec3(*rng.uniform(0.5, 3.0, 3))
    punct = (abi.PunctualLight * max(1, raw.num_punctual))()
    if raw.num_punctual:
        C.memmove(punct, raw.punctual, C.sizeof(abi.PunctualLight) * raw.num_punctual)
        for k in range(raw.num_punctual):
            p = punct[k]
            p.intensity = abi.Vec3(p.intensity.x * 1.7, p.intensity.y * 0.6, p.intensity.z)
    env = None
    if raw.env_texels:
        n = raw.env_width * raw.env_height
        env = np.ctypeslib.as_array(C.cast(raw.env_texels, C.POINTER(C.c_float)), shape=(n * 3,)).copy()
        env = (env.reshape(raw.env_height, raw.env_width, 3) * rng.uniform(0.3, 2.0, (1, 1, 3)).astype(np.float32))
        env = np.ascontiguousarray(np.roll(env, 37, axis=1), np.float32)
    new = abi.RawScene()
    C.memmove(C.byref(new), C.byref(raw), C.sizeof(abi.RawScene))
    new.materials = C.cast(mats, C.POINTER(abi.Material))
    new.punctual = C.cast(punct, C.POINTER(abi.PunctualLight))
    if env is not None:
        new.env_texels = env.ctypes.data_as(C.POINTER(abi.Vec3))
    new.env_intensity = raw.env_intensity * 1.3
    new.env_rotation = raw.env_rotation + 0.4
    return new, (mats, punct, env)


def _update_from(desc):
    u = abi.LightUpdate()
    u.materials, u.num_materials = desc.materials, desc.num_materials
    u.punctual, u.num_punctual = desc.punctual, desc.num_punctual
    u.env_texels, u.env_width, u.env_height = desc.env_texels, desc.env_width, desc.env_height
    u.env_color, u.env_intensity, u.env_rotation = desc.env_color, desc.env_intensity, desc.env_rotation
    return u


@pytest.mark.parametrize("kind,triangles", [("terrain", 262144), ("box", 36)])
def test_device_light_tables_equal_host_rebuild(kind, triangles):
    g = native.box_scene() if kind == "box" else native.terrain_scene(triangles, 1)
    before = g.build()
    raw, keep = _modified_raw(g, 5)
    after = native.BuiltScene(raw, keepalive=(g, keep))
    w, h, spp = 160, 90, 8
    cam = g.camera(w / h)
    rs = abi.render_settings(w, h, max_depth=8, seed=9)
    imgs = []
    for rebuild in (True, False):
        r = native.Renderer()
        r.upload(before.desc if rebuild else after.desc)
        r.resize(w, h)
        if rebuild:
            r.rebuild_lights(_update_from(after.desc))
        r.render(cam, rs, spp)
        imgs.append(r.download_image())
        picks = r.light_picks(cam, rs)
        imgs.append(picks)
        r.close()
    assert np.array_equal(imgs[1], imgs[3])  # light picks of the first vertex
    assert np.array_equal(imgs[0].view(np.uint32), imgs[2].view(np.uint32))
