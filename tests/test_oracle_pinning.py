"""Pins the oracle: the C restatement (oracle/photon_oracle.c) against Photon's own CPU code compiled
from its sources (oracle/_ref/libphoton_ref.so), and against the known-answer cases of Photon's
test suite (tests/test_math.cpp, test_lights.cpp, test_render.cpp, test_bvh.cpp). CPU only."""
import ctypes as C

import numpy as np
import pytest

from conftest import pixel_agreement
from oracle import oracle as O
from photon_b200 import abi, native

needs_ref = pytest.mark.skipif(not O.reference_available(), reason="Photon reference build not present")


@needs_ref
@pytest.mark.parametrize("name", ["cornell", "materials", "glass", "furnace"])
def test_restatement_is_bit_exact_on_photon_builtins(name):
    s = O.RefScene.builtin(name)
    w, h = 48, 32
    cam = s.camera(w / h)
    rs = abi.render_settings(w, h, seed=3)
    ref, _ = s.render(cam, rs, 4, threads=4)
    orc = O.orc_render(s.desc, cam, rs, 4, threads=4)
    assert np.array_equal(ref.view(np.uint32), orc.view(np.uint32))
    assert np.array_equal(s.trace_primary(cam, w, h, 2, 3).view(np.uint32), O.orc_trace_primary(s.desc, cam, w, h, 2, 3).view(np.uint32))
    assert np.array_equal(s.light_picks(cam, rs, 1), O.orc_light_picks(s.desc, cam, rs, 1))
    assert np.array_equal(s.heatmap(cam, w, h), O.orc_heatmap(s.desc, cam, w, h))


@needs_ref
@pytest.mark.parametrize("kind", ["box", "terrain"])
def test_restatement_is_bit_exact_on_generated_scenes(kind):
    g = native.box_scene() if kind == "box" else native.terrain_scene()
    b = g.build()
    w, h = (40, 40) if kind == "box" else (64, 36)
    cam = g.camera(w / h)
    rs = abi.render_settings(w, h, max_depth=8 if kind == "box" else 12, seed=1)
    ref = O.RefScene.from_desc(b.desc)
    a, _ = ref.render(cam, rs, 2, threads=4)
    o = O.orc_render(b.desc, cam, rs, 2, threads=4)
    assert np.array_equal(a.view(np.uint32), o.view(np.uint32))
    assert np.array_equal(ref.light_picks(cam, rs, 0), O.orc_light_picks(b.desc, cam, rs, 0))


@needs_ref
def test_photon_builder_and_ours_render_the_same_scene():
    # The same raw box built by Photon's Scene::build and by ours: different trees, same image
    # up to path-level float noise (same meshes, lights and environment distribution).
    g = native.box_scene()
    ours = g.build()
    theirs = O.RefScene.from_raw(g.raw)
    w, h = 32, 32
    cam = g.camera(1.0)
    rs = abi.render_settings(w, h)
    a = O.orc_render(ours.desc, cam, rs, 16, threads=4)
    b = O.orc_render(theirs.desc, cam, rs, 16, threads=4)
    frac, ma, mb = pixel_agreement(b, a)
    assert abs(ma - mb) < 0.02 * mb
    assert theirs.desc.num_tris == ours.desc.num_tris == 36
    assert abs(theirs.desc.p_emissive - ours.desc.p_emissive) < 1e-6


@needs_ref
def test_environment_distribution_matches_photon_builder():
    g = native.terrain_scene()
    ours = g.build()
    theirs = O.RefScene.from_raw(g.raw)
    d0, d1 = ours.desc, theirs.desc
    n_m = d0.env_height + 1
    n_c = d0.env_height * (d0.env_width + 1)
    m0 = np.ctypeslib.as_array(d0.env_marginal, (n_m,))
    m1 = np.ctypeslib.as_array(d1.env_marginal, (n_m,))
    c0 = np.ctypeslib.as_array(d0.env_conditional, (n_c,))
    c1 = np.ctypeslib.as_array(d1.env_conditional, (n_c,))
    assert np.array_equal(m0, m1)
    assert np.array_equal(c0, c1)
    assert d0.env_integral == d1.env_integral
    assert abs(d0.p_env - d1.p_env) < 1e-6 and abs(d0.p_punctual - d1.p_punctual) < 1e-6


# ---- known answers of Photon's own tests ---------------------------------------------------------------

def test_alias_pmf_known_answer():
    # test_math.cpp:85-103: weights {1, 0, 3, 0.5, 5.5} -> pmf w / 10 exactly; sampling reproduces it.
    w = np.array([1, 0, 3, 0.5, 5.5], np.float32)
    raw = native.box_scene().raw  # any scene; we only need the library's alias builder via a scene
    if O.reference_available():
        t = (abi.AliasEntry * 5)()
        O.reference().ref_alias_table(w, 5, t)
        for k in range(5):
            assert abs(t[k].pmf - w[k] / 10) < 1e-6
        rng = np.zeros(200000, np.float32)
        O.restatement().orc_rng_floats(9, 9, 200000, rng)
        hist = np.zeros(5)
        pmf = C.c_float()
        for u in rng[:20000]:
            k = O.restatement().orc_sample_alias(t, 5, float(u), C.byref(pmf))
            assert abs(pmf.value - w[k] / 10) < 1e-5
            hist[k] += 1
        assert np.allclose(hist / 20000, w / 10, atol=0.01)


def test_rng_known_answers():
    # test_math.cpp:28-48: uniform in [0, 1), mean 1/2; PCG32 streams differ; matches Photon's Rng.
    a = np.zeros(160000, np.float32)
    O.restatement().orc_rng_floats(42, 7, a.size, a)
    assert a.min() >= 0 and a.max() < 1
    assert abs(a.mean() - 0.5) < 0.005
    hist = np.bincount((a * 16).astype(int), minlength=16)
    chi2 = ((hist - a.size / 16) ** 2 / (a.size / 16)).sum()
    assert chi2 < 40
    if O.reference_available():
        b = np.zeros(1000, np.float32)
        O.reference().ref_rng_floats(42, 7, b.size, b)
        assert np.array_equal(a[:1000], b)
    assert O.restatement().orc_hash_u32(0) == 0
    assert O.restatement().orc_hash_u32(1) != 1


def test_offset_ray_known_answer():
    # test_math.cpp:105-115: the offset point leaves the surface along n, by little.
    rng = np.random.default_rng(11)
    n = 10000
    scale = 10.0 ** rng.uniform(-4, 4, n)
    p = ((rng.uniform(0, 1, (n, 3)) * 2 - 1) * scale[:, None]).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    q = np.zeros_like(p)
    O.restatement().orc_offset_ray(n, np.ascontiguousarray(p), np.ascontiguousarray(d), q)
    assert ((q - p) * d).sum(axis=1).min() > 0
    assert (np.linalg.norm(q - p, axis=1) < 1e-3 * np.maximum(scale, 1.0)).all()
    if O.reference_available():
        r = np.zeros_like(p)
        O.reference().ref_offset_ray(n, np.ascontiguousarray(p), np.ascontiguousarray(d), r)
        assert np.array_equal(q.view(np.uint32), r.view(np.uint32))


@needs_ref
def test_bsdf_sampling_bit_exact_against_photon():
    rng = np.random.default_rng(5)
    cases = [(0.8, 0.8, 0.8, 0, 1, 0, 1.5), (0.5, 0.2, 0.1, 0, 0.25, 0, 1.5), (0.95, 0.7, 0.3, 1, 0.3, 0, 1.5),
             (1, 1, 1, 0, 0.3, 1, 1.5), (0.7, 0.7, 0.7, 0, 0.6, 0.5, 1.5), (1, 1, 1, 0, 0, 1, 1.5)]
    for c in cases:
        p = np.array(c, np.float32)
        n = 4000
        wo = rng.normal(size=(n, 3))
        wo /= np.linalg.norm(wo, axis=1, keepdims=True)
        rows = np.zeros((n, 8), np.float32)
        rows[:, :3] = wo
        rows[:, 3:7] = rng.uniform(0, 1, (n, 4))
        a = np.zeros((n, 9), np.float32)
        b = np.zeros((n, 9), np.float32)
        O.restatement().orc_bsdf_sample(p, n, rows, a)
        O.reference().ref_bsdf_sample(p, n, rows, b)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_point_light_known_answer():
    # test_lights.cpp:127-148: point light of intensity 8 at height 2: L = 8 / 4, pdf 1, delta.
    ground = native.GeneratedScene(abi.PT_GEN_BOX)  # reuse the builder with a custom raw scene below
    pos = (abi.Vec3 * 4)(abi.Vec3(-10, 0, -10), abi.Vec3(-10, 0, 10), abi.Vec3(10, 0, 10), abi.Vec3(10, 0, -10))
    idx = (C.c_int32 * 6)(0, 1, 2, 0, 2, 3)
    tm = (C.c_int32 * 2)(0, 0)
    mat = abi.Material()
    mat.base_color = abi.Vec4(1, 1, 1, 1)
    mat.roughness, mat.ior, mat.normal_scale, mat.alpha_cutoff = 1, 1.5, 1, 0.5
    for f in ("base_color_tex", "metallic_roughness_tex", "normal_tex", "emissive_tex", "occlusion_tex"):
        setattr(mat, f, -1)
    light = abi.PunctualLight(abi.Vec3(0, 2, 0), abi.PT_LIGHT_POINT, abi.Vec3(0, -1, 0), 1, abi.Vec3(8, 8, 8), 0)
    raw = abi.RawScene()
    raw.positions, raw.num_positions = pos, 4
    raw.indices, raw.num_indices, raw.tri_material = idx, 6, tm
    raw.materials, raw.num_materials = C.pointer(mat), 1
    raw.punctual, raw.num_punctual = C.pointer(light), 1
    raw.env_intensity = 1
    b = native.BuiltScene(raw)
    out = np.zeros(12, np.float32)
    O.restatement().orc_sample_light(b.desc, np.zeros(3, np.float32), 0.5, 0.3, 0.7, 0.1, out)
    assert out[8] == 1 and abs(out[3] - 2) < 1e-5
    assert abs(0.2126 * out[4] + 0.7152 * out[5] + 0.0722 * out[6] - 2.0) < 1e-4
    assert abs(out[7] - 1.0) < 1e-6
    O.restatement().orc_sample_light(b.desc, np.array([1.5, 0, 0], np.float32), 0.5, 0.3, 0.7, 0.1, out)
    assert abs(0.2126 * out[4] + 0.7152 * out[5] + 0.0722 * out[6] - 8.0 / 6.25) < 1e-4
    del ground


@needs_ref
def test_white_furnace_known_answer():
    # test_render.cpp:30-63: flat-shaded white Lambertian sphere in a white environment, BSDF
    # sampling only, no roulette: every pixel is 1 within 1e-3.
    s = O.RefScene.builtin("furnace", flat_normals=True)
    cam = s.camera(1.0)
    rs = abi.render_settings(48, 48, max_depth=64, rr_depth=64, nee=0)
    img = O.orc_render(s.desc, cam, rs, 16, threads=4)
    lum = img @ np.array([0.2126, 0.7152, 0.0722], np.float32)
    assert np.abs(lum - 1).max() < 1e-3


@needs_ref
def test_alpha_masked_triangles_are_skipped_known_answer():
    # test_bvh.cpp:150-170: a fully masked quad in front of an opaque one: the hit is at t = 5 on
    # the second quad's material.
    pos = (abi.Vec3 * 8)(abi.Vec3(-1, -1, 1), abi.Vec3(1, -1, 1), abi.Vec3(1, 1, 1), abi.Vec3(-1, 1, 1),
                         abi.Vec3(-1, -1, 0), abi.Vec3(1, -1, 0), abi.Vec3(1, 1, 0), abi.Vec3(-1, 1, 0))
    idx = (C.c_int32 * 12)(0, 1, 2, 0, 2, 3, 4, 5, 6, 4, 6, 7)
    tm = (C.c_int32 * 4)(0, 0, 1, 1)
    mats = (abi.Material * 2)()
    for k in range(2):
        m = mats[k]
        m.base_color = abi.Vec4(1, 1, 1, 0 if k == 0 else 1)
        m.metallic, m.roughness, m.ior, m.normal_scale, m.alpha_cutoff = 1, 1, 1.5, 1, 0.5
        m.alpha_mode = abi.PT_ALPHA_MASK if k == 0 else abi.PT_ALPHA_OPAQUE
        for f in ("base_color_tex", "metallic_roughness_tex", "normal_tex", "emissive_tex", "occlusion_tex"):
            setattr(m, f, -1)
    raw = abi.RawScene()
    raw.positions, raw.num_positions = pos, 8
    raw.indices, raw.num_indices, raw.tri_material = idx, 12, tm
    raw.materials, raw.num_materials = mats, 2
    raw.env_intensity = 1
    for built in (native.BuiltScene(raw), O.RefScene.from_raw(raw)):
        d = built.desc
        cam = abi.Camera(abi.Vec3(0.1, 0.2, 5), 1e-4, abi.Vec3(0, 0, -1), 1.0, abi.Vec3(1, 0, 0), 0, abi.Vec3(0, 1, 0), 5)
        hits = O.orc_trace_primary(d, cam, 1, 1, 0, 0)
        t, tri = hits[0, 0, 0], O.hits_tri(hits)[0, 0]
        assert abs(t - 5) < 1e-4
        assert d.tris[tri].material == 1


def _raw_arrays(raw):
    """Every array of a pt_raw_scene as bytes, by name (for byte-for-byte comparison)."""
    n_pos, n_idx = raw.num_positions, raw.num_indices
    out = {}

    def take(name, ptr, count, itemsize):
        out[name] = C.string_at(ptr, count * itemsize) if ptr and count else b""

    take("positions", raw.positions, n_pos, 12)
    take("normals", raw.normals, n_pos, 12)
    take("uvs", raw.uvs, n_pos, 8)
    take("indices", raw.indices, n_idx, 4)
    take("tri_material", raw.tri_material, n_idx // 3, 4)
    take("materials", raw.materials, raw.num_materials, C.sizeof(abi.Material))
    take("punctual", raw.punctual, raw.num_punctual, C.sizeof(abi.PunctualLight))
    take("env", raw.env_texels, raw.env_width * raw.env_height, 12)
    for k in range(raw.num_textures):
        t = raw.textures[k]
        take(f"texture{k}", t.texels, t.width * t.height, 4)
        out[f"texture{k}_info"] = (t.width, t.height, t.repeat, t.srgb)
    out["scalars"] = (raw.env_width, raw.env_height, raw.env_color.x, raw.env_color.y, raw.env_color.z,
                      raw.env_intensity, raw.env_rotation)
    return out


@needs_ref
@pytest.mark.parametrize("kind,tris", [(abi.PT_GEN_BOX, 36), (abi.PT_GEN_TERRAIN, 262144), (abi.PT_GEN_TERRAIN, 70000)])
def test_reference_build_holds_the_same_scene_generator(kind, tris):
    """The benchmark's reference arm builds its scene without the product library: Photon's build
    carries its own copy of the seeded generator. Its raw meshes, materials, textures, lights and
    environment equal pt_generate_scene's byte for byte; Photon's Scene::build of them gives the
    triangle count, and its camera is Photon's Camera::view of the generator's look-at camera."""
    ours = native.GeneratedScene(kind, tris, 1)
    theirs = O.RefGeneratedRaw(kind, tris, 1)
    a, b = _raw_arrays(ours.raw), _raw_arrays(theirs.raw)
    assert a.keys() == b.keys()
    for k in a:
        assert a[k] == b[k], k
    s = O.RefScene.generated(kind, tris, 1, threads=4)
    assert s.desc.num_tris == tris
    c0, c1 = ours.camera(16 / 9), s.camera(16 / 9)
    for f in ("position", "forward", "right", "up"):
        v0, v1 = getattr(c0, f), getattr(c1, f)
        assert max(abs(v0.x - v1.x), abs(v0.y - v1.y), abs(v0.z - v1.z)) < 1e-6, f
    assert abs(c0.tan_half_fov - c1.tan_half_fov) < 1e-6 and c0.aspect == c1.aspect


@needs_ref
@pytest.mark.parametrize("name", ["materials", "terrain"])
def test_restatement_any_hit_walk_equals_photons(name):
    """The any-hit walk (Photon's occluded, traverse.h:144-147): on random rays, the restatement's
    answer, the triangle it accepts first and its node visits equal Photon's traverse<true>, including
    rays through the terrain's alpha-masked (25%) materials."""
    import scenes
    if name == "terrain":
        g = native.terrain_scene()
        b = g.build()
        ref = O.RefScene.from_desc(b.desc)
    else:
        ref = O.RefScene.builtin(name)
    rays = scenes.random_rays(ref.desc, 20000, seed=3)
    theirs = ref.occluded(rays)
    ours = O.orc_occluded(ref.desc, rays)
    assert np.array_equal(ours[:, :3], theirs[:, :3])
    assert 0.2 < ours[:, 0].mean() < 0.95
