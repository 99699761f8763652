"""Parity of the CUDA wavefront with the oracle, through the C ABI (gpu).

Bars (from the contract of this path): primary closest-hit triangle indices and the first
vertex's light picks are bit-exact; images agree within 1e-3 * max(1, max channel) per pixel
(Photon's own comparison, tests/test_gpu.cpp:58-68) on >= 99.9% of the pixels, with means within
1%. Tolerances are written next to each check."""
import numpy as np
import pytest

from conftest import pixel_agreement
from oracle import oracle as O
from photon_b200 import abi, native
import scenes

pytestmark = pytest.mark.gpu

SCENES = ["cornell", "materials", "glass", "box", "terrain"]
PIXEL_FRACTION = 0.999   # >= 99.9% of pixels within the 1e-3 relative tolerance
MEAN_REL = 0.01          # means within 1%


@pytest.fixture(scope="module")
def renderer():
    r = native.Renderer()
    yield r
    r.close()


def _settings(name, w, h, **kw):
    depth = 12 if name == "terrain" else 8
    return abi.render_settings(w, h, max_depth=kw.pop("max_depth", depth), **kw)


@pytest.mark.parametrize("name", SCENES)
def test_primary_hits_bit_exact(renderer, name):
    desc, camf, keep = scenes.scene(name)
    w, h = (320, 180) if name == "terrain" else (96, 54)
    cam = camf(w / h)
    renderer.upload(desc)
    for frame, seed in ((0, 0), (5, 7)):
        gpu = renderer.trace_primary(cam, w, h, frame, seed)
        ref = O.orc_trace_primary(desc, cam, w, h, frame, seed)
        assert np.array_equal(O.hits_tri(gpu), O.hits_tri(ref))          # triangle indices: exact
        assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32))  # t, u, v: exact bits
    assert (O.hits_tri(gpu) >= 0).mean() > 0.3


@pytest.mark.parametrize("name", SCENES)
def test_light_picks_bit_exact(renderer, name):
    desc, camf, keep = scenes.scene(name)
    w, h = (320, 180) if name == "terrain" else (96, 54)
    cam = camf(w / h)
    rs = _settings(name, w, h, seed=3)
    renderer.upload(desc)
    for frame in (0, 9):
        gpu = renderer.light_picks(cam, rs, frame)
        ref = O.orc_light_picks(desc, cam, rs, frame)
        assert np.array_equal(gpu, ref)
    assert gpu[..., 3].mean() > 0.2  # the check exercised NEE


@pytest.mark.parametrize("name", SCENES)
def test_heatmap_matches_node_visits(renderer, name):
    desc, camf, keep = scenes.scene(name)
    w, h = 64, 36
    cam = camf(w / h)
    renderer.upload(desc)
    assert np.array_equal(renderer.heatmap(cam, w, h), O.orc_heatmap(desc, cam, w, h))


@pytest.mark.parametrize("name,w,h,spp", [("cornell", 96, 54, 64), ("materials", 96, 54, 64), ("glass", 96, 54, 64),
                                          ("box", 256, 256, 64), ("terrain", 192, 108, 16)])
def test_images_agree_with_oracle(renderer, name, w, h, spp):
    """The box case is the small configuration at its stated size: the 36-triangle closed box (grey
    0.73, red and green walls, a (17, 12, 4) ceiling emitter), 256x256 at 64 spp, max depth 8, Russian
    roulette from depth 3, seed 1."""
    desc, camf, keep = scenes.scene(name)
    cam = camf(w / h)
    rs = _settings(name, w, h, seed=1)
    renderer.upload(desc)
    renderer.resize(w, h)
    renderer.render(cam, rs, spp)
    gpu = renderer.download_image()
    ref = O.orc_render(desc, cam, rs, spp)
    frac, mr, mg = pixel_agreement(ref, gpu)
    exact = float((gpu.view(np.uint32) == ref.view(np.uint32)).all(axis=-1).mean())
    print(f"{name}: {100 * frac:.3f}% of pixels within 1e-3, {100 * exact:.2f}% bit-identical, means {mr:.5f} / {mg:.5f}")
    assert frac >= PIXEL_FRACTION
    assert abs(mr - mg) <= MEAN_REL * mr
    st = renderer.stats()
    assert st.samples == spp and st.paths == w * h * spp and st.queue_overflows == 0


def test_progressive_accumulation_matches_oracle_calls(renderer):
    # Two render calls of 8 samples: the second starts at sample index 8, and the accumulation adds
    # each call's per-pixel sum (CpuRenderer::render, cpu_renderer.cpp:28-32).
    desc, camf, keep = scenes.scene("cornell")
    w, h = 64, 48
    cam = camf(w / h)
    rs = _settings("cornell", w, h)
    renderer.upload(desc)
    renderer.resize(w, h)
    renderer.render(cam, rs, 8)
    renderer.render(cam, rs, 8)
    gpu = renderer.download_image()
    s = O.orc_render_sum(desc, cam, rs, 8, frame0=0)
    s += O.orc_render_sum(desc, cam, rs, 8, frame0=8)
    ref = s * np.float32(1.0 / 16)
    frac, mr, mg = pixel_agreement(ref, gpu)
    assert frac >= PIXEL_FRACTION and abs(mr - mg) <= MEAN_REL * mr
    assert renderer.samples == 16


def test_rendering_is_deterministic(renderer):
    desc, camf, keep = scenes.scene("glass")
    cam = camf(40 / 24)
    renderer.upload(desc)
    renderer.resize(40, 24)
    imgs = []
    for seed in (5, 5, 6):
        renderer.reset()
        renderer.render(cam, _settings("glass", 40, 24, seed=seed), 4)
        imgs.append(renderer.download_image())
    assert np.array_equal(imgs[0], imgs[1])
    assert not np.array_equal(imgs[0], imgs[2])


def test_furnace_and_display(renderer):
    # test_gpu.cpp:72-103: the flat-shaded white furnace converges to 1 (< 2e-3), samples and reset
    # behave, a linear white image displays as 0xFFFFFFFF, every display mode runs.
    desc, camf, keep = scenes.photon_builtin("furnace", flat_normals=True)
    renderer.upload(desc)
    renderer.resize(64, 64)
    rs = abi.render_settings(64, 64, max_depth=64, rr_depth=64, nee=0)
    cam = camf(1.0)
    renderer.render(cam, rs, 32)
    img = renderer.download_image()
    lum = img @ np.array([0.2126, 0.7152, 0.0722], np.float32)
    assert np.abs(lum - 1).max() < 2e-3
    assert renderer.samples == 32
    renderer.reset()
    assert renderer.samples == 0
    rs.tonemap = abi.PT_TONEMAP_LINEAR
    renderer.render(cam, rs, 4)
    renderer.display(rs, abi.PT_DISPLAY_COLOR)
    px = renderer.download_display()
    assert px[32, 32] == 0xFFFFFFFF
    for m in range(1, 6):
        renderer.display(rs, m)
    assert renderer.download_display().shape == (64, 64)


def test_gbuffer_matches_oracle_primary_info(renderer):
    desc, camf, keep = scenes.scene("materials")
    w, h = 64, 36
    cam = camf(w / h)
    rs = _settings("materials", w, h)
    renderer.upload(desc)
    renderer.resize(w, h)
    renderer.render(cam, rs, 2)
    albedo, nd = renderer.download_gbuffer()
    g = O.orc_gbuffer(desc, cam, rs, frame=0)
    assert np.array_equal(albedo.view(np.uint32), g["albedo"].view(np.uint32))
    assert np.array_equal(nd.view(np.uint32), g["normal_depth"].view(np.uint32))


def test_upload_rejects_inconsistent_scenes(renderer):
    desc, camf, keep = scenes.scene("box")
    bad = abi.SceneDesc.from_buffer_copy(desc)
    bad.num_vertices = 1  # indices now point past the vertex arrays
    with pytest.raises(native.PhotonError) as e:
        renderer.upload(bad)
    assert e.value.code == abi.PT_ERR_INVALID


def test_render_before_upload_is_an_error():
    r = native.Renderer()
    r.resize(8, 8)
    with pytest.raises(native.PhotonError) as e:
        r.render(abi.Camera(), abi.render_settings(8, 8), 1)
    assert e.value.code == abi.PT_ERR_NO_SCENE
    r.close()


@pytest.mark.parametrize("name", ["box", "terrain", "cornell"])
def test_gpu_matches_golden_fixtures(renderer, name):
    # The committed fixtures were produced by Photon's own CPU build (tests/golden/make_golden.py).
    import test_golden
    z, cam, rs, spp = test_golden.load(name)
    if name == "cornell":
        keep = O.RefScene.builtin("cornell")
        desc = keep.desc
    else:
        keep = (native.box_scene() if name == "box" else native.terrain_scene())
        built = keep.build()
        desc = built.desc
    renderer.upload(desc)
    renderer.resize(rs.width, rs.height)
    assert np.array_equal(renderer.trace_primary(cam, rs.width, rs.height, 0, rs.seed).view(np.uint32), z["hits"].view(np.uint32))
    assert np.array_equal(renderer.light_picks(cam, rs, 0), z["picks"])
    renderer.render(cam, rs, spp)
    frac, ma, mb = pixel_agreement(z["image"], renderer.download_image())
    assert frac >= PIXEL_FRACTION and abs(ma - mb) <= MEAN_REL * ma


@pytest.mark.parametrize("tuning", [
    dict(packed=0),
    dict(sort_by_material=0),
    dict(sort_by_material=1, shade_block=128),
    dict(sort_by_material=2, shade_block=64),
    dict(sort_rays=3),
    dict(trace_block=64, shade_block=64),
    dict(path_capacity=1 << 14, graph_bounces=1),
    dict(tail_paths=0),
    dict(wide_shadows=1),
    dict(wide_shadows=1, packed=0, tail_paths=0),
    dict(tail_paths=1 << 30),
    dict(tail_paths=1 << 12, path_capacity=1 << 14, graph_bounces=0),
    dict(tail_paths=0, trace_refill=1, shadow_refill=1),
    dict(tail_paths=0, trace_refill=32, shadow_refill=32),
    dict(tail_paths=0, trace_refill=5, shadow_refill=27, path_capacity=1 << 13),
    dict(tail_paths=0, wide_shadows=1, shadow_refill=32, trace_block=256),
    dict(tail_paths=0, pair_walk=0),
    dict(tail_paths=0, pair_walk=1),
    dict(tail_paths=0, pair_walk=64, trace_refill=32, shadow_refill=1),
    dict(tail_paths=0, pair_walk=3, trace_block=256, path_capacity=1 << 13),
    dict(tail_paths=0, pair_walk=2, packed=0),
])
def test_tuning_variants_are_bit_identical(tuning):
    """Every autotuner knob changes how the work is scheduled, never a path's arithmetic: scalar or
    packed slab tests, material-sorted shading, ray sorting, block shapes, the path pool size, the
    graph cadence, the one-thread-per-path tail (never, always, small), the shadow rays' BVH (4-wide
    or Photon's BVH2), when a walk's warp refills its idle lanes (only once all have finished,
    whenever one has, in between) and whether leaf triangles are tested by their own lane or by the
    warp's pair pass (after 1 to 64 node visits) all give the same image bit for bit (accumulation is
    in sample order). The variants that switch the tail off make the queued kernels walk every ray."""
    desc, camf, keep = scenes.scene("terrain")
    w, h, spp = 160, 90, 4
    cam = camf(w / h)
    rs = _settings("terrain", w, h, seed=3)
    imgs = []
    for t in ({}, tuning):
        r = native.Renderer()
        r.upload(desc)
        r.resize(w, h)
        if t:
            r.set_tuning(**t)
        r.render(cam, rs, spp)
        imgs.append(r.download_image())
        r.close()
    assert np.array_equal(imgs[0], imgs[1])


def test_adaptive_tail_is_bit_identical_alone_and_concurrent():
    """The default tail threshold (-2) is chosen per render from how many renders of the process run
    on the device; it moves work between kernels only, so renders alone and renders that overlap
    on other threads give the image of a render with the tail switched off, bit for bit."""
    import threading
    desc, camf, keep = scenes.scene("terrain")
    w, h, spp = 320, 180, 2
    cam = camf(w / h)
    rs = _settings("terrain", w, h, seed=5)

    def render(tuning=None):
        r = native.Renderer()
        r.upload(desc)
        r.resize(w, h)
        if tuning:
            r.set_tuning(**tuning)
        assert r.tuning()["tail_paths"] == (tuning or {}).get("tail_paths", -2)
        r.render(cam, rs, spp)
        img = r.download_image()
        r.close()
        return img

    ref = render(dict(tail_paths=0))
    assert np.array_equal(render(), ref)
    out = [None] * 4
    threads = [threading.Thread(target=lambda k=k: out.__setitem__(k, render())) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for img in out:
        assert img is not None and np.array_equal(img, ref)


def test_resize_rejects_oversized_images_and_keeps_working():
    """Images beyond 2^30 pixels (32-bit pixel indices) are refused before anything is allocated;
    the renderer keeps its previous size and renders as before."""
    desc, camf, keep = scenes.scene("box")
    r = native.Renderer()
    r.upload(desc)
    r.resize(64, 48)
    cam = camf(64 / 48)
    rs = abi.render_settings(64, 48, seed=2)
    r.render(cam, rs, 2)
    before = r.download_image()
    with pytest.raises(native.PhotonError) as e:
        r.resize(1 << 16, 1 << 15)
    assert e.value.code == abi.PT_ERR_INVALID
    assert (r.width, r.height) == (64, 48)
    r.reset()
    r.render(cam, rs, 2)
    assert np.array_equal(r.download_image(), before)
    r.close()


@pytest.mark.parametrize("bits", [3, 4, 5])
def test_ray_sorting_is_bit_identical(bits):
    """Ray sorting (continuing rays, moved into sorted order) and the sorted walk order of the shadow
    queue run only on iterations of at least 2^21 paths (smaller ones do not pay for the scans): a
    640x360x16 frame (3.7 M paths in one pool) sorts its first bounces, and its image equals the render
    with both sorts off bit for bit (sorting reorders queues, never a path's arithmetic)."""
    desc, camf, keep = scenes.scene("terrain")
    w, h, spp = 640, 360, 16
    cam = camf(w / h)
    rs = _settings("terrain", w, h, seed=4)
    imgs = []
    for t in (dict(sort_rays=0, sort_shadows=0), dict(sort_rays=bits, sort_shadows=bits), dict(sort_rays=0, sort_shadows=bits)):
        r = native.Renderer()
        r.upload(desc)
        r.resize(w, h)
        if t:
            r.set_tuning(**t)
        r.render(cam, rs, spp)
        imgs.append(r.download_image())
        r.close()
    for img in imgs[1:]:
        assert np.array_equal(imgs[0].view(np.uint32), img.view(np.uint32))


@pytest.mark.parametrize("pair_walk", [0, 5])
@pytest.mark.parametrize("name", ["terrain", "materials", "box"])
def test_any_hit_walk_bit_exact(renderer, name, pair_walk):
    """The shadow rays' any-hit walk on the device, directly: on random rays (half of them with a
    finite tmax), whether each is occluded, the triangle its walk accepts first and its node visits (and
    for the per-lane walk its triangle tests; a pair walk's tests are done by other lanes) equal the
    oracle's (the terrain has alpha-masked materials, so the alpha test is in the walk), for the pair
    walk of the default kernels and the per-lane walk. The 4-wide walk gives the same answers."""
    desc, camf, keep = scenes.scene(name)
    renderer.upload(desc)
    before = renderer.tuning()["pair_walk"]
    renderer.set_tuning(pair_walk=pair_walk)
    rays = scenes.random_rays(desc, 50000, seed=7)
    try:
        got = renderer.occlusion_probe(rays)
    finally:
        renderer.set_tuning(pair_walk=before)  # the module's renderer is shared
    want = O.orc_occluded(desc, rays)
    if pair_walk:
        assert np.array_equal(got[:, :3], want[:, :3]) and (got[:, 3] == -1).all()
    else:
        assert np.array_equal(got, want)
    wide = renderer.occlusion_probe(rays, wide=True)
    assert np.array_equal(wide[:, 0], want[:, 0])
    assert 0.2 < got[:, 0].mean() < 0.95


def test_download_into_page_locked_memory_equals_pageable():
    """pt_download_image copies straight into a page-locked destination and through pinned staging
    into pageable memory: the same bytes either way (an image larger than one staging half)."""
    import torch
    desc, camf, keep = scenes.scene("terrain")
    w, h = 1280, 720
    r = native.Renderer()
    r.upload(desc)
    r.resize(w, h)
    r.render(camf(w / h), _settings("terrain", w, h, seed=2), 1)
    pageable = r.download_image()
    pinned = torch.empty((h, w, 3), dtype=torch.float32, pin_memory=True).numpy()
    r.download_image(out=pinned)
    r.close()
    assert np.array_equal(pageable.view(np.uint32), pinned.view(np.uint32))


def test_pair_walk_visits_the_nodes_the_lane_walk_visits():
    """The pair walks visit exactly the per-lane walks' nodes: the counted render's node visits of the
    closest-hit and any-hit walks and the closest-hit triangle tests are equal (a pair walk tests a
    node's leaf triangles together, where the per-lane any-hit walk stops at the first accepted one,
    so only the any-hit triangle tests may differ), and so is the image."""
    desc, camf, keep = scenes.scene("terrain")
    w, h = 640, 360
    counts, images = [], []
    for pw in (0, 5):
        r = native.Renderer()
        r.upload(desc)
        r.resize(w, h)
        r.set_tuning(pair_walk=pw, tail_paths=0)
        r.set_profiling(abi.PT_PROFILE_TRAVERSAL_COUNTS)
        r.render(camf(w / h), _settings("terrain", w, h, seed=4), 2)
        p = r.profile()
        counts.append((p.closest_rays, p.closest_node_visits, p.closest_tri_tests, p.shadow_rays, p.shadow_node_visits))
        images.append(r.download_image())
        r.close()
    assert counts[0] == counts[1] and counts[0][1] > 0 and counts[0][4] > 0
    assert np.array_equal(images[0].view(np.uint32), images[1].view(np.uint32))
