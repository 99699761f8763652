"""The systems forms beside the drop-in renderer (gpu): batched views in one wavefront, and the
request server with continuous batching over resident scenes. Every image must be bit-identical to
the same work rendered alone: a path depends only on (scene, camera, pixel, sample index, seed,
options), and each pixel's samples are summed in sample order."""
import threading
import time

import numpy as np
import pytest

from oracle import oracle as O
from photon_b200 import abi, native
import scenes

pytestmark = pytest.mark.gpu


def _view(cam, w, h, spp, seed, depth=8):
    return abi.View(cam, w, h, spp, seed, abi.path_options(max_depth=depth))


def test_batched_views_equal_individual_renders():
    desc, camf, keep = scenes.scene("terrain")
    sizes = [(64, 36, 4, 1), (96, 54, 1, 2), (40, 30, 16, 3), (128, 72, 2, 4), (33, 17, 8, 5)]
    views = []
    for k, (w, h, spp, seed) in enumerate(sizes):
        cam = camf(w / h)
        cam.position.x += 0.3 * k
        views.append(_view(cam, w, h, spp, seed, depth=12))
    r = native.Renderer()
    r.upload(desc)
    r.render_views(views)
    batched = [r.download_view(k, v.width, v.height) for k, v in enumerate(views)]
    for k, v in enumerate(views):
        r.resize(v.width, v.height)
        r.reset()
        r.render(v.camera, abi.RenderSettings(v.width, v.height, v.path, 1.0, abi.PT_TONEMAP_ACES, v.seed), v.spp)
        alone = r.download_image()
        assert np.array_equal(batched[k].view(np.uint32), alone.view(np.uint32)), f"view {k}"
    r.close()


def test_batched_views_with_split_passes_are_unchanged():
    # A view bigger than one pass's radiance buffer is split by sample range; the per-pixel sums
    # stay in sample order, so the image is unchanged.
    desc, camf, keep = scenes.scene("box")
    cam = camf(1.0)
    r = native.Renderer()
    r.upload(desc)
    v = _view(cam, 64, 64, 32, 9)
    r.render_views([v])
    one = r.download_view(0, 64, 64)
    r.resize(64, 64)
    r.reset()
    for _ in range(4):
        r.render(cam, abi.render_settings(64, 64, seed=9), 8)
    ref = O.orc_render(desc, cam, abi.render_settings(64, 64, seed=9), 32)
    assert np.abs(one - ref).max() < 1e-3 * max(1.0, float(ref.max()))
    r.close()


@pytest.mark.parametrize("pair_walk", [0, 5])
def test_server_walks_equal_the_renderer(pair_walk):
    """The server's multi-scene walk kernels (each ray's scene from its view), as pair walks or per-lane
    walks, give the image of the renderer's single-scene per-lane walk bit for bit. 320x180x4 paths
    exceed the server's tail threshold, so the queued walks run."""
    desc, camf, keep = scenes.scene("terrain")
    cam, path = camf(16 / 9), abi.path_options(max_depth=12)
    rr = native.Renderer()
    rr.upload(desc)
    rr.resize(320, 180)
    rr.set_tuning(pair_walk=0, tail_paths=0)
    rr.render(cam, abi.RenderSettings(320, 180, path, 1.0, abi.PT_TONEMAP_ACES, 4), 4)
    want = rr.download_image()
    rr.close()
    s = native.Server(budget_bytes=8 << 30, path_capacity=1 << 18)
    s.set_tuning(pair_walk=pair_walk)
    sid = s.add_scene(desc)
    rid = s.submit(sid, cam, 320, 180, 4, 4, path)
    s.wait(rid, 60)
    img, _ = s.fetch(rid, 320, 180)
    s.close()
    assert np.array_equal(img.view(np.uint32), want.view(np.uint32))


@pytest.fixture(scope="module")
def server_scenes():
    box = scenes.scene("box")
    terrain = scenes.scene("terrain")
    return box, terrain


def test_server_results_are_identical_alone_and_in_a_mix(server_scenes):
    (bdesc, bcam, bkeep), (tdesc, tcam, tkeep) = server_scenes
    s = native.Server(budget_bytes=8 << 30, path_capacity=1 << 18)
    sb = s.add_scene(bdesc)
    st = s.add_scene(tdesc)
    probe = dict(scene_id=st, cam=tcam(96 / 54), w=96, h=54, spp=8, seed=11, path=abi.path_options(max_depth=12))
    rid = s.submit(probe["scene_id"], probe["cam"], probe["w"], probe["h"], probe["spp"], probe["seed"], probe["path"])
    s.wait(rid, 60)
    alone, stats = s.fetch(rid, 96, 54)
    assert stats.state == abi.PT_REQ_DONE and stats.samples == 96 * 54 * 8
    # The same request among others of both scenes, submitted from several threads.
    ids = []
    lock = threading.Lock()

    def submit_many(k):
        for j in range(4):
            sid = sb if (k + j) % 2 else st
            cam = bcam(1.0) if sid == sb else tcam(16 / 9)
            w, h = (48, 48) if sid == sb else (80, 45)
            r = s.submit(sid, cam, w, h, 1 + 3 * j, 100 + 10 * k + j, abi.path_options(max_depth=8))
            with lock:
                ids.append((r, w, h))

    threads = [threading.Thread(target=submit_many, args=(k,)) for k in range(3)]
    for t in threads:
        t.start()
    rid2 = s.submit(probe["scene_id"], probe["cam"], probe["w"], probe["h"], probe["spp"], probe["seed"], probe["path"])
    for t in threads:
        t.join()
    s.wait(rid2, 120)
    mixed, _ = s.fetch(rid2, 96, 54)
    assert np.array_equal(alone.view(np.uint32), mixed.view(np.uint32))
    for r, w, h in ids:
        s.wait(r, 120)
        img, st_ = s.fetch(r, w, h)
        assert st_.state == abi.PT_REQ_DONE and np.isfinite(img).all()
    # ... and equal to the plain renderer's image of the same request.
    rr = native.Renderer()
    rr.upload(tdesc)
    rr.resize(96, 54)
    rr.render(probe["cam"], abi.RenderSettings(96, 54, probe["path"], 1.0, abi.PT_TONEMAP_ACES, 11), 8)
    assert np.array_equal(rr.download_image().view(np.uint32), alone.view(np.uint32))
    rr.close()
    stats = s.stats()
    assert stats.completed == 2 + len(ids) and stats.active == 0 and stats.queued == 0
    s.close()


def test_server_budget_cancel_and_faults(server_scenes):
    (bdesc, bcam, bkeep), _ = server_scenes
    budget = 256 << 20
    s = native.Server(budget_bytes=budget, path_capacity=1 << 16)
    sid = s.add_scene(bdesc)
    cam = bcam(1.0)
    # A request that can never fit the budget is refused at submission.
    with pytest.raises(native.PhotonError) as e:
        s.submit(sid, cam, 4096, 4096, 64)
    assert e.value.code == abi.PT_ERR_BUDGET
    assert s.stats().rejected == 1
    # Unknown scene.
    with pytest.raises(native.PhotonError) as e:
        s.submit(sid + 7, cam, 8, 8, 1)
    assert e.value.code == abi.PT_ERR_NOT_FOUND
    # Host-side fault injection: the next allocation fails; that request fails, the server stays up.
    s.fail_allocations(1)
    bad = s.submit(sid, cam, 32, 32, 1)
    with pytest.raises(native.PhotonError):
        s.wait(bad, 30)
    assert s.poll(bad) == abi.PT_REQ_FAILED
    good = s.submit(sid, cam, 32, 32, 2)
    s.wait(good, 30)
    assert s.poll(good) == abi.PT_REQ_DONE
    # A wait that runs out reports a timeout instead of hanging.
    slow = s.submit(sid, cam, 256, 256, 64)
    with pytest.raises(native.PhotonError) as e:
        s.wait(slow, 0.0)
    assert e.value.code in (abi.PT_ERR_TIMEOUT,)
    s.wait(slow, 60)
    st = s.stats()
    assert st.device_bytes_in_use <= budget
    s.close()


def test_server_device_failure_while_finishing_settles_each_request_once(server_scenes):
    """A failure raised while a finished request is being queued for its read-back (host-side
    injection, as a failing CUDA call there would) fails the requests in flight. Each request's
    device memory is given back exactly once: afterwards the server's memory in use is back to its
    pool and scenes, its budget checks still admit work, and a new request renders."""
    (bdesc, bcam, bkeep), _ = server_scenes
    budget = 1 << 30
    s = native.Server(budget_bytes=budget, path_capacity=1 << 16)
    sid = s.add_scene(bdesc)
    cam = bcam(1.0)
    idle = s.stats().device_bytes_in_use
    for _ in range(3):
        s.fail_finishing(1)
        ids = [s.submit(sid, cam, 32 + 8 * k, 32, 1 + k % 3) for k in range(6)]
        states = []
        for r in ids:
            try:
                s.wait(r, 60)
            except native.PhotonError as e:
                assert e.code == abi.PT_ERR_CUDA, e
            states.append(s.poll(r))
        assert abi.PT_REQ_FAILED in states
        assert set(states) <= {abi.PT_REQ_FAILED, abi.PT_REQ_DONE}
        for r in ids:
            try:
                s.fetch(r, 32 + 64, 32)
            except native.PhotonError:
                pass
        st = s.stats()
        assert st.active == 0 and st.queued == 0
        assert st.device_bytes_in_use == idle, (st.device_bytes_in_use, idle)
    ok = s.submit(sid, cam, 64, 64, 4)
    s.wait(ok, 60)
    assert s.poll(ok) == abi.PT_REQ_DONE
    img, _ = s.fetch(ok, 64, 64)
    assert np.isfinite(img).all() and img.mean() > 0
    assert s.stats().device_bytes_in_use == idle
    s.close()


def test_server_cancels_running_and_queued_requests(server_scenes):
    """One request runs at a time (max_active 1): a long request on the 262K scene is cancelled while
    it runs and three others while they wait; all end cancelled, their buffers are released, and the
    server goes on to finish a new request."""
    _, (tdesc, tcam, tkeep) = server_scenes
    s = native.Server(budget_bytes=4 << 30, path_capacity=1 << 18, max_active=1)
    sid = s.add_scene(tdesc)
    cam = tcam(1.0)
    deep = abi.path_options(max_depth=64, rr_depth=64)
    big = s.submit(sid, cam, 512, 512, 64, path=deep)
    more = [s.submit(sid, cam, 256, 256, 16, path=deep) for _ in range(3)]
    for r in [big] + more:
        s.cancel(r)
    for r in [big] + more:
        with pytest.raises(native.PhotonError) as e:
            s.wait(r, 60)
        assert e.value.code == abi.PT_ERR_CANCELLED
        assert s.poll(r) == abi.PT_REQ_CANCELLED
    ok = s.submit(sid, cam, 64, 64, 4)
    s.wait(ok, 60)
    assert s.poll(ok) == abi.PT_REQ_DONE
    st = s.stats()
    assert st.cancelled == 4 and st.active == 0
    s.close()


def test_server_scene_limit_holds_under_concurrent_adds(server_scenes):
    """add_scene from several threads at once: the scene table never grows past its 256 entries;
    the adds beyond it fail with PT_ERR_BUDGET, and a request still renders on a scene added last."""
    (box_desc, box_camf, box_keep), _ = server_scenes
    srv = native.Server(budget_bytes=0, path_capacity=1 << 20)
    ids, errors = [], []
    lock = threading.Lock()

    def add(k):
        for _ in range(70):
            try:
                sid = srv.add_scene(box_desc)
                with lock:
                    ids.append(sid)
            except native.PhotonError as e:
                with lock:
                    errors.append(e.code)

    threads = [threading.Thread(target=add, args=(k,)) for k in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert len(ids) == 256 and sorted(ids) == list(range(256))
    assert len(errors) == 4 * 70 - 256 and set(errors) == {abi.PT_ERR_BUDGET}
    assert srv.stats().scenes == 256
    cam = box_camf(1.0)
    rid = srv.submit(255, cam, 32, 32, 2, seed=1)
    srv.wait(rid, 60.0)
    img, _ = srv.fetch(rid, 32, 32)
    assert np.isfinite(img).all() and img.max() > 0
    srv.close()


def test_server_survives_immediate_fetches_of_many_small_requests(server_scenes):
    """Many tiny requests from several threads, each fetched the moment it is done: a fetched
    request may still be listed by a batch that the server has not read back yet, so the server must
    keep it until then (it did not, and read freed memory). Every image arrives and equals the same
    request rendered alone."""
    (box_desc, box_camf, box_keep), _ = server_scenes
    srv = native.Server(budget_bytes=0, path_capacity=1 << 20)
    sid = srv.add_scene(box_desc)
    cam = box_camf(1.0)
    failures = []

    def client(k):
        try:
            for j in range(60):
                rid = srv.submit(sid, cam, 16, 16, 1, seed=100 * k + j)
                srv.wait(rid, 60.0)
                img, st = srv.fetch(rid, 16, 16)
                if not np.isfinite(img).all():
                    failures.append((k, j, "not finite"))
                with pytest.raises(native.PhotonError):
                    srv.poll(rid)
        except Exception as e:  # noqa: BLE001 - reported below
            failures.append((k, repr(e)))

    threads = [threading.Thread(target=client, args=(k,)) for k in range(6)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not failures, failures[:3]
    rid = srv.submit(sid, cam, 16, 16, 1, seed=205)
    srv.wait(rid, 60.0)
    served, _ = srv.fetch(rid, 16, 16)
    srv.close()
    r = native.Renderer()
    r.upload(box_desc)
    r.resize(16, 16)
    r.render(cam, abi.RenderSettings(16, 16, abi.path_options(), 1.0, abi.PT_TONEMAP_ACES, 205), 1)
    assert np.array_equal(served.view(np.uint32), r.download_image().view(np.uint32))
    r.close()


def test_autotuner_record_is_used_by_batches_and_the_server():
    """pt_autotune_views tunes on a scaled-down copy of a view set: its probe rate with the chosen
    tuning is no lower than with the default, the record stays with the renderer (pt_get_tuning) and
    the last batch stays downloadable; the views render bit-identically with it; and a server given the
    record (pt_server_set_tuning) renders a request bit-identically to a server left at its defaults."""
    desc, camf, keep = scenes.scene("terrain")
    sizes = [(160, 90, 4, 1), (96, 54, 16, 2), (200, 120, 1, 3), (64, 64, 8, 4)]
    views = []
    for k, (w, h, spp, seed) in enumerate(sizes):
        cam = camf(w / h)
        cam.position.z += 0.2 * k
        views.append(_view(cam, w, h, spp, seed, depth=12))
    r = native.Renderer()
    r.upload(desc)
    r.render_views(views)
    before = [r.download_view(k, v.width, v.height) for k, v in enumerate(views)]
    chosen, default_rate, tuned_rate = r.autotune_views(views, probe_samples=1 << 18)
    assert tuned_rate >= default_rate > 0
    assert r.tuning() == chosen
    for k, v in enumerate(views):  # the autotuner's probes did not overwrite the last batch
        assert np.array_equal(r.download_view(k, v.width, v.height).view(np.uint32), before[k].view(np.uint32))
    r.render_views(views)
    for k, v in enumerate(views):
        assert np.array_equal(r.download_view(k, v.width, v.height).view(np.uint32), before[k].view(np.uint32)), f"view {k}"
    c1, d1, t1 = r.autotune(views[0].camera, abi.RenderSettings(160, 90, views[0].path, 1.0, abi.PT_TONEMAP_ACES, 1), 4,
                            probe_samples=1 << 16)
    assert t1 >= d1 > 0
    r.close()
    knobs = ("sort_by_material", "sort_rays", "packed", "wide_shadows", "trace_refill", "shadow_refill", "walk_burst", "pair_walk")
    images = []
    for record in (None, {k: chosen[k] for k in knobs}):
        s = native.Server(budget_bytes=8 << 30, path_capacity=1 << 18)
        sid = s.add_scene(desc)
        if record:
            record["sort_rays"] = min(record["sort_rays"], 4)
            s.set_tuning(**record)
        rid = s.submit(sid, views[1].camera, 96, 54, 16, seed=2, path=abi.path_options(max_depth=12))
        s.wait(rid, 60)
        img, _ = s.fetch(rid, 96, 54)
        images.append(img)
        s.close()
    assert np.array_equal(images[0].view(np.uint32), images[1].view(np.uint32))
    assert np.array_equal(images[0].view(np.uint32), before[1].view(np.uint32))


def test_server_serves_encoded_images(server_scenes):
    """The headless image endpoint: a finished request fetched as PFM is the byte stream of the float
    image in Photon's save_pfm format, and fetched as PNG the colour view of its samples (exposure, tone
    map, sRGB, RGBA8, mapped on the device at finishing). Both equal the plain renderer's image and
    display buffer of the same request. A size query keeps the request; PNG needs display = 1."""
    from test_image_io import _decode_png
    _, (tdesc, tcam, tkeep) = server_scenes
    s = native.Server(budget_bytes=8 << 30, path_capacity=1 << 18)
    sid = s.add_scene(tdesc)
    w, h, spp, seed = 96, 54, 8, 21
    cam = tcam(w / h)
    path = abi.path_options(max_depth=12)
    kw = dict(seed=seed, path=path, display=True, exposure=1.5, tonemap=abi.PT_TONEMAP_REINHARD)
    a, b = s.submit(sid, cam, w, h, spp, **kw), s.submit(sid, cam, w, h, spp, **kw)
    plain_only = s.submit(sid, cam, w, h, spp, seed=seed, path=path)
    for rid in (a, b, plain_only):
        s.wait(rid, 60)
    n = s.encoded_size(a, abi.PT_IMAGE_PFM)
    assert s.encoded_size(a, abi.PT_IMAGE_PFM) == n == len(f"PF\n{w} {h}\n-1.0\n") + w * h * 12
    pfm = s.fetch_encoded(a, abi.PT_IMAGE_PFM)
    with pytest.raises(native.PhotonError) as e:  # consumed
        s.poll(a)
    assert e.value.code == abi.PT_ERR_NOT_FOUND
    png = _decode_png(s.fetch_encoded(b, abi.PT_IMAGE_PNG))
    with pytest.raises(native.PhotonError) as e:
        s.fetch_encoded(plain_only, abi.PT_IMAGE_PNG)
    assert e.value.code == abi.PT_ERR_INVALID
    img_c, _ = s.fetch(plain_only, w, h)
    s.close()
    r = native.Renderer()
    r.upload(tdesc)
    r.resize(w, h)
    rs = abi.RenderSettings(w, h, path, 1.5, abi.PT_TONEMAP_REINHARD, seed)
    r.render(cam, rs, spp)
    img = r.download_image()
    r.display(rs, abi.PT_DISPLAY_COLOR)
    disp = r.download_display()
    r.close()
    assert np.array_equal(img.view(np.uint32), img_c.view(np.uint32))
    assert pfm == native.encode_pfm(img)
    assert np.array_equal(png, disp)


def test_server_sessions_equal_render_denoised_alone_and_under_load(server_scenes):
    """Real-time SVGF sessions served as a request class: each frame (one path per pixel, G-buffer,
    SVGF with the session's history) fetched from the server equals the same frame sequence through a
    renderer's pt_render_denoised, bit for bit. This holds for a session alone, and for frames
    submitted all at once (they run one at a time, in order) while ordinary requests flood the server
    and share its path pool. Closing a session cancels its waiting frames, and the server's memory in
    use returns to idle."""
    from photon_b200 import workloads
    _, (tdesc, tcam, tkeep) = server_scenes
    w, h, frames = 128, 72, 4
    cams = workloads.orbit_cameras(tdesc, frames, w / h)
    prev = [cams[max(f - 1, 0)] for f in range(frames)]
    rs = abi.render_settings(w, h, max_depth=12, seed=11)
    sv = abi.svgf_settings()
    r = native.Renderer()
    r.upload(tdesc)
    r.resize(w, h)
    want = []
    for f in range(frames):
        r.render_denoised(cams[f], prev[f], rs, sv)
        want.append(r.download_image())
    r.close()
    s = native.Server(budget_bytes=8 << 30, path_capacity=1 << 18, max_active=2)
    scene = s.add_scene(tdesc)
    idle = s.stats().device_bytes_in_use
    ses = s.open_session(scene, w, h, sv)
    assert s.stats().device_bytes_in_use > idle
    for f in range(frames):
        rid = s.submit_frame(ses, cams[f], prev[f], rs)
        s.wait(rid, 60)
        img, st = s.fetch(rid, w, h)
        assert st.state == abi.PT_REQ_DONE
        assert np.array_equal(img.view(np.uint32), want[f].view(np.uint32)), f"frame {f} alone"
    s.close_session(ses)
    ses = s.open_session(scene, w, h, sv)
    load = [s.submit(scene, tcam(1.0), 192, 108, 8, seed=100 + k, path=abi.path_options(max_depth=12)) for k in range(10)]
    rids = [s.submit_frame(ses, cams[f], prev[f], rs) for f in range(frames)]
    for f, rid in enumerate(rids):
        s.wait(rid, 120)
        img, _ = s.fetch(rid, w, h)
        assert np.array_equal(img.view(np.uint32), want[f].view(np.uint32)), f"frame {f} under load"
    for rid in load:
        s.wait(rid, 120)
        s.fetch(rid, 192, 108)
    s.close_session(ses)
    ses = s.open_session(scene, w, h, sv)
    queued = [s.submit_frame(ses, cams[f], prev[f], rs) for f in range(frames)]
    s.close_session(ses)
    states = []
    for rid in queued:
        try:
            s.wait(rid, 60)
        except native.PhotonError as e:
            assert e.code == abi.PT_ERR_CANCELLED
        states.append(s.poll(rid))
        try:
            s.fetch(rid, w, h)
        except native.PhotonError:
            pass
    assert states[-1] == abi.PT_REQ_CANCELLED and set(states) <= {abi.PT_REQ_DONE, abi.PT_REQ_CANCELLED}
    with pytest.raises(native.PhotonError) as e:
        s.submit_frame(ses, cams[0], prev[0], rs)
    assert e.value.code == abi.PT_ERR_NOT_FOUND
    deadline = time.time() + 30
    while s.stats().device_bytes_in_use != idle and time.time() < deadline:
        time.sleep(0.05)
    assert s.stats().device_bytes_in_use == idle
    s.close()
