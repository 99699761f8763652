"""Photon's own megakernel (src/render/gpu_renderer.cu, built unchanged for sm_100a with Photon's flags
into oracle/_ref) on the same GPU (gpu): how closely it agrees with the CPU oracle (the calibration of
the parity bar), and its throughput next to the wavefront's on the 262,144-triangle 1080p, 16 spp,
depth-12 frame (8-spp launches after a 4-spp warm-up, as `photon bench` runs it)."""
import ctypes as C
import json
import threading
import os
import time

import numpy as np
import pytest

from conftest import pixel_agreement
from oracle import oracle as O
from photon_b200 import abi, native
import scenes

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not os.path.exists(O.REF_GPU_SO), reason="Photon's CUDA build not present")]


@pytest.fixture(scope="module")
def L():
    lib = O.reference_gpu()
    if not lib.refgpu_available():
        pytest.skip("no device for Photon's renderer")
    return lib


@pytest.mark.parametrize("name", ["cornell", "materials", "glass"])
def test_photon_megakernel_agreement_with_oracle(L, name):
    s = O.RefScene.builtin(name, lib=L)
    w, h, spp = 96, 54, 64
    cam = s.camera(w / h)
    rs = abi.render_settings(w, h)
    g = L.refgpu_create()
    try:
        assert L.refgpu_upload(g, s.h)
        L.refgpu_resize(g, w, h)
        for _ in range(spp // 16):
            L.refgpu_render(g, C.byref(cam), C.byref(rs), 16)
        img = np.zeros((h, w, 3), np.float32)
        L.refgpu_download_image(g, img)
    finally:
        L.refgpu_destroy(g)
    ref = O.orc_render(s.desc, cam, rs, spp)
    frac, mr, mg = pixel_agreement(ref, img)
    print(f"Photon megakernel vs CPU, {name}: {100 * frac:.2f}% of pixels within 1e-3, means {mr:.5f} / {mg:.5f}")
    assert frac > 0.9  # Photon's own bar (tests/test_gpu.cpp:67)


def test_throughput_vs_photon_megakernel(L):
    desc, camf, keep = scenes.scene("terrain")
    W, H, SPP = 1920, 1080, 16
    cam = camf(W / H)
    rs = abi.render_settings(W, H, max_depth=12, seed=1)
    ref_scene = O.RefScene.from_desc(desc, lib=L)
    g = L.refgpu_create()
    try:
        assert L.refgpu_upload(g, ref_scene.h)
        L.refgpu_resize(g, W, H)
        L.refgpu_render(g, C.byref(cam), C.byref(rs), 4)
        L.refgpu_reset(g)
        mk_ms = 0.0
        t0 = time.perf_counter()
        for _ in range(SPP // 8):
            mk_ms += L.refgpu_render(g, C.byref(cam), C.byref(rs), 8)
        mk_wall = time.perf_counter() - t0
    finally:
        L.refgpu_destroy(g)
    r = native.Renderer()
    r.upload(desc)
    r.resize(W, H)
    r.render(cam, rs, SPP)
    r.reset()
    t0 = time.perf_counter()
    r.render(cam, rs, SPP)
    wf_wall = time.perf_counter() - t0
    wf_ms = r.last_frame_ms
    r.close()
    samples = W * H * SPP
    rec = {"megakernel_msamples_per_s": samples / (mk_ms / 1000) / 1e6, "megakernel_wall_msamples_per_s": samples / mk_wall / 1e6,
           "wavefront_msamples_per_s": samples / (wf_ms / 1000) / 1e6, "wavefront_wall_msamples_per_s": samples / wf_wall / 1e6}
    rec["speedup"] = rec["wavefront_msamples_per_s"] / rec["megakernel_msamples_per_s"]
    print("MEGAKERNEL_COMPARISON " + json.dumps(rec))
    assert rec["speedup"] > 1.0


def test_batched_views_vs_photon_megakernel(L):
    # The 64-view batched workload: one wavefront over every view, against Photon's megakernel
    # rendering each view (8-spp launches, as `photon bench`).
    from photon_b200 import workloads
    desc, camf, keep = scenes.scene("terrain")
    views = workloads.batch_views(desc, 64, seed=2)
    total = sum(v.width * v.height * v.spp for v in views)
    r = native.Renderer()
    r.upload(desc)
    r.render_views(views)
    t0 = time.perf_counter()
    r.render_views(views)
    wf = time.perf_counter() - t0
    r.close()
    ref_scene = O.RefScene.from_desc(desc, lib=L)
    g = L.refgpu_create()
    try:
        assert L.refgpu_upload(g, ref_scene.h)
        L.refgpu_resize(g, 64, 64)
        L.refgpu_render(g, C.byref(views[0].camera), C.byref(abi.render_settings(64, 64, max_depth=12)), 4)
        t0 = time.perf_counter()
        for v in views:
            L.refgpu_resize(g, v.width, v.height)
            L.refgpu_reset(g)
            rs = abi.RenderSettings(v.width, v.height, v.path, 1.0, abi.PT_TONEMAP_ACES, v.seed)
            done = 0
            while done < v.spp:
                k = min(8, v.spp - done)
                L.refgpu_render(g, C.byref(v.camera), C.byref(rs), k)
                done += k
        mk = time.perf_counter() - t0
    finally:
        L.refgpu_destroy(g)
    rec = {"batched_msamples_per_s": total / wf / 1e6, "megakernel_msamples_per_s": total / mk / 1e6, "speedup": mk / wf}
    print("BATCHED_VS_MEGAKERNEL " + json.dumps(rec))
    assert rec["speedup"] > 1.0


def test_realtime_sessions_vs_photon(L):
    """Real-time frames (1 spp + G-buffer + SVGF) on an orbit of the 262K scene at 1600x900: one
    session through pt_render_denoised against Photon's GpuRenderer::render_denoised (megakernel +
    svgf.cu); SVGF alone, ours against svgf.cu, on identical G-buffers; and eight concurrent sessions
    (host threads) of each. Frame times are wall clock of the synchronous calls; percentiles over the
    orbit's frames."""
    import torch
    from photon_b200 import workloads
    desc, camf, keep = scenes.scene("terrain")
    W, H, N = 1600, 900, 40
    cams = workloads.orbit_cameras(desc, N + 3, W / H)
    rs = abi.render_settings(W, H, max_depth=12, seed=11)
    sv = abi.svgf_settings()

    def frame_times(step):
        for f in range(3):
            step(cams[f], cams[max(f - 1, 0)])
        ts = []
        for f in range(3, N + 3):
            t0 = time.perf_counter()
            step(cams[f], cams[f - 1])
            ts.append((time.perf_counter() - t0) * 1e3)
        return np.percentile(ts, 50), np.percentile(ts, 99)

    r = native.Renderer()
    r.upload(desc)
    r.resize(W, H)
    ours = frame_times(lambda c, p: r.render_denoised(c, p, rs, sv))
    r.close()
    ref_scene = O.RefScene.from_desc(desc, lib=L)
    g = L.refgpu_create()
    try:
        assert L.refgpu_upload(g, ref_scene.h)
        L.refgpu_resize(g, W, H)
        theirs = frame_times(lambda c, p: L.refgpu_render_denoised(g, C.byref(c), C.byref(p), C.byref(rs), C.byref(sv)))
    finally:
        L.refgpu_destroy(g)
    # SVGF alone on identical G-buffers (the oracle's first-vertex G-buffer of the first orbit frame).
    gb = O.orc_gbuffer(desc, cams[0], abi.render_settings(W, H, seed=2), frame=0)
    names = ("color", "albedo", "normal_depth", "position", "emission")
    dev = {n: torch.from_numpy(gb[n]).cuda() for n in names}
    out = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    ptrs = [dev[n].data_ptr() for n in names]

    def device_ms(run, n=20):
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    ours_sv = native.Svgf(W, H)
    svgf_ours = device_ms(lambda: ours_sv.run(*ptrs, cams[0], sv, out.data_ptr()))
    ours_sv.close()
    ref = L.refsvgf_create(W, H)
    try:
        svgf_theirs = device_ms(lambda: L.refsvgf_run(ref, *ptrs, C.byref(cams[0]), C.byref(sv), out.data_ptr()))
    finally:
        L.refsvgf_destroy(ref)
    # Eight concurrent sessions (host threads), 30 frames each, 45 degrees apart on the orbit.
    from photon_b200 import sessions
    ours8 = sessions.run_sessions(desc, 8, 30, W, H)
    lat = [[] for _ in range(8)]
    gs = []
    try:
        for k in range(8):
            gk = L.refgpu_create()
            gs.append(gk)
            assert L.refgpu_upload(gk, ref_scene.h)
            L.refgpu_resize(gk, W, H)
        orbits = [workloads.orbit_cameras(desc, 33, W / H, start_deg=45.0 * k) for k in range(8)]
        barrier = threading.Barrier(9)

        def photon_session(k):
            cs = orbits[k]
            for f in range(3):
                L.refgpu_render_denoised(gs[k], C.byref(cs[f]), C.byref(cs[max(f - 1, 0)]), C.byref(rs), C.byref(sv))
            barrier.wait()
            for f in range(3, 33):
                t0 = time.perf_counter()
                L.refgpu_render_denoised(gs[k], C.byref(cs[f]), C.byref(cs[f - 1]), C.byref(rs), C.byref(sv))
                lat[k].append((time.perf_counter() - t0) * 1e3)

        threads = [threading.Thread(target=photon_session, args=(k,)) for k in range(8)]
        for t in threads:
            t.start()
        barrier.wait()
        t0 = time.perf_counter()
        for t in threads:
            t.join()
        wall = time.perf_counter() - t0
    finally:
        for gk in gs:
            L.refgpu_destroy(gk)
    all_lat = np.concatenate([np.asarray(x) for x in lat])
    rec = {"frame_p50_ms": ours[0], "frame_p99_ms": ours[1], "photon_frame_p50_ms": theirs[0], "photon_frame_p99_ms": theirs[1],
           "svgf_ms": svgf_ours, "photon_svgf_ms": svgf_theirs,
           "sessions8_p50_ms": ours8["p50_ms"], "sessions8_p99_ms": ours8["p99_ms"], "sessions8_frames_per_s": ours8["frames_per_s"],
           "photon_sessions8_p50_ms": float(np.percentile(all_lat, 50)), "photon_sessions8_p99_ms": float(np.percentile(all_lat, 99)),
           "photon_sessions8_frames_per_s": all_lat.size / wall}
    print("REALTIME_VS_PHOTON " + json.dumps(rec))
    assert svgf_ours < svgf_theirs
