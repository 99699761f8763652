"""Photon's own megakernel (src/render/gpu_renderer.cu, built unchanged for sm_100a with Photon's flags
into oracle/_ref) on the same GPU (gpu): how closely it agrees with the CPU oracle (the calibration of
the parity bar), and its throughput next to the wavefront's on the 262,144-triangle 1080p, 16 spp,
depth-12 frame (8-spp launches after a 4-spp warm-up, as `photon bench` runs it)."""
import ctypes as C
import json
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
