"""Display / tone-map parity (gpu): the wavefront's display kernel (pt_display) against Photon's own
display_kernel (gpu_renderer.cu:129-175, compiled unchanged with Photon's --use_fast_math flags into
oracle/_ref/libphoton_ref_gpu.so) on one accumulation, G-buffer and heat map of a render, for every
display mode, every tone map and two exposures; and the denoised colour view on a denoised frame.

Both device kernels are also measured against the same mapping evaluated on the host with Photon's
own host-compiled colour functions (color.h:8-41, oracle ref_display_cpu). The bar is Photon's own
agreement with its host mapping: Photon's fast-math powf and division move some 8-bit channels by one
step, so for every case the wavefront's largest channel difference from the host mapping may be no
larger than Photon's (and at most one step), its fraction of bit-identical pixels no lower, and its
largest difference from Photon's device output at most max(1, Photon's own largest difference)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from photon_b200 import abi, native
import scenes

pytestmark = pytest.mark.gpu
MODES = {abi.PT_DISPLAY_COLOR: "color", abi.PT_DISPLAY_ALBEDO: "albedo", abi.PT_DISPLAY_NORMAL: "normal",
         abi.PT_DISPLAY_DEPTH: "depth", abi.PT_DISPLAY_VARIANCE: "variance", abi.PT_DISPLAY_HEATMAP: "heatmap"}
TONEMAPS = (abi.PT_TONEMAP_LINEAR, abi.PT_TONEMAP_ACES, abi.PT_TONEMAP_REINHARD)


@pytest.fixture(scope="module")
def libs():
    if not O.reference_available():
        pytest.skip("Photon reference build not present")
    L = O.reference_gpu()
    if not L.refgpu_available():
        pytest.skip("Photon's CUDA build reports no device")
    f = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int] + [C.c_void_p] * 7
    L.refgpu_display_buffers.argtypes = f
    L.refgpu_display_buffers.restype = C.c_int
    L.ref_display_cpu.argtypes = f
    L.ref_display_cpu.restype = None
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


def _photon(L, fn, w, h, mode, rs, samples, max_depth, denoised, bufs):
    out = np.zeros((h, w), np.uint32)
    args = (w, h, mode, rs.exposure, rs.tonemap, float(samples), max_depth, 1.0 / 160.0, denoised,
            *(_ptr(bufs.get(k)) for k in ("accum", "denoised", "albedo", "nd", "variance", "heat")), out.ctypes.data)
    r = fn(*args)
    assert r in (None, 1), "Photon's display launch failed"
    return out


def _channels(px):
    return np.stack([(px >> s) & 0xFF for s in (0, 8, 16, 24)], axis=-1).astype(np.int32)


def _compare(ours, gpu, cpu, label):
    o, g, c = _channels(ours), _channels(gpu), _channels(cpu)
    d_gc, d_oc, d_og = np.abs(g - c).max(), np.abs(o - c).max(), np.abs(o - g).max()
    ex_gc = float((g == c).all(axis=-1).mean())
    ex_oc = float((o == c).all(axis=-1).mean())
    assert d_oc <= max(1, d_gc) and d_oc <= 1, f"{label}: ours vs host mapping {d_oc} steps (Photon's device: {d_gc})"
    assert ex_oc >= ex_gc, f"{label}: {ex_oc:.5f} of pixels bit-identical to the host mapping (Photon's device: {ex_gc:.5f})"
    assert d_og <= max(1, d_gc), f"{label}: ours vs Photon's display_kernel {d_og} steps"
    return ex_oc, ex_gc


def _extent(desc):
    d = np.array([desc.bounds_max.x - desc.bounds_min.x, desc.bounds_max.y - desc.bounds_min.y, desc.bounds_max.z - desc.bounds_min.z],
                 np.float32)
    return float(max(np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])), np.float32(1e-3)))


def test_display_modes_and_tone_maps_match_photon(libs):
    desc, camf, keep = scenes.scene("terrain")
    w, h, spp = 160, 90, 8
    cam = camf(w / h)
    r = native.Renderer()
    r.upload(desc)
    r.resize(w, h)
    rs = abi.render_settings(w, h, max_depth=12, seed=4)
    r.render(cam, rs, spp)
    albedo, nd = r.download_gbuffer()
    bufs = {"accum": r.download_accumulation(), "albedo": albedo, "nd": nd, "heat": r.heatmap(cam, w, h)}
    assert np.isfinite(bufs["accum"]).all() and bufs["accum"][..., 3].max() > 0
    ext = _extent(desc)
    seen = []
    for mode in MODES:
        for tm in (TONEMAPS if mode == abi.PT_DISPLAY_COLOR else (abi.PT_TONEMAP_ACES,)):
            for exposure in ((1.0, 2.5) if mode == abi.PT_DISPLAY_COLOR else (1.0,)):
                rs.tonemap, rs.exposure = tm, exposure
                r.display(rs, mode)
                ours = r.download_display()
                gpu = _photon(libs, libs.refgpu_display_buffers, w, h, mode, rs, spp, ext, 0, bufs)
                cpu = _photon(libs, libs.ref_display_cpu, w, h, mode, rs, spp, ext, 0, bufs)
                seen.append(_compare(ours, gpu, cpu, f"{MODES[mode]} tonemap {tm} exposure {exposure}"))
    r.close()
    # The views are not trivial: most pixels of every case agree exactly with the host mapping.
    assert min(e for e, _ in seen) > 0.9


def test_denoised_colour_view_matches_photon(libs):
    desc, camf, keep = scenes.scene("terrain")
    w, h = 128, 72
    cams = [camf(w / h) for _ in range(2)]
    cams[1].position.x += 0.05
    r = native.Renderer()
    r.upload(desc)
    r.resize(w, h)
    rs = abi.render_settings(w, h, max_depth=12, seed=6)
    sv = abi.svgf_settings()
    r.render_denoised(cams[0], cams[0], rs, sv)
    r.render_denoised(cams[1], cams[0], rs, sv)
    den = r.download_image()
    bufs = {"denoised": np.concatenate([den, np.zeros((h, w, 1), np.float32)], axis=-1)}
    for tm in TONEMAPS:
        rs.tonemap, rs.exposure = tm, 1.0
        r.display(rs, abi.PT_DISPLAY_COLOR)
        ours = r.download_display()
        gpu = _photon(libs, libs.refgpu_display_buffers, w, h, 0, rs, 1, 1.0, 1, bufs)
        cpu = _photon(libs, libs.ref_display_cpu, w, h, 0, rs, 1, 1.0, 1, bufs)
        _compare(ours, gpu, cpu, f"denoised colour, tonemap {tm}")
    r.close()
