"""SVGF parity (gpu): the CUDA denoiser against the oracle's C restatement and against Photon's own
svgf.cu (compiled from its sources into oracle/_ref) on identical G-buffers, frame after frame with a
moving camera; and Photon's own SVGF tests (tests/test_gpu.cpp:105-164) through pt_render_denoised.

Tolerance: outputs agree within 1e-4 relative (|a - b| <= 1e-4 * max(|b|, 1e-2) per channel) —
on every pixel against the restatement (same precise expf/powf), and on >= 99.9% of pixels against
svgf.cu, which Photon builds with --use_fast_math (approximate expf/powf/division).

svgf.cu is compared on the frames before a pixel's history reaches 4 frames: at that frame its
variance estimate switches from the spatial to the temporal one (svgf.cu:101, `len < 4`), and the
history length is exactly 4 in exact arithmetic, so the branch is decided by the last bit of
`hist_len / wsum + 1` — which fast-math division and IEEE division round differently. From then on
the two images legitimately differ; the restatement (IEEE, like this kernel) is compared on every
frame."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from photon_b200 import abi, native
import scenes

pytestmark = pytest.mark.gpu
REL = 1e-4
FLOOR = 1e-2
SWITCH_FRAME = 3  # history length 4 (the variance switch) is reached at frame index 3


def rel_err(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), FLOOR)


def moving_cameras(camf, w, h, n, step=0.05):
    cams = []
    for k in range(n):
        c = camf(w / h)
        c.position.x += step * k
        cams.append(c)
    return cams


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


def _frames(name, w, h, n):
    desc, camf, keep = scenes.scene(name)
    cams = moving_cameras(camf, w, h, n)
    rs = abi.render_settings(w, h, seed=2)
    gbufs = [O.orc_gbuffer(desc, c, rs, frame=k) for k, c in enumerate(cams)]
    return cams, gbufs, keep


def _run_device(torch, run, cams, gbufs, w, h):
    outs = []
    for k, g in enumerate(gbufs):
        dev = {n: torch.from_numpy(a).cuda() for n, a in g.items()}
        out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        prev = cams[k - 1] if k > 0 else cams[0]
        run(dev, prev, out)
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    return outs


@pytest.mark.parametrize("name", ["cornell", "materials"])
def test_svgf_matches_restatement_and_photon(torch_cuda, name):
    torch = torch_cuda
    w, h, n = 96, 64, 5
    cams, gbufs, keep = _frames(name, w, h, n)
    settings = abi.svgf_settings()
    # Ours, through the C ABI.
    ours = native.Svgf(w, h)
    got = _run_device(torch, lambda d, prev, out: ours.run(d["color"].data_ptr(), d["albedo"].data_ptr(), d["normal_depth"].data_ptr(),
                                                          d["position"].data_ptr(), d["emission"].data_ptr(), prev, settings,
                                                          out.data_ptr()), cams, gbufs, w, h)
    # The restatement on the host.
    orc = O.OrcSvgf(w, h)
    want = [orc.run(g, cams[k - 1] if k else cams[0], settings) for k, g in enumerate(gbufs)]
    for k in range(n):
        e = rel_err(got[k], want[k])
        print(f"{name} frame {k}: max rel err vs restatement {e.max():.2e}")
        assert (e <= REL).all()
    # Photon's svgf.cu (fast math).
    if not __import__("os").path.exists(O.REF_GPU_SO):
        pytest.skip("Photon's CUDA build not present")
    L = O.reference_gpu()
    ref = L.refsvgf_create(w, h)
    try:
        theirs = _run_device(torch, lambda d, prev, out: L.refsvgf_run(ref, d["color"].data_ptr(), d["albedo"].data_ptr(),
                                                                      d["normal_depth"].data_ptr(), d["position"].data_ptr(),
                                                                      d["emission"].data_ptr(), C.byref(prev), C.byref(settings),
                                                                      out.data_ptr()), cams, gbufs, w, h)
    finally:
        L.refsvgf_destroy(ref)
    for k in range(SWITCH_FRAME):
        e = rel_err(got[k], theirs[k])
        frac = float((e <= REL).all(axis=-1).mean())
        print(f"{name} frame {k}: {100 * frac:.3f}% of pixels within 1e-4 of svgf.cu, max rel err {e.max():.2e}")
        assert frac >= 0.999


def _mse(a, b):
    lum = np.array([0.2126, 0.7152, 0.0722], np.float32)
    return float(np.mean((np.minimum(a @ lum, 1.0) - np.minimum(b @ lum, 1.0)) ** 2))


def test_svgf_reduces_error():
    # tests/test_gpu.cpp:105-139 on the Cornell box at 160x160.
    desc, camf, keep = scenes.scene("cornell")
    w = h = 160
    cam = camf(1.0)
    rs = abi.render_settings(w, h)
    r = native.Renderer()
    r.upload(desc)
    r.resize(w, h)
    for _ in range(2048 // 256):
        r.render(cam, rs, 256)
    ref = r.download_image()
    r.reset()
    r.render(cam, rs, 1)
    noisy = r.download_image()
    sv = abi.svgf_settings()
    r.reset()
    r.render_denoised(cam, cam, rs, sv)
    first = r.download_image()
    for _ in range(1, 16):
        r.render_denoised(cam, cam, rs, sv)
    settled = r.download_image()
    e_noisy, e_first, e_settled = _mse(noisy, ref), _mse(first, ref), _mse(settled, ref)
    print(f"MSE: 1 spp {e_noisy:.5f}, SVGF frame 1 {e_first:.5f}, frame 16 {e_settled:.5f}")
    assert e_first < 0.5 * e_noisy
    assert e_settled < e_first
    assert np.isfinite(settled).all() and settled.min() >= 0
    lum = np.array([0.2126, 0.7152, 0.0722], np.float32)
    assert abs((settled @ lum).mean() - (ref @ lum).mean()) < 0.05 * (ref @ lum).mean()
    r.close()


def test_svgf_handles_camera_motion():
    # tests/test_gpu.cpp:141-164: the materials scene, 20 frames of a moving camera.
    desc, camf, keep = scenes.scene("materials")
    w, h = 128, 72
    r = native.Renderer()
    r.upload(desc)
    r.resize(w, h)
    rs = abi.render_settings(w, h)
    sv = abi.svgf_settings()
    cams = moving_cameras(camf, w, h, 21)
    for f in range(1, 21):
        r.render_denoised(cams[f], cams[f - 1], rs, sv)
    img = r.download_image()
    assert np.isfinite(img).all() and img.min() >= 0
    lum = np.array([0.2126, 0.7152, 0.0722], np.float32)
    assert (img @ lum).mean() > 0.05
    r.close()


def test_denoised_gbuffer_is_the_oracle_sample(torch_cuda):
    # The real-time sample's G-buffer (sample_kernel, gpu_renderer.cu:83-95) equals the oracle's.
    desc, camf, keep = scenes.scene("glass")
    w, h = 64, 48
    cam = camf(w / h)
    rs = abi.render_settings(w, h, seed=4)
    r = native.Renderer()
    r.upload(desc)
    r.resize(w, h)
    r.render_denoised(cam, cam, rs, abi.svgf_settings())
    albedo, nd = r.download_gbuffer()
    g = O.orc_gbuffer(desc, cam, rs, frame=0)
    assert np.array_equal(albedo.view(np.uint32), g["albedo"].view(np.uint32))
    assert np.array_equal(nd.view(np.uint32), g["normal_depth"].view(np.uint32))
    r.close()


@pytest.mark.parametrize("w,h,iterations", [(101, 67, 5), (96, 64, 6), (40, 24, 3)])
def test_tma_staged_passes_equal_direct_loads(torch_cuda, w, h, iterations):
    """The a-trous passes that read TMA-staged shared-memory tiles (contiguous or strided) compute
    exactly what the global-load passes compute: outputs are bit-identical frame after frame in every
    staging mode, on sizes that are not multiples of the tile grid and with a pass beyond the staged
    steps."""
    torch = torch_cuda
    cams, gbufs, keep = _frames("materials", w, h, 4)
    settings = abi.svgf_settings()
    settings.atrous_iterations = iterations
    outs = []
    for mode in (0, 1, 2, 3):
        sv = native.Svgf(w, h)
        sv.set_tma(mode)
        outs.append(_run_device(torch, lambda d, prev, out: sv.run(d["color"].data_ptr(), d["albedo"].data_ptr(), d["normal_depth"].data_ptr(),
                                                                   d["position"].data_ptr(), d["emission"].data_ptr(), prev, settings,
                                                                   out.data_ptr()), cams, gbufs, w, h))
        sv.close()
    for staged in outs[1:]:
        for a, b in zip(staged, outs[0]):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_tma_tile_wait_timeout_is_reported(torch_cuda):
    """The TMA-staged passes wait for their tiles with a bounded wait. A test hook arms each tile's
    barrier without issuing its copies and shortens the wait to 2 us, so every staged pass's wait runs
    out with nothing in flight (nothing can land late). The call after that frame reports PT_ERR_CUDA;
    with the hook off, the same session denoises again, bit-identical to a fresh session."""
    torch = torch_cuda
    w, h = 96, 64
    cams, gbufs, keep = _frames("cornell", w, h, 2)
    settings = abi.svgf_settings()
    dev = {n: torch.from_numpy(a).cuda() for n, a in gbufs[0].items()}
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")

    def run(sv):
        sv.run(dev["color"].data_ptr(), dev["albedo"].data_ptr(), dev["normal_depth"].data_ptr(), dev["position"].data_ptr(),
               dev["emission"].data_ptr(), cams[0], settings, out.data_ptr())
        torch.cuda.synchronize()
        return out.cpu().numpy()

    fresh = native.Svgf(w, h)
    want = run(fresh)
    fresh.close()
    sv = native.Svgf(w, h)
    sv.set_tma(1)  # steps 1-8 staged through TMA tiles
    sv.debug_tma_timeout(True)
    run(sv)  # every staged pass times out here; the flag is read by the next call
    with pytest.raises(native.PhotonError) as e:
        run(sv)
    assert e.value.code == abi.PT_ERR_CUDA
    sv.debug_tma_timeout(False)
    sv.reset()
    got = run(sv)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    sv.close()
