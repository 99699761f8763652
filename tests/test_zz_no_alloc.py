"""The allocation-free SVGF entry point (pt_svgf_run_noalloc), through the C ABI, for callers that
cannot allocate device memory. Its output is checked against the allocating entry point (the first
frame of a fresh pt_svgf session: the same kernels on the same G-buffers) and against the oracle's
restatement of Photon's Svgf::run on its first frame, within the SVGF tolerance
(|a - b| <= 1e-4 * max(|b|, 1e-2) per channel) on every pixel. Two calls in a row on different frames
check that the shared static scratch carries nothing from one call to the next. Collected last so it
also runs after every other test has used the device."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from photon_b200 import abi, native
import scenes

pytestmark = pytest.mark.gpu
REL = 1e-4
FLOOR = 1e-2
NAMES = ("color", "albedo", "normal_depth", "position", "emission")


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for torch")
    return torch


def _gbuffers(w, h, frames):
    desc, camf, keep = scenes.scene("cornell")
    rs = abi.render_settings(w, h, seed=5)
    out = []
    for k in range(frames):
        cam = camf(w / h)
        cam.position.x += 0.07 * k
        out.append(O.orc_gbuffer(desc, cam, rs, frame=k))
    return out, camf(w / h), keep


def _allocating(torch, dev, w, h, settings, cam):
    s = native.Svgf(w, h)
    out = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
    s.run(*(dev[n].data_ptr() for n in NAMES), cam, settings, out.data_ptr())
    torch.cuda.synchronize()
    s.close()
    return out.cpu().numpy()


@pytest.mark.parametrize("iterations", [5, 0])
def test_noalloc_matches_session_first_frame(torch_cuda, iterations):
    torch = torch_cuda
    w, h = 96, 64
    gbufs, cam, keep = _gbuffers(w, h, 2)
    settings = abi.svgf_settings()
    settings.atrous_iterations = iterations
    stream = torch.cuda.current_stream().cuda_stream
    for g in gbufs:  # two calls in a row, different inputs
        dev = {n: torch.from_numpy(g[n]).cuda() for n in NAMES}
        out = torch.full((h, w, 4), float("nan"), dtype=torch.float32, device="cuda")
        native.svgf_run_noalloc(w, h, *(dev[n].data_ptr() for n in NAMES), settings, out.data_ptr(), stream=stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = _allocating(torch, dev, w, h, settings, cam)
        assert np.isfinite(got).all()
        err = np.abs(got - want) / np.maximum(np.abs(want), FLOOR)
        assert float(err.max()) <= REL, f"max relative error {float(err.max()):.3g} against pt_svgf_run"
        # The oracle: a fresh restatement session's first frame (no history to reproject).
        oracle = O.OrcSvgf(w, h).run(g, cam, settings)
        err = np.abs(got - oracle) / np.maximum(np.abs(oracle), FLOOR)
        assert float(err.max()) <= REL, f"max relative error {float(err.max()):.3g} against the oracle"


def test_noalloc_rejects_frames_above_the_scratch(torch_cuda):
    torch = torch_cuda
    buf = torch.zeros(4, dtype=torch.float32, device="cuda")
    p = buf.data_ptr()
    settings = abi.svgf_settings()
    with pytest.raises(native.PhotonError, match="524288"):
        native.svgf_run_noalloc(1024, 513, p, p, p, p, p, settings, p)
    with pytest.raises(native.PhotonError):
        native.svgf_run_noalloc(0, 16, p, p, p, p, p, settings, p)
