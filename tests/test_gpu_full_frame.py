"""Parity at the benchmark's full size: the 262,144-triangle terrain at 1920x1080, depth 12, the
frame bench.py times (one sample per pixel here, so that Photon's CPU renderer finishes in about a
second on the host cores). Primary hits must equal Photon's bit for bit over all 2,073,600 pixels,
and the image must meet the parity bar against Photon's own CPU renderer (built from its sources)."""
import os

import numpy as np
import pytest

from conftest import pixel_agreement
from oracle import oracle as O
from photon_b200 import abi, native

pytestmark = pytest.mark.gpu
W, H, TRIS, SEED, DEPTH = 1920, 1080, 262144, 1, 12


@pytest.fixture(scope="module")
def frame():
    if not O.reference_available():
        pytest.skip("Photon's CPU build (oracle/_ref) is missing")
    g = native.terrain_scene(TRIS, SEED)
    b = g.build()
    ref = O.RefScene.from_desc(b.desc)
    return g, b, ref


def test_full_frame_primary_hits_equal_photons(frame):
    """Both closest-hit walks: the pair walk of the default kernels and the per-lane walk."""
    g, b, ref = frame
    cam = g.camera(W / H)
    theirs = ref.trace_primary(cam, W, H, 0, SEED)
    r = native.Renderer()
    r.upload(b.desc)
    for pair_walk in (5, 0):
        r.set_tuning(pair_walk=pair_walk)
        ours = r.trace_primary(cam, W, H, 0, SEED)
        assert np.array_equal(ours.view(np.uint32), theirs.view(np.uint32)), f"pair_walk={pair_walk}"
    r.close()
    assert (O.hits_tri(ours) >= 0).mean() > 0.3


def test_full_frame_image_meets_the_parity_bar(frame):
    g, b, ref = frame
    cam = g.camera(W / H)
    rs = abi.render_settings(W, H, max_depth=DEPTH, seed=SEED)
    r = native.Renderer()
    r.upload(b.desc)
    r.resize(W, H)
    r.render(cam, rs, 1)
    ours = r.download_image()
    r.close()
    theirs, _ = ref.render(cam, rs, 1, threads=os.cpu_count() or 1)
    frac, m_ref, m_ours = pixel_agreement(theirs, ours)
    exact = float((ours.view(np.uint32) == theirs.view(np.uint32)).all(axis=-1).mean())
    print(f"1920x1080: {100 * frac:.4f}% of pixels within 1e-3, {100 * exact:.3f}% bit-identical")
    assert frac >= 0.999
    assert abs(m_ref - m_ours) <= 0.01 * m_ref
