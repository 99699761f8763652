"""Photon's own GPU tests (tests/test_gpu.cpp of Photon: gpu_matches_cpu,
gpu_progressive_accumulation_converges, svgf_reduces_error, svgf_handles_camera_motion), compiled
unchanged against the drop-in header include/photon_dropin/render/gpu_renderer.h and this library
(oracle/Makefile target dropin-tests), run as a subprocess (gpu)."""
import os
import subprocess

import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(O.REF_SO), "photon_tests_dropin")


@pytest.mark.skipif(not os.path.exists(BIN), reason="the drop-in test binary is not built")
def test_photon_gpu_tests_pass_against_the_drop_in():
    r = subprocess.run([BIN, "-v", "gpu", "svgf"], capture_output=True, text=True, timeout=600)
    print(r.stdout[-3000:])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "4 passed, 0 failed, 0 skipped" in r.stdout
