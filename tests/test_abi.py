"""The C-ABI library: it loads, exports every entry point include/photon_wavefront.h declares, and its
structures have Photon's byte layouts. Runs without a GPU (no compute call)."""
import ctypes as C
import os
import re
import subprocess

from conftest import ROOT
from photon_b200 import abi, native

HEADER = os.path.join(ROOT, "include", "photon_wavefront.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("pt_create", "pt_destroy", "pt_upload_scene", "pt_update_lights", "pt_resize", "pt_reset", "pt_render",
                 "pt_render_denoised", "pt_display", "pt_download_image", "pt_download_display", "pt_server_submit",
                 "pt_svgf_run", "pt_render_views"):
        assert must in names


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (pt_[a-z0-9_]+)", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing
    for n in declared_functions():
        assert hasattr(native.lib, n)


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) == set(native.SIGNATURES)


def test_struct_layouts_match_photon():
    for t, size in abi.EXPECTED_SIZES.items():
        assert C.sizeof(t) == size, t.__name__
    assert abi.Material.alpha_cutoff.offset == 48
    assert abi.Material.occlusion_tex.offset == 76
    assert abi.BvhNode.rcount.offset == 60
    assert abi.Camera.focus_distance.offset == 60


def test_abi_version_and_no_device_errors():
    assert native.lib.pt_abi_version() == 1
    if native.device_info() is None:
        # Without a device the library reports it instead of falling back.
        h = C.c_void_p()
        assert native.lib.pt_create(0, C.byref(h)) == abi.PT_ERR_NO_DEVICE
        assert not h.value
        assert b"device" in native.lib.pt_global_error()


def test_null_arguments_are_rejected():
    assert native.lib.pt_render(None, None, None, 1) == abi.PT_ERR_INVALID
    assert native.lib.pt_resize(None, 1, 1) == abi.PT_ERR_INVALID
    assert native.lib.pt_server_submit(None, None, None) == abi.PT_ERR_INVALID
    native.lib.pt_destroy(None)


def test_ctypes_mirrors_match_the_header(tmp_path):
    """Every ctypes structure of photon_b200.abi has the size and field offsets that a C compiler gives
    the header's struct of the same name (compiled here with gcc)."""
    import shutil
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    mirrors = {
        "pt_tuning": abi.Tuning, "pt_profile": abi.Profile, "pt_kernel_time": abi.KernelTime, "pt_server_config": abi.ServerConfig,
        "pt_request": abi.Request, "pt_request_stats": abi.RequestStats, "pt_server_stats": abi.ServerStats, "pt_view": abi.View,
        "pt_stats": abi.Stats, "pt_scene_desc": abi.SceneDesc, "pt_raw_scene": abi.RawScene, "pt_texture_desc": abi.TextureDesc,
        "pt_bvh_build_options": abi.BvhBuildOptions, "pt_light_update": abi.LightUpdate,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "photon_wavefront.h"', "int main(void) {"]
    for cname, ct in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in ct._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, ct in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(ct), cname
        for fname, _ in ct._fields_:
            assert got[(cname, fname)] == getattr(ct, fname).offset, (cname, fname)
