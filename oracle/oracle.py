"""TEST INFRASTRUCTURE — Python access to the oracle.

Two libraries, both built by oracle/Makefile:
  - oracle/_build/liboracle.so: the C restatement of Photon's path tracer and SVGF (photon_oracle.c);
  - oracle/_ref/libphoton_ref.so: Photon's own CPU code compiled from its sources plus ref_shim.cpp
    (and libphoton_ref_gpu.so with Photon's CUDA megakernel and SVGF).
The restatement is pinned bit-for-bit against Photon's build by tests/test_oracle_pinning.py.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module; the
product never does.
"""
import ctypes as C
import os

import numpy as np

from photon_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libphoton_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libphoton_ref_gpu.so")

P = C.POINTER
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OrcCounters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "samples", "camera_rays", "extension_rays", "shadow_rays", "node_visits", "tri_tests", "alpha_tests",
        "shade_events", "normal_mapped_events", "nee_emissive", "nee_punctual", "nee_env", "env_lookups",
        "texture_taps")]


_orc = None
_ref = None
_refgpu = None


def restatement():
    """The C restatement (liboracle.so)."""
    global _orc
    if _orc is None:
        if not os.path.exists(RESTATEMENT_SO):
            raise RuntimeError(f"oracle restatement not built: {RESTATEMENT_SO} (run make -C oracle restatement)")
        L = C.CDLL(RESTATEMENT_SO)
        L.orc_render.argtypes = [P(abi.SceneDesc), P(abi.Camera), P(abi.RenderSettings), C.c_int, C.c_uint32, C.c_int, _f32p]
        L.orc_render_sample.argtypes = [P(abi.SceneDesc), P(abi.Camera), P(abi.RenderSettings), C.c_int, C.c_int,
                                        C.c_uint32, _f32p, C.c_void_p]
        L.orc_sample_gbuffer.argtypes = [P(abi.SceneDesc), P(abi.Camera), P(abi.RenderSettings), C.c_uint32, C.c_int,
                                         _f32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_trace_primary.argtypes = [P(abi.SceneDesc), P(abi.Camera), C.c_int, C.c_int, C.c_uint32, C.c_uint32, _f32p]
        L.orc_light_picks_primary.argtypes = [P(abi.SceneDesc), P(abi.Camera), P(abi.RenderSettings), C.c_uint32, _i32p]
        L.orc_heatmap.argtypes = [P(abi.SceneDesc), P(abi.Camera), C.c_int, C.c_int, _f32p]
        L.orc_occluded.argtypes = [P(abi.SceneDesc), _f32p, C.c_int, _i32p]
        L.orc_count.argtypes = [P(abi.SceneDesc), P(abi.Camera), P(abi.RenderSettings), C.c_int, P(OrcCounters)]
        L.orc_rng_floats.argtypes = [C.c_uint64, C.c_uint64, C.c_int, _f32p]
        L.orc_hash_u32.argtypes = [C.c_uint32]
        L.orc_hash_u32.restype = C.c_uint32
        L.orc_sample_alias.argtypes = [P(abi.AliasEntry), C.c_int, C.c_float, P(C.c_float)]
        L.orc_sample_alias.restype = C.c_int
        L.orc_offset_ray.argtypes = [C.c_int, _f32p, _f32p, _f32p]
        L.orc_bsdf_sample.argtypes = [_f32p, C.c_int, _f32p, _f32p]
        L.orc_sample_light.argtypes = [P(abi.SceneDesc), _f32p, C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
        L.orc_svgf_create.argtypes = [C.c_int, C.c_int]
        L.orc_svgf_create.restype = C.c_void_p
        L.orc_svgf_destroy.argtypes = [C.c_void_p]
        L.orc_svgf_reset.argtypes = [C.c_void_p]
        L.orc_svgf_run.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, _f32p, _f32p, P(abi.Camera), P(abi.SvgfSettings), _f32p]
        L.orc_svgf_variance.argtypes = [C.c_void_p]
        L.orc_svgf_variance.restype = P(C.c_float)
        _orc = L
    return _orc


def reference_available():
    return os.path.exists(REF_SO)


def reference():
    """Photon's own CPU build (libphoton_ref.so)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"reference build missing: {REF_SO} (run make -C oracle reference)")
        L = C.CDLL(REF_SO)
        _bind_ref(L)
        _ref = L
    return _ref


def _bind_ref(L):
    L.ref_builtin_scene.argtypes = [C.c_char_p, C.c_int]
    L.ref_builtin_scene.restype = C.c_void_p
    L.ref_scene_from_raw.argtypes = [P(abi.RawScene), C.c_int, C.c_int, C.c_int]
    L.ref_scene_from_raw.restype = C.c_void_p
    L.ref_scene_from_desc.argtypes = [P(abi.SceneDesc)]
    L.ref_scene_from_desc.restype = C.c_void_p
    L.ref_generated_scene.argtypes = [C.c_int, C.c_int64, C.c_uint64, C.c_int]
    L.ref_generated_scene.restype = C.c_void_p
    L.ref_generated_raw.argtypes = [C.c_int, C.c_int64, C.c_uint64, P(P(abi.RawScene))]
    L.ref_generated_raw.restype = C.c_void_p
    L.ref_generated_raw_free.argtypes = [C.c_void_p]
    L.ref_scene_free.argtypes = [C.c_void_p]
    L.ref_scene_desc.argtypes = [C.c_void_p]
    L.ref_scene_desc.restype = P(abi.SceneDesc)
    L.ref_scene_raw.argtypes = [C.c_void_p]
    L.ref_scene_raw.restype = P(abi.RawScene)
    L.ref_scene_camera.argtypes = [C.c_void_p, C.c_float, P(abi.Camera)]
    L.ref_camera_view.argtypes = [_f32p, _f32p, _f32p, C.c_float, C.c_float, C.c_float, C.c_float, P(abi.Camera)]
    L.ref_bvh_stats.argtypes = [C.c_void_p, P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_float), P(C.c_double)]
    L.ref_render.argtypes = [C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_int, C.c_int, C.c_void_p]
    L.ref_render.restype = C.c_double
    L.ref_render_samples.argtypes = [C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_int, _i32p, _f32p]
    L.ref_rays_per_sample.argtypes = [C.c_void_p, P(abi.Camera), P(abi.RenderSettings)]
    L.ref_rays_per_sample.restype = C.c_double
    L.ref_trace_primary.argtypes = [C.c_void_p, P(abi.Camera), C.c_int, C.c_int, C.c_uint32, C.c_uint32, _f32p]
    L.ref_light_picks_primary.argtypes = [C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_uint32, _i32p]
    L.ref_heatmap.argtypes = [C.c_void_p, P(abi.Camera), C.c_int, C.c_int, _f32p]
    L.ref_occluded.argtypes = [C.c_void_p, _f32p, C.c_int, _i32p]
    L.ref_alias_table.argtypes = [_f32p, C.c_int, P(abi.AliasEntry)]
    L.ref_rng_floats.argtypes = [C.c_uint64, C.c_uint64, C.c_int, _f32p]
    L.ref_offset_ray.argtypes = [C.c_int, _f32p, _f32p, _f32p]
    L.ref_bsdf_sample.argtypes = [_f32p, C.c_int, _f32p, _f32p]


def reference_gpu():
    """Photon's build with its CUDA megakernel and SVGF (libphoton_ref_gpu.so)."""
    global _refgpu
    if _refgpu is None:
        if not os.path.exists(REF_GPU_SO):
            raise RuntimeError(f"reference GPU build missing: {REF_GPU_SO}")
        L = C.CDLL(REF_GPU_SO)
        _bind_ref(L)
        L.refgpu_available.restype = C.c_int
        L.refgpu_create.restype = C.c_void_p
        L.refgpu_destroy.argtypes = [C.c_void_p]
        L.refgpu_upload.argtypes = [C.c_void_p, C.c_void_p]
        L.refgpu_upload.restype = C.c_int
        L.refgpu_resize.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.refgpu_reset.argtypes = [C.c_void_p]
        L.refgpu_render.argtypes = [C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_int]
        L.refgpu_render.restype = C.c_float
        L.refgpu_render_denoised.argtypes = [C.c_void_p, P(abi.Camera), P(abi.Camera), P(abi.RenderSettings),
                                             P(abi.SvgfSettings)]
        L.refgpu_render_denoised.restype = C.c_float
        L.refgpu_samples.argtypes = [C.c_void_p]
        L.refgpu_samples.restype = C.c_int
        L.refgpu_download_image.argtypes = [C.c_void_p, _f32p]
        L.refsvgf_create.argtypes = [C.c_int, C.c_int]
        L.refsvgf_create.restype = C.c_void_p
        L.refsvgf_destroy.argtypes = [C.c_void_p]
        L.refsvgf_reset.argtypes = [C.c_void_p]
        L.refsvgf_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  P(abi.Camera), P(abi.SvgfSettings), C.c_void_p]
        _refgpu = L
    return _refgpu


# ---- convenience ---------------------------------------------------------------------------------

class RefScene:
    """A scene built by Photon's own Scene::build (kept alive while referenced)."""

    def __init__(self, handle, lib):
        if not handle:
            raise RuntimeError("reference scene construction failed")
        self.h = handle
        self.lib = lib

    @classmethod
    def builtin(cls, name, flat_normals=False, lib=None):
        lib = lib or reference()
        return cls(lib.ref_builtin_scene(name.encode(), 1 if flat_normals else 0), lib)

    @classmethod
    def from_raw(cls, raw, lib=None, threads=0):
        lib = lib or reference()
        return cls(lib.ref_scene_from_raw(C.byref(raw), 0, 0, threads), lib)

    @classmethod
    def from_desc(cls, desc, lib=None):
        lib = lib or reference()
        return cls(lib.ref_scene_from_desc(C.byref(desc)), lib)

    @classmethod
    def generated(cls, kind, triangles, seed, lib=None, threads=0):
        """A benchmark scene (abi.PT_GEN_*): the seeded generator's raw meshes built by Photon's own
        Scene::build; its camera() is Photon's Camera::view of the generator's look-at camera."""
        lib = lib or reference()
        return cls(lib.ref_generated_scene(kind, triangles, seed, threads), lib)

    @property
    def desc(self):
        return self.lib.ref_scene_desc(self.h).contents

    @property
    def raw(self):
        return self.lib.ref_scene_raw(self.h).contents

    def camera(self, aspect):
        c = abi.Camera()
        self.lib.ref_scene_camera(self.h, aspect, C.byref(c))
        return c

    def bvh_stats(self):
        n, l, d = C.c_int(), C.c_int(), C.c_int()
        s, ms = C.c_float(), C.c_double()
        self.lib.ref_bvh_stats(self.h, C.byref(n), C.byref(l), C.byref(d), C.byref(s), C.byref(ms))
        return dict(nodes=n.value, leaves=l.value, depth=d.value, sah=s.value, build_ms=ms.value)

    def render(self, cam, rs, spp, threads=0):
        out = np.zeros((rs.height, rs.width, 3), np.float32)
        secs = self.lib.ref_render(self.h, C.byref(cam), C.byref(rs), spp, threads, out.ctypes.data)
        return out, secs

    def trace_primary(self, cam, w, h, frame=0, seed=0):
        out = np.zeros((h, w, 4), np.float32)
        self.lib.ref_trace_primary(self.h, C.byref(cam), w, h, frame, seed, out)
        return out

    def light_picks(self, cam, rs, frame=0):
        out = np.zeros((rs.height, rs.width, 4), np.int32)
        self.lib.ref_light_picks_primary(self.h, C.byref(cam), C.byref(rs), frame, out)
        return out

    def heatmap(self, cam, w, h):
        out = np.zeros((h, w), np.float32)
        self.lib.ref_heatmap(self.h, C.byref(cam), w, h, out)
        return out

    def occluded(self, rays8):
        """Photon's any-hit walk: (n, 4) of (occluded, accepted triangle or -1, node visits, 0)."""
        rays8 = np.ascontiguousarray(rays8, np.float32)
        out = np.zeros((rays8.shape[0], 4), np.int32)
        self.lib.ref_occluded(self.h, rays8, rays8.shape[0], out)
        return out

    def __del__(self):
        try:
            if self.h:
                self.lib.ref_scene_free(self.h)
                self.h = None
        except Exception:
            pass


class RefGeneratedRaw:
    """The generator's raw arrays as the reference library's copy of the generator makes them."""

    def __init__(self, kind, triangles, seed, lib=None):
        self.lib = lib or reference()
        p = P(abi.RawScene)()
        self.h = self.lib.ref_generated_raw(kind, triangles, seed, C.byref(p))
        if not self.h:
            raise RuntimeError("generator rejected the arguments")
        self.raw = p.contents

    def __del__(self):
        try:
            if self.h:
                self.lib.ref_generated_raw_free(self.h)
                self.h = None
        except Exception:
            pass


def orc_render(desc, cam, rs, spp, frame0=0, threads=0):
    """Average radiance (h, w, 3) of spp samples, as CpuRenderer::render + image()."""
    s = np.zeros((rs.height, rs.width, 3), np.float32)
    restatement().orc_render(C.byref(desc), C.byref(cam), C.byref(rs), spp, frame0, threads, s)
    return s * np.float32(1.0 / spp) if spp > 0 else s


def orc_render_sum(desc, cam, rs, spp, frame0=0, threads=0):
    s = np.zeros((rs.height, rs.width, 3), np.float32)
    restatement().orc_render(C.byref(desc), C.byref(cam), C.byref(rs), spp, frame0, threads, s)
    return s


def orc_trace_primary(desc, cam, w, h, frame=0, seed=0):
    out = np.zeros((h, w, 4), np.float32)
    restatement().orc_trace_primary(C.byref(desc), C.byref(cam), w, h, frame, seed, out)
    return out


def orc_light_picks(desc, cam, rs, frame=0):
    out = np.zeros((rs.height, rs.width, 4), np.int32)
    restatement().orc_light_picks_primary(C.byref(desc), C.byref(cam), C.byref(rs), frame, out)
    return out


def orc_heatmap(desc, cam, w, h):
    out = np.zeros((h, w), np.float32)
    restatement().orc_heatmap(C.byref(desc), C.byref(cam), w, h, out)
    return out


def orc_occluded(desc, rays8):
    """The restatement's any-hit walk: (n, 4) of (occluded, accepted triangle or -1, node visits,
    triangle tests)."""
    rays8 = np.ascontiguousarray(rays8, np.float32)
    out = np.zeros((rays8.shape[0], 4), np.int32)
    restatement().orc_occluded(C.byref(desc), rays8, rays8.shape[0], out)
    return out


def orc_gbuffer(desc, cam, rs, frame=0, threads=0):
    n = (rs.height, rs.width, 4)
    bufs = [np.zeros(n, np.float32) for _ in range(5)]
    restatement().orc_sample_gbuffer(C.byref(desc), C.byref(cam), C.byref(rs), frame, threads, *bufs)
    return dict(zip(("color", "albedo", "normal_depth", "position", "emission"), bufs))


def orc_count(desc, cam, rs, stride=7):
    c = OrcCounters()
    restatement().orc_count(C.byref(desc), C.byref(cam), C.byref(rs), stride, C.byref(c))
    return {n: getattr(c, n) for n, _ in OrcCounters._fields_}


class OrcSvgf:
    def __init__(self, w, h):
        self.w, self.h = w, h
        self.s = restatement().orc_svgf_create(w, h)

    def run(self, g, prev_cam, settings):
        out = np.zeros((self.h, self.w, 4), np.float32)
        restatement().orc_svgf_run(self.s, g["color"], g["albedo"], g["normal_depth"], g["position"], g["emission"],
                                   C.byref(prev_cam), C.byref(settings), out)
        return out

    def reset(self):
        restatement().orc_svgf_reset(self.s)

    def __del__(self):
        try:
            restatement().orc_svgf_destroy(self.s)
        except Exception:
            pass


def hits_tri(hits4):
    """The triangle index channel of a (t, tri, u, v) hit array (stored as int32 bits)."""
    return np.ascontiguousarray(hits4[..., 1]).view(np.int32)
