"""ctypes binding of libphoton_wavefront.so (the C ABI of include/photon_wavefront.h).

Host-side mirror of Photon's GPU renderer interface (src/render/gpu_renderer.h:36-75): the
Renderer class has its members (upload, update_lights, resize, reset, render, render_denoised,
display, download_image, download_display, width/height/samples/last_frame_ms) with the same
argument meaning; failures raise PhotonError carrying the C status code. There is no fallback:
importing this module without the built library raises.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphoton_wavefront.so")

P = C.POINTER
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


class PhotonError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{message} (status {code})")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"photon_b200: the CUDA library is not built ({LIB_PATH}); run python -m photon_b200.build")
    L = C.CDLL(LIB_PATH)
    sig = {
        "pt_abi_version": ([], C.c_int32),
        "pt_device_info": ([C.c_char_p, C.c_size_t, P(C.c_int32), P(C.c_int32), P(C.c_uint64), P(C.c_int32)], C.c_int32),
        "pt_global_error": ([], C.c_char_p),
        "pt_create": ([C.c_int32, P(C.c_void_p)], C.c_int32),
        "pt_destroy": ([C.c_void_p], None),
        "pt_last_error": ([C.c_void_p], C.c_char_p),
        "pt_upload_scene": ([C.c_void_p, P(abi.SceneDesc)], C.c_int32),
        "pt_update_lights": ([C.c_void_p, P(abi.SceneDesc)], C.c_int32),
        "pt_resize": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int32),
        "pt_reset": ([C.c_void_p], C.c_int32),
        "pt_render": ([C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_int32], C.c_int32),
        "pt_render_denoised": ([C.c_void_p, P(abi.Camera), P(abi.Camera), P(abi.RenderSettings), P(abi.SvgfSettings)], C.c_int32),
        "pt_display": ([C.c_void_p, P(abi.RenderSettings), C.c_int32, C.c_void_p], C.c_int32),
        "pt_download_image": ([C.c_void_p, _f32p, C.c_size_t], C.c_int32),
        "pt_download_display": ([C.c_void_p, _u32p, C.c_size_t], C.c_int32),
        "pt_download_gbuffer": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t], C.c_int32),
        "pt_download_accumulation": ([C.c_void_p, C.c_void_p, C.c_size_t], C.c_int32),
        "pt_display_buffer": ([C.c_void_p], C.c_void_p),
        "pt_get_stats": ([C.c_void_p, P(abi.Stats)], C.c_int32),
        "pt_renderer_stream": ([C.c_void_p], C.c_void_p),
        "pt_measure_l2_bandwidth": ([C.c_int32, C.c_size_t, C.c_int32, P(C.c_double)], C.c_int32),
        "pt_set_profiling": ([C.c_void_p, C.c_int32], C.c_int32),
        "pt_get_profile": ([C.c_void_p, P(abi.Profile)], C.c_int32),
        "pt_set_tuning": ([C.c_void_p, P(abi.Tuning)], C.c_int32),
        "pt_get_tuning": ([C.c_void_p, P(abi.Tuning)], C.c_int32),
        "pt_autotune": ([C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_int32, C.c_uint64, P(abi.Tuning),
                         P(C.c_double), P(C.c_double)], C.c_int32),
        "pt_autotune_views": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_uint64, P(abi.Tuning), P(C.c_double), P(C.c_double)],
                              C.c_int32),
        "pt_server_set_tuning": ([C.c_void_p, P(abi.Tuning)], C.c_int32),
        "pt_server_open_session": ([C.c_void_p, C.c_int32, C.c_int32, C.c_int32, P(abi.SvgfSettings), P(C.c_int32)], C.c_int32),
        "pt_server_submit_frame": ([C.c_void_p, C.c_int32, P(abi.Camera), P(abi.Camera), P(abi.RenderSettings), P(C.c_uint64)],
                                   C.c_int32),
        "pt_server_close_session": ([C.c_void_p, C.c_int32], C.c_int32),
        "pt_server_fetch_encoded": ([C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_size_t, P(C.c_size_t)], C.c_int32),
        "pt_trace_primary": ([C.c_void_p, P(abi.Camera), C.c_int32, C.c_int32, C.c_uint32, C.c_uint32, _f32p], C.c_int32),
        "pt_light_picks_primary": ([C.c_void_p, P(abi.Camera), P(abi.RenderSettings), C.c_uint32, _i32p], C.c_int32),
        "pt_heatmap": ([C.c_void_p, P(abi.Camera), C.c_int32, C.c_int32, _f32p], C.c_int32),
        "pt_occlusion_probe": ([C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p], C.c_int32),
        "pt_render_views": ([C.c_void_p, P(abi.View), C.c_int32], C.c_int32),
        "pt_download_view": ([C.c_void_p, C.c_int32, _f32p, C.c_size_t], C.c_int32),
        "pt_svgf_create": ([C.c_int32, C.c_int32, C.c_int32, P(C.c_void_p)], C.c_int32),
        "pt_svgf_destroy": ([C.c_void_p], None),
        "pt_svgf_reset": ([C.c_void_p], C.c_int32),
        "pt_svgf_run": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, P(abi.Camera),
                         P(abi.SvgfSettings), C.c_void_p], C.c_int32),
        "pt_svgf_variance": ([C.c_void_p], C.c_void_p),
        "pt_svgf_last_error": ([C.c_void_p], C.c_char_p),
        "pt_svgf_set_tma": ([C.c_void_p, C.c_int32], C.c_int32),
        "pt_svgf_debug_tma_timeout": ([C.c_void_p, C.c_int32], C.c_int32),
        "pt_rebuild_lights": ([C.c_void_p, P(abi.LightUpdate)], C.c_int32),
        "pt_encode_pfm": ([C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, P(C.c_size_t)], C.c_int32),
        "pt_encode_png": ([C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, P(C.c_size_t)], C.c_int32),
        "pt_write_pfm": ([C.c_char_p, C.c_int32, C.c_int32, C.c_void_p], C.c_int32),
        "pt_write_png": ([C.c_char_p, C.c_int32, C.c_int32, C.c_void_p], C.c_int32),
        "pt_svgf_run_noalloc": ([C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 P(abi.SvgfSettings), C.c_void_p, C.c_void_p], C.c_int32),
        "pt_server_create": ([P(abi.ServerConfig), P(C.c_void_p)], C.c_int32),
        "pt_server_destroy": ([C.c_void_p], None),
        "pt_server_last_error": ([C.c_void_p], C.c_char_p),
        "pt_server_add_scene": ([C.c_void_p, P(abi.SceneDesc), P(C.c_int32)], C.c_int32),
        "pt_server_submit": ([C.c_void_p, P(abi.Request), P(C.c_uint64)], C.c_int32),
        "pt_server_poll": ([C.c_void_p, C.c_uint64, P(C.c_int32)], C.c_int32),
        "pt_server_wait": ([C.c_void_p, C.c_uint64, C.c_double], C.c_int32),
        "pt_server_fetch": ([C.c_void_p, C.c_uint64, C.c_void_p, C.c_size_t, P(abi.RequestStats)], C.c_int32),
        "pt_server_cancel": ([C.c_void_p, C.c_uint64], C.c_int32),
        "pt_server_get_stats": ([C.c_void_p, P(abi.ServerStats)], C.c_int32),
        "pt_server_debug_fail_allocations": ([C.c_void_p, C.c_int32], C.c_int32),
        "pt_server_debug_fail_finishing": ([C.c_void_p, C.c_int32], C.c_int32),
        "pt_scene_build": ([P(abi.RawScene), P(abi.BvhBuildOptions), P(C.c_void_p)], C.c_int32),
        "pt_scene_desc_of": ([C.c_void_p], P(abi.SceneDesc)),
        "pt_scene_free": ([C.c_void_p], None),
        "pt_generate_scene": ([C.c_int32, C.c_int64, C.c_uint64, P(C.c_void_p)], C.c_int32),
        "pt_generated_raw": ([C.c_void_p], P(abi.RawScene)),
        "pt_generated_camera": ([C.c_void_p, C.c_float, P(abi.Camera)], C.c_int32),
        "pt_generated_free": ([C.c_void_p], None),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    return L, sig


lib, SIGNATURES = _load()


def _check(code, msg_fn):
    if code != abi.PT_OK:
        m = msg_fn()
        raise PhotonError(code, m.decode() if isinstance(m, bytes) else str(m))


def device_info():
    """photon::cuda_available (gpu_renderer.h:34) with its GpuInfo: None without a device."""
    name = C.create_string_buffer(256)
    major, minor, mp = C.c_int32(), C.c_int32(), C.c_int32()
    mem = C.c_uint64()
    if not lib.pt_device_info(name, 256, C.byref(major), C.byref(minor), C.byref(mem), C.byref(mp)):
        return None
    return dict(name=name.value.decode(), major=major.value, minor=minor.value, memory=mem.value, multiprocessors=mp.value)


def l2_read_bandwidth(device=0, nbytes=32 << 20, reps=64):
    """GB/s of an L2-resident read (pt_measure_l2_bandwidth)."""
    g = C.c_double()
    _check(lib.pt_measure_l2_bandwidth(device, nbytes, reps, C.byref(g)), lambda: lib.pt_global_error().decode())
    return g.value


class Renderer:
    """The wavefront drop-in for photon::GpuRenderer."""

    def __init__(self, device=0):
        h = C.c_void_p()
        _check(lib.pt_create(device, C.byref(h)), lib.pt_global_error)
        self.h = h
        self._scene_keepalive = None

    def close(self):
        if getattr(self, "h", None):
            lib.pt_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _err(self):
        return lib.pt_last_error(self.h)

    def upload(self, desc, keepalive=None):
        _check(lib.pt_upload_scene(self.h, C.byref(desc)), self._err)
        self._scene_keepalive = keepalive

    def update_lights(self, desc):
        _check(lib.pt_update_lights(self.h, C.byref(desc)), self._err)

    def resize(self, w, h):
        _check(lib.pt_resize(self.h, w, h), self._err)

    def reset(self):
        _check(lib.pt_reset(self.h), self._err)

    def render(self, cam, rs, spp):
        _check(lib.pt_render(self.h, C.byref(cam), C.byref(rs), spp), self._err)

    def rebuild_lights(self, update):
        """pt_rebuild_lights with an abi.LightUpdate."""
        _check(lib.pt_rebuild_lights(self.h, C.byref(update)), self._err)

    def render_denoised(self, cam, prev, rs, sv):
        _check(lib.pt_render_denoised(self.h, C.byref(cam), C.byref(prev), C.byref(rs), C.byref(sv)), self._err)

    def display(self, rs, mode=abi.PT_DISPLAY_COLOR, device_target=None):
        _check(lib.pt_display(self.h, C.byref(rs), mode, device_target), self._err)

    def stats(self):
        s = abi.Stats()
        _check(lib.pt_get_stats(self.h, C.byref(s)), self._err)
        return s

    @property
    def width(self):
        return self.stats().width

    @property
    def height(self):
        return self.stats().height

    @property
    def samples(self):
        return self.stats().samples

    @property
    def last_frame_ms(self):
        return self.stats().last_frame_ms

    def download_image(self, out=None):
        """The image (height, width, 3) float32; `out`, a C-contiguous float32 array of that shape, is
        filled in place when given (a reused host buffer)."""
        s = self.stats()
        if out is None:
            out = np.zeros((s.height, s.width, 3), np.float32)
        elif out.dtype != np.float32 or out.shape != (s.height, s.width, 3) or not out.flags.c_contiguous:
            raise ValueError("download_image: out must be a C-contiguous float32 array of shape (height, width, 3)")
        _check(lib.pt_download_image(self.h, out, out.size), self._err)
        return out

    def download_display(self):
        s = self.stats()
        out = np.zeros((s.height, s.width), np.uint32)
        _check(lib.pt_download_display(self.h, out, out.size), self._err)
        return out

    def download_gbuffer(self):
        s = self.stats()
        a = np.zeros((s.height, s.width, 4), np.float32)
        nd = np.zeros((s.height, s.width, 4), np.float32)
        _check(lib.pt_download_gbuffer(self.h, a.ctypes.data, nd.ctypes.data, s.width * s.height), self._err)
        return a, nd

    def download_accumulation(self):
        """Per-pixel sums (rgb radiance, squared luminance) of the samples rendered so far."""
        s = self.stats()
        a = np.zeros((s.height, s.width, 4), np.float32)
        _check(lib.pt_download_accumulation(self.h, a.ctypes.data, s.width * s.height), self._err)
        return a

    def stream(self):
        """The cudaStream_t (as an int) that orders all of this renderer's device work."""
        return lib.pt_renderer_stream(self.h)

    def set_profiling(self, flags):
        _check(lib.pt_set_profiling(self.h, flags), self._err)

    def profile(self):
        p = abi.Profile()
        _check(lib.pt_get_profile(self.h, C.byref(p)), self._err)
        return p

    def set_tuning(self, **kw):
        t = abi.Tuning(0, 0, 0, -1, -1, -1, -1, -1, -1, 0, 0, 0, -1, -1)
        for k, v in kw.items():
            setattr(t, k, v)
        _check(lib.pt_set_tuning(self.h, C.byref(t)), self._err)

    def autotune(self, cam, rs, spp, probe_samples=0):
        """Runs the autotuner; returns (chosen tuning dict, default rate, tuned rate) in samples/s."""
        t = abi.Tuning()
        d, b = C.c_double(), C.c_double()
        _check(lib.pt_autotune(self.h, C.byref(cam), C.byref(rs), spp, probe_samples, C.byref(t), C.byref(d), C.byref(b)), self._err)
        return {n: getattr(t, n) for n, _ in abi.Tuning._fields_}, d.value, b.value

    def autotune_views(self, views, probe_samples=0):
        """Runs the autotuner on a batched view set; returns (chosen tuning dict, default rate, tuned
        rate) in samples/s of the scaled-down probe."""
        arr = (abi.View * len(views))(*views)
        t = abi.Tuning()
        d, b = C.c_double(), C.c_double()
        _check(lib.pt_autotune_views(self.h, arr, len(views), probe_samples, C.byref(t), C.byref(d), C.byref(b)), self._err)
        return {n: getattr(t, n) for n, _ in abi.Tuning._fields_}, d.value, b.value

    def tuning(self):
        t = abi.Tuning()
        _check(lib.pt_get_tuning(self.h, C.byref(t)), self._err)
        return {n: getattr(t, n) for n, _ in abi.Tuning._fields_}

    def trace_primary(self, cam, w, h, frame=0, seed=0):
        out = np.zeros((h, w, 4), np.float32)
        _check(lib.pt_trace_primary(self.h, C.byref(cam), w, h, frame, seed, out), self._err)
        return out

    def light_picks(self, cam, rs, frame=0):
        out = np.zeros((rs.height, rs.width, 4), np.int32)
        _check(lib.pt_light_picks_primary(self.h, C.byref(cam), C.byref(rs), frame, out), self._err)
        return out

    def heatmap(self, cam, w, h):
        out = np.zeros((h, w), np.float32)
        _check(lib.pt_heatmap(self.h, C.byref(cam), w, h, out), self._err)
        return out

    def occlusion_probe(self, rays8, wide=False):
        """Any-hit walks of (n, 8) float32 rays (origin, tmax, direction, unused): (n, 4) int32 of
        (occluded, first accepted triangle or -1, node visits, triangle tests)."""
        rays8 = np.ascontiguousarray(rays8, np.float32)
        out = np.zeros((rays8.shape[0], 4), np.int32)
        _check(lib.pt_occlusion_probe(self.h, rays8.ctypes.data, rays8.shape[0], 1 if wide else 0, out.ctypes.data), self._err)
        return out

    def render_views(self, views):
        arr = (abi.View * len(views))(*views)
        _check(lib.pt_render_views(self.h, arr, len(views)), self._err)

    def download_view(self, i, w, h):
        out = np.zeros((h, w, 3), np.float32)
        _check(lib.pt_download_view(self.h, i, out, out.size), self._err)
        return out


class Svgf:
    """SVGF on caller G-buffers (device pointers), photon::Svgf (svgf.h:32-59)."""

    def __init__(self, w, h, device=0):
        p = C.c_void_p()
        _check(lib.pt_svgf_create(device, w, h, C.byref(p)), lib.pt_global_error)
        self.h = p
        self.w, self.hh = w, h

    def run(self, color, albedo, nd, pos, emission, prev_cam, settings, output):
        """Pointers are device addresses (ints) of width*height float4 buffers."""
        _check(lib.pt_svgf_run(self.h, color, albedo, nd, pos, emission, C.byref(prev_cam), C.byref(settings), output),
               lambda: lib.pt_svgf_last_error(self.h))

    def reset(self):
        lib.pt_svgf_reset(self.h)

    def set_tma(self, mode):
        """0 global loads, 1-3 TMA-staged tiles (pt_svgf_set_tma)."""
        _check(lib.pt_svgf_set_tma(self.h, int(mode)), lambda: lib.pt_svgf_last_error(self.h))

    def debug_tma_timeout(self, on):
        """Test hook: the TMA passes' tile wait runs out with no copy issued (pt_svgf_debug_tma_timeout)."""
        _check(lib.pt_svgf_debug_tma_timeout(self.h, 1 if on else 0), lambda: lib.pt_svgf_last_error(self.h))

    def variance_ptr(self):
        return lib.pt_svgf_variance(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib.pt_svgf_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def svgf_run_noalloc(width, height, color, albedo, normal_depth, position, emission, settings, output, stream=0, device=0):
    """The allocation-free single-frame SVGF denoise (pt_svgf_run_noalloc). Pointer arguments are
    device addresses (ints) of width*height float4 buffers; the call enqueues on `stream`."""
    _check(lib.pt_svgf_run_noalloc(device, width, height, color, albedo, normal_depth, position, emission, C.byref(settings),
                                   output, stream), lib.pt_global_error)


def encode_pfm(rgb):
    """PFM bytes of a float32 (h, w, 3) image (pt_encode_pfm)."""
    rgb = np.ascontiguousarray(rgb, np.float32)
    h, w = rgb.shape[:2]
    n = C.c_size_t()
    _check(lib.pt_encode_pfm(rgb.ctypes.data, w, h, None, 0, C.byref(n)), lib.pt_global_error)
    out = np.empty(n.value, np.uint8)
    _check(lib.pt_encode_pfm(rgb.ctypes.data, w, h, out.ctypes.data, out.size, C.byref(n)), lib.pt_global_error)
    return out.tobytes()


def encode_png(rgba, level=6):
    """PNG bytes of a uint32 (h, w) display buffer (pt_encode_png)."""
    rgba = np.ascontiguousarray(rgba, np.uint32)
    h, w = rgba.shape
    n = C.c_size_t()
    _check(lib.pt_encode_png(rgba.ctypes.data, w, h, level, None, 0, C.byref(n)), lib.pt_global_error)
    out = np.empty(n.value, np.uint8)
    _check(lib.pt_encode_png(rgba.ctypes.data, w, h, level, out.ctypes.data, out.size, C.byref(n)), lib.pt_global_error)
    return out.tobytes()


class Server:
    """The request server (continuous batching over resident scenes)."""

    def __init__(self, budget_bytes=0, device=0, path_capacity=0, max_active=0, device_wait_seconds=2.0, sort_rays=0, reserve_bytes=0):
        cfg = abi.ServerConfig(device, budget_bytes, path_capacity, max_active, device_wait_seconds, sort_rays, reserve_bytes)
        p = C.c_void_p()
        _check(lib.pt_server_create(C.byref(cfg), C.byref(p)), lib.pt_global_error)
        self.h = p
        self._keep = []

    def _err(self):
        return lib.pt_server_last_error(self.h)

    def add_scene(self, desc, keepalive=None):
        sid = C.c_int32()
        _check(lib.pt_server_add_scene(self.h, C.byref(desc), C.byref(sid)), self._err)
        return sid.value

    def submit(self, scene_id, cam, w, h, spp, seed=0, path=None, display=False, exposure=1.0, tonemap=abi.PT_TONEMAP_ACES):
        req = abi.Request(scene_id, cam, w, h, spp, seed, path or abi.path_options(), 1 if display else 0, exposure, tonemap)
        rid = C.c_uint64()
        _check(lib.pt_server_submit(self.h, C.byref(req), C.byref(rid)), self._err)
        return rid.value

    def poll(self, rid):
        st = C.c_int32()
        _check(lib.pt_server_poll(self.h, rid, C.byref(st)), self._err)
        return st.value

    def wait(self, rid, timeout_s=60.0):
        _check(lib.pt_server_wait(self.h, rid, timeout_s), self._err)

    def fetch(self, rid, w, h):
        out = np.zeros((h, w, 3), np.float32)
        st = abi.RequestStats()
        _check(lib.pt_server_fetch(self.h, rid, out.ctypes.data, out.size, C.byref(st)), self._err)
        return out, st

    def cancel(self, rid):
        _check(lib.pt_server_cancel(self.h, rid), self._err)

    def open_session(self, scene_id, w, h, svgf=None):
        """A real-time SVGF session on a resident scene (pt_server_open_session); returns its id."""
        sid = C.c_int32()
        _check(lib.pt_server_open_session(self.h, scene_id, w, h, C.byref(svgf or abi.svgf_settings()), C.byref(sid)), self._err)
        return sid.value

    def submit_frame(self, session, cam, prev, rs):
        """One frame of a session (1 spp + G-buffer + SVGF with the session's history); returns a
        request id for wait / poll / fetch."""
        rid = C.c_uint64()
        _check(lib.pt_server_submit_frame(self.h, session, C.byref(cam), C.byref(prev), C.byref(rs), C.byref(rid)), self._err)
        return rid.value

    def close_session(self, session):
        _check(lib.pt_server_close_session(self.h, session), self._err)

    def encoded_size(self, rid, fmt):
        """Size of the request's image in `fmt` (abi.PT_IMAGE_*); the request stays."""
        n = C.c_size_t()
        _check(lib.pt_server_fetch_encoded(self.h, rid, fmt, None, 0, C.byref(n)), self._err)
        return n.value

    def fetch_encoded(self, rid, fmt):
        """The request's image encoded as PFM or PNG (bytes); consumes the request."""
        n = self.encoded_size(rid, fmt)
        buf = (C.c_uint8 * n)()
        _check(lib.pt_server_fetch_encoded(self.h, rid, fmt, buf, n, C.byref(C.c_size_t())), self._err)
        return bytes(buf)

    def stats(self):
        s = abi.ServerStats()
        _check(lib.pt_server_get_stats(self.h, C.byref(s)), self._err)
        return s

    def fail_allocations(self, n):
        _check(lib.pt_server_debug_fail_allocations(self.h, n), self._err)

    def set_tuning(self, **kw):
        """Applies tuning knobs (pt_server_set_tuning); unnamed knobs keep their values."""
        t = abi.Tuning(0, 0, 0, -1, -1, -1, -1, -1, -1, 0, 0, 0, -1, -1)
        for k, v in kw.items():
            setattr(t, k, v)
        _check(lib.pt_server_set_tuning(self.h, C.byref(t)), self._err)

    def fail_finishing(self, n):
        _check(lib.pt_server_debug_fail_finishing(self.h, n), self._err)

    def close(self):
        if getattr(self, "h", None):
            lib.pt_server_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class BuiltScene:
    """Raw meshes built into a pt_scene_desc by the library's own builder."""

    def __init__(self, raw, bins=0, max_leaf=0, traversal_cost=0.0, threads=0, gpu=False, keepalive=None):
        p = C.c_void_p()
        o = abi.BvhBuildOptions(bins, max_leaf, traversal_cost, threads, 1 if gpu else 0)
        _check(lib.pt_scene_build(C.byref(raw), C.byref(o), C.byref(p)), lib.pt_global_error)
        self.h = p
        self._keep = keepalive

    @property
    def desc(self):
        return lib.pt_scene_desc_of(self.h).contents

    def close(self):
        if getattr(self, "h", None):
            lib.pt_scene_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


class GeneratedScene:
    """A procedural scene of the benchmark configurations (raw meshes + camera)."""

    def __init__(self, kind, triangles=0, seed=1):
        p = C.c_void_p()
        _check(lib.pt_generate_scene(kind, triangles, seed, C.byref(p)), lib.pt_global_error)
        self.h = p

    @property
    def raw(self):
        return lib.pt_generated_raw(self.h).contents

    def camera(self, aspect):
        c = abi.Camera()
        _check(lib.pt_generated_camera(self.h, aspect, C.byref(c)), lib.pt_global_error)
        return c

    def build(self, **kw):
        return BuiltScene(self.raw, keepalive=self, **kw)

    def close(self):
        if getattr(self, "h", None):
            lib.pt_generated_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def box_scene():
    """The 36-triangle closed box (the 256x256, 64 spp configuration's scene)."""
    return GeneratedScene(abi.PT_GEN_BOX, 36, 1)


def terrain_scene(triangles=262144, seed=1):
    """The height-field scene (262,144 triangles for the 1080p, 16 spp configuration)."""
    return GeneratedScene(abi.PT_GEN_TERRAIN, triangles, seed)
