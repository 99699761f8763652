"""ctypes mirrors of the C ABI in include/photon_wavefront.h.

The structures here have the byte layout of the header (and hence of Photon's own types, see
src/render/scene_view.h:13-150 of the Photon sources); tests check the sizes against the header.
"""
import ctypes as C

PT_OK = 0
PT_ERR_INVALID = -1
PT_ERR_CUDA = -2
PT_ERR_NO_DEVICE = -3
PT_ERR_NO_SCENE = -4
PT_ERR_BUDGET = -5
PT_ERR_TIMEOUT = -6
PT_ERR_CANCELLED = -7
PT_ERR_NOT_FOUND = -8
PT_ERR_OVERFLOW = -9
PT_ERR_ALLOC = -10

PT_TRI_ALPHA_TESTED = 1
PT_ALPHA_OPAQUE, PT_ALPHA_MASK, PT_ALPHA_BLEND = 0, 1, 2
PT_LIGHT_POINT, PT_LIGHT_SPOT, PT_LIGHT_DIRECTIONAL = 0, 1, 2
PT_TONEMAP_LINEAR, PT_TONEMAP_ACES, PT_TONEMAP_REINHARD = 0, 1, 2
(PT_DISPLAY_COLOR, PT_DISPLAY_ALBEDO, PT_DISPLAY_NORMAL, PT_DISPLAY_DEPTH, PT_DISPLAY_VARIANCE,
 PT_DISPLAY_HEATMAP) = range(6)
PT_REQ_QUEUED, PT_REQ_RUNNING, PT_REQ_DONE, PT_REQ_CANCELLED, PT_REQ_FAILED = range(5)
PT_GEN_BOX, PT_GEN_TERRAIN = 0, 1
PT_IMAGE_PFM, PT_IMAGE_PNG = 0, 1


class Vec2(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Vec4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class BvhNode(C.Structure):
    _fields_ = [("lmin", Vec3), ("left", C.c_int32), ("lmax", Vec3), ("lcount", C.c_int32),
                ("rmin", Vec3), ("right", C.c_int32), ("rmax", Vec3), ("rcount", C.c_int32)]


class TriGeom(C.Structure):
    _fields_ = [("v0", Vec3), ("material", C.c_int32), ("e1", Vec3), ("flags", C.c_int32),
                ("e2", Vec3), ("pad", C.c_int32)]


class TextureInfo(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("offset", C.c_uint32),
                ("wrap_repeat", C.c_int32), ("srgb", C.c_int32)]


class Material(C.Structure):
    _fields_ = [("base_color", Vec4), ("emission", Vec3), ("metallic", C.c_float), ("roughness", C.c_float),
                ("ior", C.c_float), ("transmission", C.c_float), ("normal_scale", C.c_float),
                ("alpha_cutoff", C.c_float), ("alpha_mode", C.c_int32), ("double_sided", C.c_int32),
                ("base_color_tex", C.c_int32), ("metallic_roughness_tex", C.c_int32), ("normal_tex", C.c_int32),
                ("emissive_tex", C.c_int32), ("occlusion_tex", C.c_int32)]


class EmissiveTri(C.Structure):
    _fields_ = [("tri", C.c_int32), ("area", C.c_float)]


class AliasEntry(C.Structure):
    _fields_ = [("prob", C.c_float), ("alias", C.c_int32), ("pmf", C.c_float), ("pad", C.c_int32)]


class PunctualLight(C.Structure):
    _fields_ = [("position", Vec3), ("type", C.c_int32), ("direction", Vec3), ("cos_inner", C.c_float),
                ("intensity", Vec3), ("cos_outer", C.c_float)]


class Camera(C.Structure):
    _fields_ = [("position", Vec3), ("tan_half_fov", C.c_float), ("forward", Vec3), ("aspect", C.c_float),
                ("right", Vec3), ("aperture", C.c_float), ("up", Vec3), ("focus_distance", C.c_float)]


class PathOptions(C.Structure):
    _fields_ = [("max_depth", C.c_int32), ("rr_depth", C.c_int32), ("clamp", C.c_float), ("nee", C.c_int32)]


class RenderSettings(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("path", PathOptions), ("exposure", C.c_float),
                ("tonemap", C.c_int32), ("seed", C.c_uint32)]


class SvgfSettings(C.Structure):
    _fields_ = [("atrous_iterations", C.c_int32), ("alpha_color", C.c_float), ("alpha_moments", C.c_float),
                ("phi_color", C.c_float), ("phi_normal", C.c_float), ("phi_depth", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("nodes", C.POINTER(BvhNode)), ("num_nodes", C.c_int32),
        ("tris", C.POINTER(TriGeom)), ("num_tris", C.c_int32),
        ("indices", C.POINTER(C.c_int32)),
        ("normals", C.POINTER(Vec3)), ("uvs", C.POINTER(Vec2)), ("tangents", C.POINTER(Vec4)),
        ("num_vertices", C.c_int32),
        ("materials", C.POINTER(Material)), ("num_materials", C.c_int32),
        ("textures", C.POINTER(TextureInfo)), ("num_textures", C.c_int32),
        ("texels", C.POINTER(C.c_uint32)), ("num_texels", C.c_uint64),
        ("srgb_lut", C.POINTER(C.c_float)),
        ("emissive", C.POINTER(EmissiveTri)), ("num_emissive", C.c_int32),
        ("tri_emissive", C.POINTER(C.c_int32)),
        ("emissive_alias", C.POINTER(AliasEntry)),
        ("emissive_power", C.c_float),
        ("punctual", C.POINTER(PunctualLight)), ("num_punctual", C.c_int32),
        ("env_texels", C.POINTER(Vec3)), ("env_width", C.c_int32), ("env_height", C.c_int32),
        ("env_marginal", C.POINTER(C.c_float)), ("env_conditional", C.POINTER(C.c_float)),
        ("env_intensity", C.c_float), ("env_rotation", C.c_float), ("env_color", Vec3), ("env_integral", C.c_float),
        ("p_env", C.c_float), ("p_emissive", C.c_float), ("p_punctual", C.c_float),
        ("bounds_min", Vec3), ("bounds_max", Vec3),
    ]


class TextureDesc(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("texels", C.POINTER(C.c_uint32)),
                ("repeat", C.c_int32), ("srgb", C.c_int32)]


class RawScene(C.Structure):
    _fields_ = [
        ("positions", C.POINTER(Vec3)), ("num_positions", C.c_int32),
        ("normals", C.POINTER(Vec3)), ("uvs", C.POINTER(Vec2)), ("tangents", C.POINTER(Vec4)),
        ("indices", C.POINTER(C.c_int32)), ("num_indices", C.c_int32),
        ("tri_material", C.POINTER(C.c_int32)),
        ("materials", C.POINTER(Material)), ("num_materials", C.c_int32),
        ("textures", C.POINTER(TextureDesc)), ("num_textures", C.c_int32),
        ("punctual", C.POINTER(PunctualLight)), ("num_punctual", C.c_int32),
        ("env_texels", C.POINTER(Vec3)), ("env_width", C.c_int32), ("env_height", C.c_int32),
        ("env_color", Vec3), ("env_intensity", C.c_float), ("env_rotation", C.c_float),
    ]


class BvhBuildOptions(C.Structure):
    _fields_ = [("bins", C.c_int32), ("max_leaf_size", C.c_int32), ("traversal_cost", C.c_float),
                ("threads", C.c_int32), ("gpu", C.c_int32)]


class LightUpdate(C.Structure):
    _fields_ = [("materials", C.POINTER(Material)), ("num_materials", C.c_int32),
                ("punctual", C.POINTER(PunctualLight)), ("num_punctual", C.c_int32),
                ("env_texels", C.POINTER(Vec3)), ("env_width", C.c_int32), ("env_height", C.c_int32),
                ("env_color", Vec3), ("env_intensity", C.c_float), ("env_rotation", C.c_float)]


class Stats(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("samples", C.c_int32), ("last_frame_ms", C.c_float),
                ("paths", C.c_uint64), ("rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("bounce_iterations", C.c_uint64), ("queue_overflows", C.c_uint64), ("device_bytes", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("path_capacity", C.c_int32), ("trace_block", C.c_int32), ("shade_block", C.c_int32),
                ("sort_by_material", C.c_int32), ("graph_bounces", C.c_int32), ("sort_rays", C.c_int32),
                ("packed", C.c_int32), ("tail_paths", C.c_int32), ("wide_shadows", C.c_int32),
                ("trace_refill", C.c_int32), ("shadow_refill", C.c_int32), ("walk_burst", C.c_int32),
                ("sort_shadows", C.c_int32), ("pair_walk", C.c_int32)]


class KernelTime(C.Structure):
    _fields_ = [("launches", C.c_uint64), ("ms", C.c_double)]


class Profile(C.Structure):
    _fields_ = [("setup", KernelTime), ("generate", KernelTime), ("trace", KernelTime), ("shade", KernelTime),
                ("shadow", KernelTime), ("accumulate", KernelTime), ("kernel_launches", C.c_uint64),
                ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("closest_node_visits", C.c_uint64),
                ("closest_tri_tests", C.c_uint64), ("shadow_node_visits", C.c_uint64), ("shadow_tri_tests", C.c_uint64),
                ("closest_lane_steps", C.c_uint64), ("closest_warp_steps", C.c_uint64), ("shadow_lane_steps", C.c_uint64),
                ("shadow_warp_steps", C.c_uint64)]


PT_PROFILE_KERNEL_TIMES, PT_PROFILE_TRAVERSAL_COUNTS = 1, 2


class View(C.Structure):
    _fields_ = [("camera", Camera), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("seed", C.c_uint32), ("path", PathOptions)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("budget_bytes", C.c_uint64), ("path_capacity", C.c_int32),
                ("max_active", C.c_int32), ("device_wait_seconds", C.c_double), ("sort_rays", C.c_int32),
                ("reserve_bytes", C.c_int64)]


class Request(C.Structure):
    _fields_ = [("scene_id", C.c_int32), ("camera", Camera), ("width", C.c_int32), ("height", C.c_int32),
                ("spp", C.c_int32), ("seed", C.c_uint32), ("path", PathOptions), ("display", C.c_int32), ("exposure", C.c_float),
                ("tonemap", C.c_int32)]


class RequestStats(C.Structure):
    _fields_ = [("submit_s", C.c_double), ("admit_s", C.c_double), ("done_s", C.c_double),
                ("samples", C.c_uint64), ("state", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("cancelled", C.c_uint64),
                ("rejected", C.c_uint64), ("samples_done", C.c_uint64), ("bounce_iterations", C.c_uint64),
                ("device_bytes_in_use", C.c_uint64), ("budget_bytes", C.c_uint64),
                ("active", C.c_int32), ("queued", C.c_int32), ("scenes", C.c_int32), ("busy_seconds", C.c_double),
                ("device_seconds", C.c_double), ("batches", C.c_uint64)]


def path_options(max_depth=8, rr_depth=3, clamp=0.0, nee=1):
    """photon::PathOptions defaults (src/render/integrator.h:21-27)."""
    return PathOptions(max_depth, rr_depth, clamp, nee)


def render_settings(width, height, max_depth=8, rr_depth=3, clamp=0.0, nee=1, exposure=1.0,
                    tonemap=PT_TONEMAP_ACES, seed=0):
    """photon::RenderSettings defaults (src/render/pixel.h:10-16)."""
    return RenderSettings(width, height, path_options(max_depth, rr_depth, clamp, nee), exposure, tonemap, seed)


def svgf_settings(atrous_iterations=5, alpha_color=0.2, alpha_moments=0.2, phi_color=4.0, phi_normal=128.0,
                  phi_depth=1.0):
    """photon::SvgfSettings defaults (src/render/gpu_renderer.h:18-25)."""
    return SvgfSettings(atrous_iterations, alpha_color, alpha_moments, phi_color, phi_normal, phi_depth)


EXPECTED_SIZES = {
    BvhNode: 64, TriGeom: 48, Material: 80, TextureInfo: 20, EmissiveTri: 8, AliasEntry: 16, PunctualLight: 48,
    Camera: 64, PathOptions: 16, RenderSettings: 36, SvgfSettings: 24,
}
