// photon::GpuRenderer over the wavefront C ABI (include/photon_wavefront.h): a header-only drop-in
// for Photon's src/render/gpu_renderer.h. Put this directory (include/photon_dropin) before Photon's
// src/ on the include path, do not compile src/render/gpu_renderer.cu or src/denoise/svgf.cu, and
// link libphoton_wavefront.so: callers (render_cli.cpp, tests/test_gpu.cpp, the viewer) compile
// unchanged. Declarations mirror gpu_renderer.h:16-75; errors follow Photon's conventions
// (upload / update_lights return false with a message, other calls throw std::runtime_error).
#pragma once

#include <cstddef>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "photon_wavefront.h"
#include "render/pixel.h"
#include "scene/scene.h"

namespace photon {

enum class DisplayMode : int { Color = 0, Albedo = 1, Normal = 2, Depth = 3, Variance = 4, Heatmap = 5 };

struct SvgfSettings {
    int atrous_iterations = 5;
    float alpha_color = 0.2f;
    float alpha_moments = 0.2f;
    float phi_color = 4.0f;
    float phi_normal = 128.0f;
    float phi_depth = 1.0f;
};

struct GpuInfo {
    std::string name;
    int compute_major = 0, compute_minor = 0;
    size_t memory = 0;
    int multiprocessors = 0;
};

inline bool cuda_available(GpuInfo* info = nullptr) {
    char name[256] = {0};
    int32_t major = 0, minor = 0, mp = 0;
    uint64_t mem = 0;
    if (!pt_device_info(name, sizeof(name), &major, &minor, &mem, &mp)) return false;
    if (info) {
        info->name = name;
        info->compute_major = major;
        info->compute_minor = minor;
        info->memory = size_t(mem);
        info->multiprocessors = mp;
    }
    return true;
}

namespace wavefront_detail {

static_assert(sizeof(CameraView) == sizeof(pt_camera), "CameraView layout");
static_assert(sizeof(BvhNode) == sizeof(pt_bvh_node) && sizeof(TriGeom) == sizeof(pt_tri_geom), "BVH layout");
static_assert(sizeof(Material) == sizeof(pt_material) && sizeof(PunctualLight) == sizeof(pt_punctual_light), "light layout");
static_assert(sizeof(AliasEntry) == sizeof(pt_alias_entry) && sizeof(EmissiveTri) == sizeof(pt_emissive_tri), "table layout");

template <typename T, typename U>
inline const T* ptr_or_null(const std::vector<U>& v) {
    return v.empty() ? nullptr : reinterpret_cast<const T*>(v.data());
}

// The built arrays of a Scene (scene.h:75-89) as a pt_scene_desc (no copies: pointer casts).
inline pt_scene_desc describe(const Scene& s) {
    pt_scene_desc d{};
    d.nodes = ptr_or_null<pt_bvh_node>(s.bvh.nodes);
    d.num_nodes = int32_t(s.bvh.nodes.size());
    d.tris = ptr_or_null<pt_tri_geom>(s.tris);
    d.num_tris = int32_t(s.tris.size());
    d.indices = ptr_or_null<int32_t>(s.bvh_indices);
    d.normals = ptr_or_null<pt_vec3>(s.normals);
    d.uvs = ptr_or_null<pt_vec2>(s.uvs);
    d.tangents = ptr_or_null<pt_vec4>(s.tangents);
    d.num_vertices = int32_t(s.positions.size());
    d.materials = ptr_or_null<pt_material>(s.materials);
    d.num_materials = int32_t(s.materials.size());
    d.textures = ptr_or_null<pt_texture_info>(s.texture_infos);
    d.num_textures = int32_t(s.texture_infos.size());
    d.texels = ptr_or_null<uint32_t>(s.texel_pool);
    d.num_texels = s.texel_pool.size();
    d.srgb_lut = ptr_or_null<float>(s.srgb_lut);
    d.emissive = ptr_or_null<pt_emissive_tri>(s.emissive);
    d.num_emissive = int32_t(s.emissive.size());
    d.tri_emissive = ptr_or_null<int32_t>(s.tri_emissive);
    d.emissive_alias = ptr_or_null<pt_alias_entry>(s.emissive_alias);
    d.emissive_power = s.emissive_power;
    d.punctual = ptr_or_null<pt_punctual_light>(s.punctual);
    d.num_punctual = int32_t(s.punctual.size());
    d.env_texels = ptr_or_null<pt_vec3>(s.env.texels);
    d.env_width = s.env.width;
    d.env_height = s.env.height;
    d.env_marginal = ptr_or_null<float>(s.env_marginal);
    d.env_conditional = ptr_or_null<float>(s.env_conditional);
    d.env_intensity = s.env.intensity;
    d.env_rotation = s.env.rotation;
    d.env_color = {s.env.color.x, s.env.color.y, s.env.color.z};
    d.env_integral = s.env_integral;
    d.p_env = s.p_env;
    d.p_emissive = s.p_emissive;
    d.p_punctual = s.p_punctual;
    d.bounds_min = {s.bvh.bounds.min.x, s.bvh.bounds.min.y, s.bvh.bounds.min.z};
    d.bounds_max = {s.bvh.bounds.max.x, s.bvh.bounds.max.y, s.bvh.bounds.max.z};
    return d;
}

inline pt_camera camera(const CameraView& c) {
    pt_camera p;
    std::memcpy(&p, &c, sizeof(p));
    return p;
}

inline pt_render_settings settings(const RenderSettings& r) {
    pt_render_settings s{};
    s.width = r.width;
    s.height = r.height;
    s.path = {r.path.max_depth, r.path.rr_depth, r.path.clamp, r.path.nee};
    s.exposure = r.exposure;
    s.tonemap = int32_t(r.tonemap);
    s.seed = r.seed;
    return s;
}

}  // namespace wavefront_detail

class GpuRenderer {
public:
    GpuRenderer() {
        if (pt_create(0, &h_) != PT_OK) throw std::runtime_error(std::string("CUDA error: ") + pt_global_error());
    }
    ~GpuRenderer() { pt_destroy(h_); }
    GpuRenderer(const GpuRenderer&) = delete;
    GpuRenderer& operator=(const GpuRenderer&) = delete;

    bool upload(const Scene& scene, std::string& error) {
        if (!scene.built) {
            error = "the scene is not built";
            return false;
        }
        pt_scene_desc d = wavefront_detail::describe(scene);
        if (pt_upload_scene(h_, &d) != PT_OK) {
            error = pt_last_error(h_);
            return false;
        }
        return true;
    }
    bool update_lights(const Scene& scene, std::string& error) {
        pt_scene_desc d = wavefront_detail::describe(scene);
        if (pt_update_lights(h_, &d) != PT_OK) {
            error = pt_last_error(h_);
            return false;
        }
        return true;
    }
    void resize(int width, int height) { check(pt_resize(h_, width, height)); }
    void reset() { check(pt_reset(h_)); }
    void render(const CameraView& camera, const RenderSettings& settings, int spp) {
        pt_camera c = wavefront_detail::camera(camera);
        pt_render_settings s = wavefront_detail::settings(settings);
        int32_t e = pt_render(h_, &c, &s, spp);
        if (e != PT_OK && e != PT_ERR_NO_SCENE) check(e);  // Photon renders nothing before upload
    }
    void render_denoised(const CameraView& camera, const CameraView& previous, const RenderSettings& settings, const SvgfSettings& svgf) {
        pt_camera c = wavefront_detail::camera(camera), p = wavefront_detail::camera(previous);
        pt_render_settings s = wavefront_detail::settings(settings);
        pt_svgf_settings v{svgf.atrous_iterations, svgf.alpha_color, svgf.alpha_moments, svgf.phi_color, svgf.phi_normal, svgf.phi_depth};
        int32_t e = pt_render_denoised(h_, &c, &p, &s, &v);
        if (e != PT_OK && e != PT_ERR_NO_SCENE) check(e);
    }
    void display(const RenderSettings& settings, DisplayMode mode, uint32_t* target = nullptr) {
        pt_render_settings s = wavefront_detail::settings(settings);
        check(pt_display(h_, &s, int32_t(mode), target));
    }
    std::vector<vec3> download_image() {
        pt_stats st{};
        pt_get_stats(h_, &st);
        std::vector<vec3> out(size_t(st.width) * size_t(st.height));
        check(pt_download_image(h_, reinterpret_cast<float*>(out.data()), out.size() * 3));
        return out;
    }
    std::vector<uint32_t> download_display() {
        pt_stats st{};
        pt_get_stats(h_, &st);
        std::vector<uint32_t> out(size_t(st.width) * size_t(st.height));
        check(pt_download_display(h_, out.data(), out.size()));
        return out;
    }
    int width() const { return stats().width; }
    int height() const { return stats().height; }
    int samples() const { return stats().samples; }
    float last_frame_ms() const { return stats().last_frame_ms; }
    uint32_t* display_buffer() const { return pt_display_buffer(h_); }

private:
    pt_stats stats() const {
        pt_stats st{};
        pt_get_stats(h_, &st);
        return st;
    }
    void check(int32_t e) const {
        if (e != PT_OK) throw std::runtime_error(std::string("CUDA error: ") + pt_last_error(h_));
    }
    pt_renderer* h_ = nullptr;
};

}  // namespace photon
