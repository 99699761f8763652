// Test-infrastructure shim over Photon's CUDA code: the one-thread-per-pixel megakernel renderer
// (src/render/gpu_renderer.cu) and the SVGF denoiser (src/denoise/svgf.cu), built unchanged with
// Photon's own flags by oracle/Makefile into oracle/_ref/libphoton_ref_gpu.so. Used only as the SVGF
// oracle (identical G-buffers in, outputs compared) and as the megakernel comparison.
#include <cstring>
#include <string>
#include <vector>

#include "denoise/svgf.h"
#include "render/gpu_renderer.h"
#include "scene/scene.h"

#include "photon_wavefront.h"

using namespace photon;

extern "C" const void* ref_scene_object(void* h);

namespace {
CameraView to_view(const pt_camera* c) {
    CameraView v;
    std::memcpy(&v, c, sizeof(v));
    return v;
}
RenderSettings to_settings(const pt_render_settings* s) {
    RenderSettings r;
    r.width = s->width;
    r.height = s->height;
    r.path.max_depth = s->path.max_depth;
    r.path.rr_depth = s->path.rr_depth;
    r.path.clamp = s->path.clamp;
    r.path.nee = s->path.nee;
    r.exposure = s->exposure;
    r.tonemap = ToneMap(s->tonemap);
    r.seed = s->seed;
    return r;
}
SvgfSettings to_svgf(const pt_svgf_settings* s) {
    SvgfSettings v;
    v.atrous_iterations = s->atrous_iterations;
    v.alpha_color = s->alpha_color;
    v.alpha_moments = s->alpha_moments;
    v.phi_color = s->phi_color;
    v.phi_normal = s->phi_normal;
    v.phi_depth = s->phi_depth;
    return v;
}
}  // namespace

extern "C" {

int refgpu_available() { return cuda_available(nullptr) ? 1 : 0; }

void* refgpu_create() { return new GpuRenderer(); }
void refgpu_destroy(void* g) { delete static_cast<GpuRenderer*>(g); }

// GpuRenderer::upload of a scene built by the reference shim (ref_builtin_scene / ref_scene_from_*).
int refgpu_upload(void* g, void* ref_scene) {
    std::string error;
    const Scene* s = static_cast<const Scene*>(ref_scene_object(ref_scene));
    return static_cast<GpuRenderer*>(g)->upload(*s, error) ? 1 : 0;
}
void refgpu_resize(void* g, int w, int h) { static_cast<GpuRenderer*>(g)->resize(w, h); }
void refgpu_reset(void* g) { static_cast<GpuRenderer*>(g)->reset(); }
// GpuRenderer::render; returns last_frame_ms (cudaEvent time of the launch).
float refgpu_render(void* g, const pt_camera* cam, const pt_render_settings* rs, int spp) {
    GpuRenderer* r = static_cast<GpuRenderer*>(g);
    r->render(to_view(cam), to_settings(rs), spp);
    return r->last_frame_ms();
}
float refgpu_render_denoised(void* g, const pt_camera* cam, const pt_camera* prev, const pt_render_settings* rs,
                             const pt_svgf_settings* sv) {
    GpuRenderer* r = static_cast<GpuRenderer*>(g);
    r->render_denoised(to_view(cam), to_view(prev), to_settings(rs), to_svgf(sv));
    return r->last_frame_ms();
}
int refgpu_samples(void* g) { return static_cast<GpuRenderer*>(g)->samples(); }
void refgpu_download_image(void* g, float* rgb) {
    std::vector<vec3> img = static_cast<GpuRenderer*>(g)->download_image();
    std::memcpy(rgb, img.data(), img.size() * sizeof(vec3));
}

// Svgf (svgf.h:32-59) on caller device buffers.
void* refsvgf_create(int w, int h) {
    Svgf* s = new Svgf();
    s->resize(w, h);
    return s;
}
void refsvgf_destroy(void* s) { delete static_cast<Svgf*>(s); }
void refsvgf_reset(void* s) { static_cast<Svgf*>(s)->reset(); }
void refsvgf_run(void* s, const float* color, const float* albedo, const float* normal_depth, const float* position,
                 const float* emission, const pt_camera* prev, const pt_svgf_settings* settings, float* output) {
    SvgfInput in{reinterpret_cast<const vec4*>(color), reinterpret_cast<const vec4*>(albedo),
                 reinterpret_cast<const vec4*>(normal_depth), reinterpret_cast<const vec4*>(position),
                 reinterpret_cast<const vec4*>(emission)};
    static_cast<Svgf*>(s)->run(in, to_view(prev), to_svgf(settings), reinterpret_cast<vec4*>(output));
}
const float* refsvgf_variance(void* s) { return reinterpret_cast<const float*>(static_cast<Svgf*>(s)->variance_buffer()); }

}  // extern "C"
