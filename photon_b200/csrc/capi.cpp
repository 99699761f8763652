// The C ABI (include/photon_wavefront.h): status codes at the boundary, exceptions inside.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "peaks.h"
#include "photon_wavefront.h"
#include "renderer.h"
#include "scene_build.h"
#include "server.h"
#include "svgf.h"

using namespace ptw;

namespace {

thread_local std::string g_error;
thread_local std::string server_error;  // pt_server_last_error of the calling thread

template <typename F>
int32_t guarded(std::string* err, F&& f) {
    try {
        f();
        if (err) err->clear();
        return PT_OK;
    } catch (const Error& e) {
        if (err) *err = e.message;
        g_error = e.message;
        return e.code;
    } catch (const std::bad_alloc&) {
        if (err) *err = "host allocation failed";
        g_error = "host allocation failed";
        return PT_ERR_ALLOC;
    } catch (const std::exception& e) {
        if (err) *err = e.what();
        g_error = e.what();
        return PT_ERR_INVALID;
    }
}

// An sm_100 device (the kernels are built for sm_100a only).
void require_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error{PT_ERR_NO_DEVICE, "no CUDA device"};
    }
    if (device < 0 || device >= count) throw Error{PT_ERR_NO_DEVICE, "device ordinal out of range"};
    cudaDeviceProp p{};
    PTW_CUDA(cudaGetDeviceProperties(&p, device));
    if (p.major != 10) throw Error{PT_ERR_NO_DEVICE, std::string("the kernels are built for sm_100a; device is ") + p.name};
}

}  // namespace

struct pt_renderer {
    std::unique_ptr<Renderer> r;
    std::string error;
};

struct pt_svgf {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::unique_ptr<SvgfDenoiser> s;
    std::string error;
    ~pt_svgf() {
        s.reset();
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

struct pt_built_scene {
    BuiltScene b;
};

struct pt_generated {
    GeneratedScene g;
};

struct pt_server {
    std::unique_ptr<Server> s;
};

extern "C" {

int32_t pt_abi_version(void) { return PT_ABI_VERSION; }

const char* pt_global_error(void) { return g_error.c_str(); }

int32_t pt_device_info(char* name, size_t name_len, int32_t* major, int32_t* minor, uint64_t* memory_bytes, int32_t* multiprocessors) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return 0;
    }
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, 0) != cudaSuccess) return 0;
    if (name && name_len) {
        std::strncpy(name, p.name, name_len - 1);
        name[name_len - 1] = 0;
    }
    if (major) *major = p.major;
    if (minor) *minor = p.minor;
    if (memory_bytes) *memory_bytes = p.totalGlobalMem;
    if (multiprocessors) *multiprocessors = p.multiProcessorCount;
    return 1;
}

// ---- renderer ------------------------------------------------------------------------------------------

int32_t pt_create(int32_t device, pt_renderer** out) {
    if (!out) return PT_ERR_INVALID;
    *out = nullptr;
    return guarded(nullptr, [&] {
        require_device(device);
        auto h = std::make_unique<pt_renderer>();
        h->r = std::make_unique<Renderer>(device);
        *out = h.release();
    });
}

void pt_destroy(pt_renderer* r) { delete r; }

const char* pt_last_error(const pt_renderer* r) { return r ? r->error.c_str() : g_error.c_str(); }

#define PT_RENDERER_CALL(r, body)                       \
    if (!(r) || !(r)->r) return PT_ERR_INVALID;         \
    return guarded(&(r)->error, [&] { body; })

int32_t pt_upload_scene(pt_renderer* r, const pt_scene_desc* scene) {
    if (!scene) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->upload(*scene, false));
}

int32_t pt_update_lights(pt_renderer* r, const pt_scene_desc* scene) {
    if (!scene) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->upload(*scene, true));
}

int32_t pt_rebuild_lights(pt_renderer* r, const pt_light_update* update) {
    if (!update) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->rebuild_lights(*update));
}

int32_t pt_resize(pt_renderer* r, int32_t width, int32_t height) { PT_RENDERER_CALL(r, r->r->resize(width, height)); }

int32_t pt_reset(pt_renderer* r) { PT_RENDERER_CALL(r, r->r->reset()); }

int32_t pt_render(pt_renderer* r, const pt_camera* camera, const pt_render_settings* settings, int32_t spp) {
    if (!camera || !settings) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->render(*camera, *settings, spp));
}

int32_t pt_render_denoised(pt_renderer* r, const pt_camera* camera, const pt_camera* previous, const pt_render_settings* settings,
                           const pt_svgf_settings* svgf) {
    if (!camera || !previous || !settings || !svgf) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->render_denoised(*camera, *previous, *settings, *svgf));
}

int32_t pt_display(pt_renderer* r, const pt_render_settings* settings, int32_t mode, uint32_t* device_target) {
    if (!settings || mode < 0 || mode > PT_DISPLAY_HEATMAP) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->display(*settings, mode, device_target));
}

int32_t pt_download_image(pt_renderer* r, float* rgb, size_t n) {
    if (!rgb && n) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->download_image(rgb, n));
}

int32_t pt_download_display(pt_renderer* r, uint32_t* rgba8, size_t n) {
    if (!rgba8 && n) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->download_display(rgba8, n));
}

int32_t pt_download_gbuffer(pt_renderer* r, float* albedo4, float* normal_depth4, size_t n_pixels) {
    PT_RENDERER_CALL(r, r->r->download_gbuffer(albedo4, normal_depth4, n_pixels));
}

int32_t pt_download_accumulation(pt_renderer* r, float* sums4, size_t n_pixels) {
    PT_RENDERER_CALL(r, r->r->download_accumulation(sums4, n_pixels));
}

uint32_t* pt_display_buffer(pt_renderer* r) { return r && r->r ? r->r->display_buffer() : nullptr; }

int32_t pt_get_stats(const pt_renderer* r, pt_stats* out) {
    if (!r || !r->r || !out) return PT_ERR_INVALID;
    r->r->stats(out);
    return PT_OK;
}

void* pt_renderer_stream(pt_renderer* r) { return r && r->r ? reinterpret_cast<void*>(r->r->stream()) : nullptr; }

int32_t pt_measure_l2_bandwidth(int32_t device, size_t bytes, int32_t reps, double* gbs) {
    if (!gbs) return PT_ERR_INVALID;
    *gbs = 0.0;
    return guarded(nullptr, [&] {
        require_device(device);
        *gbs = measure_l2_read_gbs(device, bytes, reps);
    });
}

int32_t pt_set_profiling(pt_renderer* r, int32_t flags) { PT_RENDERER_CALL(r, r->r->set_profiling(flags)); }

int32_t pt_get_profile(const pt_renderer* r, pt_profile* out) {
    if (!r || !r->r || !out) return PT_ERR_INVALID;
    r->r->get_profile(out);
    return PT_OK;
}

int32_t pt_set_tuning(pt_renderer* r, const pt_tuning* t) {
    if (!t) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->set_tuning(*t));
}

int32_t pt_autotune(pt_renderer* r, const pt_camera* camera, const pt_render_settings* settings, int32_t spp, uint64_t probe_samples,
                    pt_tuning* chosen, double* default_rate, double* tuned_rate) {
    if (!camera || !settings) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->autotune(*camera, *settings, spp, probe_samples, chosen, default_rate, tuned_rate));
}

int32_t pt_autotune_views(pt_renderer* r, const pt_view* views, int32_t n_views, uint64_t probe_samples, pt_tuning* chosen,
                          double* default_rate, double* tuned_rate) {
    if (!views || n_views <= 0) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->autotune_views(views, n_views, probe_samples, chosen, default_rate, tuned_rate));
}

int32_t pt_get_tuning(const pt_renderer* r, pt_tuning* t) {
    if (!r || !r->r || !t) return PT_ERR_INVALID;
    r->r->get_tuning(t);
    return PT_OK;
}

int32_t pt_occlusion_probe(pt_renderer* r, const float* rays8, int32_t n, int32_t wide, int32_t* out4) {
    if (!rays8 || !out4 || n < 0) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->occlusion_probe(rays8, n, wide, out4));
}

int32_t pt_trace_primary(pt_renderer* r, const pt_camera* camera, int32_t width, int32_t height, uint32_t frame, uint32_t seed, float* hits4) {
    if (!camera || !hits4) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->trace_primary(*camera, width, height, frame, seed, hits4));
}

int32_t pt_light_picks_primary(pt_renderer* r, const pt_camera* camera, const pt_render_settings* settings, uint32_t frame, int32_t* picks4) {
    if (!camera || !settings || !picks4) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->light_picks(*camera, *settings, frame, picks4));
}

int32_t pt_heatmap(pt_renderer* r, const pt_camera* camera, int32_t width, int32_t height, float* visits) {
    if (!camera || !visits) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->heatmap(*camera, width, height, visits));
}

int32_t pt_render_views(pt_renderer* r, const pt_view* views, int32_t n_views) {
    if (!views && n_views) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->render_views(views, n_views));
}

int32_t pt_download_view(pt_renderer* r, int32_t view, float* rgb, size_t n) {
    if (!rgb && n) return PT_ERR_INVALID;
    PT_RENDERER_CALL(r, r->r->download_view(view, rgb, n));
}

// ---- SVGF --------------------------------------------------------------------------------------------------

int32_t pt_svgf_create(int32_t device, int32_t width, int32_t height, pt_svgf** out) {
    if (!out || width < 0 || height < 0) return PT_ERR_INVALID;
    *out = nullptr;
    return guarded(nullptr, [&] {
        require_device(device);
        PTW_CUDA(cudaSetDevice(device));
        auto h = std::make_unique<pt_svgf>();
        h->device = device;
        PTW_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->s = std::make_unique<SvgfDenoiser>(device, h->stream);
        h->s->resize(width, height);
        *out = h.release();
    });
}

void pt_svgf_destroy(pt_svgf* s) { delete s; }

int32_t pt_svgf_reset(pt_svgf* s) {
    if (!s) return PT_ERR_INVALID;
    s->s->reset();
    return PT_OK;
}

int32_t pt_svgf_run(pt_svgf* s, const float* color, const float* albedo, const float* normal_depth, const float* position,
                    const float* emission, const pt_camera* previous, const pt_svgf_settings* settings, float* output) {
    if (!s || !color || !albedo || !normal_depth || !position || !emission || !previous || !settings || !output) return PT_ERR_INVALID;
    return guarded(&server_error, [&] {
        PTW_CUDA(cudaSetDevice(s->device));
        s->s->run(color, albedo, normal_depth, position, emission, *previous, *settings, output);
        PTW_CUDA(cudaStreamSynchronize(s->stream));
    });
}

int32_t pt_svgf_set_tma(pt_svgf* s, int32_t mode) {
    if (!s) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->set_tma(mode); });
}

int32_t pt_svgf_debug_tma_timeout(pt_svgf* s, int32_t on) {
    if (!s) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->set_tma_timeout_test(on != 0); });
}

const float* pt_svgf_variance(const pt_svgf* s) { return s ? s->s->variance() : nullptr; }

const char* pt_svgf_last_error(const pt_svgf* s) { return s ? s->error.c_str() : g_error.c_str(); }

int32_t pt_svgf_run_noalloc(int32_t device, int32_t width, int32_t height, const float* color, const float* albedo,
                            const float* normal_depth, const float* position, const float* emission, const pt_svgf_settings* settings,
                            float* output, void* stream) {
    if (!color || !albedo || !normal_depth || !position || !emission || !settings || !output) return PT_ERR_INVALID;
    return guarded(nullptr, [&] {
        svgf_run_noalloc(device, width, height, color, albedo, normal_depth, position, emission, *settings, output,
                         reinterpret_cast<cudaStream_t>(stream));
    });
}

// ---- server ------------------------------------------------------------------------------------------------

int32_t pt_server_create(const pt_server_config* cfg, pt_server** out) {
    if (!cfg || !out) return PT_ERR_INVALID;
    *out = nullptr;
    return guarded(nullptr, [&] {
        require_device(cfg->device);
        auto h = std::make_unique<pt_server>();
        h->s = std::make_unique<Server>(*cfg);
        *out = h.release();
    });
}

void pt_server_destroy(pt_server* s) { delete s; }

// The server handle is shared between threads, so its last error is kept per calling thread.
const char* pt_server_last_error(const pt_server*) { return server_error.c_str(); }

int32_t pt_server_add_scene(pt_server* s, const pt_scene_desc* scene, int32_t* scene_id) {
    if (!s || !scene || !scene_id) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { *scene_id = s->s->add_scene(*scene); });
}

int32_t pt_server_submit(pt_server* s, const pt_request* req, uint64_t* request_id) {
    if (!s || !req || !request_id) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { *request_id = s->s->submit(*req); });
}

int32_t pt_server_poll(pt_server* s, uint64_t request_id, int32_t* state) {
    if (!s || !state) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { *state = s->s->poll(request_id); });
}

int32_t pt_server_wait(pt_server* s, uint64_t request_id, double timeout_s) {
    if (!s) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->wait(request_id, timeout_s); });
}

int32_t pt_server_fetch(pt_server* s, uint64_t request_id, float* rgb, size_t n, pt_request_stats* st) {
    if (!s) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->fetch(request_id, rgb, n, st); });
}

int32_t pt_server_cancel(pt_server* s, uint64_t request_id) {
    if (!s) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->cancel(request_id); });
}

int32_t pt_server_get_stats(pt_server* s, pt_server_stats* out) {
    if (!s || !out) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->stats(out); });
}

int32_t pt_server_debug_fail_allocations(pt_server* s, int32_t count) {
    if (!s || count < 0) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->inject_allocation_failures(count); });
}

int32_t pt_server_fetch_encoded(pt_server* s, uint64_t request_id, int32_t format, uint8_t* out, size_t capacity, size_t* length) {
    if (!s || !length || (format != PT_IMAGE_PFM && format != PT_IMAGE_PNG)) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->fetch_encoded(request_id, format, out, capacity, length); });
}

int32_t pt_server_open_session(pt_server* s, int32_t scene_id, int32_t width, int32_t height, const pt_svgf_settings* svgf,
                               int32_t* session_id) {
    if (!s || !svgf || !session_id) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { *session_id = s->s->open_session(scene_id, width, height, *svgf); });
}

int32_t pt_server_submit_frame(pt_server* s, int32_t session_id, const pt_camera* camera, const pt_camera* previous,
                               const pt_render_settings* settings, uint64_t* request_id) {
    if (!s || !camera || !previous || !settings || !request_id) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { *request_id = s->s->submit_frame(session_id, *camera, *previous, *settings); });
}

int32_t pt_server_close_session(pt_server* s, int32_t session_id) {
    if (!s) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->close_session(session_id); });
}

int32_t pt_server_set_tuning(pt_server* s, const pt_tuning* t) {
    if (!s || !t) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->set_tuning(*t); });
}

int32_t pt_server_debug_fail_finishing(pt_server* s, int32_t count) {
    if (!s || count < 0) return PT_ERR_INVALID;
    return guarded(&server_error, [&] { s->s->inject_finishing_failures(count); });
}

// ---- scene construction --------------------------------------------------------------------------------

int32_t pt_scene_build(const pt_raw_scene* raw, const pt_bvh_build_options* opt, pt_built_scene** out) {
    if (!raw || !out) return PT_ERR_INVALID;
    *out = nullptr;
    return guarded(nullptr, [&] {
        auto h = std::make_unique<pt_built_scene>();
        BvhOptions o;
        if (opt) {
            if (opt->bins > 0) o.bins = opt->bins;
            if (opt->max_leaf_size > 0) o.max_leaf = opt->max_leaf_size;
            if (opt->traversal_cost > 0) o.traversal_cost = opt->traversal_cost;
            o.threads = opt->threads;
            o.gpu = opt->gpu != 0;
        }
        build_scene(*raw, o, h->b);
        *out = h.release();
    });
}

const pt_scene_desc* pt_scene_desc_of(const pt_built_scene* b) { return b ? &b->b.desc : nullptr; }

void pt_scene_free(pt_built_scene* b) { delete b; }

int32_t pt_generate_scene(int32_t kind, int64_t triangles, uint64_t seed, pt_generated** out) {
    if (!out) return PT_ERR_INVALID;
    *out = nullptr;
    return guarded(nullptr, [&] {
        auto h = std::make_unique<pt_generated>();
        generate_scene(kind, triangles, seed, h->g);
        *out = h.release();
    });
}

const pt_raw_scene* pt_generated_raw(const pt_generated* g) { return g ? &g->g.raw : nullptr; }

int32_t pt_generated_camera(const pt_generated* g, float aspect, pt_camera* out) {
    if (!g || !out || !(aspect > 0)) return PT_ERR_INVALID;
    *out = g->g.camera_view(aspect);
    return PT_OK;
}

void pt_generated_free(pt_generated* g) { delete g; }

}  // extern "C"
