/*
 * photon_wavefront.h — the C ABI of the B200 wavefront path tracer.
 *
 * This is the drop-in boundary for Photon's GPU renderer. Every entry point below replaces one member
 * of photon::GpuRenderer (src/render/gpu_renderer.h:36-75 of the Photon sources) or one of the
 * systems forms built beside it (batched views, the request server, SVGF on caller G-buffers).
 *
 * Conventions
 *  - Plain C: opaque handles, plain pointers and sizes, int status codes (PT_OK = 0). The message of
 *    the last failure on a handle is returned by pt_last_error(handle); pt_global_error() holds the
 *    message of failures that happen before a handle exists.
 *  - Scene arrays are COPIED at upload; the caller keeps ownership of every pointer it passes.
 *  - The POD types below have exactly the byte layout of the Photon types named beside them
 *    (src/render/scene_view.h:13-150, src/render/pixel.h:10-16, src/render/integrator.h:21-27), so a
 *    built photon::Scene is passed by pointer casts, without repacking.
 *  - Image buffers are row-major, pixel (x, y) at index y * width + x, RGB float triples unless said.
 *  - A renderer handle is used from one host thread at a time (as GpuRenderer). The server handle is
 *    thread-safe: pt_server_submit / poll / wait / fetch / cancel may be called from any thread.
 */
#ifndef PHOTON_WAVEFRONT_H
#define PHOTON_WAVEFRONT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------------------------- */
enum {
    PT_OK = 0,
    PT_ERR_INVALID = -1,     /* a null handle, a bad size, an inconsistent scene description */
    PT_ERR_CUDA = -2,        /* a CUDA call failed; the message names it */
    PT_ERR_NO_DEVICE = -3,   /* no CUDA device, or not an sm_100 device */
    PT_ERR_NO_SCENE = -4,    /* render before upload */
    PT_ERR_BUDGET = -5,      /* the request or scene does not fit the device-memory budget */
    PT_ERR_TIMEOUT = -6,     /* a wait ran out of time (host wait or a bounded device wait) */
    PT_ERR_CANCELLED = -7,   /* the request was cancelled */
    PT_ERR_NOT_FOUND = -8,   /* unknown request or scene id */
    PT_ERR_OVERFLOW = -9,    /* a device queue overflowed (counted on the device, never trapped) */
    PT_ERR_ALLOC = -10       /* a host or device allocation failed */
};

/* ---- POD types with Photon's layouts ------------------------------------------------------- */
typedef struct pt_vec2 { float x, y; } pt_vec2;
typedef struct pt_vec3 { float x, y, z; } pt_vec3;
typedef struct pt_vec4 { float x, y, z, w; } pt_vec4;

/* photon::BvhNode (scene_view.h:13-22), 64 bytes: the boxes of both children. A child with
 * count > 0 is a leaf over triangles [index, index + count) in BVH order; otherwise index is the
 * child node (or -1 for an empty child). */
typedef struct pt_bvh_node {
    pt_vec3 lmin; int32_t left;
    pt_vec3 lmax; int32_t lcount;
    pt_vec3 rmin; int32_t right;
    pt_vec3 rmax; int32_t rcount;
} pt_bvh_node;

/* photon::TriGeom (scene_view.h:25-32), 48 bytes: a vertex and two edges, in BVH order. */
typedef struct pt_tri_geom {
    pt_vec3 v0; int32_t material;
    pt_vec3 e1; int32_t flags;   /* PT_TRI_ALPHA_TESTED */
    pt_vec3 e2; int32_t pad;
} pt_tri_geom;
#define PT_TRI_ALPHA_TESTED 1

/* photon::TextureInfo (scene_view.h:38-44). */
typedef struct pt_texture_info {
    int32_t width, height;
    uint32_t offset;      /* into the RGBA8 texel pool */
    int32_t wrap_repeat;  /* 1 repeat, 0 clamp */
    int32_t srgb;
} pt_texture_info;

enum { PT_ALPHA_OPAQUE = 0, PT_ALPHA_MASK = 1, PT_ALPHA_BLEND = 2 };

/* photon::Material (scene_view.h:46-63), 80 bytes. */
typedef struct pt_material {
    pt_vec4 base_color;
    pt_vec3 emission;
    float metallic, roughness, ior, transmission, normal_scale, alpha_cutoff;
    int32_t alpha_mode, double_sided;
    int32_t base_color_tex, metallic_roughness_tex, normal_tex, emissive_tex, occlusion_tex;
} pt_material;

/* photon::EmissiveTri (scene_view.h:65-69) and photon::AliasEntry (:71-76). */
typedef struct pt_emissive_tri { int32_t tri; float area; } pt_emissive_tri;
typedef struct pt_alias_entry { float prob; int32_t alias; float pmf; int32_t pad; } pt_alias_entry;

enum { PT_LIGHT_POINT = 0, PT_LIGHT_SPOT = 1, PT_LIGHT_DIRECTIONAL = 2 };

/* photon::PunctualLight (scene_view.h:81-88), 48 bytes. */
typedef struct pt_punctual_light {
    pt_vec3 position; int32_t type;
    pt_vec3 direction; float cos_inner;
    pt_vec3 intensity; float cos_outer;
} pt_punctual_light;

/* photon::CameraView (scene_view.h:106-115), 64 bytes. */
typedef struct pt_camera {
    pt_vec3 position; float tan_half_fov;
    pt_vec3 forward; float aspect;
    pt_vec3 right; float aperture;
    pt_vec3 up; float focus_distance;
} pt_camera;

/* photon::PathOptions (integrator.h:21-27) without the host-only ray counter. */
typedef struct pt_path_options {
    int32_t max_depth;   /* path vertices after the camera (Photon default 8) */
    int32_t rr_depth;    /* Russian roulette from this many bounces (3) */
    float clamp;         /* luminance clamp of indirect light, 0 = off */
    int32_t nee;         /* next event estimation on/off (1) */
} pt_path_options;

enum { PT_TONEMAP_LINEAR = 0, PT_TONEMAP_ACES = 1, PT_TONEMAP_REINHARD = 2 };

/* photon::RenderSettings (pixel.h:10-16). */
typedef struct pt_render_settings {
    int32_t width, height;
    pt_path_options path;
    float exposure;
    int32_t tonemap;
    uint32_t seed;
} pt_render_settings;

/* photon::SvgfSettings (gpu_renderer.h:18-25). */
typedef struct pt_svgf_settings {
    int32_t atrous_iterations;
    float alpha_color, alpha_moments, phi_color, phi_normal, phi_depth;
} pt_svgf_settings;

/* photon::DisplayMode (gpu_renderer.h:16). */
enum { PT_DISPLAY_COLOR = 0, PT_DISPLAY_ALBEDO = 1, PT_DISPLAY_NORMAL = 2, PT_DISPLAY_DEPTH = 3,
       PT_DISPLAY_VARIANCE = 4, PT_DISPLAY_HEATMAP = 5 };

/* A built scene: the arrays photon::Scene::build produces (scene.h:75-89) and the scalars of
 * photon::SceneView (scene_view.h:117-150). Optional arrays may be NULL with a zero count. */
typedef struct pt_scene_desc {
    const pt_bvh_node* nodes; int32_t num_nodes;
    const pt_tri_geom* tris; int32_t num_tris;      /* BVH order */
    const int32_t* indices;                          /* 3 * num_tris vertex indices, BVH order */
    const pt_vec3* normals;                          /* num_vertices or NULL */
    const pt_vec2* uvs;                              /* num_vertices or NULL */
    const pt_vec4* tangents;                         /* num_vertices or NULL */
    int32_t num_vertices;
    const pt_material* materials; int32_t num_materials;
    const pt_texture_info* textures; int32_t num_textures;
    const uint32_t* texels; uint64_t num_texels;     /* RGBA8 pool */
    const float* srgb_lut;                           /* 256 entries */
    const pt_emissive_tri* emissive; int32_t num_emissive;
    const int32_t* tri_emissive;                     /* num_tris entries (index into emissive or -1) */
    const pt_alias_entry* emissive_alias;            /* num_emissive entries */
    float emissive_power;
    const pt_punctual_light* punctual; int32_t num_punctual;
    const pt_vec3* env_texels; int32_t env_width, env_height;
    const float* env_marginal;                       /* env_height + 1 */
    const float* env_conditional;                    /* env_height * (env_width + 1) */
    float env_intensity, env_rotation;
    pt_vec3 env_color;
    float env_integral;
    float p_env, p_emissive, p_punctual;
    pt_vec3 bounds_min, bounds_max;
} pt_scene_desc;

/* ---- library ------------------------------------------------------------------------------- */

/* The ABI version compiled into the library (PT_ABI_VERSION). */
int32_t pt_abi_version(void);
/* photon::cuda_available (gpu_renderer.h:34): 1 with a usable device, else 0. Fills the
 * optional outputs (name up to name_len bytes, compute capability, memory, SM count). */
int32_t pt_device_info(char* name, size_t name_len, int32_t* major, int32_t* minor, uint64_t* memory_bytes,
                       int32_t* multiprocessors);
/* The message of the last failure that had no handle to attach to. */
const char* pt_global_error(void);

/* ---- plain renderer: photon::GpuRenderer ------------------------------------------------------ */
typedef struct pt_renderer pt_renderer;

/* GpuRenderer::GpuRenderer (gpu_renderer.h:38). device = CUDA ordinal. */
int32_t pt_create(int32_t device, pt_renderer** out);
/* GpuRenderer::~GpuRenderer (gpu_renderer.h:39). NULL is accepted. */
void pt_destroy(pt_renderer* r);
/* The message of the last failed call on r (empty when none). */
const char* pt_last_error(const pt_renderer* r);

/* GpuRenderer::upload (gpu_renderer.h:44, gpu_renderer.cu:243-297): copies the built scene to the
 * device (re-laid for 128-bit loads) and resets the accumulation. */
int32_t pt_upload_scene(pt_renderer* r, const pt_scene_desc* scene);
/* GpuRenderer::update_lights (gpu_renderer.h:46, gpu_renderer.cu:299-334): re-uploads triangles,
 * materials, light tables and the environment of a scene whose BVH is unchanged. */
int32_t pt_update_lights(pt_renderer* r, const pt_scene_desc* scene);
/* GpuRenderer::resize (gpu_renderer.h:47, gpu_renderer.cu:336-351). */
int32_t pt_resize(pt_renderer* r, int32_t width, int32_t height);
/* GpuRenderer::reset (gpu_renderer.h:48, gpu_renderer.cu:353-360). */
int32_t pt_reset(pt_renderer* r);
/* GpuRenderer::render (gpu_renderer.h:51, gpu_renderer.cu:362-377): adds spp samples per pixel. */
int32_t pt_render(pt_renderer* r, const pt_camera* camera, const pt_render_settings* settings, int32_t spp);
/* GpuRenderer::render_denoised (gpu_renderer.h:53, gpu_renderer.cu:379-401): one sample per pixel
 * with the full G-buffer, denoised by SVGF against the previous camera. */
int32_t pt_render_denoised(pt_renderer* r, const pt_camera* camera, const pt_camera* previous,
                           const pt_render_settings* settings, const pt_svgf_settings* svgf);
/* GpuRenderer::display (gpu_renderer.h:56, gpu_renderer.cu:403-426): tone maps into the RGBA8
 * display buffer, or into device_target (caller-owned device memory, width*height words). */
int32_t pt_display(pt_renderer* r, const pt_render_settings* settings, int32_t mode, uint32_t* device_target);
/* GpuRenderer::download_image (gpu_renderer.h:58, gpu_renderer.cu:428-443): the average radiance,
 * 3 floats per pixel, into rgb (capacity n floats). */
int32_t pt_download_image(pt_renderer* r, float* rgb, size_t n);
/* GpuRenderer::download_display (gpu_renderer.h:59): n words. */
int32_t pt_download_display(pt_renderer* r, uint32_t* rgba8, size_t n);
/* The G-buffer of the first sample of the last pt_render (or of the last pt_render_denoised):
 * albedo (4 floats/pixel) and normal + depth (4 floats/pixel). Either pointer may be NULL. */
int32_t pt_download_gbuffer(pt_renderer* r, float* albedo4, float* normal_depth4, size_t n_pixels);
/* The accumulation as it stands (a probe, like the G-buffer): per pixel the sum of the samples'
 * radiance (rgb) and of their squared luminance (w), the inputs of pt_display's colour and variance
 * views (GpuRenderer keeps the same sums, gpu_renderer.cu:70-79). */
int32_t pt_download_accumulation(pt_renderer* r, float* sums4, size_t n_pixels);
/* GpuRenderer::display_buffer (gpu_renderer.h:65): the device address of the RGBA8 buffer. */
uint32_t* pt_display_buffer(pt_renderer* r);

typedef struct pt_stats {
    int32_t width, height, samples;
    float last_frame_ms;          /* GpuRenderer::last_frame_ms (gpu_renderer.h:64) */
    uint64_t paths;               /* paths traced by the last render */
    uint64_t rays;                /* camera + extension + shadow rays of the last render */
    uint64_t shadow_rays;
    uint64_t bounce_iterations;   /* wavefront iterations of the last render */
    uint64_t queue_overflows;     /* must stay 0 */
    uint64_t device_bytes;        /* device memory held by this renderer */
} pt_stats;
/* Accessors width/height/samples/last_frame_ms (gpu_renderer.h:61-64) plus wavefront counters. */
int32_t pt_get_stats(const pt_renderer* r, pt_stats* out);

/* Tuning of the wavefront (the autotuner's knobs). Zero fields keep the current value. */
typedef struct pt_tuning {
    int32_t path_capacity;     /* paths in flight */
    int32_t trace_block;       /* threads per block of the traversal kernels */
    int32_t shade_block;       /* threads per block of the shading kernel */
    int32_t sort_by_material;  /* k in 1-4: the shading kernel groups windows of k x shade_block paths by material
                                  class before shading them (4k x shade_block on iterations whose rays
                                  are sorted afterwards); 0: queue order; -1 keep */
    int32_t graph_bounces;     /* bounce iterations captured per CUDA graph launch */
    int32_t sort_rays;         /* 0 off, 1-6: sort continuing rays by direction octant + Morton origin cell
                                  with this many bits per axis before tracing them, on iterations of at
                                  least 2,097,152 paths (4: the renderer's default; the server: 0); -1 keep */
    int32_t packed;            /* 1: f32x2 (packed FP32) slab tests in traversal, 0: scalar; -1 keep */
    int32_t tail_paths;        /* once no new paths remain and at most this many are queued, one kernel finishes
                                  them (a thread per path, every bounce); 0 never; -1 keep; -2 (default)
                                  131,072 for a render that starts while no other render of this process
                                  runs on the device, 65,536 otherwise and in the server */
    int32_t wide_shadows;      /* 1: shadow rays walk a 4-wide BVH collapsed from the scene's BVH2 (same
                                  answers), 0 (default): the BVH2; -1 keep */
    int32_t trace_refill;      /* 1-32: a warp of the closest-hit walk claims new rays for its idle lanes
                                  once fewer than this many lanes hold a ray (1: only when all have
                                  finished, 32 rays at a time); <= 0 keep */
    int32_t shadow_refill;     /* the same for the shadow (any-hit) walk; <= 0 keep */
    int32_t walk_burst;        /* walk steps each lane takes between two refill checks of its warp (1 to 2^20);
                                  <= 0 keep */
    int32_t sort_shadows;      /* 0 off (the default), 1-6: walk the shadow rays of iterations of at least
                                  2,097,152 paths ordered by direction octant + Morton origin cell (this
                                  many bits per axis); -1 keep */
    int32_t pair_walk;         /* 0: each lane walks its ray through node visits and triangle tests on its own;
                                  1-64 (default 5): pair walks, with the leaf triangles a warp's rays reach
                                  tested by all its lanes together after up to this many node visits per
                                  lane (same hits and answers; packed slab tests and the BVH2 only, so
                                  packed = 0 and the 4-wide shadow walk use the per-lane walks); -1 keep */
} pt_tuning;
int32_t pt_set_tuning(pt_renderer* r, const pt_tuning* t);
int32_t pt_get_tuning(const pt_renderer* r, pt_tuning* t);
/* The autotuner: picks path capacity, block shapes, material sorting, graph cadence, ray sorting, the
 * tail size and the walk knobs (4-wide shadows, refill thresholds, burst, shadow order, pair walks) for
 * the uploaded scene by coordinate descent, timing probe renders of `camera` (at most `probe_samples`
 * paths each, into private buffers: the accumulation is untouched). A knob moves for a gain above 2%,
 * and the final pick is kept only if it still beats the starting tuning by 2% when both are timed
 * again. Applies the kept tuning, returns it in `chosen` (optional) and the probe throughput of the
 * starting and kept tunings (samples/s). */
int32_t pt_autotune(pt_renderer* r, const pt_camera* camera, const pt_render_settings* settings, int32_t spp,
                    uint64_t probe_samples, pt_tuning* chosen, double* default_rate, double* tuned_rate);

/* ---- measurement ---------------------------------------------------------------------------- */

/* The CUDA stream (a cudaStream_t) on which every device operation of this renderer is ordered, so
 * that callers can time it with their own events. */
void* pt_renderer_stream(pt_renderer* r);

/* Read bandwidth (GB/s) of an L2-resident buffer of `bytes` (1 MiB to 64 MiB) read `reps` times per
 * launch with loads that bypass L1; the best of five launches. The denominator for kernels whose
 * data stays in L2 (the BVH walk). No counterpart in Photon (a measurement helper). */
int32_t pt_measure_l2_bandwidth(int32_t device, size_t bytes, int32_t reps, double* gbs);

enum { PT_PROFILE_KERNEL_TIMES = 1, PT_PROFILE_TRAVERSAL_COUNTS = 2 };
typedef struct pt_kernel_time { uint64_t launches; double ms; } pt_kernel_time;
typedef struct pt_profile {
    pt_kernel_time setup, generate, trace, shade, shadow, accumulate;
    uint64_t kernel_launches;                       /* every kernel this renderer launched */
    uint64_t closest_rays, shadow_rays;             /* rays traced (camera + extension, shadow) */
    uint64_t closest_node_visits, closest_tri_tests;/* with PT_PROFILE_TRAVERSAL_COUNTS */
    uint64_t shadow_node_visits, shadow_tri_tests;
    /* SIMT use of the trace and shadow walks (with PT_PROFILE_TRAVERSAL_COUNTS): lane steps (a node
     * visit or triangle test of one ray) and warp steps (walk-loop iterations of a warp with a live
     * lane); lane_steps / warp_steps = live lanes per step, out of 32. The tail kernel is not counted. */
    uint64_t closest_lane_steps, closest_warp_steps, shadow_lane_steps, shadow_warp_steps;
} pt_profile;
/* flags: PT_PROFILE_KERNEL_TIMES records CUDA events between the kernels of every bounce iteration
 * (inside the captured graphs) and sums each kernel's device time; PT_PROFILE_TRAVERSAL_COUNTS
 * counts node visits and triangle tests (slower kernels: for a separate, untimed render). */
int32_t pt_set_profiling(pt_renderer* r, int32_t flags);
/* Totals since the last pt_set_profiling call. */
int32_t pt_get_profile(const pt_renderer* r, pt_profile* out);

/* ---- parity probes (the integrator's discrete decisions, for bit-exact checks) -------------- */

/* Primary closest hits of pixel centres + the first random jitter of sample `frame`, exactly the
 * camera rays of render_sample (pixel.h:18-24): per pixel (t, tri, u, v) into hits4 (4 * w * h floats;
 * tri is stored as a float bit pattern of the int32, -1 on a miss). Walked as the renderer's rendering
 * walks them: the pair walk unless its tuning sets pair_walk = 0 (or packed = 0). */
int32_t pt_trace_primary(pt_renderer* r, const pt_camera* camera, int32_t width, int32_t height, uint32_t frame,
                         uint32_t seed, float* hits4);
/* The light pick of next event estimation at the first vertex of every pixel's sample `frame`
 * (integrator.h:206-209 with lights.h:139-202): per pixel 4 int32 = group (0 emissive, 1 punctual,
 * 2 environment, -1 none), index (emissive entry, punctual light, or env row*width+col), alias bin,
 * 1 if NEE ran at that vertex. */
int32_t pt_light_picks_primary(pt_renderer* r, const pt_camera* camera, const pt_render_settings* settings,
                               uint32_t frame, int32_t* picks4);
/* BVH node visits of the primary ray through each pixel centre (heatmap_kernel,
 * gpu_renderer.cu:98-106), w * h floats. */
int32_t pt_heatmap(pt_renderer* r, const pt_camera* camera, int32_t width, int32_t height, float* visits);
/* Any-hit walks (traverse.h:144-147, occluded; the shadow rays' walk) of n caller rays, 8 floats each
 * (origin, tmax, direction, unused): out4 per ray = (occluded, first triangle accepted in the walk's
 * order or -1, node visits, triangle tests). Walked as the renderer's shadow rays are: the pair walk
 * unless its tuning sets pair_walk = 0 (or packed = 0); a pair walk's triangle tests are made by other
 * lanes and reported as -1. wide = 1 walks the 4-wide BVH where the scene has one (then only
 * `occluded` is Photon's, the counts are of the 4-wide walk). */
int32_t pt_occlusion_probe(pt_renderer* r, const float* rays8, int32_t n, int32_t wide, int32_t* out4);

/* ---- batched views (one persistent launch over many views) --------------------------------- */
typedef struct pt_view {
    pt_camera camera;
    int32_t width, height, spp;
    uint32_t seed;
    pt_path_options path;
} pt_view;
/* Renders every view into its own accumulation in one wavefront: work items of all views share
 * the path pool, bounce iterations run as captured CUDA graphs. Results: pt_download_view. */
int32_t pt_render_views(pt_renderer* r, const pt_view* views, int32_t n_views);
int32_t pt_download_view(pt_renderer* r, int32_t view, float* rgb, size_t n);
/* The autotuner for a batched view set (pt_render_views): the probe is the set itself with every
 * view's resolution scaled by one factor to about `probe_samples` paths in all (0: 2^25). The chosen
 * tuning stays with the renderer (its record for the resident scene), so later pt_render_views and
 * pt_render calls use it; pt_get_tuning reads it back (pt_server_set_tuning applies it to a server). The
 * results of the last pt_render_views stay downloadable. No counterpart in Photon (fixed 16x8 blocks,
 * gpu_renderer.cu:60-80). */
int32_t pt_autotune_views(pt_renderer* r, const pt_view* views, int32_t n_views, uint64_t probe_samples, pt_tuning* chosen,
                          double* default_rate, double* tuned_rate);

/* ---- SVGF on caller G-buffers (svgf.h:24-42) --------------------------------------------------
 * A denoiser session with its own history. Inputs are device pointers to width*height float4:
 * color, albedo, normal_depth, position (w = material id, -1 miss), emission — the layout of
 * photon::SvgfInput. output receives the denoised radiance (float4, w = 1). */
typedef struct pt_svgf pt_svgf;
int32_t pt_svgf_create(int32_t device, int32_t width, int32_t height, pt_svgf** out);
void pt_svgf_destroy(pt_svgf* s);
int32_t pt_svgf_reset(pt_svgf* s);
int32_t pt_svgf_run(pt_svgf* s, const float* color, const float* albedo, const float* normal_depth,
                    const float* position, const float* emission, const pt_camera* previous,
                    const pt_svgf_settings* settings, float* output);
/* The variance estimate of the last run (Svgf::variance_buffer, svgf.h:44): a device pointer. */
/* How the a-trous passes read their 5x5 taps: 0 from global memory; 1 (default) from shared-memory
 * tiles that the Tensor Memory Accelerator stages, contiguous tiles for steps 1-8 and global loads
 * beyond; 2 as 1 plus a strided tile (one residue class of x, y mod 8) for step 16; 3 strided tiles
 * for steps 1-16. Every mode gives the same output bit for bit. */
int32_t pt_svgf_set_tma(pt_svgf* s, int32_t mode);
/* Test hook for the TMA passes' bounded wait (no counterpart in Photon): with on = 1 they arm their
 * tile barrier without issuing the tile copies and wait 2 us, so the wait runs out with no copy in
 * flight; the timeout is reported as PT_ERR_CUDA by the next pt_svgf_run, and the frame is invalid. */
int32_t pt_svgf_debug_tma_timeout(pt_svgf* s, int32_t on);
const float* pt_svgf_variance(const pt_svgf* s);
const char* pt_svgf_last_error(const pt_svgf* s);

/* An allocation-free SVGF denoise of one frame, for callers that cannot call cudaMalloc: an engine
 * whose frame loop must not allocate (allocation synchronises the device and stalls the frame), a
 * caller whose device memory is owned by its own caching allocator, or code that runs where the
 * CUDA allocator may not be called. No counterpart in Photon (its Svgf allocates its buffers in
 * Svgf::resize, svgf.cu:225-236).
 * The frame is denoised without history, as the first frame of a session (demodulate, spatial
 * variance, `settings->atrous_iterations` a-trous passes, remodulate); inputs and output are caller
 * device pointers to width*height float4 in the layout of pt_svgf_run. The intermediates live in one
 * static device array of 40 MiB (524,288 pixels x 5 float4) that every GPU loading the library keeps
 * until the process exits; frames above 524,288 pixels are rejected with PT_ERR_INVALID. The first
 * call on a device looks up that array's device address (cudaGetSymbolAddress), so make it before any
 * stream capture; the address is kept for the life of the process, so a device reset
 * (cudaDeviceReset) after that first call is not supported. The call only enqueues work on `stream` (a cudaStream_t, 0 = legacy default stream)
 * and allocates nothing; every call shares the one array, so calls whose work overlaps on the GPU
 * (other streams, other threads) race — order them on one stream. */
int32_t pt_svgf_run_noalloc(int32_t device, int32_t width, int32_t height, const float* color, const float* albedo,
                            const float* normal_depth, const float* position, const float* emission,
                            const pt_svgf_settings* settings, float* output, void* stream);

/* Light tables rebuilt on the device (no counterpart call in Photon, whose update_lights takes a scene
 * rebuilt on the host: gpu_renderer.cu:299-334 after scene.cpp:113-210). New materials (same count,
 * same per-triangle assignment), punctual lights and environment for the uploaded scene; the
 * emissive-triangle list, its alias table, the light-group probabilities and the environment's
 * sampling distribution are computed on the device, equal to what pt_scene_build computes for the
 * same inputs. env_texels NULL: a constant environment of env_color. */
typedef struct pt_light_update {
    const pt_material* materials; int32_t num_materials;
    const pt_punctual_light* punctual; int32_t num_punctual;
    const pt_vec3* env_texels; int32_t env_width, env_height;
    pt_vec3 env_color; float env_intensity, env_rotation;
} pt_light_update;
int32_t pt_rebuild_lights(pt_renderer* r, const pt_light_update* update);

/* ---- result encoders (host) --------------------------------------------------------------------- */
/* PFM of a float rgb image (row-major, top row first), in the format of Photon's save_pfm
 * (src/scene/image.cpp:88-96): "PF\n<w> <h>\n-1.0\n", then little-endian float rgb rows, bottom row
 * first. With out == NULL only *length (the encoded size) is set; a capacity below it is
 * PT_ERR_INVALID. */
int32_t pt_encode_pfm(const float* rgb, int32_t width, int32_t height, uint8_t* out, size_t capacity, size_t* length);
/* PNG (8-bit RGBA, zlib `level` 0-9) of a display buffer (pt_download_display's packing: each uint32's
 * bytes in memory order are R, G, B, A), the image Photon's save_pfm counterpart save_png writes
 * (image.cpp:84-86). Size query as pt_encode_pfm. */
int32_t pt_encode_png(const uint32_t* rgba, int32_t width, int32_t height, int32_t level, uint8_t* out, size_t capacity,
                      size_t* length);
/* The file forms of the two encoders (photon::save_pfm / photon::save_png). */
int32_t pt_write_pfm(const char* path, int32_t width, int32_t height, const float* rgb);
int32_t pt_write_png(const char* path, int32_t width, int32_t height, const uint32_t* rgba);

/* ---- request server (continuous batching over resident scenes) ------------------------------ */
typedef struct pt_server pt_server;
typedef struct pt_server_config {
    int32_t device;
    uint64_t budget_bytes;     /* device memory for scenes + requests + path pool */
    int32_t path_capacity;     /* shared path pool (0: 16,777,216 paths) */
    int32_t max_active;        /* requests on the device at once (0: 16; negative: unbounded, budget only) */
    double device_wait_seconds;/* bound of every device-side wait (0: 2 s) */
    int32_t sort_rays;         /* ray sorting of iterations of at least 2,097,152 paths, bits per axis of the
                                  origin cell (1-6); 0: the default (4, while that many paths are
                                  pending); -1: off */
    int64_t reserve_bytes;     /* device memory reserved up front for request buffers (0: min(32 GiB, half
                                  the free memory, what the budget leaves beside the path pool);
                                  negative: none, the pool grows on demand) */
} pt_server_config;
typedef struct pt_request {
    int32_t scene_id;
    pt_camera camera;
    int32_t width, height, spp;
    uint32_t seed;
    pt_path_options path;
    /* display = 1: the finished image is also mapped for display on the device (the colour view of
     * pt_display: exposure, tone map, sRGB, RGBA8) for pt_server_fetch_encoded's PNG; 0 (zero-filled
     * requests): the float image only. */
    int32_t display;
    float exposure;
    int32_t tonemap;           /* PT_TONEMAP_* */
} pt_request;
enum { PT_REQ_QUEUED = 0, PT_REQ_RUNNING = 1, PT_REQ_DONE = 2, PT_REQ_CANCELLED = 3, PT_REQ_FAILED = 4 };
typedef struct pt_request_stats {
    double submit_s, admit_s, done_s;  /* server clock, seconds */
    uint64_t samples;
    int32_t state;
} pt_request_stats;
typedef struct pt_server_stats {
    uint64_t submitted, completed, cancelled, rejected;
    uint64_t samples_done;
    uint64_t bounce_iterations;
    uint64_t device_bytes_in_use, budget_bytes;
    int32_t active, queued, scenes;
    double busy_seconds;
    double device_seconds;     /* device time of the bounce-iteration batches (CUDA events), for the busy fraction */
    uint64_t batches;          /* batches of bounce iterations launched */
} pt_server_stats;
int32_t pt_server_create(const pt_server_config* cfg, pt_server** out);
void pt_server_destroy(pt_server* s);
/* The message of the calling thread's last failed call on a server (the handle is shared between
 * threads, so each thread reads its own). */
const char* pt_server_last_error(const pt_server* s);
/* Makes a scene resident (copied) and returns its id. PT_ERR_BUDGET when it does not fit. */
int32_t pt_server_add_scene(pt_server* s, const pt_scene_desc* scene, int32_t* scene_id);
/* Non-blocking. Fails with PT_ERR_BUDGET when the request alone can never fit the budget. */
int32_t pt_server_submit(pt_server* s, const pt_request* req, uint64_t* request_id);
int32_t pt_server_poll(pt_server* s, uint64_t request_id, int32_t* state);
/* Waits up to timeout_s for the request to finish (PT_ERR_TIMEOUT otherwise). */
int32_t pt_server_wait(pt_server* s, uint64_t request_id, double timeout_s);
/* Copies a finished request's average radiance (3 floats/pixel) and releases it. */
int32_t pt_server_fetch(pt_server* s, uint64_t request_id, float* rgb, size_t n, pt_request_stats* st);
int32_t pt_server_cancel(pt_server* s, uint64_t request_id);
/* The headless image endpoint: a finished request's image encoded in a wire format, instead of raw
 * floats. PT_IMAGE_PFM: the float rgb image in the format of Photon's save_pfm (image.cpp:88-96);
 * PT_IMAGE_PNG: the request's display image (it must have been submitted with display = 1), RGBA8 as
 * Photon's save_png writes a display buffer (image.cpp:84-86). With out == NULL only *length is set
 * and the request stays (the encoding is kept for the next call); otherwise the bytes are copied
 * (capacity >= *length, else PT_ERR_INVALID) and the request is consumed as by pt_server_fetch. */
enum { PT_IMAGE_PFM = 0, PT_IMAGE_PNG = 1 };
int32_t pt_server_fetch_encoded(pt_server* s, uint64_t request_id, int32_t format, uint8_t* out, size_t capacity, size_t* length);
int32_t pt_server_get_stats(pt_server* s, pt_server_stats* out);
/* Real-time SVGF sessions served beside the requests (GpuRenderer::render_denoised, gpu_renderer.cu:
 * 379-401, as a request class of the server). A session holds a G-buffer and a denoiser history on
 * the server's device (counted against its budget). Each frame is one path per pixel of `camera`
 * (sample index = the session's frame number, seed and path options from `settings`), whose first
 * vertex writes the G-buffer and the denoiser's records (reprojection into `previous`), then denoised
 * by SVGF (temporal, variance, `atrous_iterations` a-trous passes) with the session's history. Frames
 * go through a lane of their own: the waiting frames of all sessions are rendered together by a second
 * wavefront on a stream of the device's highest priority, beside the request stream, so a frame does
 * not wait for the requests' bounce iterations. The result is the denoised image: pt_server_poll /
 * wait / fetch take the returned request id as for any request; it equals the image of the same frame
 * sequence through pt_render_denoised. A session's frames are rendered one at a time in submission
 * order (a frame waits for its predecessor's denoise). Closing a session cancels its frames still
 * waiting; one on the device finishes first. */
int32_t pt_server_open_session(pt_server* s, int32_t scene_id, int32_t width, int32_t height, const pt_svgf_settings* svgf,
                               int32_t* session_id);
int32_t pt_server_submit_frame(pt_server* s, int32_t session_id, const pt_camera* camera, const pt_camera* previous,
                               const pt_render_settings* settings, uint64_t* request_id);
int32_t pt_server_close_session(pt_server* s, int32_t session_id);
/* Applies a tuning record (as pt_autotune / pt_autotune_views chose it for a scene) to the server's
 * wavefront from its next batch: the material-sort window, ray-sort bits (at most the configured
 * sort_rays), packed slab tests, 4-wide shadow BVH, walk refill and burst. Its pool size, block
 * shapes, graph cadence and tail size are ignored (the pool is set by pt_server_config). Images do not
 * change with any of them. Thread-safe. */
int32_t pt_server_set_tuning(pt_server* s, const pt_tuning* t);
/* Test hook (host-side fault injection): the next `count` device allocations of request buffers
 * fail, so the affected requests end in PT_REQ_FAILED without touching the GPU. */
int32_t pt_server_debug_fail_allocations(pt_server* s, int32_t count);
/* Test hook (host-side fault injection): the next `count` finishing steps (a finished request's
 * image being summed and queued for its copy to host memory) raise an error as a failing CUDA call
 * would; the server fails the requests in flight, settles each one's device-memory accounting
 * exactly once and goes on serving. */
int32_t pt_server_debug_fail_finishing(pt_server* s, int32_t count);

/* ---- scene construction (host) ----------------------------------------------------------------
 * Photon builds scenes on the host (Scene::build, scene.cpp:212-255). The library carries its own
 * builder so that servers and benchmarks can admit procedural scenes without Photon's host code:
 * pt_scene_build turns raw meshes into the pt_scene_desc arrays (binned SAH BVH with 2-child 64-byte
 * nodes, alias table, environment CDFs). */
typedef struct pt_texture_desc {
    int32_t width, height;
    const uint32_t* texels;  /* RGBA8, row 0 at the top */
    int32_t repeat, srgb;
} pt_texture_desc;
typedef struct pt_raw_scene {
    const pt_vec3* positions; int32_t num_positions;
    const pt_vec3* normals;   /* num_positions or NULL */
    const pt_vec2* uvs;       /* num_positions or NULL */
    const pt_vec4* tangents;  /* num_positions or NULL */
    const int32_t* indices; int32_t num_indices;
    const int32_t* tri_material;   /* num_indices / 3 */
    const pt_material* materials; int32_t num_materials;
    const pt_texture_desc* textures; int32_t num_textures;
    const pt_punctual_light* punctual; int32_t num_punctual;
    const pt_vec3* env_texels; int32_t env_width, env_height;
    pt_vec3 env_color; float env_intensity, env_rotation;
} pt_raw_scene;
typedef struct pt_built_scene pt_built_scene;
/* BVH build options (0 fields: defaults). gpu = 1 builds on the current CUDA device: the same tree
 * and triangle order as the host build, bit for bit (the admission cost of a large scene in serving). */
typedef struct pt_bvh_build_options { int32_t bins, max_leaf_size; float traversal_cost; int32_t threads; int32_t gpu; } pt_bvh_build_options;
int32_t pt_scene_build(const pt_raw_scene* raw, const pt_bvh_build_options* opt, pt_built_scene** out);
/* The built arrays; valid until pt_scene_free. */
const pt_scene_desc* pt_scene_desc_of(const pt_built_scene* b);
void pt_scene_free(pt_built_scene* b);

/* Procedural scenes of the benchmark configurations. kind:
 *   PT_GEN_BOX      the closed box: 5 walls, 2 rotated boxes, a ceiling emitter (36 triangles);
 *   PT_GEN_TERRAIN  the height-field scene: value-noise terrain, instanced spheres and cylinders
 *                   (10% mirrored), 64 materials (25% alpha-masked checker), 64 emissive triangles,
 *                   4 point/spot lights, a 1024x512 HDR sky with 3 lobes. triangles = total count
 *                   (262144 for the 262K scene; larger counts scale the tessellation). */
enum { PT_GEN_BOX = 0, PT_GEN_TERRAIN = 1 };
typedef struct pt_generated pt_generated;
int32_t pt_generate_scene(int32_t kind, int64_t triangles, uint64_t seed, pt_generated** out);
const pt_raw_scene* pt_generated_raw(const pt_generated* g);
/* The scene's default camera for an aspect ratio. */
int32_t pt_generated_camera(const pt_generated* g, float aspect, pt_camera* out);
void pt_generated_free(pt_generated* g);

#ifdef __cplusplus
}
#endif

#endif /* PHOTON_WAVEFRONT_H */
