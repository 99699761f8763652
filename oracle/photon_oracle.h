/*
 * photon_oracle.h — TEST INFRASTRUCTURE, not part of the product.
 *
 * A plain-C restatement of Photon's path-tracing hot path (render_sample → trace_path with BVH2
 * traversal, the glTF BSDF, NEE + MIS light sampling, Russian roulette) and of its SVGF denoiser, on
 * the scene arrays of include/photon_wavefront.h. It is the oracle the CUDA path is compared with.
 * Every function cites the Photon source it restates (paths relative to the Photon repository).
 *
 * Pinning: tests/test_oracle_pinning.py checks this restatement bit-for-bit against Photon's own CPU
 * code compiled from its sources (oracle/_ref/libphoton_ref.so) on the same scenes, cameras and
 * seeds, and against the known-answer cases of Photon's test suite.
 *
 * Only tests/, the smoke check and the CPU-baseline leg of bench.py may load this library.
 */
#ifndef PHOTON_ORACLE_H
#define PHOTON_ORACLE_H

#include "photon_wavefront.h"

#ifdef __cplusplus
extern "C" {
#endif

/* CpuRenderer::render (cpu_renderer.cpp:20-39): for every pixel, acc = sum over s < spp of
 * render_sample(frame = frame0 + s), then sum_rgb[pixel] += acc. threads = 0: all cores. */
void orc_render(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, int spp, uint32_t frame0,
                int threads, float* sum_rgb);

/* render_sample (pixel.h:18-29) of one (x, y, frame); primary16 (optional) receives PrimaryInfo
 * (integrator.h:30-37) as position(3), depth, normal(3), material(as float), albedo(3), emission(3),
 * pad(2). */
void orc_render_sample(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, int x, int y,
                       uint32_t frame, float* L3, float* primary16);

/* The sample_kernel G-buffer (gpu_renderer.cu:83-95) of one frame, float4 per pixel each. */
void orc_sample_gbuffer(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, uint32_t frame,
                        int threads, float* color4, float* albedo4, float* normal_depth4, float* position4,
                        float* emission4);

/* Primary closest hit of every pixel's sample `frame` (t, tri as int bits, u, v). */
void orc_trace_primary(const pt_scene_desc* s, const pt_camera* cam, int w, int h, uint32_t frame, uint32_t seed,
                       float* hits4);

/* Light pick at the first vertex (group, index, alias bin, nee-ran), as pt_light_picks_primary. */
void orc_light_picks_primary(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs,
                             uint32_t frame, int32_t* picks4);

/* Node visits of the pixel-centre primary ray (gpu_renderer.cu:98-106). */
void orc_heatmap(const pt_scene_desc* s, const pt_camera* cam, int w, int h, float* visits);
/* Any-hit walks of n rays (origin, tmax, direction, unused): (occluded, first accepted triangle or -1,
 * node visits, triangle tests) per ray. */
void orc_occluded(const pt_scene_desc* s, const float* rays8, int n, int32_t* out4);

/* Work counts of the path tracer, for the algorithmic-bytes model (rays, node visits, triangle
 * tests, alpha tests, shading events, NEE picks per group, texture taps), accumulated over every
 * `stride`-th pixel's sample 0 (as `photon bench` counts rays, render_cli.cpp:307-318). */
typedef struct orc_counters {
    uint64_t samples, camera_rays, extension_rays, shadow_rays;
    uint64_t node_visits, tri_tests, alpha_tests, shade_events, normal_mapped_events;
    uint64_t nee_emissive, nee_punctual, nee_env, env_lookups, texture_taps;
} orc_counters;
void orc_count(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, int stride,
               orc_counters* out);

/* Known-answer helpers. */
void orc_rng_floats(uint64_t seed, uint64_t stream, int n, float* out);              /* sampling.h:9-34 */
uint32_t orc_hash_u32(uint32_t x);                                                  /* sampling.h:37-44 */
int orc_sample_alias(const pt_alias_entry* t, int n, float u, float* pmf);         /* lights.h:22-30 */
void orc_offset_ray(int n, const float* p, const float* nrm, float* out);          /* integrator.h:61-69 */
void orc_bsdf_sample(const float* params7, int n, const float* rows8, float* out9); /* bsdf.h:255-281 */
/* sample_light (lights.h:139-202): out = wi(3), dist, radiance(3), pdf, delta, tri, bary(2). */
void orc_sample_light(const pt_scene_desc* s, const float* p3, float u_group, float u0, float u1, float u_light,
                      float* out12);

/* SVGF (svgf.cu:37-255) on host float4 buffers, with its own history. */
typedef struct orc_svgf orc_svgf;
orc_svgf* orc_svgf_create(int w, int h);
void orc_svgf_destroy(orc_svgf* s);
void orc_svgf_reset(orc_svgf* s);
void orc_svgf_run(orc_svgf* s, const float* color4, const float* albedo4, const float* normal_depth4,
                  const float* position4, const float* emission4, const pt_camera* prev, const pt_svgf_settings* st,
                  float* out4);
const float* orc_svgf_variance(const orc_svgf* s);

#ifdef __cplusplus
}
#endif

#endif
