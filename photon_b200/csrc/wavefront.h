// Host-side interface of the wavefront kernels (wavefront.cu): the device structures shared by the
// kernels and the renderer, and the launch wrappers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "pt_types.h"

namespace ptw {

// One unit of batched work: a camera over an image, spp samples per pixel starting at sample index
// frame0. Every (sample, pixel) pair is one path; paths of all views share the path pool.
struct DevView {
    float cam[16];            // pt_camera: position, tan_half_fov, forward, aspect, right, aperture, up, focus
    int width, height, spp, scene;
    uint32_t seed, frame0;
    int max_depth, rr_depth;
    int nee;
    float clamp;
    int gbuffer;              // 1: sample 0 writes the first-hit G-buffer
    int realtime;             // 1: the accumulate step also writes `color` (sample 0)
    unsigned long long work_begin, work_count;
    unsigned long long local_base;   // index of the view's first work item within its image's samples
    float4* sample_out;       // work_count radiance values, indexed by (sample * pixels + tile slot)
    float4* accum;            // rgb sum + luminance^2 sum per pixel
    float4* acc_pass;         // running per-call sum across passes (may be null for single-pass calls)
    float4* g_albedo;
    float4* g_normal_depth;
    float4* g_position;
    float4* g_emission;
    float4* g_color;
    float4* g_edge;           // the denoiser's edge and motion records (see gbuffer.cuh), optional
    float4* g_motion;
    float prev_cam[16];       // pt_camera of the previous frame, for the motion records
    int has_prev;
    unsigned long long* done_counter;  // optional: paths finished (for serving progress)
};

// Device counters of one wavefront run. The kernels read the iteration's sizes from here, so a
// bounce iteration is a fixed launch sequence that a CUDA graph can replay.
struct Counters {
    uint32_t parity;                 // buffer holding this iteration's paths (the sort step sets it so
                                     // that the next setup finds the sorted paths)
    uint32_t count[2];               // paths in each buffer
    uint32_t shadow_count;
    uint32_t gen_base, gen_n;        // slots filled by this iteration's generate step
    uint32_t fetch[6];               // work-claim counters: generate, trace, shade, shadow, sort scatter, tail
    uint32_t overflow;
    uint32_t tail;                   // 1: this iteration finishes every queued path in k_tail
    uint32_t tail_limit;             // queued paths at or below which k_tail takes over (host-set per render)
    uint32_t sorting;                // 1: this iteration's continuing rays are sorted (sort_bits > 0, enough paths)
    uint32_t shadow_sorting;         // 1: this iteration's shadow rays are walked in sorted order (shadow_sort_bits > 0)
    uint32_t gen_view;               // first view whose work is not all generated (views are in work order)
    uint32_t iterations;
    unsigned long long work_base, work_next, work_total;
    unsigned long long rays, shadow_rays, paths_done;
    unsigned long long node_visits, tri_tests;
    unsigned long long shadow_node_visits, shadow_tri_tests;
    // SIMT use of the queue walks (k_trace, k_shadow), counted with the traversal counters: lane
    // steps (one node visit or triangle test of one ray) and warp steps (iterations of a warp's walk
    // loop with a live lane); lane steps / warp steps = live lanes per step out of 32.
    unsigned long long trace_lane_steps, trace_warp_steps, shadow_lane_steps, shadow_warp_steps;
};

struct PathBuffers {
    float4* o[2];      // (origin, prev_pdf)
    float4* d[2];      // (direction, flags: depth | prev_delta << 16)
    float4* beta[2];   // (beta, L.x)
    float4* lr[2];     // (L.y, L.z, rng state lo, rng state hi)
    uint4* id[2];      // (view, local work index, pixel, sample in pass)
    float4* hit;       // (t, tri, u, v)
    float4* sh0;       // shadow queue: (origin, tmax)
    float4* sh1;       // (direction, target)
    float4* sh2;       // (contribution, view | terminal flag)
    uint32_t capacity;
};

struct WfParams {
    const DevScene* scenes;
    const DevView* views;
    int num_views;
    int single_scene;          // >= 0: every view uses this scene slot
    const float4* single_nodes;   // with single_scene >= 0: that scene's BVH2, 4-wide BVH (or null) and
    const float4* single_nodes4;  // triangles, so that the walks take the array bases from the launch
    const float4* single_tris;    // parameters instead of holding them in registers
    PathBuffers pb;
    Counters* ctr;
    int count_work;            // 1: count node visits / triangle tests (stats runs)
    int packed;                // 1: f32x2 slab tests in the traversal kernels
    uint32_t tail_paths;       // > 0: once no new paths remain and at most Counters::tail_limit are queued,
                               // finish them in one kernel (one thread per path, all bounces)
    int wide_shadows;          // 1: shadow rays walk the 4-wide BVH where the scene has one
    uint32_t trace_refill;     // 1-32: a trace warp claims new rays once fewer of its lanes hold one
    uint32_t shadow_refill;    // the same for the shadow walk
    uint32_t walk_burst;       // walk steps each lane takes between two looks at its warp (>= 1)
    uint32_t pair_visits;      // > 0: the BVH2 walks are pair walks with up to this many node visits per
                               //      warp step (packed slab tests only); 0: per-lane walks
    int sort_material;         // 1: the shade kernel groups each block's paths by material class
    int sort_bits;             // > 0: sort continuing paths by direction octant + Morton origin cell
                               //      (this many bits per axis) before they are traced
    uint32_t* keys;            // capacity entries (sort keys of the shade output)
    uint32_t* hist;            // 8 << (3 * sort_bits) bucket counts (zero between iterations)
    uint32_t* offsets;         // bucket write positions of the scatter
    int shadow_sort_bits;      // > 0: walk the shadow queue ordered by direction octant + Morton origin cell
    uint32_t* shadow_keys;     // capacity entries (sort keys of the shadow queue)
    uint32_t* shadow_hist;     // 8 << (3 * shadow_sort_bits) bucket counts (zero between iterations)
    uint32_t* shadow_offsets;
    uint32_t* shadow_perm;     // capacity entries: the shadow queue's order for the walk
};

// A camera passed by value to the probe kernels (pt_camera as 16 floats).
struct CameraArg {
    float c[16];
};

struct LaunchShape {
    int sms;
    int gen_grid, gen_block;
    int trace_grid, trace_block;
    int shade_grid, shade_block;
    int shadow_grid, shadow_block;
    int pair_trace_grid, pair_shadow_grid;  // the pair walks (more shared memory per block)
};

// Fills grid sizes from the occupancy of each kernel on `device` (block sizes as requested).
cudaError_t wf_launch_shape(int device, int trace_block, int shade_block, LaunchShape* out);
// One bounce iteration: setup, generate, [tail], trace, shade, shadow [, the three ray-sort kernels].
// With `events` (6 entries), an event is recorded before the first kernel and after each of the five
// stages (the tail counts with trace, the sort kernels with shadow).
cudaError_t wf_iteration(const WfParams& p, const LaunchShape& ls, cudaStream_t stream, cudaEvent_t* events = nullptr);
// Iterations with fewer queued paths are not ray-sorted (the scan and scatter would cost more than the
// coherence gains).
constexpr uint32_t kSortMinPaths = 1u << 21;
// Kernels wf_iteration launches for these parameters.
inline int wf_kernels_per_iteration(const WfParams& p) {
    return 5 + (p.tail_paths > 0 ? 1 : 0) + (p.sort_bits > 0 ? 3 : 0) + (p.shadow_sort_bits > 0 ? 2 : 0);
}
// Sums the samples of every pixel of a view in sample order (after a pass).
cudaError_t wf_accumulate(const DevView* d_view, const DevView& h_view, int first_pass, int last_pass, cudaStream_t stream);
// rgb[3 i + c] = accum[i].c * scale for n pixels (a finished image, averaged over its samples).
// rgb[3i..3i+2] = accum[i].xyz * scale (or the plain xyz when apply_scale is false).
cudaError_t wf_resolve(const float4* accum, uint32_t n, float scale, bool apply_scale, float* rgb, cudaStream_t stream);

// Probes (same device functions as the wavefront). With pair_visits > 0 the walks are the pair walks
// of the wavefront's default kernels, over a queue counted in `claim` (one device word).
cudaError_t wf_trace_primary(const DevScene* scene, const float* cam16, int w, int h, uint32_t frame, uint32_t seed,
                             float4* out, uint32_t* claim, uint32_t pair_visits, cudaStream_t stream);
cudaError_t wf_light_picks(const DevScene* scene, const DevView* view, int4* out, int w, int h, cudaStream_t stream);
cudaError_t wf_heatmap(const DevScene* scene, const float* cam16, int w, int h, float* out, cudaStream_t stream);
// Any-hit walks of n rays (2 float4 each: origin + tmax, direction + unused): out[i] = (occluded,
// first accepted triangle or -1, node visits, triangle tests).
cudaError_t wf_occlusion_probe(const DevScene* scene, const float4* rays, int n, int wide, int4* out, uint32_t* claim, uint32_t pair_visits,
                               cudaStream_t stream);

struct DisplayParams {
    int w, h, mode;
    float exposure;
    int tonemap;
    float inv_samples, samples, max_depth, heat_scale;
    int denoised;
};
cudaError_t wf_display(const DisplayParams& p, const float4* accum, const float4* denoised, const float4* albedo,
                       const float4* normal_depth, const float4* variance, const float* heat, uint32_t* out,
                       cudaStream_t stream);

}  // namespace ptw
