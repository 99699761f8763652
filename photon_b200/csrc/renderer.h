// The wavefront engine and the drop-in renderer built on it (host side).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "device_scene.h"
#include "wavefront.h"

namespace ptw {

class SvgfDenoiser;

// tail_paths value that picks the threshold per render: kTailAlone while no other render of this
// process runs on the device, kTailShared otherwise. A render alone is bound by its longest paths,
// which the tail finishes without an iteration barrier per bounce; renders that share the GPU are
// bound by throughput, where the wavefront's sorted iterations use the SMs better than the tail's
// one path per thread (1600x900 real-time frames: one session 3.6 -> 3.1 ms with the larger
// threshold, eight concurrent sessions 12.6 -> 15.5 ms).
constexpr int kTailAuto = -2;
constexpr int kTailAlone = 1 << 17;
constexpr int kTailShared = 1 << 16;

// Tunable launch parameters (the autotuner's knobs).
struct Tuning {
    int path_capacity = 1 << 24;   // paths in flight (the pool grows to what a render needs, up to this)
    int trace_block = 128;
    int shade_block = 256;
    int sort_by_material = 4;      // shade windows of 4 x shade_block paths grouped by material class
    int graph_bounces = 4;         // iterations per CUDA graph launch
    int sort_rays = 4;             // origin bits per axis of the ray-sort key (0: no sorting); iterations of
                                   // at least 2M paths only
    int packed = 1;                // f32x2 slab tests
    int wide_shadows = 0;          // 1: shadow rays walk the 4-wide BVH (measured slower on the 262K scene:
                                   // as a pair walk 13.2 ms against 11.0 per 1080p frame)
    int tail_paths = kTailAuto;    // finish the last queued paths one thread each below this many (0: never)
    int trace_refill = 24;         // a closest-hit warp claims new rays once fewer than this many lanes hold one
    int shadow_refill = 24;        // the same for the shadow walk
    int walk_burst = 16;           // walk steps a lane takes between two refill checks of its warp
    int pair_walk = 5;             // > 0: pair walks (leaf triangles of a warp tested together) with up to
                                   // this many node visits per warp step; 0: per-lane walks. On the 262K
                                   // scene's 1080p frame: trace 28.2 -> 24.0 ms, shadow 13.7 -> 11.0 ms
                                   // (4 to 6 visits within noise; 2: 26.1 ms, 10: 25.6 ms)
    int sort_shadows = 0;          // origin bits per axis of the shadow-queue walk order (0: queue order);
                                   // iterations of at least 2M paths only. Off: on the 262K scene's 1080p
                                   // frame the shadow walk took 13.65 ms sorted against 13.63 unsorted (the
                                   // shade order already groups them) and the keys cost shade 0.3 ms
};

// Runs wavefront passes over a table of views on one device stream. Owns the path pool, the
// counters and the captured iteration graph.
class WavefrontEngine {
public:
    WavefrontEngine(int device, cudaStream_t stream);
    ~WavefrontEngine();

    void set_tuning(const Tuning& t);
    const Tuning& tuning() const { return tuning_; }

    // Makes sure the pool holds at least min(capacity, needed) paths.
    void reserve_paths(uint64_t needed);
    // Frees the path pool and the sort buffers (the next run allocates them again).
    void release_paths();

    // Renders one pass: every work item of `views` (device table of n views, work ranges
    // contiguous from 0) until all paths finished. scenes: device table; single_scene >= 0 when
    // all views share that slot, whose host copy is `single` (its device array pointers). Blocks the
    // host until done (bounded by max_iterations).
    void run(const DevScene* scenes, int single_scene, const DevScene* single, const DevView* views, int n_views,
             uint64_t total_work, bool count_work = false);

    // Continuous mode (the request server): prepare once, then alternate iterate() with host-side
    // admission of new work (append_work) and completion checks (counters()).
    void begin(const DevScene* scenes, const DevView* views, int n_views);
    void set_views(const DevView* views, int n_views);
    void append_work(uint64_t new_total);   // raises work_total (stream-ordered)
    void iterate(int iterations);           // launches iterations and copies the counters back
    const Counters& counters() const { return *h_ctr_; }  // valid after sync()
    void sync();
    // Pipelined continuous mode: launches `iterations` bounce iterations and nothing else; the caller
    // copies the counters (device_counters) itself and raises work_total with a stream-ordered copy
    // from its own staging memory (set_work_total_async).
    void launch(int iterations);
    Counters* device_counters() const { return ctr_.ptr; }
    // Queued paths at or below which an iteration hands everything to the tail (0: never), as set by
    // the last begin().
    uint32_t tail_limit_in_use() const { return tail_limit_; }
    void set_work_total_async(const unsigned long long* pinned_value);
    // Continuous mode: whether the next launches carry the ray-sort kernels (the tuning's sort_rays;
    // the kernels still sort only iterations of at least kSortMinPaths paths).
    void set_continuous_sorting(bool on) {
        cont_params_.sort_bits = on ? tuning_.sort_rays : 0;
        cont_params_.shadow_sort_bits = on ? tuning_.sort_shadows : 0;
    }
    // Continuous mode: takes the knobs of `t` that only change what the next launches are given
    // (material-sort window, ray-sort bits up to those the buffers were sized for, packed slab tests,
    // 4-wide shadow BVH, walk refill and burst). Pool size, block shapes, graph cadence and the tail
    // stay as they were set before begin().
    void update_scheduling(const Tuning& t);

    const Counters& last() const { return last_; }

    // Profiling (pt_set_profiling): per-kernel device time recorded by events inside the graphs,
    // and traversal counters in the kernels.
    void set_profiling(int flags);
    int profiling() const { return profile_flags_; }
    // Device milliseconds per kernel (setup, generate, trace, shade, shadow) and launch counts.
    double kernel_ms[5] = {0, 0, 0, 0, 0};
    uint64_t kernel_launches = 0, iteration_launches = 0;
    size_t device_bytes() const;
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    uint64_t bytes_per_path() const;

private:
    void ensure_shape();
    void capture(const WfParams& p);
    WfParams params(const DevScene* scenes, int single, const DevScene* single_host, const DevView* views, int n, bool count) const;

    int device_;
    cudaStream_t stream_;
    Tuning tuning_;
    LaunchShape shape_{};
    bool shape_ok_ = false;
    PathBuffers pb_{};
    DeviceBuffer<float4> bufs_[12];
    DeviceBuffer<uint4> ids_[2];
    DeviceBuffer<Counters> ctr_;
    DeviceBuffer<uint32_t> keys_, hist_, offsets_;
    DeviceBuffer<uint32_t> shadow_keys_, shadow_hist_, shadow_offsets_, shadow_perm_;
    Counters* h_ctr_ = nullptr;
    Counters last_{};
    cudaGraphExec_t graph_ = nullptr;
    WfParams graph_params_{};
    int graph_iters_ = 0;
    cudaEvent_t ev_ = nullptr;
    // continuous mode
    WfParams cont_params_{};
    int profile_flags_ = 0;
    std::vector<cudaEvent_t> prof_ev_;
    uint32_t tail_limit_ = 0;
    void collect_kernel_times(int iterations);
};

// The drop-in for photon::GpuRenderer (src/render/gpu_renderer.h:36-75).
class Renderer {
public:
    explicit Renderer(int device);
    ~Renderer();

    void upload(const pt_scene_desc& d, bool lights_only);
    void rebuild_lights(const pt_light_update& u);
    void resize(int w, int h);
    void reset();
    void render(const pt_camera& cam, const pt_render_settings& rs, int spp);
    void render_denoised(const pt_camera& cam, const pt_camera& prev, const pt_render_settings& rs, const pt_svgf_settings& sv);
    void display(const pt_render_settings& rs, int mode, uint32_t* target);
    void download_image(float* rgb, size_t n);
    void download_display(uint32_t* out, size_t n);
    void download_gbuffer(float* albedo4, float* nd4, size_t n);
    void download_accumulation(float* sums4, size_t n);
    uint32_t* display_buffer() const { return display_.ptr; }
    void stats(pt_stats* out) const;
    void set_tuning(const pt_tuning& t);
    void get_tuning(pt_tuning* t) const;
    void autotune(const pt_camera& cam, const pt_render_settings& rs, int spp, uint64_t probe_samples, pt_tuning* chosen,
                  double* default_rate, double* tuned_rate);
    void autotune_views(const pt_view* views, int n, uint64_t probe_samples, pt_tuning* chosen, double* default_rate, double* tuned_rate);

    void trace_primary(const pt_camera& cam, int w, int h, uint32_t frame, uint32_t seed, float* hits4);
    void light_picks(const pt_camera& cam, const pt_render_settings& rs, uint32_t frame, int32_t* picks4);
    void heatmap(const pt_camera& cam, int w, int h, float* out);
    void occlusion_probe(const float* rays8, int n, int wide, int32_t* out4);

    void set_profiling(int flags);
    void get_profile(pt_profile* out) const;
    cudaStream_t stream() const { return stream_; }

    void render_views(const pt_view* views, int n);
    void download_view(int v, float* rgb, size_t n);

    std::string error;

private:
    void fill_view(DevView& v, const pt_camera& cam, int w, int h, int spp, uint32_t seed, const pt_path_options& po,
                   uint32_t frame0) const;
    void render_pass_set(std::vector<DevView>& views, int spp_total, std::vector<int>& spp_each, std::vector<uint32_t>& frame0);
    void tune_on(const std::vector<pt_view>& probe, pt_tuning* chosen, double* default_rate, double* tuned_rate);

    int device_;
    cudaStream_t stream_ = nullptr;
    std::unique_ptr<WavefrontEngine> engine_;
    DeviceScene scene_;
    DeviceBuffer<DevScene> scene_table_;
    int width_ = 0, height_ = 0, samples_ = 0;
    uint32_t frame_ = 0;
    float last_ms_ = 0;
    bool denoised_ = false;
    DeviceBuffer<float4> accum_, acc_pass_, albedo_, normal_depth_, edge_, motion_, emission_, color_, denoised_buf_;
    DeviceBuffer<float> heat_;
    DeviceBuffer<uint32_t> display_;
    DeviceBuffer<uint32_t> probe_claim_;  // the pair-walk probes' queue counter
    DeviceBuffer<float4> sample_out_;
    DeviceBuffer<DevView> d_views_;
    pt_camera last_camera_{};
    bool heat_valid_ = false;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    uint64_t sample_cap_ = uint64_t(1) << 26;  // radiance slots per pass (1 GiB)
    std::unique_ptr<SvgfDenoiser> svgf_;
    // batched views
    std::vector<pt_view> batch_views_;
    std::vector<DeviceBuffer<float4>> batch_accum_;
    std::vector<DeviceBuffer<float4>> batch_pass_;   // per-view pass sums when a view is split into passes
    Counters last_ctr_{};
    pt_profile profile_{};
    cudaEvent_t acc_ev_[2] = {nullptr, nullptr};
    // Downloads: the image resolved on the device, then copied out through two pinned halves so
    // that the device-to-host copy of one chunk overlaps the host copy of the previous one.
    DeviceBuffer<float> rgb_dev_;
    float* stage_[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev_[2] = {nullptr, nullptr};
    void resolve_and_copy_out(const float4* src, size_t npix, float scale, bool apply_scale, float* rgb);
};

}  // namespace ptw
