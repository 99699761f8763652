// The wavefront engine (path pool, device counters, CUDA-graph iterations) and the drop-in renderer
// that replaces photon::GpuRenderer (src/render/gpu_renderer.cu:177-454 of Photon).
#include "renderer.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstring>

#include "svgf.h"

namespace ptw {

// ---- WavefrontEngine ------------------------------------------------------------------------------------

namespace {

// Renders of this process in progress per device (WavefrontEngine::run), for the kTailAuto choice.
constexpr int kMaxDevices = 64;
std::atomic<int> g_renders[kMaxDevices];

struct RenderCount {
    int device;
    int others;  // other renders in progress on the device when this one started
    explicit RenderCount(int d) : device(d >= 0 && d < kMaxDevices ? d : -1), others(0) {
        if (device >= 0) others = g_renders[device].fetch_add(1);
    }
    ~RenderCount() {
        if (device >= 0) g_renders[device].fetch_sub(1);
    }
};

uint32_t tail_limit(int tail_paths, bool alone) {
    if (tail_paths == kTailAuto) return uint32_t(alone ? kTailAlone : kTailShared);
    return tail_paths > 0 ? uint32_t(tail_paths) : 0u;
}

}  // namespace

WavefrontEngine::WavefrontEngine(int device, cudaStream_t stream) : device_(device), stream_(stream) {
    PTW_CUDA(cudaMallocHost(reinterpret_cast<void**>(&h_ctr_), sizeof(Counters)));
    std::memset(h_ctr_, 0, sizeof(Counters));
    PTW_CUDA(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming));
    ctr_.allocate(1);
}

WavefrontEngine::~WavefrontEngine() {
    if (graph_) cudaGraphExecDestroy(graph_);
    for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
    if (ev_) cudaEventDestroy(ev_);
    if (h_ctr_) cudaFreeHost(h_ctr_);
}

void WavefrontEngine::set_tuning(const Tuning& t) {
    bool reshape = t.trace_block != tuning_.trace_block || t.shade_block != tuning_.shade_block;
    bool realloc = t.path_capacity != tuning_.path_capacity;
    tuning_ = t;
    if (reshape) shape_ok_ = false;
    if (realloc) {
        for (auto& b : bufs_) b.release();
        for (auto& b : ids_) b.release();
        pb_ = PathBuffers{};
    }
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
}

void WavefrontEngine::set_profiling(int flags) {
    profile_flags_ = flags;
    for (double& m : kernel_ms) m = 0;
    kernel_launches = iteration_launches = 0;
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    int need = 6 * std::max(1, tuning_.graph_bounces);
    while (int(prof_ev_.size()) < need) {
        cudaEvent_t e;
        PTW_CUDA(cudaEventCreate(&e));
        prof_ev_.push_back(e);
    }
}

void WavefrontEngine::collect_kernel_times(int iterations) {
    for (int k = 0; k < iterations; k++)
        for (int j = 0; j < 5; j++) {
            float ms = 0;
            PTW_CUDA(cudaEventElapsedTime(&ms, prof_ev_[size_t(6 * k + j)], prof_ev_[size_t(6 * k + j + 1)]));
            kernel_ms[j] += ms;
        }
}

uint64_t WavefrontEngine::bytes_per_path() const { return 12 * 16 + 2 * 16; }

void WavefrontEngine::reserve_paths(uint64_t needed) {
    uint64_t want = std::min<uint64_t>(uint64_t(tuning_.path_capacity), (needed + 1023) / 1024 * 1024);
    if (want < 1024) want = 1024;
    if (pb_.capacity >= want) return;
    for (auto& b : bufs_) b.allocate(want);
    for (auto& b : ids_) b.allocate(want);
    for (int k = 0; k < 2; k++) {
        pb_.o[k] = bufs_[0 + k].ptr;
        pb_.d[k] = bufs_[2 + k].ptr;
        pb_.beta[k] = bufs_[4 + k].ptr;
        pb_.lr[k] = bufs_[6 + k].ptr;
        pb_.id[k] = ids_[k].ptr;
    }
    pb_.hit = bufs_[8].ptr;
    pb_.sh0 = bufs_[9].ptr;
    pb_.sh1 = bufs_[10].ptr;
    pb_.sh2 = bufs_[11].ptr;
    keys_.allocate(want);
    shadow_keys_.allocate(want);
    shadow_perm_.allocate(want);
    pb_.capacity = uint32_t(want);
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
}

void WavefrontEngine::release_paths() {
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    for (auto& b : bufs_) b.release();
    for (auto& b : ids_) b.release();
    for (DeviceBuffer<uint32_t>* b : {&keys_, &hist_, &offsets_, &shadow_keys_, &shadow_hist_, &shadow_offsets_, &shadow_perm_}) b->release();
    pb_ = PathBuffers{};
}

size_t WavefrontEngine::device_bytes() const {
    size_t b = ctr_.bytes() + keys_.bytes() + hist_.bytes() + offsets_.bytes() + shadow_keys_.bytes() + shadow_hist_.bytes() +
               shadow_offsets_.bytes() + shadow_perm_.bytes();
    for (const auto& x : bufs_) b += x.bytes();
    for (const auto& x : ids_) b += x.bytes();
    return b;
}

void WavefrontEngine::ensure_shape() {
    if (tuning_.sort_rays > 0 && hist_.count < (size_t(8) << (3 * tuning_.sort_rays))) {
        size_t buckets = size_t(8) << (3 * tuning_.sort_rays);
        hist_.allocate(buckets);
        offsets_.allocate(buckets);
        hist_.zero(stream_);
        PTW_CUDA(cudaStreamSynchronize(stream_));
    }
    if (tuning_.sort_shadows > 0 && shadow_hist_.count < (size_t(8) << (3 * tuning_.sort_shadows))) {
        size_t buckets = size_t(8) << (3 * tuning_.sort_shadows);
        shadow_hist_.allocate(buckets);
        shadow_offsets_.allocate(buckets);
        shadow_hist_.zero(stream_);
        PTW_CUDA(cudaStreamSynchronize(stream_));
    }
    if (shape_ok_) return;
    PTW_CUDA(wf_launch_shape(device_, tuning_.trace_block, tuning_.shade_block, &shape_));
    shape_ok_ = true;
}

WfParams WavefrontEngine::params(const DevScene* scenes, int single, const DevScene* single_host, const DevView* views, int n,
                                 bool count) const {
    WfParams p;
    std::memset(&p, 0, sizeof(p));  // padding too: captured graphs are matched by comparing the bytes
    p.scenes = scenes;
    p.views = views;
    p.num_views = n;
    p.single_scene = single;
    if (single >= 0) {
        if (!single_host) throw Error{PT_ERR_INVALID, "a single-scene pass needs the scene's host copy"};
        p.single_nodes = single_host->nodes;
        p.single_nodes4 = single_host->nodes4;
        p.single_tris = single_host->tris;
    }
    p.pb = pb_;
    p.ctr = ctr_.ptr;
    p.count_work = count ? 1 : 0;
    p.packed = tuning_.packed ? 1 : 0;
    p.sort_bits = tuning_.sort_rays;
    p.sort_material = tuning_.sort_by_material;
    p.tail_paths = tuning_.tail_paths == kTailAuto ? 1u : uint32_t(std::max(0, tuning_.tail_paths));
    p.wide_shadows = tuning_.wide_shadows;
    p.trace_refill = uint32_t(std::clamp(tuning_.trace_refill, 1, 32));
    p.shadow_refill = uint32_t(std::clamp(tuning_.shadow_refill, 1, 32));
    p.walk_burst = uint32_t(std::clamp(tuning_.walk_burst, 1, 1 << 20));
    p.pair_visits = uint32_t(std::clamp(tuning_.pair_walk, 0, 64));
    p.keys = keys_.ptr;
    p.hist = hist_.ptr;
    p.offsets = offsets_.ptr;
    p.shadow_sort_bits = tuning_.sort_shadows;
    p.shadow_keys = shadow_keys_.ptr;
    p.shadow_hist = shadow_hist_.ptr;
    p.shadow_offsets = shadow_offsets_.ptr;
    p.shadow_perm = shadow_perm_.ptr;
    return p;
}

void WavefrontEngine::capture(const WfParams& p) {
    if (graph_) {
        cudaGraphExecDestroy(graph_);
        graph_ = nullptr;
    }
    int iters = std::max(1, tuning_.graph_bounces);
    cudaGraph_t g = nullptr;
    bool timed = (profile_flags_ & PT_PROFILE_KERNEL_TIMES) && int(prof_ev_.size()) >= 6 * iters;
    PTW_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    cudaError_t inner = cudaSuccess;
    for (int k = 0; k < iters && inner == cudaSuccess; k++) inner = wf_iteration(p, shape_, stream_, timed ? &prof_ev_[size_t(6 * k)] : nullptr);
    if (inner == cudaSuccess) inner = cudaMemcpyAsync(h_ctr_, ctr_.ptr, sizeof(Counters), cudaMemcpyDeviceToHost, stream_);
    cudaError_t e = cudaStreamEndCapture(stream_, &g);
    if (inner != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        throw Error{PT_ERR_CUDA, std::string("graph capture: a captured launch failed: ") + cudaGetErrorString(inner)};
    }
    if (e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        throw Error{PT_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e)};
    }
    e = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        graph_ = nullptr;
        throw Error{PT_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(e)};
    }
    graph_params_ = p;
    graph_iters_ = iters;
}

void WavefrontEngine::run(const DevScene* scenes, int single_scene, const DevScene* single, const DevView* views, int n_views,
                          uint64_t total_work, bool count_work) {
    if (total_work == 0) return;
    cudaError_t stale = cudaGetLastError();
    if (stale != cudaSuccess) throw Error{PT_ERR_CUDA, std::string("an earlier CUDA call failed: ") + cudaGetErrorString(stale)};
    reserve_paths(total_work);
    ensure_shape();
    RenderCount busy(device_);
    std::memset(h_ctr_, 0, sizeof(Counters));
    h_ctr_->parity = 1;
    h_ctr_->work_total = total_work;
    h_ctr_->tail_limit = tail_limit(tuning_.tail_paths, busy.others == 0);
    PTW_CUDA(cudaMemcpyAsync(ctr_.ptr, h_ctr_, sizeof(Counters), cudaMemcpyHostToDevice, stream_));
    WfParams p = params(scenes, single_scene, single, views, n_views, count_work || (profile_flags_ & PT_PROFILE_TRAVERSAL_COUNTS));
    // A render too small for any iteration to reach the sorting threshold launches no sort kernels.
    if (std::min<uint64_t>(total_work, uint64_t(tuning_.path_capacity)) < kSortMinPaths) {
        p.sort_bits = 0;
        p.shadow_sort_bits = 0;
    }
    bool use_graph = tuning_.graph_bounces > 0;
    bool timed = (profile_flags_ & PT_PROFILE_KERNEL_TIMES) != 0;
    if (use_graph && (!graph_ || std::memcmp(&graph_params_, &p, sizeof(p)) != 0 || graph_iters_ != tuning_.graph_bounces)) capture(p);
    const uint64_t max_launches = 1u << 22;
    for (uint64_t launch = 0;; launch++) {
        int iters = use_graph ? graph_iters_ : 1;
        if (use_graph) {
            PTW_CUDA(cudaGraphLaunch(graph_, stream_));
        } else {
            PTW_CUDA(wf_iteration(p, shape_, stream_, timed ? prof_ev_.data() : nullptr));
            PTW_CUDA(cudaMemcpyAsync(h_ctr_, ctr_.ptr, sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
        }
        PTW_CUDA(cudaEventRecord(ev_, stream_));
        PTW_CUDA(cudaEventSynchronize(ev_));
        kernel_launches += uint64_t(iters) * uint64_t(wf_kernels_per_iteration(p));
        iteration_launches += uint64_t(iters);
        if (timed) collect_kernel_times(iters);
        const Counters& h = *h_ctr_;
        if (h.count[h.parity ^ 1u] == 0 && h.work_next >= h.work_total) break;
        if (launch > max_launches) throw Error{PT_ERR_TIMEOUT, "wavefront did not drain"};
    }
    last_ = *h_ctr_;
}

void WavefrontEngine::begin(const DevScene* scenes, const DevView* views, int n_views) {
    ensure_shape();
    std::memset(h_ctr_, 0, sizeof(Counters));
    h_ctr_->parity = 1;
    h_ctr_->tail_limit = tail_limit(tuning_.tail_paths, false);  // a server shares the GPU between requests
    tail_limit_ = h_ctr_->tail_limit;
    PTW_CUDA(cudaMemcpyAsync(ctr_.ptr, h_ctr_, sizeof(Counters), cudaMemcpyHostToDevice, stream_));
    cont_params_ = params(scenes, -1, nullptr, views, n_views, false);
}

void WavefrontEngine::update_scheduling(const Tuning& t) {
    if (t.sort_rays > 0 && hist_.count < (size_t(8) << (3 * t.sort_rays)))
        throw Error{PT_ERR_INVALID, "sort_rays above the bits the running wavefront was sized for"};
    tuning_.sort_by_material = t.sort_by_material;
    tuning_.sort_rays = t.sort_rays;
    tuning_.packed = t.packed;
    tuning_.wide_shadows = t.wide_shadows;
    tuning_.trace_refill = t.trace_refill;
    tuning_.shadow_refill = t.shadow_refill;
    tuning_.walk_burst = t.walk_burst;
    tuning_.pair_walk = t.pair_walk;
    const WfParams fresh = params(cont_params_.scenes, -1, nullptr, cont_params_.views, cont_params_.num_views, false);
    cont_params_.sort_material = fresh.sort_material;
    cont_params_.packed = fresh.packed;
    cont_params_.wide_shadows = fresh.wide_shadows;
    cont_params_.trace_refill = fresh.trace_refill;
    cont_params_.shadow_refill = fresh.shadow_refill;
    cont_params_.walk_burst = fresh.walk_burst;
    cont_params_.pair_visits = fresh.pair_visits;
    if (cont_params_.sort_bits > 0) cont_params_.sort_bits = tuning_.sort_rays;
}

void WavefrontEngine::set_views(const DevView* views, int n_views) {
    cont_params_.views = views;
    cont_params_.num_views = n_views;
    cont_params_.pb = pb_;
}

void WavefrontEngine::append_work(uint64_t new_total) {
    static_assert(sizeof(unsigned long long) == 8, "counter width");
    // A stream-ordered write of work_total between iterations (the kernels read it in setup).
    // The value is staged in a pinned slot so that the copy reads it at execution time.
    h_ctr_->work_total = new_total;
    PTW_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctr_.ptr) + offsetof(Counters, work_total), &h_ctr_->work_total,
                             sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void WavefrontEngine::iterate(int iterations) {
    for (int k = 0; k < iterations; k++) PTW_CUDA(wf_iteration(cont_params_, shape_, stream_));
    kernel_launches += uint64_t(iterations) * uint64_t(wf_kernels_per_iteration(cont_params_));
    iteration_launches += uint64_t(iterations);
    PTW_CUDA(cudaMemcpyAsync(h_ctr_, ctr_.ptr, sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
}

void WavefrontEngine::launch(int iterations) {
    for (int k = 0; k < iterations; k++) PTW_CUDA(wf_iteration(cont_params_, shape_, stream_));
    kernel_launches += uint64_t(iterations) * uint64_t(wf_kernels_per_iteration(cont_params_));
    iteration_launches += uint64_t(iterations);
}

void WavefrontEngine::set_work_total_async(const unsigned long long* pinned_value) {
    PTW_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(ctr_.ptr) + offsetof(Counters, work_total), pinned_value, sizeof(unsigned long long),
                             cudaMemcpyHostToDevice, stream_));
}

void WavefrontEngine::sync() {
    PTW_CUDA(cudaEventRecord(ev_, stream_));
    PTW_CUDA(cudaEventSynchronize(ev_));
}

// ---- Renderer ----------------------------------------------------------------------------------------------

Renderer::Renderer(int device) : device_(device) {
    PTW_CUDA(cudaSetDevice(device));
    PTW_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    engine_ = std::make_unique<WavefrontEngine>(device, stream_);
    PTW_CUDA(cudaEventCreate(&ev0_));
    PTW_CUDA(cudaEventCreate(&ev1_));
    PTW_CUDA(cudaEventCreate(&acc_ev_[0]));
    PTW_CUDA(cudaEventCreate(&acc_ev_[1]));
    d_views_.allocate(1);
}

Renderer::~Renderer() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    svgf_.reset();
    engine_.reset();
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    for (cudaEvent_t e : acc_ev_)
        if (e) cudaEventDestroy(e);
    for (int k = 0; k < 2; k++) {
        if (stage_ev_[k]) cudaEventDestroy(stage_ev_[k]);
        if (stage_[k]) cudaFreeHost(stage_[k]);
    }
    if (stream_) cudaStreamDestroy(stream_);
}

void Renderer::upload(const pt_scene_desc& d, bool lights_only) {
    PTW_CUDA(cudaSetDevice(device_));
    scene_.upload(d, stream_, lights_only);
    if (width_ > 0) reset();
    else {
        samples_ = 0;
        frame_ = 0;
        denoised_ = false;
    }
}

void Renderer::rebuild_lights(const pt_light_update& u) {
    PTW_CUDA(cudaSetDevice(device_));
    scene_.rebuild_lights(u, stream_);
    if (width_ > 0) reset();
}

void Renderer::resize(int w, int h) {
    if (w < 0 || h < 0) throw Error{PT_ERR_INVALID, "negative image size"};
    // Pixel indices are 32-bit in the kernels.
    if (uint64_t(w) * uint64_t(h) > (uint64_t(1) << 30)) throw Error{PT_ERR_INVALID, "image larger than 2^30 pixels"};
    if (w == width_ && h == height_ && accum_.count) return;
    PTW_CUDA(cudaSetDevice(device_));
    // No image until every buffer is sized: a failed allocation leaves a renderer that renders
    // nothing rather than one whose buffers are smaller than its image.
    width_ = 0;
    height_ = 0;
    // The per-pixel buffers only grow, so a renderer that serves images of several sizes does not
    // free and allocate (each a device-wide synchronisation) on every size change. The denoiser's
    // buffers are sized on the first real-time frame.
    size_t n = size_t(w) * size_t(h);
    for (DeviceBuffer<float4>* b : {&accum_, &albedo_, &normal_depth_, &edge_, &motion_, &emission_, &color_, &denoised_buf_}) {
        b->reserve(n);
        if (n) PTW_CUDA(cudaMemsetAsync(b->ptr, 0, n * sizeof(float4), stream_));
    }
    heat_.reserve(n);
    display_.reserve(n);
    if (n) PTW_CUDA(cudaMemsetAsync(display_.ptr, 0, n * sizeof(uint32_t), stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
    width_ = w;
    height_ = h;
    reset();
}

void Renderer::reset() {
    samples_ = 0;
    frame_ = 0;
    denoised_ = false;
    heat_valid_ = false;
    accum_.zero(stream_);
    if (svgf_) svgf_->reset();
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::fill_view(DevView& v, const pt_camera& cam, int w, int h, int spp, uint32_t seed, const pt_path_options& po,
                         uint32_t frame0) const {
    // The path depth lives in 16 bits of the path state.
    if (po.max_depth < 0 || po.max_depth > 65535) throw Error{PT_ERR_INVALID, "max_depth must be in [0, 65535]"};
    if (w < 0 || h < 0 || spp < 0) throw Error{PT_ERR_INVALID, "negative image size or spp"};
    std::memset(&v, 0, sizeof(v));
    std::memcpy(v.cam, &cam, sizeof(v.cam));
    v.width = w;
    v.height = h;
    v.spp = spp;
    v.scene = 0;
    v.seed = seed;
    v.frame0 = frame0;
    v.max_depth = po.max_depth;
    v.rr_depth = po.rr_depth;
    v.nee = po.nee;
    v.clamp = po.clamp;
}

// Renders a set of views (each with its own spp and first sample index) in passes that fit the
// radiance buffer: work units are (view, sample range) packed in order; each unit's samples are
// summed into its view's accumulation in sample order after its pass.
void Renderer::render_pass_set(std::vector<DevView>& views, int /*spp_total*/, std::vector<int>& spp_each, std::vector<uint32_t>& frame0) {
    struct Unit {
        int view, s0, s1;
    };
    std::vector<std::vector<Unit>> passes(1);
    uint64_t used = 0;
    for (size_t vi = 0; vi < views.size(); vi++) {
        uint64_t npix = uint64_t(views[vi].width) * uint64_t(views[vi].height);
        if (npix == 0 || spp_each[vi] <= 0) continue;
        int s = 0;
        while (s < spp_each[vi]) {
            uint64_t room = sample_cap_ > used ? sample_cap_ - used : 0;
            int take = int(std::min<uint64_t>(uint64_t(spp_each[vi] - s), room / npix));
            if (take <= 0) {
                if (used == 0) take = 1;  // a single sample row larger than the cap: one pass of its own
                else {
                    passes.emplace_back();
                    used = 0;
                    continue;
                }
            }
            passes.back().push_back({int(vi), s, s + take});
            used += uint64_t(take) * npix;
            s += take;
        }
    }
    for (const auto& pass : passes) {
        if (pass.empty()) continue;
        std::vector<DevView> table;
        uint64_t work = 0;
        for (const Unit& u : pass) {
            DevView v = views[size_t(u.view)];
            uint64_t npix = uint64_t(v.width) * uint64_t(v.height);
            v.spp = u.s1 - u.s0;
            v.frame0 = frame0[size_t(u.view)] + uint32_t(u.s0);
            v.gbuffer = (u.s0 == 0) ? v.gbuffer : 0;
            v.realtime = (u.s0 == 0) ? v.realtime : 0;
            v.work_begin = work;
            v.work_count = npix * uint64_t(v.spp);
            table.push_back(v);
            work += v.work_count;
        }
        sample_out_.reserve(work);
        uint64_t off = 0;
        for (DevView& v : table) {
            v.sample_out = sample_out_.ptr + off;
            off += v.work_count;
        }
        if (d_views_.count < table.size()) d_views_.allocate(table.size());
        PTW_CUDA(cudaMemcpyAsync(d_views_.ptr, table.data(), table.size() * sizeof(DevView), cudaMemcpyHostToDevice, stream_));
        engine_->run(scene_.device_view(), 0, &scene_.view(), d_views_.ptr, int(table.size()), work);
        last_ctr_ = engine_->last();
        profile_.closest_rays += last_ctr_.rays;
        profile_.shadow_rays += last_ctr_.shadow_rays;
        profile_.closest_node_visits += last_ctr_.node_visits;
        profile_.closest_tri_tests += last_ctr_.tri_tests;
        profile_.shadow_node_visits += last_ctr_.shadow_node_visits;
        profile_.shadow_tri_tests += last_ctr_.shadow_tri_tests;
        profile_.closest_lane_steps += last_ctr_.trace_lane_steps;
        profile_.closest_warp_steps += last_ctr_.trace_warp_steps;
        profile_.shadow_lane_steps += last_ctr_.shadow_lane_steps;
        profile_.shadow_warp_steps += last_ctr_.shadow_warp_steps;
        bool timed = engine_->profiling() & PT_PROFILE_KERNEL_TIMES;
        cudaError_t stale = cudaGetLastError();
        if (stale != cudaSuccess) throw Error{PT_ERR_CUDA, std::string("after the wavefront pass: ") + cudaGetErrorString(stale)};
        if (timed) PTW_CUDA(cudaEventRecord(acc_ev_[0], stream_));
        for (size_t k = 0; k < table.size(); k++) {
            const Unit& u = pass[k];
            int first = u.s0 == 0, last = u.s1 == spp_each[size_t(u.view)];
            PTW_CUDA(wf_accumulate(d_views_.ptr + k, table[k], first, last, stream_));
        }
        profile_.accumulate.launches += table.size();
        profile_.kernel_launches += table.size();
        if (timed) PTW_CUDA(cudaEventRecord(acc_ev_[1], stream_));
        PTW_CUDA(cudaStreamSynchronize(stream_));
        if (timed) {
            float ms = 0;
            cudaEventElapsedTime(&ms, acc_ev_[0], acc_ev_[1]);
            profile_.accumulate.ms += ms;
        }
    }
}

void Renderer::render(const pt_camera& cam, const pt_render_settings& rs, int spp) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "render before upload"};
    if (width_ == 0 || height_ == 0 || spp <= 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    if (denoised_) reset();
    uint64_t npix = uint64_t(width_) * uint64_t(height_);
    DevView v;
    fill_view(v, cam, width_, height_, spp, rs.seed, rs.path, uint32_t(samples_));
    v.gbuffer = 1;
    v.accum = accum_.ptr;
    v.g_albedo = albedo_.ptr;
    v.g_normal_depth = normal_depth_.ptr;
    if (uint64_t(spp) * npix > sample_cap_) {
        acc_pass_.reserve(npix);
        v.acc_pass = acc_pass_.ptr;
    }
    std::vector<DevView> views{v};
    std::vector<int> spps{spp};
    std::vector<uint32_t> f0{uint32_t(samples_)};
    PTW_CUDA(cudaEventRecord(ev0_, stream_));
    render_pass_set(views, spp, spps, f0);
    PTW_CUDA(cudaEventRecord(ev1_, stream_));
    PTW_CUDA(cudaEventSynchronize(ev1_));
    PTW_CUDA(cudaEventElapsedTime(&last_ms_, ev0_, ev1_));
    samples_ += spp;
    last_camera_ = cam;
    heat_valid_ = false;
}

void Renderer::render_denoised(const pt_camera& cam, const pt_camera& prev, const pt_render_settings& rs, const pt_svgf_settings& sv) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "render before upload"};
    if (width_ == 0 || height_ == 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    if (!svgf_) svgf_ = std::make_unique<SvgfDenoiser>(device_, stream_);
    svgf_->resize(width_, height_);
    if (!denoised_) {
        samples_ = 0;
        svgf_->reset();
    }
    denoised_ = true;
    DevView v;
    fill_view(v, cam, width_, height_, 1, rs.seed, rs.path, frame_);
    v.gbuffer = 1;
    v.realtime = 1;
    // The real-time sample is not accumulated: its radiance goes to `color` only.
    acc_pass_.reserve(size_t(width_) * size_t(height_));
    v.accum = acc_pass_.ptr;
    v.g_albedo = albedo_.ptr;
    v.g_normal_depth = normal_depth_.ptr;
    v.g_emission = emission_.ptr;
    v.g_color = color_.ptr;
    // The denoiser's own records: octahedral normal + depth + material, and the reprojection into
    // the previous camera's image.
    v.g_edge = edge_.ptr;
    v.g_motion = motion_.ptr;
    static_assert(sizeof(v.prev_cam) == sizeof(pt_camera), "camera layout");
    std::memcpy(v.prev_cam, &prev, sizeof(v.prev_cam));
    v.has_prev = 1;
    std::vector<DevView> views{v};
    std::vector<int> spps{1};
    std::vector<uint32_t> f0{frame_};
    PTW_CUDA(cudaEventRecord(ev0_, stream_));
    render_pass_set(views, 1, spps, f0);
    svgf_->run_frame(reinterpret_cast<const float*>(color_.ptr), reinterpret_cast<const float*>(albedo_.ptr),
                     reinterpret_cast<const float*>(emission_.ptr), reinterpret_cast<const float*>(edge_.ptr),
                     reinterpret_cast<const float*>(motion_.ptr), sv, reinterpret_cast<float*>(denoised_buf_.ptr));
    PTW_CUDA(cudaEventRecord(ev1_, stream_));
    PTW_CUDA(cudaEventSynchronize(ev1_));
    cudaEventElapsedTime(&last_ms_, ev0_, ev1_);
    frame_++;
    samples_ = 1;
    last_camera_ = cam;
    heat_valid_ = false;
}

void Renderer::display(const pt_render_settings& rs, int mode, uint32_t* target) {
    if (width_ == 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    if (mode == PT_DISPLAY_HEATMAP && !heat_valid_ && scene_.ready()) {
        PTW_CUDA(wf_heatmap(scene_.device_view(), reinterpret_cast<const float*>(&last_camera_), width_, height_, heat_.ptr, stream_));
        heat_valid_ = true;
    }
    DisplayParams p;
    p.w = width_;
    p.h = height_;
    p.mode = mode;
    p.exposure = rs.exposure;
    p.tonemap = rs.tonemap;
    p.samples = float(samples_);
    p.inv_samples = samples_ > 0 ? 1.0f / float(samples_) : 0.0f;
    p.max_depth = scene_.extent();
    p.heat_scale = 1.0f / 160.0f;
    p.denoised = denoised_ ? 1 : 0;
    const float4* variance = svgf_ && svgf_->width() == width_ && svgf_->height() == height_
                                 ? reinterpret_cast<const float4*>(svgf_->variance())
                                 : nullptr;
    PTW_CUDA(wf_display(p, accum_.ptr, denoised_buf_.ptr, albedo_.ptr, normal_depth_.ptr, variance, heat_.ptr,
                        target ? target : display_.ptr, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::download_image(float* rgb, size_t n) {
    size_t npix = size_t(width_) * size_t(height_);
    if (n < 3 * npix) throw Error{PT_ERR_INVALID, "download_image: buffer too small"};
    if (npix == 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    // vec3 * (1 / samples), as GpuRenderer::download_image and CpuRenderer::image (one IEEE multiply
    // per channel, on the device); the denoised image is copied as it is.
    float inv = samples_ > 0 ? 1.0f / float(samples_) : 0.0f;
    resolve_and_copy_out(denoised_ ? denoised_buf_.ptr : accum_.ptr, npix, inv, !denoised_, rgb);
}

void Renderer::resolve_and_copy_out(const float4* src, size_t npix, float scale, bool apply_scale, float* rgb) {
    constexpr size_t kChunk = size_t(1) << 21;  // floats per pinned half (8 MiB)
    const size_t n = 3 * npix;
    rgb_dev_.reserve(n);
    PTW_CUDA(wf_resolve(src, uint32_t(npix), scale, apply_scale, rgb_dev_.ptr, stream_));
    // A page-locked destination takes one direct copy at the link's rate; pageable memory goes
    // through the pinned halves below.
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, rgb) == cudaSuccess && attr.type == cudaMemoryTypeHost) {
        PTW_CUDA(cudaMemcpyAsync(rgb, rgb_dev_.ptr, n * sizeof(float), cudaMemcpyDeviceToHost, stream_));
        PTW_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    cudaGetLastError();  // (an unknown pointer is not an error here)
    for (int k = 0; k < 2; k++) {
        if (!stage_[k]) PTW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&stage_[k]), kChunk * sizeof(float), cudaHostAllocDefault));
        if (!stage_ev_[k]) PTW_CUDA(cudaEventCreateWithFlags(&stage_ev_[k], cudaEventDisableTiming));
    }
    const size_t chunks = (n + kChunk - 1) / kChunk;
    auto issue = [&](size_t c) {
        size_t off = c * kChunk, len = std::min(kChunk, n - off);
        PTW_CUDA(cudaMemcpyAsync(stage_[c & 1], rgb_dev_.ptr + off, len * sizeof(float), cudaMemcpyDeviceToHost, stream_));
        PTW_CUDA(cudaEventRecord(stage_ev_[c & 1], stream_));
    };
    issue(0);
    for (size_t c = 0; c < chunks; c++) {
        // Chunk c + 1 goes to the half that chunk c - 1 used, whose host copy has finished.
        if (c + 1 < chunks) issue(c + 1);
        PTW_CUDA(cudaEventSynchronize(stage_ev_[c & 1]));
        size_t off = c * kChunk, len = std::min(kChunk, n - off);
        std::memcpy(rgb + off, stage_[c & 1], len * sizeof(float));
    }
}

void Renderer::download_display(uint32_t* out, size_t n) {
    size_t npix = size_t(width_) * size_t(height_);
    if (n < npix) throw Error{PT_ERR_INVALID, "download_display: buffer too small"};
    if (npix) {
        PTW_CUDA(cudaMemcpyAsync(out, display_.ptr, npix * 4, cudaMemcpyDeviceToHost, stream_));
        PTW_CUDA(cudaStreamSynchronize(stream_));
    }
}

void Renderer::download_gbuffer(float* albedo4, float* nd4, size_t n) {
    size_t npix = size_t(width_) * size_t(height_);
    if (n < npix) throw Error{PT_ERR_INVALID, "download_gbuffer: buffer too small"};
    if (albedo4) PTW_CUDA(cudaMemcpyAsync(albedo4, albedo_.ptr, npix * 16, cudaMemcpyDeviceToHost, stream_));
    if (nd4) PTW_CUDA(cudaMemcpyAsync(nd4, normal_depth_.ptr, npix * 16, cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::download_accumulation(float* sums4, size_t n) {
    size_t npix = size_t(width_) * size_t(height_);
    if (n < npix) throw Error{PT_ERR_INVALID, "download_accumulation: buffer too small"};
    if (npix == 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    PTW_CUDA(cudaMemcpyAsync(sums4, accum_.ptr, npix * sizeof(float4), cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::stats(pt_stats* out) const {
    std::memset(out, 0, sizeof(*out));
    out->width = width_;
    out->height = height_;
    out->samples = samples_;
    out->last_frame_ms = last_ms_;
    out->paths = last_ctr_.work_total;
    out->rays = last_ctr_.rays + last_ctr_.shadow_rays;
    out->shadow_rays = last_ctr_.shadow_rays;
    out->bounce_iterations = last_ctr_.iterations;
    out->queue_overflows = last_ctr_.overflow;
    size_t b = scene_.device_bytes() + engine_->device_bytes() + sample_out_.bytes() + heat_.bytes() + display_.bytes();
    for (const DeviceBuffer<float4>* x : {&accum_, &acc_pass_, &albedo_, &normal_depth_, &edge_, &motion_, &emission_, &color_, &denoised_buf_}) b += x->bytes();
    out->device_bytes = b;
}

void Renderer::set_profiling(int flags) {
    engine_->set_profiling(flags);
    profile_ = pt_profile{};
}

void Renderer::get_profile(pt_profile* out) const {
    *out = profile_;
    const WavefrontEngine& e = *engine_;
    pt_kernel_time* k[5] = {&out->setup, &out->generate, &out->trace, &out->shade, &out->shadow};
    for (int j = 0; j < 5; j++) {
        k[j]->launches = e.iteration_launches;
        k[j]->ms = e.kernel_ms[j];
    }
    out->kernel_launches = profile_.kernel_launches + e.kernel_launches;
}

void Renderer::set_tuning(const pt_tuning& t) {
    Tuning cur = engine_->tuning();
    if (t.path_capacity > 0) cur.path_capacity = t.path_capacity;
    if (t.trace_block > 0) {
        if (t.trace_block % 32 || t.trace_block > 256) throw Error{PT_ERR_INVALID, "trace_block must be a multiple of 32, at most 256"};
        cur.trace_block = t.trace_block;
    }
    if (t.shade_block > 0) {
        if (t.shade_block % 32 || t.shade_block > 256) throw Error{PT_ERR_INVALID, "shade_block must be a multiple of 32, at most 256"};
        cur.shade_block = t.shade_block;
    }
    if (t.sort_by_material >= 0) {
        if (t.sort_by_material > 4) throw Error{PT_ERR_INVALID, "sort_by_material must be in [0, 4]"};
        cur.sort_by_material = t.sort_by_material;
    }
    if (t.graph_bounces >= 0) cur.graph_bounces = t.graph_bounces;
    if (t.sort_rays >= 0) {
        if (t.sort_rays > 6) throw Error{PT_ERR_INVALID, "sort_rays must be in [0, 6]"};
        cur.sort_rays = t.sort_rays;
    }
    if (t.packed >= 0) cur.packed = t.packed ? 1 : 0;
    if (t.tail_paths >= 0 || t.tail_paths == kTailAuto) cur.tail_paths = t.tail_paths;
    if (t.wide_shadows >= 0) cur.wide_shadows = t.wide_shadows ? 1 : 0;
    if (t.trace_refill > 32 || t.shadow_refill > 32) throw Error{PT_ERR_INVALID, "trace_refill and shadow_refill must be in [1, 32]"};
    if (t.trace_refill > 0) cur.trace_refill = t.trace_refill;
    if (t.shadow_refill > 0) cur.shadow_refill = t.shadow_refill;
    if (t.walk_burst > (1 << 20)) throw Error{PT_ERR_INVALID, "walk_burst must be in [1, 2^20]"};
    if (t.walk_burst > 0) cur.walk_burst = t.walk_burst;
    if (t.sort_shadows >= 0) {
        if (t.sort_shadows > 6) throw Error{PT_ERR_INVALID, "sort_shadows must be in [0, 6]"};
        cur.sort_shadows = t.sort_shadows;
    }
    if (t.pair_walk >= 0) {
        if (t.pair_walk > 64) throw Error{PT_ERR_INVALID, "pair_walk must be in [0, 64]"};
        cur.pair_walk = t.pair_walk;
    }
    engine_->set_tuning(cur);
}

void Renderer::get_tuning(pt_tuning* t) const {
    const Tuning& c = engine_->tuning();
    t->path_capacity = c.path_capacity;
    t->trace_block = c.trace_block;
    t->shade_block = c.shade_block;
    t->sort_by_material = c.sort_by_material;
    t->graph_bounces = c.graph_bounces;
    t->sort_rays = c.sort_rays;
    t->packed = c.packed;
    t->tail_paths = c.tail_paths;
    t->wide_shadows = c.wide_shadows;
    t->trace_refill = c.trace_refill;
    t->shadow_refill = c.shadow_refill;
    t->walk_burst = c.walk_burst;
    t->sort_shadows = c.sort_shadows;
    t->pair_walk = c.pair_walk;
}

// Coordinate descent over the knobs, one at a time, each candidate timed on the same probe view set.
// Every probe runs twice and keeps the faster time, after a warm-up render with the candidate (graph
// capture and buffer growth are not timed). A knob moves only for a gain above 2%. The probe renders
// into the batched-view buffers, whose previous contents are put back afterwards.
void Renderer::tune_on(const std::vector<pt_view>& probe, pt_tuning* chosen, double* default_rate, double* tuned_rate) {
    uint64_t samples = 0;
    for (const pt_view& v : probe) samples += uint64_t(v.width) * uint64_t(v.height) * uint64_t(v.spp);
    if (samples == 0) throw Error{PT_ERR_INVALID, "autotune: the probe has no samples"};
    std::vector<pt_view> saved_views;
    std::vector<DeviceBuffer<float4>> saved_accum, saved_pass;
    saved_views.swap(batch_views_);
    saved_accum.swap(batch_accum_);
    saved_pass.swap(batch_pass_);
    auto restore = [&]() {
        batch_views_.swap(saved_views);
        batch_accum_.swap(saved_accum);
        batch_pass_.swap(saved_pass);
    };
    try {
        auto time_probe = [&]() {
            render_views(probe.data(), int(probe.size()));  // warm-up (graph capture, buffer growth)
            float best = 1e30f;
            for (int k = 0; k < 2; k++) {
                render_views(probe.data(), int(probe.size()));
                best = std::min(best, last_ms_);
            }
            return double(samples) / (double(best) / 1000.0);
        };
        Tuning base = engine_->tuning();
        engine_->set_tuning(base);
        double best_rate = time_probe();
        const double base_rate = best_rate;
        if (default_rate) *default_rate = best_rate;
        Tuning best = base;
        auto try_knob = [&](auto setter, std::initializer_list<int> values) {
            Tuning start = best;
            for (int val : values) {
                Tuning t = start;
                setter(t, val);
                engine_->set_tuning(t);
                double rate = time_probe();
                if (rate > best_rate * 1.02) {
                    best_rate = rate;
                    best = t;
                }
            }
            engine_->set_tuning(best);
        };
        try_knob([](Tuning& t, int v) { t.path_capacity = v; }, {1 << 20, 1 << 21, 1 << 22, 1 << 23, 1 << 24});
        try_knob([](Tuning& t, int v) { t.trace_block = v; }, {64, 128, 256});
        try_knob([](Tuning& t, int v) { t.shade_block = v; }, {64, 128, 256});
        try_knob([](Tuning& t, int v) { t.sort_by_material = v; }, {0, 1, 2, 4});
        try_knob([](Tuning& t, int v) { t.graph_bounces = v; }, {2, 4, 8});
        try_knob([](Tuning& t, int v) { t.sort_rays = v; }, {0, 3, 4, 5});
        try_knob([](Tuning& t, int v) { t.tail_paths = v; }, {0, 1 << 16, 1 << 17, 1 << 18, 1 << 20});
        try_knob([](Tuning& t, int v) { t.wide_shadows = v; }, {0, 1});
        try_knob([](Tuning& t, int v) { t.trace_refill = v; }, {1, 8, 16, 24, 32});
        try_knob([](Tuning& t, int v) { t.shadow_refill = v; }, {1, 8, 16, 24, 32});
        try_knob([](Tuning& t, int v) { t.walk_burst = v; }, {4, 8, 16, 32, 64});
        try_knob([](Tuning& t, int v) { t.sort_shadows = v; }, {0, 3, 4, 5});
        try_knob([](Tuning& t, int v) { t.pair_walk = v; }, {0, 3, 5, 8});
        // The chosen record against the starting one, timed once more each: a pick that does not
        // still win by 2% was noise, and the starting record stays.
        engine_->set_tuning(base);
        const double base_again = time_probe();
        engine_->set_tuning(best);
        const double best_again = time_probe();
        if (!(best_again > base_again * 1.02)) {
            best = base;
            best_rate = std::max(base_again, base_rate);  // the kept record's rate: its faster timing
            engine_->set_tuning(base);
        }
        if (tuned_rate) *tuned_rate = best_rate;
        if (chosen) get_tuning(chosen);
    } catch (...) {
        restore();
        throw;
    }
    restore();
}

// The single-view autotuner: the probe is the camera's view at a reduced resolution that holds about
// probe_samples paths.
void Renderer::autotune(const pt_camera& cam, const pt_render_settings& rs, int spp, uint64_t probe_samples, pt_tuning* chosen,
                        double* default_rate, double* tuned_rate) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "autotune before upload"};
    if (spp <= 0 || rs.width <= 0 || rs.height <= 0) throw Error{PT_ERR_INVALID, "autotune: bad view"};
    if (probe_samples == 0) probe_samples = uint64_t(1) << 23;
    double full = double(rs.width) * double(rs.height) * double(spp);
    double scale = std::min(1.0, std::sqrt(double(probe_samples) / full));
    pt_view v{};
    v.camera = cam;
    v.width = std::max(8, int(rs.width * scale));
    v.height = std::max(8, int(rs.height * scale));
    v.spp = spp;
    v.seed = rs.seed;
    v.path = rs.path;
    tune_on({v}, chosen, default_rate, tuned_rate);
}

// The batched form's autotuner: the probe is the view set itself with every view's resolution scaled
// by one factor so that the set holds about probe_samples paths (spp, cameras and options kept).
void Renderer::autotune_views(const pt_view* views, int n, uint64_t probe_samples, pt_tuning* chosen, double* default_rate,
                              double* tuned_rate) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "autotune before upload"};
    if (n <= 0 || !views) throw Error{PT_ERR_INVALID, "autotune: no views"};
    if (probe_samples == 0) probe_samples = uint64_t(1) << 25;
    double full = 0;
    for (int i = 0; i < n; i++) full += double(views[i].width) * double(views[i].height) * double(views[i].spp);
    if (full <= 0) throw Error{PT_ERR_INVALID, "autotune: the views have no samples"};
    double scale = std::min(1.0, std::sqrt(double(probe_samples) / full));
    std::vector<pt_view> probe(views, views + n);
    for (pt_view& v : probe) {
        v.width = std::max(8, int(v.width * scale));
        v.height = std::max(8, int(v.height * scale));
    }
    tune_on(probe, chosen, default_rate, tuned_rate);
}

void Renderer::trace_primary(const pt_camera& cam, int w, int h, uint32_t frame, uint32_t seed, float* hits4) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "trace before upload"};
    if (w <= 0 || h <= 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    DeviceBuffer<float4> out;
    out.allocate(size_t(w) * size_t(h));
    probe_claim_.reserve(1);
    const Tuning& t = engine_->tuning();
    const uint32_t pairs = t.packed ? uint32_t(std::clamp(t.pair_walk, 0, 64)) : 0u;  // the render's closest-hit walk
    PTW_CUDA(wf_trace_primary(scene_.device_view(), reinterpret_cast<const float*>(&cam), w, h, frame, seed, out.ptr, probe_claim_.ptr, pairs,
                              stream_));
    PTW_CUDA(cudaMemcpyAsync(hits4, out.ptr, out.bytes(), cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::light_picks(const pt_camera& cam, const pt_render_settings& rs, uint32_t frame, int32_t* picks4) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "probe before upload"};
    if (rs.width <= 0 || rs.height <= 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    DevView v;
    fill_view(v, cam, rs.width, rs.height, 1, rs.seed, rs.path, frame);
    DeviceBuffer<DevView> dv;
    dv.upload(&v, 1, stream_);
    DeviceBuffer<int4> out;
    out.allocate(size_t(rs.width) * size_t(rs.height));
    PTW_CUDA(wf_light_picks(scene_.device_view(), dv.ptr, out.ptr, rs.width, rs.height, stream_));
    PTW_CUDA(cudaMemcpyAsync(picks4, out.ptr, out.bytes(), cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::heatmap(const pt_camera& cam, int w, int h, float* out) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "probe before upload"};
    if (w <= 0 || h <= 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    DeviceBuffer<float> buf;
    buf.allocate(size_t(w) * size_t(h));
    PTW_CUDA(wf_heatmap(scene_.device_view(), reinterpret_cast<const float*>(&cam), w, h, buf.ptr, stream_));
    PTW_CUDA(cudaMemcpyAsync(out, buf.ptr, buf.bytes(), cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::occlusion_probe(const float* rays8, int n, int wide, int32_t* out4) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "probe before upload"};
    if (n <= 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    DeviceBuffer<float4> rays;
    rays.upload(reinterpret_cast<const float4*>(rays8), size_t(n) * 2, stream_);
    DeviceBuffer<int4> out;
    out.allocate(size_t(n));
    probe_claim_.reserve(1);
    const Tuning& t = engine_->tuning();
    const uint32_t pairs = t.packed ? uint32_t(std::clamp(t.pair_walk, 0, 64)) : 0u;  // the render's any-hit walk
    PTW_CUDA(wf_occlusion_probe(scene_.device_view(), rays.ptr, n, wide, out.ptr, probe_claim_.ptr, pairs, stream_));
    PTW_CUDA(cudaMemcpyAsync(out4, out.ptr, out.bytes(), cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
}

void Renderer::render_views(const pt_view* views, int n) {
    if (!scene_.ready()) throw Error{PT_ERR_NO_SCENE, "render before upload"};
    if (n < 0) throw Error{PT_ERR_INVALID, "negative view count"};
    PTW_CUDA(cudaSetDevice(device_));
    batch_views_.assign(views, views + n);
    batch_accum_.resize(size_t(n));
    std::vector<DevView> table(static_cast<size_t>(n));
    std::vector<int> spps(static_cast<size_t>(n));
    std::vector<uint32_t> f0(size_t(n), 0);
    batch_pass_.resize(size_t(n));
    for (int i = 0; i < n; i++) {
        const pt_view& pv = views[i];
        if (pv.width < 0 || pv.height < 0 || pv.spp < 0) throw Error{PT_ERR_INVALID, "bad view size"};
        if (uint64_t(pv.width) * uint64_t(pv.height) > (uint64_t(1) << 30)) throw Error{PT_ERR_INVALID, "view larger than 2^30 pixels"};
        size_t npix = size_t(pv.width) * size_t(pv.height);
        batch_accum_[size_t(i)].allocate(npix);
        batch_accum_[size_t(i)].zero(stream_);
        fill_view(table[size_t(i)], pv.camera, pv.width, pv.height, pv.spp, pv.seed, pv.path, 0);
        table[size_t(i)].accum = batch_accum_[size_t(i)].ptr;
        if (uint64_t(pv.spp) * npix > sample_cap_) {
            batch_pass_[size_t(i)].reserve(npix);
            table[size_t(i)].acc_pass = batch_pass_[size_t(i)].ptr;
        }
        spps[size_t(i)] = pv.spp;
    }
    // One pass when it fits: the radiance buffer may take up to half of the free device memory.
    uint64_t total = 0;
    for (int i = 0; i < n; i++) total += uint64_t(views[i].width) * uint64_t(views[i].height) * uint64_t(views[i].spp);
    size_t free_b = 0, total_b = 0;
    PTW_CUDA(cudaMemGetInfo(&free_b, &total_b));
    uint64_t saved_cap = sample_cap_;
    uint64_t room = uint64_t(free_b / 2) / sizeof(float4) + sample_out_.count;
    sample_cap_ = std::max<uint64_t>(saved_cap, std::min<uint64_t>(total, room));
    PTW_CUDA(cudaEventRecord(ev0_, stream_));
    try {
        render_pass_set(table, 0, spps, f0);
    } catch (...) {
        sample_cap_ = saved_cap;
        throw;
    }
    sample_cap_ = saved_cap;
    PTW_CUDA(cudaEventRecord(ev1_, stream_));
    PTW_CUDA(cudaEventSynchronize(ev1_));
    PTW_CUDA(cudaEventElapsedTime(&last_ms_, ev0_, ev1_));
}

void Renderer::download_view(int v, float* rgb, size_t n) {
    if (v < 0 || size_t(v) >= batch_views_.size()) throw Error{PT_ERR_NOT_FOUND, "no such view"};
    const pt_view& pv = batch_views_[size_t(v)];
    size_t npix = size_t(pv.width) * size_t(pv.height);
    if (n < 3 * npix) throw Error{PT_ERR_INVALID, "download_view: buffer too small"};
    if (npix == 0) return;
    PTW_CUDA(cudaSetDevice(device_));
    float inv = pv.spp > 0 ? 1.0f / float(pv.spp) : 0.0f;
    resolve_and_copy_out(batch_accum_[size_t(v)].ptr, npix, inv, true, rgb);
}

}  // namespace ptw
