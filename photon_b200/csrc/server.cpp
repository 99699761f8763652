// The request server (continuous batching over resident scenes).
//
// A server thread owns one device stream and one wavefront engine in continuous mode. Requests are
// admitted in arrival order while they fit the device-memory budget: each admitted request becomes
// a view (camera, size, spp, seed, scene slot) whose work range is appended to the running
// wavefront, so its paths share the path pool with every other request in flight, whatever their
// scene, resolution or spp. Between graph-sized batches of bounce iterations the thread reads the
// per-view finished-path counters; a request whose paths have all finished is summed in sample
// order (so its image is the same alone or in any mix), copied to the host and released.
// The device never waits on anything: kernels claim work with atomics and return, so a stalled
// request cannot hang the GPU; host waits are all bounded.
#include "server.h"

#include <algorithm>
#include <chrono>
#include <cstring>

namespace ptw {

namespace {
constexpr int kMaxScenes = 256;
constexpr int kItersPerCheck = 2;
}  // namespace

Server::Server(const pt_server_config& cfg) : cfg_(cfg), device_(cfg.device) {
    t0_ = std::chrono::steady_clock::now();
    PTW_CUDA(cudaSetDevice(device_));
    PTW_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    engine_ = std::make_unique<WavefrontEngine>(device_, stream_);
    Tuning t;
    if (cfg.path_capacity > 0) t.path_capacity = cfg.path_capacity;
    engine_->set_tuning(t);
    engine_->reserve_paths(uint64_t(t.path_capacity));
    pool_bytes_ = engine_->device_bytes();
    d_scenes_.allocate(kMaxScenes);
    d_views_.allocate(1024);
    d_done_.allocate(1024);
    d_done_.zero(stream_);
    PTW_CUDA(cudaStreamSynchronize(stream_));
    st_.budget_bytes = cfg.budget_bytes;
    if (cfg_.budget_bytes && pool_bytes_ > cfg_.budget_bytes) throw Error{PT_ERR_BUDGET, "the path pool alone exceeds the budget"};
    thread_ = std::thread([this] { loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    if (thread_.joinable()) thread_.join();
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    requests_.clear();
    engine_.reset();
    scenes_.clear();
    cudaStreamDestroy(stream_);
}

double Server::now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count(); }

size_t Server::request_bytes(const pt_request& r) const {
    size_t npix = size_t(r.width) * size_t(r.height);
    return npix * size_t(r.spp) * sizeof(float4) + npix * sizeof(float4) + sizeof(DevView) + sizeof(unsigned long long);
}

int32_t Server::add_scene(const pt_scene_desc& d) {
    size_t est = DeviceScene::estimate_bytes(d);
    {
        std::lock_guard<std::mutex> g(mu_);
        if (int(scenes_.size()) >= kMaxScenes) throw Error{PT_ERR_BUDGET, "too many resident scenes"};
        if (cfg_.budget_bytes && bytes_in_use_ + pool_bytes_ + scene_bytes_ + est > cfg_.budget_bytes)
            throw Error{PT_ERR_BUDGET, "the scene does not fit the device-memory budget"};
    }
    PTW_CUDA(cudaSetDevice(device_));
    cudaStream_t s;
    PTW_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    auto scene = std::make_unique<DeviceScene>();
    try {
        scene->upload(d, s, false);
    } catch (...) {
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    std::lock_guard<std::mutex> g(mu_);
    scene_bytes_ += scene->device_bytes();
    scenes_.push_back(std::move(scene));
    scenes_dirty_ = true;
    st_.scenes = int(scenes_.size());
    cv_work_.notify_all();
    return int32_t(scenes_.size()) - 1;
}

uint64_t Server::submit(const pt_request& r) {
    if (r.width <= 0 || r.height <= 0 || r.spp <= 0) throw Error{PT_ERR_INVALID, "request: width, height and spp must be positive"};
    if (r.path.max_depth < 0 || r.path.max_depth > 65535) throw Error{PT_ERR_INVALID, "request: max_depth must be in [0, 65535]"};
    if (uint64_t(r.width) * uint64_t(r.height) * uint64_t(r.spp) >= (uint64_t(1) << 32))
        throw Error{PT_ERR_INVALID, "request: more than 2^32 samples"};
    std::lock_guard<std::mutex> g(mu_);
    if (r.scene_id < 0 || r.scene_id >= int(scenes_.size())) throw Error{PT_ERR_NOT_FOUND, "request: unknown scene"};
    size_t need = request_bytes(r);
    if (cfg_.budget_bytes && need + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes) {
        st_.rejected++;
        throw Error{PT_ERR_BUDGET, "request: larger than the device-memory budget"};
    }
    auto q = std::make_unique<Request>();
    q->id = next_id_++;
    q->req = r;
    q->submit_s = now();
    q->bytes = need;
    q->work = uint64_t(r.width) * uint64_t(r.height) * uint64_t(r.spp);
    uint64_t id = q->id;
    requests_[id] = std::move(q);
    queue_.push_back(id);
    st_.submitted++;
    cv_work_.notify_all();
    return id;
}

int32_t Server::poll(uint64_t id) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    return it->second->state;
}

void Server::wait(uint64_t id, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    auto deadline = std::chrono::steady_clock::now() + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                                            std::chrono::duration<double>(std::max(0.0, timeout_s)));
    for (;;) {
        auto it = requests_.find(id);
        if (it == requests_.end()) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
        int s = it->second->state;
        if (s == PT_REQ_DONE) return;
        if (s == PT_REQ_CANCELLED) throw Error{PT_ERR_CANCELLED, "request cancelled"};
        if (s == PT_REQ_FAILED) throw Error{PT_ERR_CUDA, "request failed: " + it->second->error};
        if (cv_done_.wait_until(lk, deadline) == std::cv_status::timeout) {
            auto it2 = requests_.find(id);
            if (it2 != requests_.end() && it2->second->state == PT_REQ_DONE) return;
            throw Error{PT_ERR_TIMEOUT, "wait timed out"};
        }
    }
}

void Server::fetch(uint64_t id, float* rgb, size_t n, pt_request_stats* st) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    Request& r = *it->second;
    if (r.state == PT_REQ_QUEUED || r.state == PT_REQ_RUNNING) throw Error{PT_ERR_INVALID, "request not finished"};
    if (st) {
        st->submit_s = r.submit_s;
        st->admit_s = r.admit_s;
        st->done_s = r.done_s;
        st->samples = r.work;
        st->state = r.state;
    }
    if (r.state == PT_REQ_DONE && rgb) {
        if (n < r.result.size()) throw Error{PT_ERR_INVALID, "fetch: buffer too small"};
        std::memcpy(rgb, r.result.data(), r.result.size() * sizeof(float));
    }
    int state = r.state;
    requests_.erase(it);
    if (state == PT_REQ_CANCELLED) throw Error{PT_ERR_CANCELLED, "request cancelled"};
}

void Server::cancel(uint64_t id) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end()) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    Request& r = *it->second;
    if (r.state == PT_REQ_QUEUED) {
        queue_.erase(std::remove(queue_.begin(), queue_.end(), id), queue_.end());
        r.state = PT_REQ_CANCELLED;
        r.done_s = now();
        st_.cancelled++;
        cv_done_.notify_all();
    } else if (r.state == PT_REQ_RUNNING) {
        r.cancel = true;
        cv_work_.notify_all();
    }
}

void Server::stats(pt_server_stats* out) {
    std::lock_guard<std::mutex> g(mu_);
    *out = st_;
    out->device_bytes_in_use = bytes_in_use_ + pool_bytes_ + scene_bytes_;
    out->budget_bytes = cfg_.budget_bytes;
    out->active = int(active_.size());
    out->queued = int(queue_.size());
    out->scenes = int(scenes_.size());
}

void Server::inject_allocation_failures(int n) {
    std::lock_guard<std::mutex> g(mu_);
    inject_failures_ = n;
}

void Server::upload_scene_table() {
    std::vector<DevScene> table;
    for (const auto& s : scenes_) table.push_back(s->view());
    PTW_CUDA(cudaMemcpyAsync(d_scenes_.ptr, table.data(), table.size() * sizeof(DevScene), cudaMemcpyHostToDevice, stream_));
    scenes_dirty_ = false;
}

// Called with the lock held: allocates the request's buffers and appends its view.
bool Server::try_admit(Request& r) {
    if (cfg_.max_active > 0 && int(active_.size()) >= cfg_.max_active) return false;
    if (cfg_.budget_bytes && bytes_in_use_ + r.bytes + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes) return false;
    size_t npix = size_t(r.req.width) * size_t(r.req.height);
    try {
        if (inject_failures_ > 0) {
            inject_failures_--;
            throw Error{PT_ERR_ALLOC, "injected allocation failure"};
        }
        r.sample_out.allocate(npix * size_t(r.req.spp));
        r.accum.allocate(npix);
        r.accum.zero(stream_);
    } catch (const Error& e) {
        r.sample_out.release();
        r.accum.release();
        r.state = PT_REQ_FAILED;
        r.error = e.message;
        r.done_s = now();
        cv_done_.notify_all();
        return true;  // consumed (failed), not retried
    }
    // Grow the view table (and the finished-path counters) by doubling.
    if (views_.size() + 1 > d_views_.count) {
        size_t cap = d_views_.count * 2;
        DeviceBuffer<DevView> nv;
        nv.allocate(cap);
        DeviceBuffer<unsigned long long> nd;
        nd.allocate(cap);
        nd.zero(stream_);
        PTW_CUDA(cudaMemcpyAsync(nd.ptr, d_done_.ptr, d_done_.bytes(), cudaMemcpyDeviceToDevice, stream_));
        PTW_CUDA(cudaStreamSynchronize(stream_));
        d_views_ = std::move(nv);
        d_done_ = std::move(nd);
        for (size_t k = 0; k < views_.size(); k++) views_[k].done_counter = d_done_.ptr + k;
        views_uploaded_ = 0;  // re-upload everything
    }
    DevView v;
    std::memset(&v, 0, sizeof(v));
    std::memcpy(v.cam, &r.req.camera, sizeof(v.cam));
    v.width = r.req.width;
    v.height = r.req.height;
    v.spp = r.req.spp;
    v.scene = r.req.scene_id;
    v.seed = r.req.seed;
    v.frame0 = 0;
    v.max_depth = r.req.path.max_depth;
    v.rr_depth = r.req.path.rr_depth;
    v.nee = r.req.path.nee;
    v.clamp = r.req.path.clamp;
    v.work_begin = work_total_;
    v.work_count = r.work;
    v.sample_out = r.sample_out.ptr;
    v.accum = r.accum.ptr;
    v.done_counter = d_done_.ptr + views_.size();
    r.view = int(views_.size());
    views_.push_back(v);
    work_total_ += r.work;
    bytes_in_use_ += r.bytes;
    r.state = PT_REQ_RUNNING;
    r.admit_s = now();
    active_.push_back(r.id);
    return true;
}

// Sums a finished request's samples in order and copies its image to the host (lock released).
void Server::finish(Request& r) {
    const DevView& v = views_[size_t(r.view)];
    PTW_CUDA(wf_accumulate(d_views_.ptr + r.view, v, 1, 1, stream_));
    size_t npix = size_t(r.req.width) * size_t(r.req.height);
    std::vector<float4> raw(npix);
    PTW_CUDA(cudaMemcpyAsync(raw.data(), r.accum.ptr, npix * sizeof(float4), cudaMemcpyDeviceToHost, stream_));
    PTW_CUDA(cudaStreamSynchronize(stream_));
    r.result.resize(3 * npix);
    float inv = 1.0f / float(r.req.spp);
    for (size_t i = 0; i < npix; i++) {
        r.result[3 * i] = raw[i].x * inv;
        r.result[3 * i + 1] = raw[i].y * inv;
        r.result[3 * i + 2] = raw[i].z * inv;
    }
}

void Server::loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    double busy_since = -1;
    while (!stop_) {
        try {
            // Admission in arrival order while the budget allows.
            while (!queue_.empty()) {
                Request& r = *requests_[queue_.front()];
                if (!try_admit(r)) break;
                queue_.pop_front();
            }
            if (scenes_dirty_) upload_scene_table();
            if (views_uploaded_ < views_.size()) {
                PTW_CUDA(cudaMemcpyAsync(d_views_.ptr + views_uploaded_, views_.data() + views_uploaded_,
                                         (views_.size() - views_uploaded_) * sizeof(DevView), cudaMemcpyHostToDevice, stream_));
                views_uploaded_ = views_.size();
                if (!engine_started_) {
                    engine_->begin(d_scenes_.ptr, d_views_.ptr, int(views_.size()));
                    engine_started_ = true;
                }
                engine_->set_views(d_views_.ptr, int(views_.size()));
                engine_->append_work(work_total_);
            }
            // Cancelled running requests: their remaining paths end at their first vertex.
            for (uint64_t id : active_) {
                Request& r = *requests_[id];
                if (r.cancel && views_[size_t(r.view)].max_depth != 0) {
                    views_[size_t(r.view)].max_depth = 0;
                    PTW_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(d_views_.ptr + r.view) + offsetof(DevView, max_depth),
                                             &views_[size_t(r.view)].max_depth, sizeof(int), cudaMemcpyHostToDevice, stream_));
                    PTW_CUDA(cudaStreamSynchronize(stream_));
                }
            }
            if (active_.empty()) {
                if (busy_since >= 0) {
                    st_.busy_seconds += now() - busy_since;
                    busy_since = -1;
                }
                cv_work_.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
            if (busy_since < 0) busy_since = now();
            // A batch of bounce iterations with the lock released.
            std::vector<Request*> active;
            for (uint64_t id : active_) active.push_back(requests_[id].get());
            lk.unlock();
            engine_->iterate(kItersPerCheck);
            engine_->sync();
            if (h_done_.size() < views_.size()) h_done_.resize(views_.size());
            size_t lo = views_.size(), hi = 0;
            for (Request* r : active) {
                size_t vi = size_t(r->view);
                lo = std::min(lo, vi);
                hi = std::max(hi, vi + 1);
            }
            PTW_CUDA(cudaMemcpyAsync(h_done_.data() + lo, d_done_.ptr + lo, (hi - lo) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
            PTW_CUDA(cudaStreamSynchronize(stream_));
            std::vector<Request*> finished;
            for (Request* r : active)
                if (h_done_[size_t(r->view)] >= r->work) finished.push_back(r);
            for (Request* r : finished)
                if (!r->cancel) finish(*r);
            lk.lock();
            st_.bounce_iterations = engine_->counters().iterations;
            for (Request* r : finished) {
                r->state = r->cancel ? PT_REQ_CANCELLED : PT_REQ_DONE;
                r->done_s = now();
                if (r->cancel) st_.cancelled++;
                else {
                    st_.completed++;
                    st_.samples_done += r->work;
                }
                bytes_in_use_ -= r->bytes;
                r->sample_out.release();
                r->accum.release();
                active_.erase(std::remove(active_.begin(), active_.end(), r->id), active_.end());
            }
            if (!finished.empty()) cv_done_.notify_all();
        } catch (const Error& e) {
            if (!lk.owns_lock()) lk.lock();
            // A device failure fails every running request; the server keeps its handle valid.
            for (uint64_t id : active_) {
                Request& r = *requests_[id];
                r.state = PT_REQ_FAILED;
                r.error = e.message;
                r.done_s = now();
                bytes_in_use_ -= r.bytes;
            }
            active_.clear();
            cv_done_.notify_all();
        }
    }
}

}  // namespace ptw
