// The request server (continuous batching over resident scenes).
//
// A server thread owns one device stream and one wavefront engine in continuous mode. Requests are
// admitted in arrival order while they fit the device-memory budget; an admitted request's paths are
// handed to the running wavefront in chunks, so they share the path pool with every other request
// in flight, whatever their scene, resolution or spp. The thread keeps about one pool's worth of
// handed-over paths ahead of generation and fills it shortest-remaining-request first, so a small
// request that arrives behind a large one waits for one chunk, not for the whole large image.
// Each chunk is a view (camera, size, spp, seed, scene slot) over a range of the image's work items;
// all chunks of a request count into one finished-path counter. Between batches of bounce
// iterations the thread reads the counters; a request whose paths have all finished is summed in
// sample order (so its image is the same alone or in any mix), copied to the host and released.
// Request buffers come from a private stream-ordered memory pool, so admissions and releases never
// synchronise the device.
// The device never waits on anything: kernels claim work with atomics and return, so a stalled
// request cannot hang the GPU; host waits are all bounded.
#include "server.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>

#include "image_io.h"

namespace ptw {

namespace {
constexpr int kMaxScenes = 256;
constexpr uint64_t kChunkPaths = uint64_t(1) << 20;  // paths per chunk handed to the wavefront
// Requests admitted at once when the configuration leaves it open. More do not feed the wavefront
// any better (it takes chunks of a few of them at a time) but hold device memory for their sample
// buffers: on the four-scene stream at 200 req/s, an open limit gave 970-1,530 Msamples/s and
// p50 10-46 s, a limit of 16 gave 1,893 Msamples/s and p50 9.8 s (32: 1,805 and 10.1 s).
constexpr int kDefaultMaxActive = 16;
}  // namespace

Server::Server(const pt_server_config& cfg) : cfg_(cfg), device_(cfg.device) {
    t0_ = std::chrono::steady_clock::now();
    PTW_CUDA(cudaSetDevice(device_));
    PTW_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    engine_ = std::make_unique<WavefrontEngine>(device_, stream_);
    // The pool of a plain render (16M paths) and its ray sorting: on the four-scene stream at a
    // saturating 500 req/s they took the server from 1,842 (8M paths, unsorted) to 2,383 Msamples/s.
    // The sort kernels are launched only while at least kSortMinPaths paths are pending (loop()), so a
    // lightly loaded server does not pay for them.
    Tuning t;
    t.path_capacity = cfg.path_capacity > 0 ? cfg.path_capacity : (1 << 24);
    if (cfg.sort_rays < -1 || cfg.sort_rays > 6) throw Error{PT_ERR_INVALID, "sort_rays must be in [-1, 6]"};
    t.sort_rays = cfg.sort_rays > 0 ? cfg.sort_rays : (cfg.sort_rays == 0 ? 4 : 0);
    created_sort_rays_ = t.sort_rays;
    engine_->set_tuning(t);
    engine_->reserve_paths(uint64_t(t.path_capacity));
    pool_bytes_ = engine_->device_bytes();
    d_scenes_.allocate(kMaxScenes);
    d_views_.allocate(1024);
    d_done_.allocate(1024);
    d_done_.zero(stream_);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device_;
    PTW_CUDA(cudaMemPoolCreate(&mem_pool_, &props));
    uint64_t keep = ~uint64_t(0);  // freed request buffers stay in the pool for the next admissions
    PTW_CUDA(cudaMemPoolSetAttribute(mem_pool_, cudaMemPoolAttrReleaseThreshold, &keep));
    // Reserve the pool's working set now: growing it while requests run maps memory on the loop's
    // thread between batches, and the device idles meanwhile (a fresh server's first saturating
    // stream ran at 0.60 of the device's time, the same stream again at 0.89). Up to 32 GiB, half the
    // free memory, and what the budget leaves beside the path pool.
    {
        size_t free_b = 0, total_b = 0;
        PTW_CUDA(cudaMemGetInfo(&free_b, &total_b));
        size_t reserve = std::min<size_t>(size_t(32) << 30, free_b / 2);
        if (cfg.budget_bytes) reserve = std::min<size_t>(reserve, cfg.budget_bytes > pool_bytes_ ? cfg.budget_bytes - pool_bytes_ : 0);
        if (cfg.reserve_bytes > 0) reserve = std::min<size_t>(size_t(cfg.reserve_bytes), free_b / 2);
        if (cfg.reserve_bytes < 0) reserve = 0;
        if (reserve >= (size_t(1) << 20)) {
            void* p = nullptr;
            if (cudaMallocFromPoolAsync(&p, reserve, mem_pool_, stream_) == cudaSuccess) PTW_CUDA(cudaFreeAsync(p, stream_));
            else cudaGetLastError();  // no reservation: the pool grows on demand
        }
    }
    PTW_CUDA(cudaStreamCreateWithFlags(&fin_stream_, cudaStreamNonBlocking));
    {
        int least = 0, greatest = 0;
        PTW_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        PTW_CUDA(cudaStreamCreateWithPriority(&session_stream_, cudaStreamNonBlocking, greatest));
        session_engine_ = std::make_unique<WavefrontEngine>(device_, session_stream_);
        Tuning st;
        st.path_capacity = 1 << 23;  // grown on the first frames to what they need, up to this
        session_engine_->set_tuning(st);
        lane_idle_bytes_ = session_engine_->device_bytes();
    }
    for (Batch& b : batch_) {
        PTW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&b.ctr), sizeof(Counters), cudaHostAllocDefault));
        PTW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&b.work_total), sizeof(unsigned long long), cudaHostAllocDefault));
        PTW_CUDA(cudaEventCreate(&b.ev));
        PTW_CUDA(cudaEventCreate(&b.ev_start));
        std::memset(b.ctr, 0, sizeof(Counters));
    }
    PTW_CUDA(cudaStreamSynchronize(stream_));
    st_.budget_bytes = cfg.budget_bytes;
    if (cfg_.budget_bytes && pool_bytes_ > cfg_.budget_bytes) throw Error{PT_ERR_BUDGET, "the path pool alone exceeds the budget"};
    thread_ = std::thread([this] { loop(); });
    session_thread_ = std::thread([this] { session_loop(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> g(mu_);
        stop_ = true;
    }
    cv_work_.notify_all();
    cv_frames_.notify_all();
    if (thread_.joinable()) thread_.join();
    if (session_thread_.joinable()) session_thread_.join();
    cudaSetDevice(device_);
    cudaStreamSynchronize(session_stream_);
    cudaStreamSynchronize(stream_);
    cudaStreamSynchronize(fin_stream_);
    for (auto& kv : requests_) release_buffers(*kv.second, stream_);
    for (Finishing& f : finishing_) cudaEventDestroy(f.ev);
    for (auto& kv : requests_)
        if (kv.second->result) cudaFreeAsync(kv.second->result, stream_);
    cudaStreamSynchronize(stream_);
    for (Batch& b : batch_) {
        cudaFreeHost(b.ctr);
        cudaFreeHost(b.work_total);
        if (b.done) cudaFreeHost(b.done);
        if (b.views) cudaFreeHost(b.views);
        cudaEventDestroy(b.ev);
        cudaEventDestroy(b.ev_start);
    }
    requests_.clear();
    sessions_.clear();
    session_engine_.reset();
    engine_.reset();
    scenes_.clear();
    if (mem_pool_) cudaMemPoolDestroy(mem_pool_);
    cudaStreamDestroy(fin_stream_);
    cudaStreamDestroy(session_stream_);
    cudaStreamDestroy(stream_);
}

double Server::now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count(); }

size_t Server::request_bytes(const pt_request& r) const {
    // (The display image, when asked for, goes into the sample buffer after the float image.)
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
    // Checked again under the lock that publishes the scene: concurrent add_scene calls all passed the
    // first check before any of them was counted, and the device scene table holds kMaxScenes entries.
    if (int(scenes_.size()) >= kMaxScenes) throw Error{PT_ERR_BUDGET, "too many resident scenes"};
    if (cfg_.budget_bytes && bytes_in_use_ + pool_bytes_ + scene_bytes_ + scene->device_bytes() > cfg_.budget_bytes)
        throw Error{PT_ERR_BUDGET, "the scene does not fit the device-memory budget"};
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
    if (r.display != 0 && (r.display != 1 || r.tonemap < 0 || r.tonemap > 2 || !std::isfinite(r.exposure)))
        throw Error{PT_ERR_INVALID, "request: display must be 0 or 1, with a tone map in [0, 2] and a finite exposure"};
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
    if (it == requests_.end() || it->second->fetched) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    return it->second->state;
}

void Server::wait(uint64_t id, double timeout_s) {
    std::unique_lock<std::mutex> lk(mu_);
    auto deadline = std::chrono::steady_clock::now() + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                                                            std::chrono::duration<double>(std::max(0.0, timeout_s)));
    for (;;) {
        auto it = requests_.find(id);
        if (it == requests_.end() || it->second->fetched) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
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

// Copies part of a finished request's device result into caller memory, on the calling thread (with
// the server's device current for the copy, the caller's restored after it).
void Server::read_result(const Request& r, void* dst, size_t offset, size_t bytes) {
    int previous = 0;
    PTW_CUDA(cudaGetDevice(&previous));
    PTW_CUDA(cudaSetDevice(device_));
    cudaError_t e = cudaMemcpyAsync(dst, reinterpret_cast<const char*>(r.result) + offset, bytes, cudaMemcpyDeviceToHost, cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
    cudaSetDevice(previous);
    PTW_CUDA(e);
}

void Server::fetch(uint64_t id, float* rgb, size_t n, pt_request_stats* st) {
    std::unique_lock<std::mutex> g(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end() || it->second->fetched) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    Request& r = *it->second;
    if (r.state == PT_REQ_QUEUED || r.state == PT_REQ_RUNNING) throw Error{PT_ERR_INVALID, "request not finished"};
    if (r.reading) throw Error{PT_ERR_INVALID, "fetch: another call is reading this request"};
    if (st) {
        st->submit_s = r.submit_s;
        st->admit_s = r.admit_s;
        st->done_s = r.done_s;
        st->samples = r.work;
        st->state = r.state;
    }
    if (r.state == PT_REQ_DONE && rgb) {
        const size_t bytes = 3 * size_t(r.req.width) * size_t(r.req.height) * sizeof(float);
        if (n < 3 * size_t(r.req.width) * size_t(r.req.height)) throw Error{PT_ERR_INVALID, "fetch: buffer too small"};
        // The copy out of device memory runs outside the lock (the server loop goes on meanwhile); no
        // other call can release the request while `reading` is set.
        r.reading = true;
        g.unlock();
        try {
            read_result(r, rgb, 0, bytes);
        } catch (...) {
            g.lock();
            r.reading = false;
            throw;
        }
        g.lock();
        r.reading = false;
    }
    int state = r.state;
    if (r.result) {
        PTW_CUDA(cudaFreeAsync(r.result, fin_stream_));
        bytes_in_use_ -= r.result_bytes;
    }
    r.result = nullptr;
    r.fetched = true;
    if (r.batch_refs == 0) requests_.erase(it);  // else the loop erases it after its last batch
    if (state == PT_REQ_CANCELLED) throw Error{PT_ERR_CANCELLED, "request cancelled"};
}

void Server::fetch_encoded(uint64_t id, int format, uint8_t* out, size_t capacity, size_t* length) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end() || it->second->fetched) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    Request& r = *it->second;
    if (r.state == PT_REQ_QUEUED || r.state == PT_REQ_RUNNING) throw Error{PT_ERR_INVALID, "request not finished"};
    if (r.state == PT_REQ_CANCELLED) throw Error{PT_ERR_CANCELLED, "request cancelled"};
    if (r.state == PT_REQ_FAILED) throw Error{PT_ERR_CUDA, "request failed: " + r.error};
    if (r.reading) throw Error{PT_ERR_INVALID, "fetch: another call is reading this request"};
    if (format == PT_IMAGE_PNG && !r.req.display) throw Error{PT_ERR_INVALID, "PNG: the request was not submitted with display = 1"};
    if (r.encoded_format != format) {
        // The copy out and the encoding (PNG: zlib) take milliseconds: they run outside the lock.
        // The request cannot go away meanwhile: fetches refuse a request that is being read.
        r.reading = true;
        const int w = r.req.width, h = r.req.height;
        const size_t npix = size_t(w) * size_t(h);
        lk.unlock();
        std::vector<uint8_t> enc;
        bool ok = true;
        try {
            if (format == PT_IMAGE_PFM) {
                std::vector<float> rgb(3 * npix);
                read_result(r, rgb.data(), 0, rgb.size() * sizeof(float));
                enc = encode_pfm(rgb.data(), w, h);
            } else {
                std::vector<uint32_t> rgba(npix);
                read_result(r, rgba.data(), 3 * npix * sizeof(float), npix * sizeof(uint32_t));
                ok = encode_png(rgba.data(), w, h, 6, enc);
            }
        } catch (const std::bad_alloc&) {
            ok = false;
        } catch (...) {
            lk.lock();
            r.reading = false;
            throw;
        }
        lk.lock();
        r.reading = false;
        if (!ok) throw Error{PT_ERR_ALLOC, "fetch: encoding failed"};
        r.encoded = std::move(enc);
        r.encoded_format = format;
    }
    *length = r.encoded.size();
    if (!out) return;  // a size query keeps the request
    if (capacity < r.encoded.size()) throw Error{PT_ERR_INVALID, "fetch: buffer too small"};
    std::memcpy(out, r.encoded.data(), r.encoded.size());
    if (r.result) {
        PTW_CUDA(cudaFreeAsync(r.result, fin_stream_));
        bytes_in_use_ -= r.result_bytes;
    }
    r.result = nullptr;
    r.encoded = std::vector<uint8_t>();
    r.fetched = true;
    if (r.batch_refs == 0) requests_.erase(it);  // else the loop erases it after its last batch
}

int32_t Server::open_session(int32_t scene_id, int w, int h, const pt_svgf_settings& sv) {
    if (w <= 0 || h <= 0 || uint64_t(w) * uint64_t(h) > (uint64_t(1) << 30))
        throw Error{PT_ERR_INVALID, "session: width and height must be positive, at most 2^30 pixels"};
    if (sv.atrous_iterations < 0 || sv.atrous_iterations > 30) throw Error{PT_ERR_INVALID, "session: atrous_iterations out of range"};
    const size_t npix = size_t(w) * size_t(h);
    // G-buffer (6), denoised image, and the denoiser's own eight buffers (with tile padding).
    const size_t estimate = 16 * npix * sizeof(float4) + (size_t(1) << 20);
    {
        std::lock_guard<std::mutex> g(mu_);
        if (scene_id < 0 || scene_id >= int(scenes_.size())) throw Error{PT_ERR_NOT_FOUND, "session: unknown scene"};
        if (cfg_.budget_bytes && bytes_in_use_ + estimate + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes)
            throw Error{PT_ERR_BUDGET, "session: does not fit the device-memory budget"};
    }
    auto s = std::make_unique<Session>();
    s->scene = scene_id;
    s->w = w;
    s->h = h;
    s->sv = sv;
    PTW_CUDA(cudaSetDevice(device_));
    for (DeviceBuffer<float4>* b : {&s->albedo, &s->normal_depth, &s->emission, &s->color, &s->edge, &s->motion, &s->denoised}) {
        b->allocate(npix);
        PTW_CUDA(cudaMemsetAsync(b->ptr, 0, npix * sizeof(float4), session_stream_));
    }
    s->svgf = std::make_unique<SvgfDenoiser>(device_, session_stream_);
    s->svgf->resize(w, h);
    s->bytes = 7 * npix * sizeof(float4) + s->svgf->device_bytes();
    // (The session lane's path pool, grown with the first frames, counts in the server's pool bytes.)
    std::lock_guard<std::mutex> g(mu_);
    if (cfg_.budget_bytes && bytes_in_use_ + s->bytes + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes)
        throw Error{PT_ERR_BUDGET, "session: does not fit the device-memory budget"};
    s->id = next_session_++;
    bytes_in_use_ += s->bytes;
    const int32_t id = s->id;
    sessions_[id] = std::move(s);
    return id;
}

// Called with the lock held.
void Server::free_session_if_closed(Session& s) {
    if (!s.closed || s.busy) return;
    bytes_in_use_ -= s.bytes;
    sessions_.erase(s.id);  // no frame of it is on the device: its buffers are idle
}

// Called with the lock held, once a session frame has left the device (finished, cancelled, failed).
void Server::session_frame_ended(Request& r) {
    if (!r.ses) return;
    Session* s = r.ses;
    r.ses = nullptr;
    s->busy = false;
    free_session_if_closed(*s);
    cv_frames_.notify_all();  // its next frame may go
}

void Server::close_session(int32_t session) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = sessions_.find(session);
    if (it == sessions_.end() || it->second->closed) throw Error{PT_ERR_NOT_FOUND, "unknown session"};
    Session& s = *it->second;
    s.closed = true;
    // Frames still waiting end cancelled; a frame on the device finishes first.
    for (auto q = frame_queue_.begin(); q != frame_queue_.end();) {
        Request& r = *requests_[*q];
        if (r.session != session) {
            ++q;
            continue;
        }
        r.state = PT_REQ_CANCELLED;
        r.done_s = now();
        st_.cancelled++;
        q = frame_queue_.erase(q);
    }
    cv_done_.notify_all();
    free_session_if_closed(s);
}

uint64_t Server::submit_frame(int32_t session, const pt_camera& cam, const pt_camera& prev, const pt_render_settings& rs) {
    if (rs.path.max_depth < 0 || rs.path.max_depth > 65535) throw Error{PT_ERR_INVALID, "frame: max_depth must be in [0, 65535]"};
    std::lock_guard<std::mutex> g(mu_);
    auto it = sessions_.find(session);
    if (it == sessions_.end() || it->second->closed) throw Error{PT_ERR_NOT_FOUND, "unknown session"};
    Session& s = *it->second;
    auto q = std::make_unique<Request>();
    q->id = next_id_++;
    q->req = pt_request{};
    q->req.scene_id = s.scene;
    q->req.camera = cam;
    q->req.width = s.w;
    q->req.height = s.h;
    q->req.spp = 1;
    q->req.seed = rs.seed;
    q->req.path = rs.path;
    q->session = session;
    q->prev = prev;
    q->frame = s.frames++;
    q->submit_s = now();
    q->bytes = request_bytes(q->req);
    q->work = uint64_t(s.w) * uint64_t(s.h);
    if (cfg_.budget_bytes && q->bytes + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes) {
        st_.rejected++;
        throw Error{PT_ERR_BUDGET, "frame: larger than the device-memory budget"};
    }
    const uint64_t id = q->id;
    requests_[id] = std::move(q);
    frame_queue_.push_back(id);
    st_.submitted++;
    cv_frames_.notify_all();
    return id;
}

// The session lane's thread: takes the oldest waiting frame of every session (a session's next frame
// waits for this one: its denoiser history), renders them together as one batched wavefront pass on
// the session stream (their paths share that lane's pool; the tail kernel finishes the last ones),
// then per frame sums its sample, denoises it with its session's history and resolves the image into
// a device result buffer.
void Server::session_loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    while (!stop_) {
        std::vector<Request*> frames;
        size_t need = 0;
        for (uint64_t id : frame_queue_) {
            Request& r = *requests_[id];
            bool taken = false;
            for (const Request* f : frames) taken = taken || f->session == r.session;
            auto it = sessions_.find(r.session);
            if (taken || it == sessions_.end()) continue;
            if (cfg_.budget_bytes && bytes_in_use_ + need + r.bytes + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes) break;
            r.ses = it->second.get();
            frames.push_back(&r);
            need += r.bytes;
        }
        if (frames.empty()) {
            if (sessions_.empty() && lane_bytes_ > 0) {
                // No session left: give the lane's path pool back (the next session's frames grow it again).
                session_engine_->release_paths();
                pool_bytes_ -= lane_bytes_;
                lane_bytes_ = 0;
            }
            cv_frames_.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        for (Request* r : frames) {
            frame_queue_.erase(std::find(frame_queue_.begin(), frame_queue_.end(), r->id));
            r->state = PT_REQ_RUNNING;
            r->admit_s = now();
            r->ses->busy = true;
        }
        bytes_in_use_ += need;
        std::vector<DevScene> table;
        for (const auto& s : scenes_) table.push_back(s->view());
        lk.unlock();

        std::string failure;
        try {
            std::vector<DevView> views(frames.size());
            uint64_t work = 0;
            int single = frames.front()->req.scene_id;
            for (size_t k = 0; k < frames.size(); k++) {
                Request& r = *frames[k];
                Session& ses = *r.ses;
                const size_t npix = size_t(r.req.width) * size_t(r.req.height);
                if (r.req.scene_id != single) single = -1;
                PTW_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.sample_out), npix * sizeof(float4), mem_pool_, session_stream_));
                PTW_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.accum), npix * sizeof(float4), mem_pool_, session_stream_));
                PTW_CUDA(cudaMemsetAsync(r.accum, 0, npix * sizeof(float4), session_stream_));
                // pt_render_denoised's frame: one path per pixel whose first vertex writes the G-buffer
                // and the denoiser's records; the sample index is the frame number.
                DevView& v = views[k];
                std::memset(&v, 0, sizeof(v));
                std::memcpy(v.cam, &r.req.camera, sizeof(v.cam));
                v.width = r.req.width;
                v.height = r.req.height;
                v.spp = 1;
                v.scene = r.req.scene_id;
                v.seed = r.req.seed;
                v.frame0 = r.frame;
                v.max_depth = r.req.path.max_depth;
                v.rr_depth = r.req.path.rr_depth;
                v.nee = r.req.path.nee;
                v.clamp = r.req.path.clamp;
                v.sample_out = r.sample_out;
                v.accum = r.accum;
                v.gbuffer = 1;
                v.realtime = 1;
                v.g_albedo = ses.albedo.ptr;
                v.g_normal_depth = ses.normal_depth.ptr;
                v.g_emission = ses.emission.ptr;
                v.g_color = ses.color.ptr;
                v.g_edge = ses.edge.ptr;
                v.g_motion = ses.motion.ptr;
                static_assert(sizeof(v.prev_cam) == sizeof(pt_camera), "camera layout");
                std::memcpy(v.prev_cam, &r.prev, sizeof(v.prev_cam));
                v.has_prev = 1;
                v.work_begin = work;
                v.work_count = npix;
                work += npix;
            }
            if (session_scenes_.count < table.size()) session_scenes_.allocate(std::max<size_t>(table.size(), 16));
            if (session_views_.count < views.size()) session_views_.allocate(std::max<size_t>(views.size(), 16));
            PTW_CUDA(cudaMemcpyAsync(session_scenes_.ptr, table.data(), table.size() * sizeof(DevScene), cudaMemcpyHostToDevice,
                                     session_stream_));
            PTW_CUDA(cudaMemcpyAsync(session_views_.ptr, views.data(), views.size() * sizeof(DevView), cudaMemcpyHostToDevice,
                                     session_stream_));
            session_engine_->run(session_scenes_.ptr, single, single >= 0 ? &table[size_t(single)] : nullptr, session_views_.ptr,
                                 int(views.size()), work);
            for (size_t k = 0; k < frames.size(); k++) {
                Request& r = *frames[k];
                Session& ses = *r.ses;
                const uint32_t npix = uint32_t(r.req.width) * uint32_t(r.req.height);
                PTW_CUDA(wf_accumulate(session_views_.ptr + k, views[k], 1, 1, session_stream_));  // writes the colour
                ses.svgf->run_frame(reinterpret_cast<const float*>(ses.color.ptr), reinterpret_cast<const float*>(ses.albedo.ptr),
                                    reinterpret_cast<const float*>(ses.emission.ptr), reinterpret_cast<const float*>(ses.edge.ptr),
                                    reinterpret_cast<const float*>(ses.motion.ptr), ses.sv, reinterpret_cast<float*>(ses.denoised.ptr));
                r.result_bytes = size_t(npix) * 3 * sizeof(float);
                PTW_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.result), r.result_bytes, mem_pool_, session_stream_));
                PTW_CUDA(wf_resolve(ses.denoised.ptr, npix, 1.0f, false, r.result, session_stream_));
                release_buffers(r, session_stream_);
            }
            PTW_CUDA(cudaStreamSynchronize(session_stream_));
        } catch (const Error& e) {
            failure = e.message;
            cudaStreamSynchronize(session_stream_);
            cudaGetLastError();
        }

        lk.lock();
        size_t lane = session_engine_->device_bytes() - lane_idle_bytes_;
        pool_bytes_ = pool_bytes_ - lane_bytes_ + lane;
        lane_bytes_ = lane;
        for (Request* r : frames) {
            bytes_in_use_ -= r->bytes;
            r->done_s = now();
            if (!failure.empty() || r->cancel) {
                release_buffers(*r, session_stream_);
                if (r->result) cudaFreeAsync(r->result, session_stream_);
                r->result = nullptr;
                r->state = failure.empty() ? PT_REQ_CANCELLED : PT_REQ_FAILED;
                r->error = failure;
                if (failure.empty()) st_.cancelled++;
            } else {
                r->state = PT_REQ_DONE;
                bytes_in_use_ += r->result_bytes;  // its result, until fetched
                st_.completed++;
                st_.samples_done += r->work;
            }
            session_frame_ended(*r);
        }
        cv_done_.notify_all();
    }
}

void Server::cancel(uint64_t id) {
    std::lock_guard<std::mutex> g(mu_);
    auto it = requests_.find(id);
    if (it == requests_.end() || it->second->fetched) throw Error{PT_ERR_NOT_FOUND, "unknown request"};
    Request& r = *it->second;
    if (r.state == PT_REQ_QUEUED) {
        queue_.erase(std::remove(queue_.begin(), queue_.end(), id), queue_.end());
        frame_queue_.erase(std::remove(frame_queue_.begin(), frame_queue_.end(), id), frame_queue_.end());
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

void Server::inject_finishing_failures(int n) { inject_finish_failures_.store(n); }

void Server::set_tuning(const pt_tuning& t) {
    std::lock_guard<std::mutex> g(mu_);
    Tuning cur = tuning_pending_ ? pending_tuning_ : engine_->tuning();
    if (t.sort_by_material >= 0) {
        if (t.sort_by_material > 4) throw Error{PT_ERR_INVALID, "sort_by_material must be in [0, 4]"};
        cur.sort_by_material = t.sort_by_material;
    }
    if (t.sort_rays >= 0) {
        if (t.sort_rays > created_sort_rays_) throw Error{PT_ERR_INVALID, "sort_rays above the server's configured sort_rays"};
        cur.sort_rays = t.sort_rays;
    }
    if (t.packed >= 0) cur.packed = t.packed ? 1 : 0;
    if (t.wide_shadows >= 0) cur.wide_shadows = t.wide_shadows ? 1 : 0;
    if (t.trace_refill > 32 || t.shadow_refill > 32) throw Error{PT_ERR_INVALID, "trace_refill and shadow_refill must be in [1, 32]"};
    if (t.walk_burst > (1 << 20)) throw Error{PT_ERR_INVALID, "walk_burst must be in [1, 2^20]"};
    if (t.trace_refill > 0) cur.trace_refill = t.trace_refill;
    if (t.shadow_refill > 0) cur.shadow_refill = t.shadow_refill;
    if (t.walk_burst > 0) cur.walk_burst = t.walk_burst;
    if (t.pair_walk > 64) throw Error{PT_ERR_INVALID, "pair_walk must be in [0, 64]"};
    if (t.pair_walk >= 0) cur.pair_walk = t.pair_walk;
    pending_tuning_ = cur;  // (the shadow-queue order is not taken: the server's wavefront has no buffers for it)
    tuning_pending_ = true;
    cv_work_.notify_all();
}

// Called with the lock held: drops the references of a completed batch's snapshot, erasing the
// requests that were fetched meanwhile.
void Server::release_batch_refs(const std::vector<Request*>& reqs) {
    for (Request* r : reqs) {
        if (--r->batch_refs == 0 && r->fetched) requests_.erase(r->id);
    }
}

void Server::upload_scene_table() {
    std::vector<DevScene> table;
    for (const auto& s : scenes_) table.push_back(s->view());
    PTW_CUDA(cudaMemcpyAsync(d_scenes_.ptr, table.data(), table.size() * sizeof(DevScene), cudaMemcpyHostToDevice, stream_));
    scenes_dirty_ = false;
}

void Server::release_buffers(Request& r, cudaStream_t s) {
    if (r.sample_out) cudaFreeAsync(r.sample_out, s);
    if (r.accum) cudaFreeAsync(r.accum, s);
    r.sample_out = r.accum = nullptr;
}

// Called with the lock held: allocates the request's buffers and its finished-path counter. Its work
// is handed to the wavefront later, chunk by chunk (append_chunks).
bool Server::try_admit(Request& r) {
    const int max_active = cfg_.max_active > 0 ? cfg_.max_active : (cfg_.max_active == 0 ? kDefaultMaxActive : 0);
    if (max_active > 0 && int(active_.size()) >= max_active) return false;
    if (cfg_.budget_bytes && bytes_in_use_ + r.bytes + pool_bytes_ + scene_bytes_ > cfg_.budget_bytes) return false;
    size_t npix = size_t(r.req.width) * size_t(r.req.height);
    try {
        if (inject_failures_ > 0) {
            inject_failures_--;
            throw Error{PT_ERR_ALLOC, "injected allocation failure"};
        }
        PTW_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.sample_out), npix * size_t(r.req.spp) * sizeof(float4), mem_pool_,
                                         stream_));
        PTW_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r.accum), npix * sizeof(float4), mem_pool_, stream_));
        PTW_CUDA(cudaMemsetAsync(r.accum, 0, npix * sizeof(float4), stream_));
    } catch (const Error& e) {
        cudaGetLastError();
        release_buffers(r, stream_);
        r.state = PT_REQ_FAILED;
        r.error = e.message;
        r.done_s = now();
        cv_done_.notify_all();
        return true;  // consumed (failed), not retried
    }
    // Grow the finished-path counters by doubling.
    if (size_t(done_slots_) + 1 > d_done_.count) {
        DeviceBuffer<unsigned long long> nd;
        nd.allocate(d_done_.count * 2);
        nd.zero(stream_);
        PTW_CUDA(cudaMemcpyAsync(nd.ptr, d_done_.ptr, d_done_.bytes(), cudaMemcpyDeviceToDevice, stream_));
        PTW_CUDA(cudaStreamSynchronize(stream_));
        d_done_ = std::move(nd);
        for (auto& kv : requests_) {
            Request& q = *kv.second;
            if (q.done_slot < 0) continue;
            q.tmpl.done_counter = d_done_.ptr + q.done_slot;
            for (int vi : q.views) views_[size_t(vi)].done_counter = q.tmpl.done_counter;
        }
        views_uploaded_ = 0;  // re-upload everything
    }
    r.done_slot = done_slots_++;
    DevView& v = r.tmpl;
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
    v.sample_out = r.sample_out;
    v.accum = r.accum;
    v.done_counter = d_done_.ptr + r.done_slot;
    bytes_in_use_ += r.bytes;
    r.state = PT_REQ_RUNNING;
    r.admit_s = now();
    active_.push_back(r.id);
    return true;
}

// Called with the lock held: hands chunks of the running requests' work to the wavefront, shortest
// remaining request first, until about one path pool's worth waits ahead of generation.
void Server::append_chunks() {
    const uint64_t generated = generated_;
    // Two batches run between a counter read and the next append: keep both supplied.
    const uint64_t target = (2 * uint64_t(iters_per_batch_) + 1) * uint64_t(engine_->tuning().path_capacity);
    while (work_total_ < generated + target) {
        Request* best = nullptr;
        for (uint64_t id : active_) {
            Request& r = *requests_[id];
            if (r.cancel || r.appended >= r.work) continue;
            if (!best || r.work - r.appended < best->work - best->appended) best = &r;
        }
        if (!best) break;
        const uint64_t n = std::min(best->work - best->appended, kChunkPaths);
        if (views_.size() + 1 > d_views_.count) {
            DeviceBuffer<DevView> nv;
            nv.allocate(d_views_.count * 2);
            d_views_ = std::move(nv);
            views_uploaded_ = 0;  // re-upload everything
        }
        DevView v = best->tmpl;
        v.work_begin = work_total_;
        v.work_count = n;
        v.local_base = best->appended;
        best->views.push_back(int(views_.size()));
        views_.push_back(v);
        best->appended += n;
        work_total_ += n;
    }
}

void Server::loop() {
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    double busy_since = -1;
    int cur = 0;
    while (!stop_) {
        std::vector<Request*> released;  // a read-back batch's snapshot, dropped under the lock
        std::vector<Request*> done;      // requests whose image has landed in host memory this turn
        try {
            // Admission in arrival order while the budget allows, then chunks of work.
            // Admission in arrival order while the budget and the limit on requests at once allow.
            while (!queue_.empty()) {
                Request& r = *requests_[queue_.front()];
                if (!try_admit(r)) break;
                queue_.pop_front();
            }
            append_chunks();
            if (scenes_dirty_) upload_scene_table();
            if (tuning_pending_ && engine_started_) {
                engine_->update_scheduling(pending_tuning_);
                tuning_pending_ = false;
            }
            Batch& B = batch_[cur];
            Batch& P = batch_[cur ^ 1];
            if (views_uploaded_ < views_.size()) {
                // New view-table entries go up through B's pinned staging (B's previous batch has
                // completed): a copy from pageable memory could hold this thread until the stream
                // drains, and the device would idle while the host turns around.
                const size_t n_new = views_.size() - views_uploaded_;
                if (n_new > B.views_cap) {
                    if (B.views) PTW_CUDA(cudaFreeHost(B.views));
                    B.views = nullptr;
                    B.views_cap = 0;
                    const size_t cap = std::max<size_t>(2 * n_new, 4096);
                    PTW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&B.views), cap * sizeof(DevView), cudaHostAllocDefault));
                    B.views_cap = cap;
                }
                std::memcpy(B.views, views_.data() + views_uploaded_, n_new * sizeof(DevView));
                PTW_CUDA(cudaMemcpyAsync(d_views_.ptr + views_uploaded_, B.views, n_new * sizeof(DevView), cudaMemcpyHostToDevice, stream_));
                views_uploaded_ = views_.size();
                if (!engine_started_) {
                    if (tuning_pending_) {  // set before the first request: the wavefront starts with it
                        engine_->set_tuning(pending_tuning_);
                        tuning_pending_ = false;
                    }
                    engine_->begin(d_scenes_.ptr, d_views_.ptr, int(views_.size()));
                    engine_started_ = true;
                }
                engine_->set_views(d_views_.ptr, int(views_.size()));
                *B.work_total = work_total_;  // B's previous batch has completed: its staging is free
                engine_->set_work_total_async(B.work_total);
            }
            // Cancelled running requests: no further chunks, and the paths of those handed over end at
            // their first vertex.
            for (uint64_t id : active_) {
                Request& r = *requests_[id];
                if (!r.cancel) continue;
                for (int vi : r.views) {
                    if (views_[size_t(vi)].max_depth == 0) continue;
                    views_[size_t(vi)].max_depth = 0;
                    PTW_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(d_views_.ptr + vi) + offsetof(DevView, max_depth),
                                             &views_[size_t(vi)].max_depth, sizeof(int), cudaMemcpyHostToDevice, stream_));
                    PTW_CUDA(cudaStreamSynchronize(stream_));
                }
            }
            const bool launch = !active_.empty();
            if (!launch && !P.in_flight && finishing_.empty()) {
                if (busy_since >= 0) {
                    st_.busy_seconds += now() - busy_since;
                    busy_since = -1;
                }
                cv_work_.wait_for(lk, std::chrono::milliseconds(20));
                continue;
            }
            if (busy_since < 0) busy_since = now();
            // Snapshot of this batch's requests and their counter range.
            B.reqs.clear();
            B.need.clear();
            size_t lo = size_t(done_slots_), hi = 0;
            for (uint64_t id : active_) {
                Request* r = requests_[id].get();
                r->batch_refs++;
                B.reqs.push_back(r);
                B.need.push_back(r->cancel ? r->appended : r->work);
                lo = std::min(lo, size_t(r->done_slot));
                hi = std::max(hi, size_t(r->done_slot) + 1);
            }
            if (hi < lo) hi = lo;
            B.lo = lo;
            B.n = hi - lo;
            if (B.n > B.done_cap) {
                if (B.done) PTW_CUDA(cudaFreeHost(B.done));
                B.done_cap = std::max<size_t>(B.n * 2, 1024);
                PTW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&B.done), B.done_cap * sizeof(unsigned long long), cudaHostAllocDefault));
            }
            const unsigned long long* d_done = d_done_.ptr;
            lk.unlock();

            // Launch this batch, then read the previous one's results while it runs.
            if (launch) {
                // Work not yet generated plus paths queued can only shrink between batches (apart from
                // new chunks, counted in work_total_), so if even this stale count fits the tail,
                // the next iteration finishes everything and the rest of a batch would be empty.
                const uint64_t pending = (work_total_ - generated_) + queued_;
                const uint32_t tail = engine_->tail_limit_in_use();
                B.iterations = (tail > 0 && pending <= tail) ? 1 : iters_per_batch_;
                engine_->set_continuous_sorting(pending >= kSortMinPaths);
                PTW_CUDA(cudaEventRecord(B.ev_start, stream_));
                engine_->launch(B.iterations);
                batches_++;
                PTW_CUDA(cudaMemcpyAsync(B.ctr, engine_->device_counters(), sizeof(Counters), cudaMemcpyDeviceToHost, stream_));
                if (B.n)
                    PTW_CUDA(cudaMemcpyAsync(B.done, d_done + B.lo, B.n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_));
                PTW_CUDA(cudaEventRecord(B.ev, stream_));
                B.in_flight = true;
            }
            std::vector<Request*> finished, cancelled;
            if (P.in_flight) {
                PTW_CUDA(cudaEventSynchronize(P.ev));
                P.in_flight = false;
                generated_ = P.ctr->work_next;
                queued_ = P.ctr->count[P.ctr->parity ^ 1u];
                iterations_ = P.ctr->iterations;
                // Aim for batches of about a millisecond of device time: long enough that the host's
                // turn between batches stays hidden, short enough that finished requests and new
                // arrivals are seen soon.
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, P.ev_start, P.ev) == cudaSuccess && ms > 0.0f) {
                    device_ms_ += ms;
                    double want = double(P.iterations) * (1.0 / double(ms));
                    iters_per_batch_ = std::max(1, std::min(16, int(want + 0.5)));
                }
                for (size_t k = 0; k < P.reqs.size(); k++) {
                    Request* r = P.reqs[k];
                    if (r->finishing || P.done[size_t(r->done_slot) - P.lo] < P.need[k]) continue;
                    r->finishing = true;  // the batch launched meanwhile also lists it: finish once
                    (r->cancel ? cancelled : finished).push_back(r);
                }
                // Sum each finished request's samples in order and resolve its image into a device
                // result buffer that fetch copies out, on the second stream after the batch that
                // finished it; release its sample buffers behind it. (Results stay on the device: an
                // allocation of pinned host memory here would stall this thread and idle the device.)
                for (Request* r : finished) {
                    const uint32_t npix = uint32_t(r->req.width) * uint32_t(r->req.height);
                    const int first = r->views.front();  // carries the whole image's spp and buffers
                    PTW_CUDA(cudaStreamWaitEvent(fin_stream_, P.ev, 0));
                    PTW_CUDA(wf_accumulate(d_views_.ptr + first, views_[size_t(first)], 1, 1, fin_stream_));
                    r->result_bytes = size_t(npix) * (3 * sizeof(float) + (r->req.display ? sizeof(uint32_t) : 0));
                    PTW_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&r->result), r->result_bytes, mem_pool_, fin_stream_));
                    float* rgb = r->result;
                    PTW_CUDA(wf_resolve(r->accum, npix, 1.0f / float(r->req.spp), true, rgb, fin_stream_));
                    if (r->req.display) {
                        // The colour view of pt_display on the summed samples, after the float image.
                        DisplayParams dp{};
                        dp.w = r->req.width;
                        dp.h = r->req.height;
                        dp.mode = PT_DISPLAY_COLOR;
                        dp.exposure = r->req.exposure;
                        dp.tonemap = r->req.tonemap;
                        dp.samples = float(r->req.spp);
                        dp.inv_samples = 1.0f / float(r->req.spp);
                        dp.max_depth = 1.0f;
                        dp.heat_scale = 1.0f / 160.0f;
                        uint32_t* rgba = reinterpret_cast<uint32_t*>(rgb + 3 * size_t(npix));
                        PTW_CUDA(wf_display(dp, r->accum, nullptr, nullptr, nullptr, nullptr, nullptr, rgba, fin_stream_));
                    }
                    release_buffers(*r, fin_stream_);
                    Finishing f{r, nullptr};
                    PTW_CUDA(cudaEventCreateWithFlags(&f.ev, cudaEventDisableTiming));
                    PTW_CUDA(cudaEventRecord(f.ev, fin_stream_));
                    finishing_.push_back(f);
                    if (inject_finish_failures_.load() > 0 && inject_finish_failures_.fetch_sub(1) > 0)
                        throw Error{PT_ERR_CUDA, "injected failure while finishing a request"};
                }
                for (Request* r : cancelled) release_buffers(*r, stream_);
                released = std::move(P.reqs);
                P.reqs.clear();
            }
            // Images whose copy has landed: normalise by the sample count. With nothing else to do,
            // wait for the oldest copy instead of polling.
            if (!launch && !finishing_.empty() && finished.empty()) PTW_CUDA(cudaEventSynchronize(finishing_.front().ev));
            for (size_t k = 0; k < finishing_.size();) {
                Finishing& f = finishing_[k];
                cudaError_t q = cudaEventQuery(f.ev);
                if (q == cudaErrorNotReady) {
                    k++;
                    continue;
                }
                PTW_CUDA(q);
                cudaEventDestroy(f.ev);
                done.push_back(f.r);
                finishing_.erase(finishing_.begin() + std::ptrdiff_t(k));
            }
            lk.lock();
            st_.bounce_iterations = iterations_;
            st_.device_seconds = device_ms_ / 1000.0;
            st_.batches = batches_;
            // A request leaves the active list once its image is being finished (the next batches no
            // longer carry it); its memory counts against the budget until the copy has landed.
            auto deactivate = [&](Request* r) { active_.erase(std::remove(active_.begin(), active_.end(), r->id), active_.end()); };
            for (Request* r : finished) deactivate(r);
            for (Request* r : cancelled) {
                deactivate(r);
                r->state = PT_REQ_CANCELLED;
                r->done_s = now();
                bytes_in_use_ -= r->bytes;
                st_.cancelled++;
            }
            for (Request* r : done) {
                r->state = PT_REQ_DONE;
                r->done_s = now();
                bytes_in_use_ -= r->bytes;
                bytes_in_use_ += r->result_bytes;  // its result, until fetched
                st_.completed++;
                st_.samples_done += r->work;
            }
            if (!done.empty() || !cancelled.empty()) cv_done_.notify_all();
            release_batch_refs(released);
            released.clear();
            cur ^= 1;
        } catch (const Error& e) {
            if (!lk.owns_lock()) lk.lock();
            release_batch_refs(released);
            cudaStreamSynchronize(stream_);
            cudaStreamSynchronize(fin_stream_);
            cudaGetLastError();
            for (Batch& b : batch_) {
                b.in_flight = false;
                release_batch_refs(b.reqs);
                b.reqs.clear();
            }
            // Each request is settled exactly once, whichever of the lists below hold it: a request
            // finished in this turn sits both in finishing_ and (until the lock is taken) in active_,
            // and one whose copy landed in this turn has already left finishing_ for `done`.
            for (Request* r : done) {
                if (r->state != PT_REQ_RUNNING) continue;
                r->state = PT_REQ_DONE;  // its image is complete
                r->done_s = now();
                bytes_in_use_ -= r->bytes;
                bytes_in_use_ += r->result_bytes;
                st_.completed++;
                st_.samples_done += r->work;
            }
            for (Finishing& f : finishing_) {
                cudaEventDestroy(f.ev);
                if (f.r->state != PT_REQ_RUNNING) continue;
                f.r->state = PT_REQ_FAILED;
                f.r->error = e.message;
                f.r->done_s = now();
                bytes_in_use_ -= f.r->bytes;
                if (f.r->result) cudaFreeAsync(f.r->result, fin_stream_);
                f.r->result = nullptr;
            }
            finishing_.clear();
            // A device failure fails every running request; the server keeps its handle valid.
            for (uint64_t id : active_) {
                Request& r = *requests_[id];
                if (r.state != PT_REQ_RUNNING) {  // settled above
                    release_buffers(r, stream_);
                    continue;
                }
                r.state = PT_REQ_FAILED;
                r.error = e.message;
                r.done_s = now();
                bytes_in_use_ -= r.bytes;
                release_buffers(r, stream_);
                if (r.result) cudaFreeAsync(r.result, fin_stream_);  // allocated before the failure
                r.result = nullptr;
            }
            active_.clear();
            cv_done_.notify_all();
        }
    }
}

}  // namespace ptw
