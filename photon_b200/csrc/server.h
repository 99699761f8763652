// The request server: resident scenes, continuous batching of render requests into one shared
// wavefront, admission by device-memory budget.
#pragma once

#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "photon_wavefront.h"
#include "renderer.h"

namespace ptw {

class Server {
public:
    explicit Server(const pt_server_config& cfg);
    ~Server();

    int32_t add_scene(const pt_scene_desc& d);
    uint64_t submit(const pt_request& r);
    int32_t poll(uint64_t id);
    void wait(uint64_t id, double timeout_s);
    void fetch(uint64_t id, float* rgb, size_t n, pt_request_stats* st);
    void cancel(uint64_t id);
    void stats(pt_server_stats* out);

    // Host-side fault injection for tests: the next `n` device allocations of request buffers fail.
    void inject_allocation_failures(int n);

private:
    struct Request {
        uint64_t id;
        pt_request req;
        int state = PT_REQ_QUEUED;
        double submit_s = 0, admit_s = 0, done_s = 0;
        uint64_t work = 0;
        size_t bytes = 0;
        int view = -1;          // index in the view table once admitted
        bool cancel = false;
        std::string error;
        DeviceBuffer<float4> sample_out, accum;
        std::vector<float> result;  // rgb, filled when done
    };

    void loop();
    double now() const;
    size_t request_bytes(const pt_request& r) const;
    bool try_admit(Request& r);
    void finish(Request& r);
    void upload_scene_table();

    pt_server_config cfg_;
    int device_;
    cudaStream_t stream_ = nullptr;
    std::unique_ptr<WavefrontEngine> engine_;

    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    bool stop_ = false;
    std::thread thread_;

    std::vector<std::unique_ptr<DeviceScene>> scenes_;
    bool scenes_dirty_ = false;
    DeviceBuffer<DevScene> d_scenes_;
    size_t scene_bytes_ = 0;

    std::map<uint64_t, std::unique_ptr<Request>> requests_;
    std::deque<uint64_t> queue_;
    std::vector<uint64_t> active_;
    uint64_t next_id_ = 1;

    // The view table grows by one entry per admitted request; work ranges are contiguous.
    std::vector<DevView> views_;
    DeviceBuffer<DevView> d_views_;
    DeviceBuffer<unsigned long long> d_done_;
    std::vector<unsigned long long> h_done_;
    size_t views_uploaded_ = 0;
    uint64_t work_total_ = 0;
    size_t bytes_in_use_ = 0;
    size_t pool_bytes_ = 0;
    bool engine_started_ = false;
    int inject_failures_ = 0;

    pt_server_stats st_{};
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace ptw
