// The request server: resident scenes, continuous batching of render requests into one shared
// wavefront, admission by device-memory budget.
#pragma once

#include <atomic>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "photon_wavefront.h"
#include "renderer.h"
#include "svgf.h"

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
    void fetch_encoded(uint64_t id, int format, uint8_t* out, size_t capacity, size_t* length);
    void cancel(uint64_t id);
    void stats(pt_server_stats* out);

    // Host-side fault injection for tests: the next `n` device allocations of request buffers fail.
    void inject_allocation_failures(int n);
    // Host-side fault injection for tests: the next `n` finishing steps fail (an error thrown right
    // after a finished request has been queued for its read-back, as a failing CUDA call would).
    void inject_finishing_failures(int n);
    // A tuning record (pt_server_set_tuning): its scheduling knobs apply from the next batch.
    void set_tuning(const pt_tuning& t);

    // Real-time SVGF sessions served beside the requests (pt_server_open_session and friends).
    int32_t open_session(int32_t scene_id, int w, int h, const pt_svgf_settings& sv);
    void close_session(int32_t session);
    uint64_t submit_frame(int32_t session, const pt_camera& cam, const pt_camera& prev, const pt_render_settings& rs);

private:
    // A session: the G-buffer of its frames and its denoiser history, on the server's device. Its
    // frames are requests of one path per pixel whose first vertex writes the G-buffer and whose
    // finishing step denoises it; one frame is on the device at a time, in submission order.
    struct Session {
        int id = 0, scene = 0, w = 0, h = 0;
        pt_svgf_settings sv{};
        std::unique_ptr<SvgfDenoiser> svgf;  // on the session stream
        DeviceBuffer<float4> albedo, normal_depth, emission, color, edge, motion, denoised;
        uint32_t frames = 0;  // frames submitted: the next frame's sample index
        bool busy = false;    // a frame is admitted and not finished
        bool closed = false;
        size_t bytes = 0;
    };

    struct Request {
        uint64_t id;
        pt_request req;
        int state = PT_REQ_QUEUED;
        double submit_s = 0, admit_s = 0, done_s = 0;
        uint64_t work = 0;
        size_t bytes = 0;
        uint64_t appended = 0;  // paths handed to the wavefront so far
        std::vector<int> views; // its chunks in the view table (the first also serves the accumulation)
        int done_slot = -1;     // its finished-path counter
        DevView tmpl{};         // the view of the whole image; chunks differ in work range only
        std::atomic<bool> cancel{false};
        bool finishing = false;  // its image is being summed and copied out
        // Batches whose snapshot lists this request. A fetched request is erased only once none
        // does, since the loop reads a batch's requests after the batch completes, without the lock.
        int batch_refs = 0;
        bool fetched = false;
        std::string error;
        float4* sample_out = nullptr;  // stream-ordered allocations from the server's memory pool
        float4* accum = nullptr;
        int session = -1;         // a session frame: its session id, previous camera and sample index
        pt_camera prev{};
        uint32_t frame = 0;
        Session* ses = nullptr;   // set at admission (the session lives while a frame of it runs)
        float* result = nullptr;  // the finished image on the device (from the request pool): rgb floats,
                                  // and with req.display the RGBA8 display image after them; held until
                                  // fetched (counted against the budget meanwhile)
        size_t result_bytes = 0;
        std::vector<uint8_t> encoded;  // the image in encoded_format, kept by a size query
        int encoded_format = -1;
        bool reading = false;          // a fetch is copying its result out, outside the lock
    };

    void loop();
    void session_loop();
    double now() const;
    size_t request_bytes(const pt_request& r) const;
    bool try_admit(Request& r);
    void session_frame_ended(Request& r);  // with the lock held: the session may take its next frame
    void free_session_if_closed(Session& s);
    void append_chunks();
    void release_buffers(Request& r, cudaStream_t s);
    void read_result(const Request& r, void* dst, size_t offset, size_t bytes);  // device -> caller memory
    void upload_scene_table();
    void release_batch_refs(const std::vector<Request*>& reqs);

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
    std::map<int32_t, std::unique_ptr<Session>> sessions_;
    int32_t next_session_ = 1;
    // The session lane: session frames are rendered by a wavefront of their own on a stream of the
    // device's highest priority, driven by their own thread, so that a frame does not wait for the
    // request stream's bounce iterations (which hold the whole path pool at saturation).
    std::deque<uint64_t> frame_queue_;
    std::condition_variable cv_frames_;
    std::thread session_thread_;
    cudaStream_t session_stream_ = nullptr;
    std::unique_ptr<WavefrontEngine> session_engine_;
    DeviceBuffer<DevScene> session_scenes_;
    DeviceBuffer<DevView> session_views_;
    std::deque<uint64_t> queue_;
    std::vector<uint64_t> active_;
    uint64_t next_id_ = 1;

    // The view table grows by one entry per appended chunk; work ranges are contiguous.
    std::vector<DevView> views_;
    DeviceBuffer<DevView> d_views_;
    DeviceBuffer<unsigned long long> d_done_;   // one finished-path counter per admitted request
    std::vector<unsigned long long> h_done_;
    int done_slots_ = 0;
    cudaMemPool_t mem_pool_ = nullptr;
    // Pipelining: while the device runs one batch of bounce iterations, the host reads the counters
    // of the previous one (pinned copies, one staging set per batch) and finishes requests on a
    // second stream.
    struct Batch {
        Counters* ctr = nullptr;                 // pinned
        unsigned long long* done = nullptr;      // pinned, finished-path counters [lo, lo + n)
        size_t done_cap = 0, lo = 0, n = 0;
        unsigned long long* work_total = nullptr;  // pinned staging of the work total
        DevView* views = nullptr;                // pinned staging of the view-table entries it uploads
        size_t views_cap = 0;
        std::vector<Request*> reqs;              // active requests when the batch was launched
        std::vector<uint64_t> need;              // their paths to finish (all, or those handed over if cancelled)
        cudaEvent_t ev = nullptr, ev_start = nullptr;
        int iterations = 0;
        bool in_flight = false;
    };
    Batch batch_[2];
    struct Finishing {
        Request* r;
        cudaEvent_t ev;  // its image is complete in r->result
    };
    std::vector<Finishing> finishing_;
    int iters_per_batch_ = 2;  // adapted so that a batch keeps the device busy for about a millisecond
    cudaStream_t fin_stream_ = nullptr;
    uint64_t generated_ = 0;       // work items generated, as of the last completed batch
    uint64_t queued_ = 0;          // paths queued for the next iteration, as of the last completed batch
    uint64_t iterations_ = 0;
    double device_ms_ = 0;         // device time of completed batches
    uint64_t batches_ = 0;
    size_t views_uploaded_ = 0;
    uint64_t work_total_ = 0;
    size_t bytes_in_use_ = 0;
    size_t pool_bytes_ = 0;         // the request pool and, while sessions run, the session lane's (lane_bytes_)
    size_t lane_bytes_ = 0;         // the session lane's path pool and sort buffers
    size_t lane_idle_bytes_ = 0;    // the lane engine's own buffers (its counters), not counted
    bool engine_started_ = false;
    int inject_failures_ = 0;
    bool tuning_pending_ = false;  // under mu_: pending_tuning_ waits for the loop
    int created_sort_rays_ = 0;    // the ray-sort bits the wavefront's buffers are sized for
    Tuning pending_tuning_;
    std::atomic<int> inject_finish_failures_{0};  // read by the loop outside the lock

    pt_server_stats st_{};
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace ptw
