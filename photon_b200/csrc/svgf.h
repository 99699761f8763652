// SVGF denoiser (host side): replaces photon::Svgf (src/denoise/svgf.h:32-59 of Photon).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

#include "device_scene.h"
#include "photon_wavefront.h"

namespace ptw {

// How one a-trous pass stages its taps: rank 0 = global loads, 2 = a contiguous TMA tile, 5 = a
// strided TMA tile (one residue class of x, y mod e); r = step / e grid cells between taps.
struct TmaPass {
    int rank, e, r;
};

class SvgfDenoiser {
public:
    SvgfDenoiser(int device, cudaStream_t stream);
    ~SvgfDenoiser();
    SvgfDenoiser(const SvgfDenoiser&) = delete;
    SvgfDenoiser& operator=(const SvgfDenoiser&) = delete;
    void resize(int w, int h);
    // How the a-trous passes stage their taps (pt_svgf_set_tma): 0 global loads; 1-3 TMA-staged
    // shared-memory tiles for some steps (see tma_passes_for_mode in svgf.cu).
    void set_tma(int mode);
    bool tma_active() const { return maps_ok_; }
    // Test hook: the TMA passes arm their tile barrier without issuing the copies and wait 2 us, so
    // their bounded wait runs out with no copy in flight; the next call reports PT_ERR_CUDA.
    void set_tma_timeout_test(bool on) { tma_test_ = on; }
    void reset() { has_history_ = false; }
    // Svgf::run (svgf.cu:238-255): inputs and output are device float4 buffers of width*height in
    // Photon's SvgfInput layout (colour, albedo, normal + depth, position + material, emission).
    void run(const float* color, const float* albedo, const float* normal_depth, const float* position, const float* emission,
             const pt_camera& prev, const pt_svgf_settings& s, float* output);
    // The same on the denoiser's own layout: colour, albedo, emission, edge records (octahedral normal
    // x, y, depth, int32 material id) and motion records (offset to the previous frame's pixel, distance
    // from the previous camera, valid flag), float4 each.
    void run_frame(const float* color, const float* albedo, const float* emission, const float* edge, const float* motion,
                   const pt_svgf_settings& s, float* output);
    // Svgf::variance_buffer (svgf.h:44).
    const float* variance() const { return reinterpret_cast<const float*>(filter_[0].ptr); }
    int width() const { return w_; }
    int height() const { return h_; }
    cudaStream_t stream() const { return stream_; }
    size_t device_bytes() const;

private:
    void check_status();
    void build_tma_plan();

    int device_;
    cudaStream_t stream_;
    int w_ = 0, h_ = 0;
    bool has_history_ = false;
    int tma_mode_ = 1;
    bool tma_test_ = false;
    bool maps_ok_ = false;
    std::vector<CUtensorMap> maps_;    // [edge, filter 0, filter 1][pass]
    TmaPass passes_[5];
    int* status_host_ = nullptr;       // set by a TMA pass whose tile load timed out (mapped host memory)
    int* status_dev_ = nullptr;
    DeviceBuffer<float4> prev_illum_, prev_moments_, prev_edge_, edge_, illum_, moments_, filter_[2];
};

// The allocation-free single-frame denoise (pt_svgf_run_noalloc): scratch in a static device array.
constexpr int kNoAllocMaxPixels = 1 << 19;  // 524,288 pixels (e.g. 960x540 or 1024x512)
constexpr int kNoAllocMaxDevices = 64;
void svgf_run_noalloc(int device, int w, int h, const float* color, const float* albedo, const float* normal_depth, const float* position,
                      const float* emission, const pt_svgf_settings& s, float* output, cudaStream_t stream);

}  // namespace ptw
