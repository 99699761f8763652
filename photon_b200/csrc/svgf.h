// SVGF denoiser (host side): replaces photon::Svgf (src/denoise/svgf.h:32-59 of Photon).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.h"
#include "photon_wavefront.h"

namespace ptw {

class SvgfDenoiser {
public:
    SvgfDenoiser(int device, cudaStream_t stream);
    void resize(int w, int h);
    void reset() { has_history_ = false; }
    // Svgf::run (svgf.cu:238-255): inputs and output are device float4 buffers of width*height.
    void run(const float* color, const float* albedo, const float* normal_depth, const float* position, const float* emission,
             const pt_camera& prev, const pt_svgf_settings& s, float* output);
    // Svgf::variance_buffer (svgf.h:44).
    const float* variance() const { return reinterpret_cast<const float*>(filter_[0].ptr); }
    int width() const { return w_; }
    int height() const { return h_; }
    cudaStream_t stream() const { return stream_; }
    size_t device_bytes() const;

private:
    int device_;
    cudaStream_t stream_;
    int w_ = 0, h_ = 0;
    bool has_history_ = false;
    DeviceBuffer<float4> prev_illum_, prev_moments_, prev_nd_, prev_pos_, illum_, moments_, filter_[2];
};

// The allocation-free single-frame denoise (pt_svgf_run_noalloc): scratch in a static device array.
constexpr int kNoAllocMaxPixels = 1 << 19;  // 524,288 pixels (e.g. 960x540 or 1024x512)
constexpr int kNoAllocMaxDevices = 64;
void svgf_run_noalloc(int device, int w, int h, const float* color, const float* albedo, const float* normal_depth, const float* position,
                      const float* emission, const pt_svgf_settings& s, float* output, cudaStream_t stream);

}  // namespace ptw
