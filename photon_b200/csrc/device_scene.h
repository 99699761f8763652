// Device memory helpers and the device-resident scene (host side).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "photon_wavefront.h"
#include "pt_error.h"
#include "pt_types.h"

namespace ptw {

#define PTW_CUDA(x)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess)                                                                        \
            throw ::ptw::Error{PT_ERR_CUDA, std::string("CUDA error: ") + cudaGetErrorString(e_) + " (" #x ")"}; \
    } while (0)

// An owning device allocation (counts bytes against an optional budget).
template <typename T>
struct DeviceBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), count(o.count) {
        o.ptr = nullptr;
        o.count = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            count = o.count;
            o.ptr = nullptr;
            o.count = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    void allocate(size_t n) {
        if (n == count && ptr) return;
        release();
        if (n == 0) return;
        PTW_CUDA(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)));
        count = n;
    }
    // Grows (never shrinks) to at least n elements; returns true when the allocation changed.
    bool reserve(size_t n) {
        if (n <= count && ptr) return false;
        allocate(n);
        return true;
    }
    void upload(const T* src, size_t n, cudaStream_t s = 0) {
        allocate(n);
        if (n) PTW_CUDA(cudaMemcpyAsync(ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void zero(cudaStream_t s = 0) {
        if (ptr) PTW_CUDA(cudaMemsetAsync(ptr, 0, count * sizeof(T), s));
    }
    size_t bytes() const { return count * sizeof(T); }
};

// A scene copied to the device and re-laid for 128-bit loads (see DevScene in pt_scene.cuh).
class DeviceScene {
public:
    // Validates and uploads; throws Error. update_lights_only re-uploads the arrays that
    // GpuRenderer::update_lights touches (triangles, materials, light tables, environment).
    void upload(const pt_scene_desc& d, cudaStream_t stream, bool update_lights_only = false);
    const DevScene& view() const { return view_; }
    const DevScene* device_view() const { return d_view_.ptr; }
    bool ready() const { return ready_; }
    size_t device_bytes() const;
    float extent() const { return extent_; }
    // Bytes a scene will occupy on the device (for admission before upload).
    static size_t estimate_bytes(const pt_scene_desc& d);
    // pt_rebuild_lights: new materials, punctual lights and environment; the light tables are built
    // on the device (light_build.cu).
    void rebuild_lights(const pt_light_update& u, cudaStream_t stream);

private:
    DeviceBuffer<float4> nodes4_;
    DeviceBuffer<float4> nodes_, tris_, normals_, tangents_, materials_, alias_, punctual_, env_texels_;
    DeviceBuffer<int4> tri_idx_, textures_;
    DeviceBuffer<float2> uvs_;
    DeviceBuffer<uint32_t> texels_;
    DeviceBuffer<uint8_t> shade_keys_;
    DeviceBuffer<float> srgb_lut_, env_marginal_, env_conditional_, env_row_sin_;
    DeviceBuffer<int2> emissive_;
    DeviceBuffer<DevScene> d_view_;
    DevScene view_{};
    bool ready_ = false;
    float extent_ = 1.0f;
    int32_t num_vertices_ = 0;
    int32_t num_materials_ = 0;
    void upload_shade_keys(const pt_material* materials, int32_t n, cudaStream_t s);
    float bounds_[6] = {0, 0, 0, 0, 0, 0};  // the scene box (lo xyz, hi xyz), for the light-group weights
};

// Checks a scene description for internal consistency; throws Error(PT_ERR_INVALID).
void validate_scene(const pt_scene_desc& d, bool lights_only);

}  // namespace ptw
