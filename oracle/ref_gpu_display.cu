// Test infrastructure: Photon's display_kernel (src/render/gpu_renderer.cu:129-175) run on caller
// buffers, so that the wavefront's display kernel can be compared with it on one accumulation.
//
// display_kernel and its DisplayParams live in an unnamed namespace of gpu_renderer.cu, so they can
// only be launched from that translation unit. This file is that translation unit: it compiles
// Photon's gpu_renderer.cu unchanged, included from where it lies (oracle/Makefile builds it with
// Photon's own CUDA flags in place of gpu_renderer.cu's separate object, into
// oracle/_ref/libphoton_ref_gpu.so), and adds one launcher after it. Nothing of Photon's is modified.
#include "render/gpu_renderer.cu"

#include "photon_wavefront.h"

extern "C" {

// One display_kernel launch, with GpuRenderer::display's block shape and its inv_samples rule
// (gpu_renderer.cu:403-423), over host copies of the buffers (width * height float4 each; `heat`
// one float per pixel). Writes the packed RGBA8 pixels to `out` (host). Returns 1 on success.
int refgpu_display_buffers(int w, int h, int mode, float exposure, int tonemap, float samples, float max_depth, float heat_scale,
                           int denoised, const float* accum4, const float* denoised4, const float* albedo4, const float* normal_depth4,
                           const float* variance4, const float* heat, uint32_t* out) {
    using namespace photon;
    const size_t n = size_t(w) * size_t(h);
    if (n == 0) return 1;
    DeviceBuffer<vec4> d_acc, d_den, d_alb, d_nd, d_var;
    DeviceBuffer<float> d_heat;
    DeviceBuffer<uint32_t> d_out;
    try {
        d_acc.allocate(n);
        d_den.allocate(n);
        d_alb.allocate(n);
        d_nd.allocate(n);
        d_var.allocate(n);
        d_heat.allocate(n);
        d_out.allocate(n);
    } catch (const std::exception&) {
        return 0;
    }
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return src ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) : cudaMemset(dst, 0, bytes);
    };
    if (up(d_acc.ptr, accum4, n * 16) || up(d_den.ptr, denoised4, n * 16) || up(d_alb.ptr, albedo4, n * 16) ||
        up(d_nd.ptr, normal_depth4, n * 16) || up(d_var.ptr, variance4, n * 16) || up(d_heat.ptr, heat, n * 4))
        return 0;
    DisplayParams p;
    p.w = w;
    p.h = h;
    p.mode = DisplayMode(mode);
    p.exposure = exposure;
    p.tonemap = ToneMap(tonemap);
    p.samples = samples;
    p.inv_samples = samples > 0 ? 1.0f / samples : 0.0f;
    p.max_depth = max_depth;
    p.heat_scale = heat_scale;
    p.denoised = denoised != 0;
    dim3 block(kBlockX, kBlockY), grid((w + kBlockX - 1) / kBlockX, (h + kBlockY - 1) / kBlockY);
    display_kernel<<<grid, block>>>(p, d_acc.ptr, d_den.ptr, d_alb.ptr, d_nd.ptr, d_var.ptr, d_heat.ptr, d_out.ptr);
    if (cudaGetLastError() != cudaSuccess) return 0;
    if (cudaMemcpy(out, d_out.ptr, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    return 1;
}

}  // extern "C"
