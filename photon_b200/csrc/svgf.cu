// SVGF (Schied et al. 2017) on the device, following Photon's src/denoise/svgf.cu:
// demodulation + temporal reprojection with moments, the variance estimate, and the a-trous passes
// with luminance / normal / depth edge-stopping. The history copy (svgf.cu:188-197) is fused into the
// epilogue of a-trous pass 0 and the remodulation (svgf.cu:199-210) into the last pass, so a frame is
// 2 + iterations launches instead of 4 + iterations. Arithmetic follows the reference's expression
// order with precise expf / powf (Photon builds its svgf.cu with --use_fast_math).
#include "svgf.h"

#include <cstring>
#include <mutex>

#include "pt_math.cuh"

namespace ptw {

namespace {

struct PrevCamera {
    float c[16];  // pt_camera
};

struct Frame5 {
    const float4 *color, *albedo, *nd, *pos, *emission;
};

__device__ __forceinline__ V3 demodulate(V3 color, V3 emission, V3 albedo) {
    V3 il = vmax(color - emission, v3(0));
    return {il.x / fmaxf(albedo.x, 1e-3f), il.y / fmaxf(albedo.y, 1e-3f), il.z / fmaxf(albedo.z, 1e-3f)};
}

// project (svgf.cu:25-35): a world position in the previous frame's pixel coordinates.
__device__ __forceinline__ bool project(const PrevCamera& pc, V3 p, int w, int h, float& px, float& py, float& dist) {
    const float* c = pc.c;
    V3 d = p - V3{c[0], c[1], c[2]};
    float z = dot(d, V3{c[4], c[5], c[6]});
    if (z <= 1e-4f) return false;
    float sx = dot(d, V3{c[8], c[9], c[10]}) / (z * c[3] * c[7]);
    float sy = dot(d, V3{c[12], c[13], c[14]}) / (z * c[3]);
    px = (sx + 1.0f) * 0.5f * float(w) - 0.5f;
    py = (1.0f - sy) * 0.5f * float(h) - 0.5f;
    dist = length(d);
    return true;
}

// temporal_kernel (svgf.cu:37-92).
__global__ void k_temporal(Frame5 in, PrevCamera prev, int w, int h, int has_history, float alpha_c, float alpha_m,
                           const float4* __restrict__ prev_illum, const float4* __restrict__ prev_moments, const float4* __restrict__ prev_nd,
                           const float4* __restrict__ prev_pos, float4* __restrict__ out_illum, float4* __restrict__ out_moments) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 pos = __ldg(in.pos + i);
    V3 cur = demodulate(xyz(__ldg(in.color + i)), xyz(__ldg(in.emission + i)), xyz(__ldg(in.albedo + i)));
    float lum = luminance(cur);
    V3 hist_c = v3(0);
    float hm0 = 0, hm1 = 0, hist_len = 0, wsum = 0;
    if (has_history && pos.w >= 0) {
        float px, py, dist;
        if (project(prev, xyz(pos), w, h, px, py, dist)) {
            V3 n = xyz(__ldg(in.nd + i));
            int x0 = int(floorf(px)), y0 = int(floorf(py));
            float fx = px - float(x0), fy = py - float(y0);
            for (int k = 0; k < 4; k++) {
                int xx = x0 + (k & 1), yy = y0 + (k >> 1);
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                int j = yy * w + xx;
                float4 pp = __ldg(prev_pos + j);
                float4 pn = __ldg(prev_nd + j);
                if (pp.w != pos.w) continue;
                if (fabsf(pn.w - dist) > 0.05f * dist + 0.01f) continue;
                if (dot(xyz(pn), n) < 0.9f) continue;
                float bw = ((k & 1) ? fx : 1 - fx) * ((k >> 1) ? fy : 1 - fy);
                float4 pi = __ldg(prev_illum + j);
                float4 pm = __ldg(prev_moments + j);
                hist_c = hist_c + xyz(pi) * bw;
                hm0 = hm0 + pm.x * bw;
                hm1 = hm1 + pm.y * bw;
                hist_len += pi.w * bw;
                wsum += bw;
            }
        }
    }
    V3 c;
    float m0, m1, len;
    if (wsum > 1e-3f) {
        hist_c = hist_c / wsum;
        float inv = 1.0f / wsum;
        hm0 = hm0 * inv;
        hm1 = hm1 * inv;
        len = fminf(hist_len / wsum + 1.0f, 64.0f);
        float ac = fmaxf(alpha_c, 1.0f / len), am = fmaxf(alpha_m, 1.0f / len);
        c = lerp(hist_c, cur, ac);
        m0 = lerpf(hm0, lum, am);
        m1 = lerpf(hm1, lum * lum, am);
    } else {
        len = 1.0f;
        c = cur;
        m0 = lum;
        m1 = lum * lum;
    }
    float variance = fmaxf(0.0f, m1 - m0 * m0);
    out_illum[i] = make_float4(c.x, c.y, c.z, len);
    out_moments[i] = make_float4(m0, m1, variance, 0.0f);
}

// variance_kernel (svgf.cu:96-132): from the moments, or a 7x7 bilateral estimate while the
// history is shorter than 4 frames.
__global__ void k_variance(Frame5 in, int w, int h, const float4* __restrict__ illum, const float4* __restrict__ moments,
                           float phi_normal, float4* __restrict__ out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 cc = __ldg(illum + i);
    V3 c = xyz(cc);
    float len = cc.w;
    float variance = __ldg(moments + i).z;
    float mat = __ldg(in.pos + i).w;
    if (len < 4.0f && mat >= 0) {
        float4 ndc = __ldg(in.nd + i);
        V3 n = xyz(ndc);
        float z = ndc.w;
        float wsum = 0, m1 = 0, m2 = 0;
        V3 acc = v3(0);
        for (int dy = -3; dy <= 3; dy++)
            for (int dx = -3; dx <= 3; dx++) {
                int xx = x + dx, yy = y + dy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                int j = yy * w + xx;
                if (__ldg(in.pos + j).w != mat) continue;
                float4 nd = __ldg(in.nd + j);
                float wn = powf(fmaxf(0.0f, dot(n, xyz(nd))), phi_normal);
                float wz = expf(-fabsf(nd.w - z) / (0.05f * z + 1e-3f));
                float wt = wn * wz;
                float4 m = __ldg(moments + j);
                m1 += m.x * wt;
                m2 += m.y * wt;
                acc = acc + xyz(__ldg(illum + j)) * wt;
                wsum += wt;
            }
        if (wsum > 0) {
            m1 /= wsum;
            m2 /= wsum;
            variance = fmaxf(0.0f, m2 - m1 * m1) * (4.0f / len);
            c = acc / wsum;
        }
    }
    out[i] = make_float4(c.x, c.y, c.z, variance);
}

struct AtrousEpilogue {
    // Pass 0: the history of the next frame (svgf.cu:188-197).
    float4 *prev_illum, *prev_moments, *prev_nd, *prev_pos;
    const float4 *illum, *moments;
    // Last pass: remodulation into the output (svgf.cu:199-210).
    float4* output;
};

// atrous_kernel (svgf.cu:134-186) with the fused epilogues.
__global__ void k_atrous(Frame5 in, int w, int h, int step, float phi_color, float phi_normal, float phi_depth,
                         const float4* __restrict__ src, float4* __restrict__ dst, AtrousEpilogue ep) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 center = __ldg(src + i);
    float mat = __ldg(in.pos + i).w;
    float4 result = center;
    if (mat >= 0) {
        float var = 0, vw = 0;
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                int xx = min(max(x + dx, 0), w - 1), yy = min(max(y + dy, 0), h - 1);
                float k = (dx == 0 && dy == 0) ? 0.25f : ((dx == 0 || dy == 0) ? 0.125f : 0.0625f);
                var += __ldg(src + yy * w + xx).w * k;
                vw += k;
            }
        var /= vw;
        float4 ndc = __ldg(in.nd + i);
        V3 n = xyz(ndc);
        float z = ndc.w;
        float zx = __ldg(in.nd + y * w + min(x + 1, w - 1)).w - __ldg(in.nd + y * w + max(x - 1, 0)).w;
        float zy = __ldg(in.nd + min(y + 1, h - 1) * w + x).w - __ldg(in.nd + max(y - 1, 0) * w + x).w;
        float grad = 0.5f * fmaxf(fabsf(zx), fabsf(zy));
        float lum_c = luminance(xyz(center));
        float sigma_l = phi_color * sqrtf(fmaxf(var, 0.0f)) + 1e-4f;
        const float kernel[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
        V3 sum = v3(0);
        float wsum = 0, vsum = 0;
        for (int dy = -2; dy <= 2; dy++)
            for (int dx = -2; dx <= 2; dx++) {
                int xx = x + dx * step, yy = y + dy * step;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                int j = yy * w + xx;
                if (__ldg(in.pos + j).w != mat) continue;
                float4 s = __ldg(src + j);
                float4 nd = __ldg(in.nd + j);
                float k = kernel[abs(dx)] * kernel[abs(dy)];
                float wl = expf(-fabsf(luminance(xyz(s)) - lum_c) / sigma_l);
                float wn = powf(fmaxf(0.0f, dot(n, xyz(nd))), phi_normal);
                float dist = sqrtf(float(dx * dx + dy * dy)) * float(step);
                float wz = expf(-fabsf(nd.w - z) / (phi_depth * grad * dist + 1e-3f * z + 1e-4f));
                float wt = k * wl * wn * wz;
                sum = sum + xyz(s) * wt;
                vsum += wt * wt * s.w;
                wsum += wt;
            }
        if (wsum > 0) {
            V3 r = sum / wsum;
            result = make_float4(r.x, r.y, r.z, vsum / (wsum * wsum));
        }
    }
    dst[i] = result;
    if (ep.prev_illum) {
        ep.prev_illum[i] = make_float4(result.x, result.y, result.z, __ldg(ep.illum + i).w);
        ep.prev_moments[i] = __ldg(ep.moments + i);
        ep.prev_nd[i] = __ldg(in.nd + i);
        ep.prev_pos[i] = __ldg(in.pos + i);
    }
    if (ep.output) {
        if (mat < 0) {
            ep.output[i] = __ldg(in.color + i);
        } else {
            V3 a = xyz(__ldg(in.albedo + i));
            V3 c = xyz(result) * vmax(a, v3(1e-3f)) + xyz(__ldg(in.emission + i));
            ep.output[i] = make_float4(c.x, c.y, c.z, 1.0f);
        }
    }
}

// History + remodulation without any a-trous pass (atrous_iterations == 0).
__global__ void k_history_remodulate(Frame5 in, int w, int h, const float4* __restrict__ filtered, AtrousEpilogue ep) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 f = __ldg(filtered + i);
    ep.prev_illum[i] = make_float4(f.x, f.y, f.z, __ldg(ep.illum + i).w);
    ep.prev_moments[i] = __ldg(ep.moments + i);
    ep.prev_nd[i] = __ldg(in.nd + i);
    ep.prev_pos[i] = __ldg(in.pos + i);
    if (__ldg(in.pos + i).w < 0) {
        ep.output[i] = __ldg(in.color + i);
    } else {
        V3 a = xyz(__ldg(in.albedo + i));
        V3 c = xyz(f) * vmax(a, v3(1e-3f)) + xyz(__ldg(in.emission + i));
        ep.output[i] = make_float4(c.x, c.y, c.z, 1.0f);
    }
}

// Remodulation alone (svgf.cu:199-210), for zero a-trous iterations without history.
__global__ void k_remodulate_only(Frame5 in, int w, int h, const float4* __restrict__ filtered, float4* __restrict__ out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    if (__ldg(in.pos + i).w < 0) {
        out[i] = __ldg(in.color + i);
        return;
    }
    V3 a = xyz(__ldg(in.albedo + i));
    V3 c = xyz(__ldg(filtered + i)) * vmax(a, v3(1e-3f)) + xyz(__ldg(in.emission + i));
    out[i] = make_float4(c.x, c.y, c.z, 1.0f);
}

}  // namespace

SvgfDenoiser::SvgfDenoiser(int device, cudaStream_t stream) : device_(device), stream_(stream) {}

size_t SvgfDenoiser::device_bytes() const {
    return prev_illum_.bytes() + prev_moments_.bytes() + prev_nd_.bytes() + prev_pos_.bytes() + illum_.bytes() + moments_.bytes() +
           filter_[0].bytes() + filter_[1].bytes();
}

void SvgfDenoiser::resize(int w, int h) {
    if (w == w_ && h == h_ && illum_.ptr) return;
    w_ = w;
    h_ = h;
    size_t n = size_t(w) * size_t(h);
    for (DeviceBuffer<float4>* b : {&prev_illum_, &prev_moments_, &prev_nd_, &prev_pos_, &illum_, &moments_, &filter_[0], &filter_[1]}) {
        b->allocate(n);
        b->zero(stream_);
    }
    PTW_CUDA(cudaStreamSynchronize(stream_));
    has_history_ = false;
}

void SvgfDenoiser::run(const float* color, const float* albedo, const float* nd, const float* pos, const float* emission,
                       const pt_camera& prev, const pt_svgf_settings& s, float* output) {
    if (w_ == 0 || h_ == 0) return;
    if (s.atrous_iterations < 0 || s.atrous_iterations > 30) throw Error{PT_ERR_INVALID, "atrous_iterations out of range"};
    Frame5 in{reinterpret_cast<const float4*>(color), reinterpret_cast<const float4*>(albedo), reinterpret_cast<const float4*>(nd),
              reinterpret_cast<const float4*>(pos), reinterpret_cast<const float4*>(emission)};
    PrevCamera pc;
    static_assert(sizeof(pt_camera) == sizeof(pc.c), "camera layout");
    std::memcpy(pc.c, &prev, sizeof(pc.c));
    dim3 block(32, 4), grid((w_ + 31) / 32, (h_ + 3) / 4);
    k_temporal<<<grid, block, 0, stream_>>>(in, pc, w_, h_, has_history_ ? 1 : 0, s.alpha_color, s.alpha_moments, prev_illum_.ptr,
                                             prev_moments_.ptr, prev_nd_.ptr, prev_pos_.ptr, illum_.ptr, moments_.ptr);
    k_variance<<<grid, block, 0, stream_>>>(in, w_, h_, illum_.ptr, moments_.ptr, s.phi_normal, filter_[0].ptr);
    AtrousEpilogue hist{prev_illum_.ptr, prev_moments_.ptr, prev_nd_.ptr, prev_pos_.ptr, illum_.ptr, moments_.ptr, nullptr};
    int src = 0;
    for (int it = 0; it < s.atrous_iterations; it++) {
        AtrousEpilogue ep{};
        if (it == 0) ep = hist;
        if (it == s.atrous_iterations - 1) ep.output = reinterpret_cast<float4*>(output);
        k_atrous<<<grid, block, 0, stream_>>>(in, w_, h_, 1 << it, s.phi_color, s.phi_normal, s.phi_depth, filter_[src].ptr,
                                              filter_[1 - src].ptr, ep);
        src = 1 - src;
    }
    if (s.atrous_iterations == 0) {
        hist.output = reinterpret_cast<float4*>(output);
        k_history_remodulate<<<grid, block, 0, stream_>>>(in, w_, h_, filter_[src].ptr, hist);
    }
    PTW_CUDA(cudaGetLastError());
    has_history_ = true;
}

// ---- the allocation-free single-frame denoise ------------------------------------------------------------
// For callers that cannot allocate device memory (pt_svgf_run_noalloc): a frame is denoised without
// history (the first frame of a session: demodulation, the spatial variance estimate, the a-trous
// passes, remodulation) by the same kernels as SvgfDenoiser::run, with their four intermediate
// buffers carved out of one file-scope device array instead of allocations.
namespace {

// illum, moments and the two a-trous buffers, kNoAllocMaxPixels float4 each: 32 MiB per device.
static __device__ __align__(256) float4 g_noalloc_scratch[4 * size_t(kNoAllocMaxPixels)];

std::mutex g_noalloc_mu;
float4* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// The device address of the scratch array on the current device (host code must not use the
// symbol's host-side name as a device pointer). Looked up once per device.
float4* noalloc_scratch(int device) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
        void* p = nullptr;
        PTW_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[device] = static_cast<float4*>(p);
    }
    return g_noalloc_ptr[device];
}

}  // namespace

void svgf_run_noalloc(int device, int w, int h, const float* color, const float* albedo, const float* nd, const float* pos,
                      const float* emission, const pt_svgf_settings& s, float* output, cudaStream_t stream) {
    if (w <= 0 || h <= 0) throw Error{PT_ERR_INVALID, "svgf_run_noalloc: width and height must be positive"};
    if (int64_t(w) * int64_t(h) > kNoAllocMaxPixels)
        throw Error{PT_ERR_INVALID, "svgf_run_noalloc: the frame has more than 524288 pixels (the size of the static scratch)"};
    if (s.atrous_iterations < 0 || s.atrous_iterations > 30) throw Error{PT_ERR_INVALID, "atrous_iterations out of range"};
    if (device < 0 || device >= kNoAllocMaxDevices) throw Error{PT_ERR_INVALID, "svgf_run_noalloc: device ordinal out of range"};
    int previous = 0;
    PTW_CUDA(cudaGetDevice(&previous));
    PTW_CUDA(cudaSetDevice(device));
    try {
        float4* base = noalloc_scratch(device);
        float4 *illum = base, *moments = base + kNoAllocMaxPixels, *f0 = base + 2 * size_t(kNoAllocMaxPixels),
               *f1 = base + 3 * size_t(kNoAllocMaxPixels);
        Frame5 in{reinterpret_cast<const float4*>(color), reinterpret_cast<const float4*>(albedo), reinterpret_cast<const float4*>(nd),
                  reinterpret_cast<const float4*>(pos), reinterpret_cast<const float4*>(emission)};
        PrevCamera pc{};  // unused without history
        dim3 block(32, 4), grid((w + 31) / 32, (h + 3) / 4);
        // Without history the temporal step reads nothing from earlier calls, and every scratch
        // element a kernel reads was written earlier in this call: nothing needs clearing.
        k_temporal<<<grid, block, 0, stream>>>(in, pc, w, h, 0, s.alpha_color, s.alpha_moments, nullptr, nullptr, nullptr, nullptr, illum,
                                               moments);
        k_variance<<<grid, block, 0, stream>>>(in, w, h, illum, moments, s.phi_normal, f0);
        float4* bufs[2] = {f0, f1};
        int src = 0;
        for (int it = 0; it < s.atrous_iterations; it++) {
            AtrousEpilogue ep{};
            if (it == s.atrous_iterations - 1) ep.output = reinterpret_cast<float4*>(output);
            k_atrous<<<grid, block, 0, stream>>>(in, w, h, 1 << it, s.phi_color, s.phi_normal, s.phi_depth, bufs[src], bufs[1 - src], ep);
            src = 1 - src;
        }
        if (s.atrous_iterations == 0) k_remodulate_only<<<grid, block, 0, stream>>>(in, w, h, bufs[src], reinterpret_cast<float4*>(output));
        PTW_CUDA(cudaGetLastError());
    } catch (...) {
        cudaSetDevice(previous);
        throw;
    }
    PTW_CUDA(cudaSetDevice(previous));
}

}  // namespace ptw
