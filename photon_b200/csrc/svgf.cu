// SVGF (Schied et al. 2017) on the device, following Photon's src/denoise/svgf.cu:
// demodulation + temporal reprojection with moments, the variance estimate, and the a-trous passes
// with luminance / normal / depth edge-stopping. The history copy (svgf.cu:188-197) is fused into the
// epilogue of a-trous pass 0 and the remodulation (svgf.cu:199-210) into the last pass, so a frame is
// 2 + iterations launches instead of 4 + iterations. Arithmetic follows the reference's expression
// order with precise expf / powf (Photon builds its svgf.cu with --use_fast_math).
#include "svgf.h"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "gbuffer.cuh"
#include "pt_math.cuh"

namespace ptw {

namespace {


// Photon's SvgfInput (svgf.h:24-30): five float4 per pixel.
struct Frame5 {
    const float4 *color, *albedo, *nd, *pos, *emission;
};

// The denoiser's own inputs. Per pixel, besides colour, albedo and emission (float4, rgb):
//   edge:   the octahedral-encoded normal (x, y), the depth, the material id (int32 bits; -1: no surface)
//   motion: offset to the pixel's position in the previous frame (dx, dy), its distance from the
//           previous camera, and 1 when it projects into the previous frame (else 0)
// The a-trous passes, the bulk of the work, read 32 bytes per tap (filtered colour + edge) instead of
// the 48 of Photon's layout.
struct SvgfFrame {
    const float4 *color, *albedo, *emission, *edge, *motion;
};

// The octahedral map's unnormalised direction; oct_decode normalises it (the fast reciprocal square
// root is accurate to a few ulp, far inside the filter's tolerances).
__device__ __forceinline__ V3 oct_direction(float ex, float ey) {
    V3 v{ex, ey, 1.0f - fabsf(ex) - fabsf(ey)};
    if (v.z < 0.0f) {
        float qx = (1.0f - fabsf(ey)) * sign_nz(ex), qy = (1.0f - fabsf(ex)) * sign_nz(ey);
        v.x = qx;
        v.y = qy;
    }
    return v;
}
__device__ __forceinline__ V3 oct_decode(float ex, float ey) {
    V3 v = oct_direction(ex, ey);
    return v * rsqrtf(dot(v, v));
}
// max(0, n . decode(e))^phi as exp(phi * log(.)), for the edge weights: pow(0, phi) = 0 for phi > 0
// and 1 for phi = 0, as powf.
__device__ __forceinline__ float log_normal_weight(V3 n, float ex, float ey, float phi) {
    V3 v = oct_direction(ex, ey);
    float c = fmaxf(0.0f, dot(n, v) * rsqrtf(dot(v, v)));
    return c > 0.0f ? phi * __logf(c) : (phi > 0.0f ? -kInf : 0.0f);
}
__device__ __forceinline__ int edge_material(float4 e) { return __float_as_int(e.w); }

__device__ __forceinline__ V3 demodulate(V3 color, V3 emission, V3 albedo) {
    V3 il = vmax(color - emission, v3(0));
    return {il.x / fmaxf(albedo.x, 1e-3f), il.y / fmaxf(albedo.y, 1e-3f), il.z / fmaxf(albedo.z, 1e-3f)};
}

struct History {
    const float4 *illum, *moments, *edge;  // the previous frame's
};

// temporal_kernel (svgf.cu:37-92). FromPhoton: the inputs are Photon's five buffers; the kernel
// derives this frame's edge records and the reprojection from the world position and the previous
// camera. Otherwise it reads the edge and motion records. Either way the edge records go to edge_out.
template <bool FromPhoton>
__global__ void __launch_bounds__(128) k_temporal(Frame5 in5, SvgfFrame in, PrevCamera prev, int w, int h, int has_history, float alpha_c,
                                                  float alpha_m, History hist, float4* __restrict__ edge_out, float4* __restrict__ out_illum,
                                                  float4* __restrict__ out_moments) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    V3 color, albedo, emission;
    float4 edge;
    bool reproject = false;
    float px = 0, py = 0, dist = 0;
    if (FromPhoton) {
        float4 nd = __ldg(in5.nd + i), pos = __ldg(in5.pos + i);
        edge = edge_record(xyz(nd), nd.w, int(pos.w));
        edge_out[i] = edge;
        color = xyz(__ldg(in5.color + i));
        albedo = xyz(__ldg(in5.albedo + i));
        emission = xyz(__ldg(in5.emission + i));
        reproject = has_history && pos.w >= 0 && project(prev, xyz(pos), w, h, px, py, dist);
    } else {
        edge = __ldg(in.edge + i);
        edge_out[i] = edge;  // the denoiser's own (padded) copy, which the a-trous tensor maps cover
        float4 m = __ldg(in.motion + i);
        color = xyz(__ldg(in.color + i));
        albedo = xyz(__ldg(in.albedo + i));
        emission = xyz(__ldg(in.emission + i));
        reproject = has_history && edge_material(edge) >= 0 && m.w != 0.0f;
        px = float(x) + m.x;
        py = float(y) + m.y;
        dist = m.z;
    }
    V3 cur = demodulate(color, emission, albedo);
    float lum = luminance(cur);
    V3 hist_c = v3(0);
    float hm0 = 0, hm1 = 0, hist_len = 0, wsum = 0;
    if (reproject) {
        V3 n = oct_decode(edge.x, edge.y);
        int mat = edge_material(edge);
        int x0 = int(floorf(px)), y0 = int(floorf(py));
        float fx = px - float(x0), fy = py - float(y0);
        for (int k = 0; k < 4; k++) {
            int xx = x0 + (k & 1), yy = y0 + (k >> 1);
            if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
            int j = yy * w + xx;
            float4 pe = __ldg(hist.edge + j);
            if (edge_material(pe) != mat) continue;
            if (fabsf(pe.z - dist) > 0.05f * dist + 0.01f) continue;
            if (dot(oct_decode(pe.x, pe.y), n) < 0.9f) continue;
            float bw = ((k & 1) ? fx : 1 - fx) * ((k >> 1) ? fy : 1 - fy);
            float4 pi = __ldg(hist.illum + j);
            float4 pm = __ldg(hist.moments + j);
            hist_c = hist_c + xyz(pi) * bw;
            hm0 = hm0 + pm.x * bw;
            hm1 = hm1 + pm.y * bw;
            hist_len += pi.w * bw;
            wsum += bw;
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
// history is shorter than 4 frames. The edge-stopping weights use the fast exp / pow that Photon's
// build (--use_fast_math) gives svgf.cu.
__global__ void __launch_bounds__(128) k_variance(const float4* __restrict__ edge, int w, int h, const float4* __restrict__ illum,
                                                  const float4* __restrict__ moments, float phi_normal, float4* __restrict__ out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 cc = __ldg(illum + i);
    V3 c = xyz(cc);
    float len = cc.w;
    float variance = __ldg(moments + i).z;
    float4 e = __ldg(edge + i);
    int mat = edge_material(e);
    if (len < 4.0f && mat >= 0) {
        V3 n = oct_decode(e.x, e.y);
        float z = e.z;
        float inv_dz = __fdividef(1.0f, 0.05f * z + 1e-3f);
        float wsum = 0, m1 = 0, m2 = 0;
        V3 acc = v3(0);
        for (int dy = -3; dy <= 3; dy++)
            for (int dx = -3; dx <= 3; dx++) {
                int xx = x + dx, yy = y + dy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                int j = yy * w + xx;
                float4 ej = __ldg(edge + j);
                if (edge_material(ej) != mat) continue;
                float wt = __expf(log_normal_weight(n, ej.x, ej.y, phi_normal) - fabsf(ej.z - z) * inv_dz);
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
    float4 *prev_illum, *prev_moments, *prev_edge;
    const float4 *illum, *moments;
    // Last pass: remodulation into the output (svgf.cu:199-210).
    float4* output;
    const float4 *color, *albedo, *emission;
};

__device__ __forceinline__ float4 remodulate(const AtrousEpilogue& ep, int i, int mat, float4 filtered) {
    if (mat < 0) return __ldg(ep.color + i);
    V3 a = xyz(__ldg(ep.albedo + i));
    V3 c = xyz(filtered) * vmax(a, v3(1e-3f)) + xyz(__ldg(ep.emission + i));
    return make_float4(c.x, c.y, c.z, 1.0f);
}

// atrous_kernel (svgf.cu:134-186) with the fused epilogues. The three edge-stopping weights of a tap
// (luminance, normal, depth) are multiplied as one exponential of the summed log-weights, with fast
// exp / log / reciprocal as in Photon's build of svgf.cu (--use_fast_math).
__global__ void __launch_bounds__(128) k_atrous(const float4* __restrict__ edge, int w, int h, int step, float phi_color, float phi_normal,
                                                float phi_depth, const float4* __restrict__ src, float4* __restrict__ dst, AtrousEpilogue ep) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 center = __ldg(src + i);
    float4 e = __ldg(edge + i);
    int mat = edge_material(e);
    float4 result = center;
    if (mat >= 0) {
        float var = 0, vw = 0;
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                int xx = min(max(x + dx, 0), w - 1), yy = min(max(y + dy, 0), h - 1);
                float k = (dx == 0 && dy == 0) ? 0.25f : ((dx == 0 || dy == 0) ? 0.125f : 0.0625f);
                var += __ldg(src + yy * w + xx).w * k;
                vw += k;
            }
        var /= vw;
        V3 n = oct_decode(e.x, e.y);
        float z = e.z;
        float zx = __ldg(edge + y * w + min(x + 1, w - 1)).z - __ldg(edge + y * w + max(x - 1, 0)).z;
        float zy = __ldg(edge + min(y + 1, h - 1) * w + x).z - __ldg(edge + max(y - 1, 0) * w + x).z;
        float grad = 0.5f * fmaxf(fabsf(zx), fabsf(zy));
        float lum_c = luminance(xyz(center));
        float sigma_l = phi_color * sqrtf(fmaxf(var, 0.0f)) + 1e-4f;
        float inv_sigma = __fdividef(1.0f, sigma_l);
        // The depth term's denominator depends on the tap only through its distance, one of
        // 0, 1, sqrt 2, 2, sqrt 5, sqrt 8 (x step) in the 5x5 footprint.
        const float gs = phi_depth * grad * float(step), dz0 = 1e-3f * z + 1e-4f;
        const float inv_dz[6] = {__fdividef(1.0f, dz0), __fdividef(1.0f, gs + dz0), __fdividef(1.0f, gs * 1.41421356f + dz0),
                                 __fdividef(1.0f, gs * 2.0f + dz0), __fdividef(1.0f, gs * 2.23606798f + dz0),
                                 __fdividef(1.0f, gs * 2.82842712f + dz0)};
        const float kernel[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
        V3 sum = v3(0);
        float wsum = 0, vsum = 0;
#pragma unroll
        for (int dy = -2; dy <= 2; dy++)
#pragma unroll
            for (int dx = -2; dx <= 2; dx++) {
                int xx = x + dx * step, yy = y + dy * step;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                int j = yy * w + xx;
                float4 ej = __ldg(edge + j);
                if (edge_material(ej) != mat) continue;
                float4 s = __ldg(src + j);
                const int r2 = dx * dx + dy * dy;
                const int di = r2 == 0 ? 0 : r2 == 1 ? 1 : r2 == 2 ? 2 : r2 == 4 ? 3 : r2 == 5 ? 4 : 5;
                float k = kernel[abs(dx)] * kernel[abs(dy)];
                // wl * wn * wz of svgf.cu:168-175 as one exponential.
                float arg = log_normal_weight(n, ej.x, ej.y, phi_normal) - fabsf(luminance(xyz(s)) - lum_c) * inv_sigma -
                            fabsf(ej.z - z) * inv_dz[di];
                float wt = k * __expf(arg);
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
        ep.prev_edge[i] = e;
    }
    if (ep.output) ep.output[i] = remodulate(ep, i, mat, result);
}

// ---- a-trous passes with TMA-staged tiles ------------------------------------------------------------------
// A pass with step s reads, for each pixel, the 5 x 5 taps at offsets (dx, dy) * s. A block takes a
// 16 x 16 tile of pixels on a grid of spacing e (e = 1: a contiguous tile) whose taps lie r = s / e
// grid cells apart, so all of them fall in a (16 + 4r)^2 box of the same grid. The Tensor Memory
// Accelerator copies that box of both inputs (filtered colour, edge records) into shared memory, one
// tiled load each, and every tap reads shared memory instead of L1/L2.
//   Contiguous tiles (e = 1, r = s) use a 2-D tensor map (floats of a row, rows).
//   Strided tiles (e = 8, one residue class (x mod 8, y mod 8) per block) use a 5-D view of the buffer
//   (float lane, x mod e, x / e, y mod e, y / e) whose box is lanes 4, 1, 16 + 4r, 1, 16 + 4r.
constexpr int kTmaTile = 16;
constexpr int kTmaPasses = 5;   // steps 1, 2, 4, 8, 16 may be staged
constexpr unsigned long long kTmaWaitNs = 200000000ull;    // 0.2 s: far beyond any tile load
constexpr unsigned long long kTmaDrainNs = 2000000000ull;  // after a timeout: the copies' last chance to land
constexpr unsigned long long kTmaTestWaitNs = 2000ull;     // the test mode's waits (no copy is issued)

__host__ __device__ constexpr int tma_box_side(int r) { return kTmaTile + 4 * r; }
size_t tma_smem_bytes(int r) { return 2 * size_t(tma_box_side(r)) * size_t(tma_box_side(r)) * sizeof(float4) + 16; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase 0 of the tile barrier for at most `limit_ns`.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned long long limit_ns) {
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, 0))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

template <int Rank>
__global__ void __launch_bounds__(kTmaTile * kTmaTile) k_atrous_tma(const __grid_constant__ CUtensorMap map_src,
                                                                    const __grid_constant__ CUtensorMap map_edge,
                                                                    const float4* __restrict__ src, const float4* __restrict__ edge,
                                                                    int w, int h, int e, int r, float phi_color, float phi_normal,
                                                                    float phi_depth, float4* __restrict__ dst, AtrousEpilogue ep,
                                                                    int* status, int test_no_copy) {
    extern __shared__ __align__(128) float4 tile_smem[];
    const int n = tma_box_side(r);  // box side in grid cells
    float4* t_src = tile_smem;
    float4* t_edge = tile_smem + n * n;
    uint64_t* bar = reinterpret_cast<uint64_t*>(tile_smem + 2 * n * n);
    const int rx = int(blockIdx.z) % e, ry = int(blockIdx.z) / e;
    const int cx0 = int(blockIdx.x) * kTmaTile, cy0 = int(blockIdx.y) * kTmaTile;
    const bool leader = threadIdx.x == 0 && threadIdx.y == 0;
    if (leader) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    // Test mode (test_no_copy): the barrier is armed for the tiles but no copy is issued, so the wait
    // below runs out with nothing in flight and the timeout path is exercised without any risk.
    if (leader) {
        const uint32_t bytes = uint32_t(2 * n * n * sizeof(float4));
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    }
    if (leader && !test_no_copy) {
        const int bx = cx0 - 2 * r, by = cy0 - 2 * r;
        if (Rank == 2) {
            // Innermost coordinate in floats: 4 * bx, a multiple of 4 floats = 16 bytes.
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                    smem_u32(t_src)),
                "l"(&map_src), "r"(4 * bx), "r"(by), "r"(smem_u32(bar))
                : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
                    smem_u32(t_edge)),
                "l"(&map_edge), "r"(4 * bx), "r"(by), "r"(smem_u32(bar))
                : "memory");
        } else {
            asm volatile(
                "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(
                    smem_u32(t_src)),
                "l"(&map_src), "r"(0), "r"(rx), "r"(bx), "r"(ry), "r"(by), "r"(smem_u32(bar))
                : "memory");
            asm volatile(
                "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(
                    smem_u32(t_edge)),
                "l"(&map_edge), "r"(0), "r"(rx), "r"(bx), "r"(ry), "r"(by), "r"(smem_u32(bar))
                : "memory");
        }
    }
    if (!mbar_wait_bounded(bar, test_no_copy ? kTmaTestWaitNs : kTmaWaitNs)) {
        // The tiles did not land in time: report it (the host then fails the call and discards the
        // frame) and wait once more, ten times longer, for the copies in flight, so that the block
        // does not leave while they may still write its shared memory. Copies of valid coordinates
        // into this block's own tile complete unless the device itself has failed; only then can the
        // second wait also run out, and the block leaves so that the kernel ends.
        if (leader) atomicOr(status, 1);
        mbar_wait_bounded(bar, test_no_copy ? kTmaTestWaitNs : kTmaDrainNs);
        return;
    }
    const int tx = int(threadIdx.x), ty = int(threadIdx.y);
    const int x = rx + e * (cx0 + tx), y = ry + e * (cy0 + ty);
    if (x >= w || y >= h) return;
    const int i = y * w + x, step = e * r;
    const int ci = (ty + 2 * r) * n + (tx + 2 * r);
    float4 center = t_src[ci];
    float4 ec = t_edge[ci];
    int mat = edge_material(ec);
    float4 result = center;
    if (mat >= 0) {
        float var = 0, vw = 0;
#pragma unroll
        for (int dy = -1; dy <= 1; dy++)
#pragma unroll
            for (int dx = -1; dx <= 1; dx++) {
                int xx = min(max(x + dx, 0), w - 1), yy = min(max(y + dy, 0), h - 1);
                float k = (dx == 0 && dy == 0) ? 0.25f : ((dx == 0 || dy == 0) ? 0.125f : 0.0625f);
                var += __ldg(src + yy * w + xx).w * k;
                vw += k;
            }
        var /= vw;
        V3 nrm = oct_decode(ec.x, ec.y);
        float z = ec.z;
        float zx = __ldg(edge + y * w + min(x + 1, w - 1)).z - __ldg(edge + y * w + max(x - 1, 0)).z;
        float zy = __ldg(edge + min(y + 1, h - 1) * w + x).z - __ldg(edge + max(y - 1, 0) * w + x).z;
        float grad = 0.5f * fmaxf(fabsf(zx), fabsf(zy));
        float lum_c = luminance(xyz(center));
        float sigma_l = phi_color * sqrtf(fmaxf(var, 0.0f)) + 1e-4f;
        float inv_sigma = __fdividef(1.0f, sigma_l);
        const float gs = phi_depth * grad * float(step), dz0 = 1e-3f * z + 1e-4f;
        const float inv_dz[6] = {__fdividef(1.0f, dz0), __fdividef(1.0f, gs + dz0), __fdividef(1.0f, gs * 1.41421356f + dz0),
                                 __fdividef(1.0f, gs * 2.0f + dz0), __fdividef(1.0f, gs * 2.23606798f + dz0),
                                 __fdividef(1.0f, gs * 2.82842712f + dz0)};
        const float kernel[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
        V3 sum = v3(0);
        float wsum = 0, vsum = 0;
#pragma unroll
        for (int dy = -2; dy <= 2; dy++)
#pragma unroll
            for (int dx = -2; dx <= 2; dx++) {
                int xx = x + dx * step, yy = y + dy * step;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                int tj = ci + dy * r * n + dx * r;
                float4 ej = t_edge[tj];
                if (edge_material(ej) != mat) continue;
                float4 sj = t_src[tj];
                const int r2 = dx * dx + dy * dy;
                const int di = r2 == 0 ? 0 : r2 == 1 ? 1 : r2 == 2 ? 2 : r2 == 4 ? 3 : r2 == 5 ? 4 : 5;
                float k = kernel[abs(dx)] * kernel[abs(dy)];
                float arg = log_normal_weight(nrm, ej.x, ej.y, phi_normal) - fabsf(luminance(xyz(sj)) - lum_c) * inv_sigma -
                            fabsf(ej.z - z) * inv_dz[di];
                float wt = k * __expf(arg);
                sum = sum + xyz(sj) * wt;
                vsum += wt * wt * sj.w;
                wsum += wt;
            }
        if (wsum > 0) {
            V3 rr = sum / wsum;
            result = make_float4(rr.x, rr.y, rr.z, vsum / (wsum * wsum));
        }
    }
    dst[i] = result;
    if (ep.prev_illum) {
        ep.prev_illum[i] = make_float4(result.x, result.y, result.z, __ldg(ep.illum + i).w);
        ep.prev_moments[i] = __ldg(ep.moments + i);
        ep.prev_edge[i] = ec;
    }
    if (ep.output) ep.output[i] = remodulate(ep, i, mat, result);
}

// History and/or remodulation without any a-trous pass (atrous_iterations == 0).
__global__ void __launch_bounds__(128) k_history_remodulate(const float4* __restrict__ edge, int w, int h,
                                                            const float4* __restrict__ filtered, AtrousEpilogue ep) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    int i = y * w + x;
    float4 f = __ldg(filtered + i);
    float4 e = __ldg(edge + i);
    if (ep.prev_illum) {
        ep.prev_illum[i] = make_float4(f.x, f.y, f.z, __ldg(ep.illum + i).w);
        ep.prev_moments[i] = __ldg(ep.moments + i);
        ep.prev_edge[i] = e;
    }
    ep.output[i] = remodulate(ep, i, edge_material(e), f);
}

// One frame: temporal, variance, a-trous passes with the fused epilogues. `hist_out` is the
// history epilogue (null members: none); scratch: illum, moments and the two a-trous buffers.
// Tensor maps of the TMA passes: [buffer: edge, f0, f1][pass 0..kTmaPasses-1], or none.
struct TmaPlan {
    const CUtensorMap* maps;
    const TmaPass* passes;  // [kTmaPasses]
    int* status;
    int test_no_copy;       // the timeout test mode (SvgfDenoiser::set_tma_timeout_test)
};

template <bool FromPhoton>
void denoise(const Frame5& in5, const SvgfFrame& in, const PrevCamera& pc, int w, int h, bool has_history, const History& hist,
             float4* edge_out, const AtrousEpilogue& hist_out, float4* illum, float4* moments, float4* f0, float4* f1,
             const pt_svgf_settings& s, float* output, const TmaPlan& tma, cudaStream_t stream) {
    dim3 block(32, 4), grid((w + 31) / 32, (h + 3) / 4);
    const float4* edge = edge_out;
    k_temporal<FromPhoton><<<grid, block, 0, stream>>>(in5, in, pc, w, h, has_history ? 1 : 0, s.alpha_color, s.alpha_moments, hist,
                                                       edge_out, illum, moments);
    k_variance<<<grid, block, 0, stream>>>(edge, w, h, illum, moments, s.phi_normal, f0);
    AtrousEpilogue last{};
    last.output = reinterpret_cast<float4*>(output);
    last.color = FromPhoton ? in5.color : in.color;
    last.albedo = FromPhoton ? in5.albedo : in.albedo;
    last.emission = FromPhoton ? in5.emission : in.emission;
    float4* bufs[2] = {f0, f1};
    int src = 0;
    for (int it = 0; it < s.atrous_iterations; it++) {
        AtrousEpilogue ep{};
        if (it == 0) ep = hist_out;
        if (it == s.atrous_iterations - 1) {
            ep.output = last.output;
            ep.color = last.color;
            ep.albedo = last.albedo;
            ep.emission = last.emission;
        }
        if (tma.maps && it < kTmaPasses && tma.passes[it].rank != 0) {
            const TmaPass& tp = tma.passes[it];
            const int gx = (w + tp.e - 1) / tp.e, gy = (h + tp.e - 1) / tp.e;
            dim3 tgrid((gx + kTmaTile - 1) / kTmaTile, (gy + kTmaTile - 1) / kTmaTile, tp.e * tp.e);
            const CUtensorMap& ms = tma.maps[(1 + src) * kTmaPasses + it];
            const CUtensorMap& me = tma.maps[it];
            if (tp.rank == 2)
                k_atrous_tma<2><<<tgrid, dim3(kTmaTile, kTmaTile), tma_smem_bytes(tp.r), stream>>>(
                    ms, me, bufs[src], edge, w, h, tp.e, tp.r, s.phi_color, s.phi_normal, s.phi_depth, bufs[1 - src], ep, tma.status,
                    tma.test_no_copy);
            else
                k_atrous_tma<5><<<tgrid, dim3(kTmaTile, kTmaTile), tma_smem_bytes(tp.r), stream>>>(
                    ms, me, bufs[src], edge, w, h, tp.e, tp.r, s.phi_color, s.phi_normal, s.phi_depth, bufs[1 - src], ep, tma.status,
                    tma.test_no_copy);
        } else {
            k_atrous<<<grid, block, 0, stream>>>(edge, w, h, 1 << it, s.phi_color, s.phi_normal, s.phi_depth, bufs[src], bufs[1 - src],
                                                 ep);
        }
        src = 1 - src;
    }
    if (s.atrous_iterations == 0) {
        AtrousEpilogue ep = hist_out;
        ep.output = last.output;
        ep.color = last.color;
        ep.albedo = last.albedo;
        ep.emission = last.emission;
        k_history_remodulate<<<grid, block, 0, stream>>>(edge, w, h, bufs[src], ep);
    }
    PTW_CUDA(cudaGetLastError());
}

}  // namespace

SvgfDenoiser::SvgfDenoiser(int device, cudaStream_t stream) : device_(device), stream_(stream) {
    PTW_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&status_host_), sizeof(int), cudaHostAllocMapped));
    *status_host_ = 0;
    PTW_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&status_dev_), status_host_, 0));
}

SvgfDenoiser::~SvgfDenoiser() {
    if (status_host_) cudaFreeHost(status_host_);
}

size_t SvgfDenoiser::device_bytes() const {
    return prev_illum_.bytes() + prev_moments_.bytes() + prev_edge_.bytes() + edge_.bytes() + illum_.bytes() + moments_.bytes() +
           filter_[0].bytes() + filter_[1].bytes();
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Elements a buffer needs so that every address a pass's tensor map can reach lies inside it: the
// 5-D view reaches up to e - 1 pixels past a row's end and e rows past the last row.
size_t tma_buffer_elements(int w, int h) { return (size_t(h) + 9) * size_t(w) + 16; }

}  // namespace

void SvgfDenoiser::resize(int w, int h) {
    if (w == w_ && h == h_ && illum_.ptr) return;
    if (w <= 0 || h <= 0 || uint64_t(w) * uint64_t(h) > (uint64_t(1) << 30))
        throw Error{PT_ERR_INVALID, "svgf: width and height must be positive, at most 2^30 pixels"};
    // The size is recorded once every buffer has it, so a failed allocation cannot leave buffers
    // smaller than the recorded frame.
    w_ = 0;
    h_ = 0;
    size_t n = size_t(w) * size_t(h), np = tma_buffer_elements(w, h);
    for (DeviceBuffer<float4>* b : {&prev_illum_, &prev_moments_, &prev_edge_, &illum_, &moments_}) {
        b->allocate(n);
        b->zero(stream_);
    }
    for (DeviceBuffer<float4>* b : {&edge_, &filter_[0], &filter_[1]}) {
        b->allocate(np);
        b->zero(stream_);
    }
    PTW_CUDA(cudaStreamSynchronize(stream_));
    w_ = w;
    h_ = h;
    has_history_ = false;
    // Tensor maps of the TMA a-trous passes over edge_, filter_[0], filter_[1]; without them (no
    // encoder in the CUDA driver, or a shape it rejects) the passes read global memory directly.
    build_tma_plan();
}

// The staging of each a-trous pass for a TMA mode (pt_svgf_set_tma):
//   1: contiguous tiles for steps 1-8, global loads from step 16 on;
//   2: contiguous tiles for steps 1-8, a strided tile for step 16;
//   3: strided tiles (x, y mod min(step, 8)) for steps 1-16.
static void tma_passes_for_mode(int mode, TmaPass* out) {
    for (int it = 0; it < kTmaPasses; it++) {
        const int step = 1 << it;
        if (mode == 3 || (mode == 2 && step == 16)) {
            const int e = step < 8 ? step : 8;
            out[it] = TmaPass{5, e, step / e};
        } else if ((mode == 1 || mode == 2) && step <= 8) {
            out[it] = TmaPass{2, 1, step};
        } else {
            out[it] = TmaPass{0, 1, step};
        }
    }
}

void SvgfDenoiser::build_tma_plan() {
    maps_.assign(3 * kTmaPasses, CUtensorMap{});
    maps_ok_ = false;
    tma_passes_for_mode(tma_mode_, passes_);
    if (tma_mode_ == 0 || w_ == 0) return;
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return;
    {
        // Kernel attributes belong to a device: set them once on each device that runs the passes.
        // Up to 2 x 48 x 48 float4 of tiles (contiguous, step 8) per block.
        static std::mutex attr_mu;
        static std::vector<int> attr_done;
        int dev = 0;
        PTW_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> g(attr_mu);
        if (size_t(dev) >= attr_done.size()) attr_done.resize(size_t(dev) + 1, 0);
        if (!attr_done[size_t(dev)]) {
            PTW_CUDA(cudaFuncSetAttribute(k_atrous_tma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem_bytes(8))));
            PTW_CUDA(cudaFuncSetAttribute(k_atrous_tma<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tma_smem_bytes(8))));
            attr_done[size_t(dev)] = 1;
        }
    }
    float4* bufs[3] = {edge_.ptr, filter_[0].ptr, filter_[1].ptr};
    const int w = w_, h = h_;
    for (int b = 0; b < 3; b++)
        for (int it = 0; it < kTmaPasses; it++) {
            const TmaPass& tp = passes_[it];
            if (tp.rank == 0) continue;
            const cuuint32_t n = cuuint32_t(tma_box_side(tp.r));
            CUresult res;
            if (tp.rank == 2) {
                const cuuint64_t dims[2] = {4 * cuuint64_t(w), cuuint64_t(h)};
                const cuuint64_t strides[1] = {16 * cuuint64_t(w)};
                const cuuint32_t box[2] = {4 * n, n};
                const cuuint32_t estr[2] = {1, 1};
                res = encode(&maps_[size_t(b) * kTmaPasses + it], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, bufs[b], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            } else {
                const cuuint64_t e = cuuint64_t(tp.e);
                const cuuint64_t dims[5] = {4, e, (cuuint64_t(w) + e - 1) / e, e, (cuuint64_t(h) + e - 1) / e};
                const cuuint64_t strides[4] = {16, 16 * e, 16 * cuuint64_t(w), 16 * cuuint64_t(w) * e};
                const cuuint32_t box[5] = {4, 1, n, 1, n};
                const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
                res = encode(&maps_[size_t(b) * kTmaPasses + it], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, bufs[b], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            }
            if (res != CUDA_SUCCESS) return;
        }
    maps_ok_ = true;
}

void SvgfDenoiser::set_tma(int mode) {
    if (mode < 0 || mode > 3) throw Error{PT_ERR_INVALID, "TMA mode must be in [0, 3]"};
    tma_mode_ = mode;
    build_tma_plan();
}

static void check_settings(const pt_svgf_settings& s) {
    if (s.atrous_iterations < 0 || s.atrous_iterations > 30) throw Error{PT_ERR_INVALID, "atrous_iterations out of range"};
}

void SvgfDenoiser::check_status() {
    if (*reinterpret_cast<volatile int*>(status_host_)) {
        *status_host_ = 0;
        throw Error{PT_ERR_CUDA, "SVGF: a shared-memory tile load did not complete in time"};
    }
}

void SvgfDenoiser::run(const float* color, const float* albedo, const float* nd, const float* pos, const float* emission,
                       const pt_camera& prev, const pt_svgf_settings& s, float* output) {
    if (w_ == 0 || h_ == 0) return;
    check_settings(s);
    check_status();
    Frame5 in5{reinterpret_cast<const float4*>(color), reinterpret_cast<const float4*>(albedo), reinterpret_cast<const float4*>(nd),
               reinterpret_cast<const float4*>(pos), reinterpret_cast<const float4*>(emission)};
    PrevCamera pc;
    static_assert(sizeof(pt_camera) == sizeof(pc.c), "camera layout");
    std::memcpy(pc.c, &prev, sizeof(pc.c));
    History hist{prev_illum_.ptr, prev_moments_.ptr, prev_edge_.ptr};
    AtrousEpilogue hist_out{prev_illum_.ptr, prev_moments_.ptr, prev_edge_.ptr, illum_.ptr, moments_.ptr, nullptr, nullptr, nullptr, nullptr};
    TmaPlan plan{maps_ok_ ? maps_.data() : nullptr, passes_, status_dev_, tma_test_ ? 1 : 0};
    denoise<true>(in5, SvgfFrame{}, pc, w_, h_, has_history_, hist, edge_.ptr, hist_out, illum_.ptr, moments_.ptr, filter_[0].ptr,
                  filter_[1].ptr, s, output, plan, stream_);
    has_history_ = true;
}

void SvgfDenoiser::run_frame(const float* color, const float* albedo, const float* emission, const float* edge, const float* motion,
                             const pt_svgf_settings& s, float* output) {
    if (w_ == 0 || h_ == 0) return;
    check_settings(s);
    check_status();
    SvgfFrame in{reinterpret_cast<const float4*>(color), reinterpret_cast<const float4*>(albedo), reinterpret_cast<const float4*>(emission),
                 reinterpret_cast<const float4*>(edge), reinterpret_cast<const float4*>(motion)};
    History hist{prev_illum_.ptr, prev_moments_.ptr, prev_edge_.ptr};
    AtrousEpilogue hist_out{prev_illum_.ptr, prev_moments_.ptr, prev_edge_.ptr, illum_.ptr, moments_.ptr, nullptr, nullptr, nullptr, nullptr};
    TmaPlan plan{maps_ok_ ? maps_.data() : nullptr, passes_, status_dev_, tma_test_ ? 1 : 0};
    denoise<false>(Frame5{}, in, PrevCamera{}, w_, h_, has_history_, hist, edge_.ptr, hist_out, illum_.ptr, moments_.ptr, filter_[0].ptr,
                   filter_[1].ptr, s, output, plan, stream_);
    has_history_ = true;
}

// ---- the allocation-free single-frame denoise ------------------------------------------------------------
// For callers that cannot allocate device memory (pt_svgf_run_noalloc): a frame is denoised without
// history (the first frame of a session: demodulation, the spatial variance estimate, the a-trous
// passes, remodulation) by the same kernels as SvgfDenoiser::run, with their five intermediate
// buffers carved out of one file-scope device array instead of allocations.
namespace {

// edge records, illum, moments and the two a-trous buffers, kNoAllocMaxPixels float4 each: 40 MiB
// per device.
static __device__ __align__(256) float4 g_noalloc_scratch[5 * size_t(kNoAllocMaxPixels)];

std::mutex g_noalloc_mu;
float4* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// The device address of the scratch array on the current device (host code must not use the
// symbol's host-side name as a device pointer). Looked up once per device and kept for the life of
// the process: after a cudaDeviceReset the module may load elsewhere, so a reset after the first call
// is not supported (the header says so).
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
    check_settings(s);
    if (device < 0 || device >= kNoAllocMaxDevices) throw Error{PT_ERR_INVALID, "svgf_run_noalloc: device ordinal out of range"};
    int previous = 0;
    PTW_CUDA(cudaGetDevice(&previous));
    PTW_CUDA(cudaSetDevice(device));
    try {
        float4* base = noalloc_scratch(device);
        const size_t n = kNoAllocMaxPixels;
        float4 *edge = base, *illum = base + n, *moments = base + 2 * n, *f0 = base + 3 * n, *f1 = base + 4 * n;
        Frame5 in5{reinterpret_cast<const float4*>(color), reinterpret_cast<const float4*>(albedo), reinterpret_cast<const float4*>(nd),
                   reinterpret_cast<const float4*>(pos), reinterpret_cast<const float4*>(emission)};
        // Without history the temporal step reads nothing from earlier calls, and every scratch
        // element a kernel reads was written earlier in this call: nothing needs clearing.
        denoise<true>(in5, SvgfFrame{}, PrevCamera{}, w, h, false, History{}, edge, AtrousEpilogue{}, illum, moments, f0, f1, s, output,
                      TmaPlan{nullptr, nullptr, nullptr, 0}, stream);
    } catch (...) {
        cudaSetDevice(previous);
        throw;
    }
    PTW_CUDA(cudaSetDevice(previous));
}

}  // namespace ptw
