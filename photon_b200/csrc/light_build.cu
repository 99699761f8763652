// Light tables built on the device (pt_rebuild_lights): the emissive-triangle list and its alias
// table, the light-group probabilities and the environment's sampling distribution, computed from new
// materials / lights / environment for a scene already on the device. The definitions, and the order
// of every floating-point operation, are those of the host builder (scene_build.cpp), so the tables
// equal the ones pt_scene_build produces for the same inputs; the parallel steps are those whose
// results do not depend on order (per triangle, per row), the sums that do are taken by one thread
// in the host's order.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstring>
#include <vector>

#include "device_scene.h"
#include "pt_math.cuh"

namespace ptw {

namespace {

constexpr float kPiF = 3.14159265358979323846f;

__device__ __forceinline__ float lum3(float x, float y, float z) { return 0.2126f * x + 0.7152f * y + 0.0722f * z; }

struct TexArgs {
    const int4* textures;  // (width, height, offset, repeat | srgb << 1)
    const uint32_t* texels;
    const float* lut;
    int num_textures;
};

// Bilinear RGB lookup (scene_build.cpp host_tex_rgb).
__device__ V3 tex_rgb(const TexArgs& T, int ti, float u, float v) {
    const int4 t = T.textures[ti];
    const int w = t.x, h = t.y;
    const bool repeat = (t.w & 1) != 0, srgb = (t.w & 2) != 0;
    float x = u * float(w) - 0.5f, y = v * float(h) - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    if (!(fabsf(fx) < 1e8f) || !(fabsf(fy) < 1e8f)) return V3{0, 0, 0};
    int x0 = int(fx), y0 = int(fy);
    float tx = x - fx, ty = y - fy;
    auto wrap = [&](int i, int n) {
        if (repeat) {
            i %= n;
            return i < 0 ? i + n : i;
        }
        return i < 0 ? 0 : (i >= n ? n - 1 : i);
    };
    int xa = wrap(x0, w), xb = wrap(x0 + 1, w), ya = wrap(y0, h), yb = wrap(y0 + 1, h);
    auto texel = [&](int xx, int yy) {
        uint32_t p = T.texels[uint32_t(t.z) + uint32_t(yy * w + xx)];
        if (srgb) return V3{T.lut[p & 0xFF], T.lut[(p >> 8) & 0xFF], T.lut[(p >> 16) & 0xFF]};
        const float s = 1.0f / 255.0f;
        return V3{float(p & 0xFF) * s, float((p >> 8) & 0xFF) * s, float((p >> 16) & 0xFF) * s};
    };
    V3 top = texel(xa, ya) * (1 - tx) + texel(xb, ya) * tx;
    V3 bot = texel(xa, yb) * (1 - tx) + texel(xb, yb) * tx;
    return top * (1 - ty) + bot * ty;
}

// Per triangle: the alpha-test flag from its material, and whether it emits (with its area and
// power, as the host builder's "emissive triangles by power").
__global__ void k_light_tris(const float4* __restrict__ materials, float4* __restrict__ tris, const int4* __restrict__ tri_idx,
                             const float2* __restrict__ uvs, TexArgs T, int n, int* __restrict__ flag, float* __restrict__ area_out,
                             float* __restrict__ power_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4* g = tris + kTriStride * size_t(i);
    const int mi = __float_as_int(g[0].w);
    const float4* m = materials + 5 * size_t(mi);
    const float4 m1 = m[1], m3 = m[3], m4 = m[4];
    const int alpha_mode = __float_as_int(m3.y), double_sided = __float_as_int(m3.z), emissive_tex = __float_as_int(m4.z);
    g[1].w = __int_as_float(alpha_mode != PT_ALPHA_OPAQUE ? PT_TRI_ALPHA_TESTED : 0);
    flag[i] = 0;
    float l = lum3(m1.x, m1.y, m1.z);
    if (l <= 0) return;
    if (emissive_tex >= 0 && emissive_tex < T.num_textures && uvs) {
        const float pts[7][2] = {{1.f / 3, 1.f / 3}, {0.1f, 0.1f}, {0.8f, 0.1f}, {0.1f, 0.8f}, {0.45f, 0.1f}, {0.45f, 0.45f}, {0.1f, 0.45f}};
        const int4 idx = tri_idx[i];
        const float2 a = uvs[idx.x], b = uvs[idx.y], c = uvs[idx.z];
        float sum = 0;
        for (int k = 0; k < 7; k++) {
            float w0 = 1 - pts[k][0] - pts[k][1];
            float u = a.x * w0 + b.x * pts[k][0] + c.x * pts[k][1];
            float v = a.y * w0 + b.y * pts[k][0] + c.y * pts[k][1];
            V3 tc = tex_rgb(T, emissive_tex, u, v);
            sum += lum3(m1.x * tc.x, m1.y * tc.y, m1.z * tc.z);
        }
        l = sum / 7.0f;
        if (l <= 1e-4f) return;
    }
    const V3 e1 = xyz(g[1]), e2 = xyz(g[2]);
    const V3 cr{e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x};
    const float area = 0.5f * sqrtf(cr.x * cr.x + cr.y * cr.y + cr.z * cr.z);
    if (area <= 0) return;
    flag[i] = 1;
    area_out[i] = area;
    power_out[i] = area * l * kPiF * (double_sided ? 2.0f : 1.0f);
}

// Emitters in triangle order: the list (triangle, area bits), each triangle's entry (or -1), powers.
__global__ void k_light_scatter(const int* __restrict__ flag, const int* __restrict__ pos, const float* __restrict__ area,
                                const float* __restrict__ power, int n, int4* __restrict__ tri_idx, int2* __restrict__ emissive,
                                float* __restrict__ power_c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int e = -1;
    if (flag[i]) {
        e = pos[i];
        emissive[e] = make_int2(i, __float_as_int(area[i]));
        power_c[e] = power[i];
    }
    tri_idx[i].w = e;
}

// The host builder's alias_table (Walker / Vose, both worklists consumed in index order) and the
// total emissive power, by one thread in the host's order.
__global__ void k_light_alias(const float* __restrict__ w, int n, float4* __restrict__ table, double* __restrict__ fill,
                              int* __restrict__ under, int* __restrict__ over, float* __restrict__ total_power) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float power = 0;
    for (int i = 0; i < n; i++) power += w[i];
    *total_power = power;
    if (n == 0) return;
    double sum = 0;
    for (int i = 0; i < n; i++) sum += w[i] > 0 ? double(w[i]) : 0.0;
    int nu = 0, no = 0;
    for (int i = 0; i < n; i++) {
        double pmf = sum > 0 ? (w[i] > 0 ? double(w[i]) : 0.0) / sum : 1.0 / double(n);
        table[i] = make_float4(1.0f, __int_as_float(i), float(pmf), 0.0f);
        fill[i] = pmf * double(n);
        if (fill[i] < 1.0) under[nu++] = i;
        else over[no++] = i;
    }
    // `under` grows while it is consumed: an over-full entry that drops below one joins its end.
    int u = 0, o = 0;
    while (u < nu && o < no) {
        int lo = under[u++], hi = over[o];
        table[lo].x = float(fill[lo]);
        table[lo].y = __int_as_float(hi);
        fill[hi] -= 1.0 - fill[lo];
        if (fill[hi] < 1.0) {
            o++;
            under[nu++] = hi;
        }
    }
    for (; u < nu; u++) table[under[u]].x = 1.0f;
    for (; o < no; o++) table[over[o]].x = 1.0f;
}

// Environment texels with their luminance, and each row's conditional CDF (one thread per row, in
// the host's order).
__global__ void k_env_texels(const float* __restrict__ rgb, size_t n, float4* __restrict__ out) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = rgb[3 * i], y = rgb[3 * i + 1], z = rgb[3 * i + 2];
    out[i] = make_float4(x, y, z, lum3(x, y, z));
}

__global__ void k_env_rows(const float4* __restrict__ texels, int w, int h, const float* __restrict__ row_sin, float* __restrict__ cond,
                           double* __restrict__ row_total) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= h) return;
    const float sin_theta = row_sin[y];
    const float4* row = texels + size_t(y) * size_t(w);
    double rs = 0;
    for (int x = 0; x < w; x++) rs = rs + double(row[x].w) * sin_theta;
    row_total[y] = rs;
    float* cdf = cond + size_t(y) * size_t(w + 1);
    cdf[0] = 0.0f;
    double prefix = 0;
    for (int x = 1; x <= w; x++) {
        prefix = prefix + double(row[x - 1].w) * sin_theta;
        cdf[x] = rs > 0 ? float(double(float(prefix)) / rs) : float(x) / float(w);
    }
}

// The marginal CDF, the integral and the mean luminance (one thread, the host's order).
__global__ void k_env_marginal(const float4* __restrict__ texels, int w, int h, const double* __restrict__ row_total,
                               float* __restrict__ marginal, float* __restrict__ scalars) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double all = 0;
    marginal[0] = 0.0f;
    for (int y = 0; y < h; y++) {
        all = all + row_total[y];
        marginal[y + 1] = float(all);  // the prefix, normalised below
    }
    for (int y = 1; y <= h; y++) marginal[y] = all > 0 ? float(double(marginal[y]) / all) : float(y) / float(h);
    scalars[0] = float(all / (double(w) * double(h)));
    double s = 0;
    const size_t n = size_t(w) * size_t(h);
    for (size_t i = 0; i < n; i++) s += texels[i].w;
    scalars[1] = float(s / double(n));
}

float lum_h(const pt_vec3& c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

}  // namespace

void DeviceScene::rebuild_lights(const pt_light_update& u, cudaStream_t s) {
    if (!ready_) throw Error{PT_ERR_NO_SCENE, "rebuild_lights before upload"};
    if (!u.materials || u.num_materials != num_materials_)
        throw Error{PT_ERR_INVALID, "rebuild_lights: the material count must stay the scene's"};
    if (u.num_punctual < 0 || (u.num_punctual > 0 && !u.punctual)) throw Error{PT_ERR_INVALID, "rebuild_lights: punctual lights missing"};
    if (u.env_texels && (u.env_width <= 0 || u.env_height <= 0)) throw Error{PT_ERR_INVALID, "rebuild_lights: environment size"};
    const int num_textures = int(textures_.count);
    for (int32_t m = 0; m < u.num_materials; m++) {
        const pt_material& mm = u.materials[m];
        const int32_t tex[5] = {mm.base_color_tex, mm.metallic_roughness_tex, mm.normal_tex, mm.emissive_tex, mm.occlusion_tex};
        for (int32_t t : tex)
            if (t >= num_textures) throw Error{PT_ERR_INVALID, "rebuild_lights: material texture out of range"};
    }
    const int n = view_.num_tris;
    materials_.upload(reinterpret_cast<const float4*>(u.materials), size_t(u.num_materials) * 5, s);
    upload_shade_keys(u.materials, u.num_materials, s);
    // Emissive triangles, in triangle order.
    DeviceBuffer<int> flag, pos;
    DeviceBuffer<float> area, power, power_c;
    flag.allocate(size_t(n) + 1);
    pos.allocate(size_t(n) + 1);
    area.allocate(size_t(n) + 1);
    power.allocate(size_t(n) + 1);
    TexArgs T{textures_.ptr, texels_.ptr, srgb_lut_.ptr, num_textures};
    int ne = 0;
    if (n > 0) {
        k_light_tris<<<(n + 255) / 256, 256, 0, s>>>(materials_.ptr, tris_.ptr, tri_idx_.ptr, uvs_.ptr, T, n, flag.ptr, area.ptr, power.ptr);
        PTW_CUDA(cudaGetLastError());
        size_t temp = 0;
        PTW_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, flag.ptr, pos.ptr, n + 1, s));
        DeviceBuffer<uint8_t> tmp;
        tmp.allocate(temp + 1);
        PTW_CUDA(cudaMemsetAsync(flag.ptr + n, 0, sizeof(int), s));
        PTW_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, temp, flag.ptr, pos.ptr, n + 1, s));
        PTW_CUDA(cudaMemcpyAsync(&ne, pos.ptr + n, sizeof(int), cudaMemcpyDeviceToHost, s));
        PTW_CUDA(cudaStreamSynchronize(s));
    }
    emissive_.allocate(size_t(ne));
    alias_.allocate(size_t(ne));
    power_c.allocate(size_t(ne) + 1);
    if (n > 0) {
        k_light_scatter<<<(n + 255) / 256, 256, 0, s>>>(flag.ptr, pos.ptr, area.ptr, power.ptr, n, tri_idx_.ptr, emissive_.ptr, power_c.ptr);
        PTW_CUDA(cudaGetLastError());
    }
    DeviceBuffer<double> fill;
    DeviceBuffer<int> under, over;
    DeviceBuffer<float> scalars;
    fill.allocate(size_t(ne) + 1);
    under.allocate(size_t(ne) + 1);
    over.allocate(size_t(ne) + 1);
    scalars.allocate(4);
    k_light_alias<<<1, 32, 0, s>>>(power_c.ptr, ne, alias_.ptr, fill.ptr, under.ptr, over.ptr, scalars.ptr + 2);
    PTW_CUDA(cudaGetLastError());
    // Environment.
    const bool has_env_image = u.env_texels != nullptr;
    if (has_env_image) {
        const int w = u.env_width, h = u.env_height;
        const size_t texn = size_t(w) * size_t(h);
        DeviceBuffer<float> rgb;
        rgb.upload(reinterpret_cast<const float*>(u.env_texels), 3 * texn, s);
        env_texels_.allocate(texn);
        k_env_texels<<<unsigned((texn + 255) / 256), 256, 0, s>>>(rgb.ptr, texn, env_texels_.ptr);
        std::vector<float> row_sin(static_cast<size_t>(h));
        for (int y = 0; y < h; y++) row_sin[size_t(y)] = std::sin((float(y) + 0.5f) / float(h) * kPiF);
        env_row_sin_.upload(row_sin.data(), row_sin.size(), s);
        env_conditional_.allocate(size_t(h) * size_t(w + 1));
        env_marginal_.allocate(size_t(h) + 1);
        DeviceBuffer<double> row_total;
        row_total.allocate(size_t(h));
        k_env_rows<<<(h + 127) / 128, 128, 0, s>>>(env_texels_.ptr, w, h, env_row_sin_.ptr, env_conditional_.ptr, row_total.ptr);
        k_env_marginal<<<1, 32, 0, s>>>(env_texels_.ptr, w, h, row_total.ptr, env_marginal_.ptr, scalars.ptr);
        PTW_CUDA(cudaGetLastError());
        PTW_CUDA(cudaStreamSynchronize(s));
    } else {
        env_texels_.release();
        env_marginal_.release();
        env_conditional_.release();
        env_row_sin_.release();
    }
    float sc[4] = {0, 0, 0, 0};
    PTW_CUDA(cudaMemcpyAsync(sc, scalars.ptr, sizeof(sc), cudaMemcpyDeviceToHost, s));
    punctual_.upload(reinterpret_cast<const float4*>(u.punctual), size_t(u.num_punctual) * 3, s);
    PTW_CUDA(cudaStreamSynchronize(s));
    const float env_integral = has_env_image ? sc[0] : 0.0f;
    const float mean_env = has_env_image ? sc[1] : lum_h(u.env_color);
    const float emissive_power = sc[2];
    // Light-group probabilities (the host builder's definition and arithmetic).
    const float dx = bounds_[3] - bounds_[0], dy = bounds_[4] - bounds_[1], dz = bounds_[5] - bounds_[2];
    const float r = view_.num_tris == 0 ? 1.0f : 0.5f * std::sqrt(dx * dx + dy * dy + dz * dz);
    float group_power[3];
    group_power[0] = mean_env * u.env_intensity * kPiF * kPiF * r * r * 4.0f;
    group_power[1] = emissive_power;
    group_power[2] = 0;
    for (int32_t k = 0; k < u.num_punctual; k++) {
        const pt_punctual_light& l = u.punctual[k];
        group_power[2] += l.type == PT_LIGHT_DIRECTIONAL ? lum_h(l.intensity) * kPiF * r * r : lum_h(l.intensity) * 4.0f * kPiF;
    }
    float prob[3] = {0, 0, 0};
    const float total = group_power[0] + group_power[1] + group_power[2];
    if (total > 0) {
        for (int g = 0; g < 3; g++) {
            prob[g] = group_power[g] / total;
            if (group_power[g] > 0 && prob[g] < 0.05f) prob[g] = 0.05f;
        }
        const float norm = prob[0] + prob[1] + prob[2];
        for (float& p : prob) p /= norm;
    }
    DevScene& v = view_;
    v.materials = materials_.ptr;
    v.emissive = emissive_.ptr;
    v.alias = alias_.ptr;
    v.punctual = punctual_.ptr;
    v.env_texels = env_texels_.ptr;
    v.env_marginal = env_marginal_.ptr;
    v.env_conditional = env_conditional_.ptr;
    v.env_row_sin = env_row_sin_.ptr;
    v.num_emissive = ne;
    v.num_punctual = u.num_punctual;
    v.env_width = has_env_image ? u.env_width : 0;
    v.env_height = has_env_image ? u.env_height : 0;
    v.env_intensity = u.env_intensity;
    v.env_integral = env_integral;
    v.env_cos_neg = std::cos(-u.env_rotation);
    v.env_sin_neg = std::sin(-u.env_rotation);
    v.env_cos_pos = std::cos(u.env_rotation);
    v.env_sin_pos = std::sin(u.env_rotation);
    v.env_color_x = u.env_color.x;
    v.env_color_y = u.env_color.y;
    v.env_color_z = u.env_color.z;
    v.p_env = prob[0];
    v.p_emissive = prob[1];
    v.p_punctual = prob[2];
    v.has_lights = (prob[0] + prob[1] + prob[2]) > 0 ? 1 : 0;
    d_view_.upload(&v, 1, s);
    PTW_CUDA(cudaStreamSynchronize(s));
}

}  // namespace ptw
