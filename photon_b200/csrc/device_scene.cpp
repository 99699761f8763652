// Upload of a built scene to the device (replaces GpuRenderer::upload / update_lights,
// src/render/gpu_renderer.cu:243-334 of Photon): validation, re-layout and copies.
//
// Values that Photon's integrator computes from per-scene constants are precomputed here with the
// host's libm, exactly as Photon's CPU build evaluates them: cosf/sinf of the environment rotation
// (lights.h:34-37) and the per-row sinf of the environment distribution (lights.h:70,94), plus the
// luminance of each environment texel (math.h:112), so the device never needs those transcendentals.
#include "device_scene.h"
#include "wide_bvh.h"

#include <cmath>
#include <cstring>

namespace ptw {

namespace {

constexpr float kPiHost = 3.14159265358979323846f;

float lum_host(const pt_vec3& c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

[[noreturn]] void invalid(const std::string& m) { throw Error{PT_ERR_INVALID, "invalid scene: " + m}; }

}  // namespace

void validate_scene(const pt_scene_desc& d, bool lights_only) {
    if (d.num_tris < 0 || d.num_nodes < 0 || d.num_vertices < 0 || d.num_materials < 0) invalid("negative count");
    if (!lights_only) {
        if (d.num_nodes < 1 || !d.nodes) invalid("a BVH needs at least its root node");
        if (d.num_tris > 0 && (!d.tris || !d.indices)) invalid("triangles without geometry or indices");
        for (int32_t i = 0; i < d.num_nodes; i++) {
            const pt_bvh_node& n = d.nodes[i];
            const int32_t idx[2] = {n.left, n.right}, cnt[2] = {n.lcount, n.rcount};
            for (int k = 0; k < 2; k++) {
                if (cnt[k] > 0) {
                    if (idx[k] < 0 || int64_t(idx[k]) + cnt[k] > d.num_tris) invalid("leaf range outside the triangles");
                } else if (idx[k] >= d.num_nodes) {
                    invalid("child node index out of range");
                } else if (idx[k] >= 0 && idx[k] <= i) {
                    invalid("child node index does not follow its parent (depth-first order)");
                }
            }
        }
        for (int64_t i = 0; i < int64_t(d.num_tris) * 3; i++)
            if (d.indices[i] < 0 || d.indices[i] >= d.num_vertices) invalid("vertex index out of range");
    }
    if (d.num_materials < 1 || !d.materials) invalid("no materials");
    for (int32_t t = 0; t < d.num_tris; t++)
        if (d.tris[t].material < 0 || d.tris[t].material >= d.num_materials) invalid("triangle material out of range");
    if (d.num_textures > 0 && !d.textures) invalid("textures missing");
    for (int32_t i = 0; i < d.num_textures; i++) {
        const pt_texture_info& t = d.textures[i];
        if (t.width <= 0 || t.height <= 0 || uint64_t(t.offset) + uint64_t(t.width) * uint64_t(t.height) > d.num_texels)
            invalid("texture outside the texel pool");
    }
    for (int32_t m = 0; m < d.num_materials; m++) {
        const pt_material& mm = d.materials[m];
        const int32_t tex[5] = {mm.base_color_tex, mm.metallic_roughness_tex, mm.normal_tex, mm.emissive_tex, mm.occlusion_tex};
        for (int32_t t : tex)
            if (t >= d.num_textures) invalid("material texture out of range");
    }
    if (d.num_textures > 0 && !d.srgb_lut) invalid("textures need the sRGB table");
    if (d.num_emissive > 0 && (!d.emissive || !d.emissive_alias || !d.tri_emissive)) invalid("emissive tables missing");
    for (int32_t k = 0; k < d.num_emissive; k++) {
        if (d.emissive[k].tri < 0 || d.emissive[k].tri >= d.num_tris) invalid("emissive triangle out of range");
        if (d.emissive_alias[k].alias < 0 || d.emissive_alias[k].alias >= d.num_emissive) invalid("alias entry out of range");
    }
    if (d.tri_emissive)
        for (int32_t t = 0; t < d.num_tris; t++)
            if (d.tri_emissive[t] >= d.num_emissive) invalid("triangle emissive entry out of range");
    if (d.num_punctual > 0 && !d.punctual) invalid("punctual lights missing");
    if (d.env_texels) {
        if (d.env_width <= 0 || d.env_height <= 0 || !d.env_marginal || !d.env_conditional) invalid("environment tables missing");
    }
}

size_t DeviceScene::estimate_bytes(const pt_scene_desc& d) {
    size_t b = 0;
    b += size_t(d.num_nodes) * 64 + size_t(d.num_tris) * (16 * kTriStride + 16);
    b += size_t(d.num_vertices) * ((d.normals ? 16 : 0) + (d.uvs ? 8 : 0) + (d.tangents ? 16 : 0));
    b += size_t(d.num_materials) * 80 + size_t(d.num_textures) * 16 + size_t(d.num_texels) * 4 + 1024;
    b += size_t(d.num_emissive) * 24 + size_t(d.num_punctual) * 48;
    if (d.env_texels) b += size_t(d.env_width) * d.env_height * 16 + (size_t(d.env_height) + 1) * 4 + size_t(d.env_height) * (d.env_width + 1) * 4 + size_t(d.env_height) * 4;
    return b + sizeof(DevScene);
}

size_t DeviceScene::device_bytes() const {
    return nodes_.bytes() + nodes4_.bytes() + tris_.bytes() + normals_.bytes() + tangents_.bytes() + materials_.bytes() + alias_.bytes() +
           punctual_.bytes() + env_texels_.bytes() + tri_idx_.bytes() + textures_.bytes() + uvs_.bytes() + texels_.bytes() +
           srgb_lut_.bytes() + env_marginal_.bytes() + env_conditional_.bytes() + env_row_sin_.bytes() + emissive_.bytes() +
           shade_keys_.bytes() + d_view_.bytes();
}

// Shading classes: materials of one class take the same branches through the BSDF, texture and
// emission code, so the shade kernel groups a block's paths by class.
void DeviceScene::upload_shade_keys(const pt_material* materials, int32_t n, cudaStream_t s) {
    std::vector<uint8_t> keys(static_cast<size_t>(n));
    for (size_t m = 0; m < keys.size(); m++) {
        const pt_material& mm = materials[m];
        int k = 1;
        if (mm.metallic > 0.0f) k += 1;
        if (mm.transmission > 0.0f) k += 2;
        if (mm.base_color_tex >= 0 || mm.metallic_roughness_tex >= 0) k += 4;
        if (mm.normal_tex >= 0) k += 8;
        if (mm.emission.x > 0.0f || mm.emission.y > 0.0f || mm.emission.z > 0.0f || mm.emissive_tex >= 0) k += 16;
        keys[m] = uint8_t(k);
    }
    shade_keys_.upload(keys.data(), keys.size(), s);
    PTW_CUDA(cudaStreamSynchronize(s));
}

void DeviceScene::upload(const pt_scene_desc& d, cudaStream_t s, bool lights_only) {
    if (lights_only && !ready_) lights_only = false;
    if (lights_only && d.num_tris != view_.num_tris) throw Error{PT_ERR_INVALID, "update_lights: the triangle count changed"};
    validate_scene(d, lights_only);
    if (!lights_only) {
        nodes_.upload(reinterpret_cast<const float4*>(d.nodes), size_t(d.num_nodes) * 4, s);
        // The 4-wide BVH for any-hit rays, collapsed from the same tree (absent if it does not fit
        // the walk's stack or leaf encoding; the shadow rays then walk the BVH2).
        std::vector<Bvh4Node> wide;
        int depth = 0;
        if (build_bvh4(d.nodes, d.num_nodes, d.num_tris, wide, &depth)) {
            nodes4_.upload(reinterpret_cast<const float4*>(wide.data()), wide.size() * 8, s);
            PTW_CUDA(cudaStreamSynchronize(s));
        } else {
            nodes4_.release();
        }
        num_vertices_ = d.num_vertices;
        if (d.normals) {
            std::vector<float4> n(size_t(d.num_vertices));
            for (size_t i = 0; i < n.size(); i++) n[i] = make_float4(d.normals[i].x, d.normals[i].y, d.normals[i].z, 0.0f);
            normals_.upload(n.data(), n.size(), s);
            PTW_CUDA(cudaStreamSynchronize(s));
        } else {
            normals_.release();
        }
        if (d.uvs) uvs_.upload(reinterpret_cast<const float2*>(d.uvs), size_t(d.num_vertices), s);
        else uvs_.release();
        if (d.tangents) tangents_.upload(reinterpret_cast<const float4*>(d.tangents), size_t(d.num_vertices), s);
        else tangents_.release();
        std::vector<int4> tex(size_t(d.num_textures));
        for (size_t i = 0; i < tex.size(); i++) {
            const pt_texture_info& t = d.textures[i];
            tex[i] = make_int4(t.width, t.height, int(t.offset), (t.wrap_repeat ? 1 : 0) | (t.srgb ? 2 : 0));
        }
        textures_.upload(tex.data(), tex.size(), s);
        texels_.upload(d.texels, size_t(d.num_texels), s);
        if (d.srgb_lut) srgb_lut_.upload(d.srgb_lut, 256, s);
        else srgb_lut_.release();
        punctual_.upload(reinterpret_cast<const float4*>(d.punctual), size_t(d.num_punctual) * 3, s);
        PTW_CUDA(cudaStreamSynchronize(s));
    }
    // What update_lights re-uploads (gpu_renderer.cu:303-310): triangles, materials, light tables
    // and the environment.
    {
        // Photon's 48-byte TriGeom records, each padded to 64 bytes (kTriStride float4); the padding
        // carries the vertex indices for the alpha test.
        std::vector<float4> padded(size_t(d.num_tris) * kTriStride, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
        const float4* src = reinterpret_cast<const float4*>(d.tris);
        for (size_t t = 0; t < size_t(d.num_tris); t++) {
            for (int k = 0; k < 3; k++) padded[t * kTriStride + size_t(k)] = src[t * 3 + size_t(k)];
            int32_t vi[4] = {d.indices[3 * t], d.indices[3 * t + 1], d.indices[3 * t + 2], 0};
            std::memcpy(&padded[t * kTriStride + 3], vi, sizeof(vi));
        }
        tris_.upload(padded.data(), padded.size(), s);
        PTW_CUDA(cudaStreamSynchronize(s));
    }
    materials_.upload(reinterpret_cast<const float4*>(d.materials), size_t(d.num_materials) * 5, s);
    num_materials_ = d.num_materials;
    upload_shade_keys(d.materials, d.num_materials, s);
    std::vector<int4> idx(size_t(d.num_tris));
    for (size_t t = 0; t < idx.size(); t++)
        idx[t] = make_int4(d.indices[3 * t], d.indices[3 * t + 1], d.indices[3 * t + 2], d.tri_emissive ? d.tri_emissive[t] : -1);
    tri_idx_.upload(idx.data(), idx.size(), s);
    emissive_.upload(reinterpret_cast<const int2*>(d.emissive), size_t(d.num_emissive), s);
    alias_.upload(reinterpret_cast<const float4*>(d.emissive_alias), size_t(d.num_emissive), s);
    std::vector<float4> env;
    std::vector<float> row_sin;
    if (d.env_texels) {
        size_t n = size_t(d.env_width) * size_t(d.env_height);
        env.resize(n);
        for (size_t i = 0; i < n; i++) env[i] = make_float4(d.env_texels[i].x, d.env_texels[i].y, d.env_texels[i].z, lum_host(d.env_texels[i]));
        env_texels_.upload(env.data(), n, s);
        env_marginal_.upload(d.env_marginal, size_t(d.env_height) + 1, s);
        env_conditional_.upload(d.env_conditional, size_t(d.env_height) * size_t(d.env_width + 1), s);
        row_sin.resize(size_t(d.env_height));
        for (int y = 0; y < d.env_height; y++) row_sin[size_t(y)] = std::sin((float(y) + 0.5f) / float(d.env_height) * kPiHost);
        env_row_sin_.upload(row_sin.data(), row_sin.size(), s);
    } else {
        env_texels_.release();
        env_marginal_.release();
        env_conditional_.release();
        env_row_sin_.release();
    }

    DevScene& v = view_;
    v = DevScene{};
    v.nodes = nodes_.ptr;
    v.nodes4 = nodes4_.ptr;
    v.tris = tris_.ptr;
    v.tri_idx = tri_idx_.ptr;
    v.normals = normals_.ptr;
    v.uvs = uvs_.ptr;
    v.tangents = tangents_.ptr;
    v.materials = materials_.ptr;
    v.shade_keys = shade_keys_.ptr;
    v.textures = textures_.ptr;
    v.texels = texels_.ptr;
    v.srgb_lut = srgb_lut_.ptr;
    v.emissive = emissive_.ptr;
    v.alias = alias_.ptr;
    v.punctual = punctual_.ptr;
    v.env_texels = env_texels_.ptr;
    v.env_marginal = env_marginal_.ptr;
    v.env_conditional = env_conditional_.ptr;
    v.env_row_sin = env_row_sin_.ptr;
    v.num_tris = d.num_tris;
    v.num_nodes = int(nodes_.count / 4);
    v.num_emissive = d.num_emissive;
    v.num_punctual = int(punctual_.count / 3);
    v.env_width = d.env_width;
    v.env_height = d.env_height;
    v.env_intensity = d.env_intensity;
    v.env_integral = d.env_integral;
    v.env_cos_neg = std::cos(-d.env_rotation);
    v.env_sin_neg = std::sin(-d.env_rotation);
    v.env_cos_pos = std::cos(d.env_rotation);
    v.env_sin_pos = std::sin(d.env_rotation);
    v.env_color_x = d.env_color.x;
    v.env_color_y = d.env_color.y;
    v.env_color_z = d.env_color.z;
    v.p_env = d.p_env;
    v.p_emissive = d.p_emissive;
    v.p_punctual = d.p_punctual;
    v.has_lights = (d.p_env + d.p_emissive + d.p_punctual) > 0 ? 1 : 0;
    v.bvh_depth = 0;
    {
        float lo[3] = {d.bounds_min.x, d.bounds_min.y, d.bounds_min.z}, hi[3] = {d.bounds_max.x, d.bounds_max.y, d.bounds_max.z};
        float inv[3];
        for (int k = 0; k < 3; k++) {
            float e = hi[k] - lo[k];
            if (!(e > 0) || !std::isfinite(e)) {
                lo[k] = 0;
                e = 1;
            }
            inv[k] = 1.0f / e;
        }
        v.bounds_lo_x = lo[0];
        v.bounds_lo_y = lo[1];
        v.bounds_lo_z = lo[2];
        v.inv_extent_x = inv[0];
        v.inv_extent_y = inv[1];
        v.inv_extent_z = inv[2];
    }
    d_view_.upload(&v, 1, s);
    PTW_CUDA(cudaStreamSynchronize(s));
    bounds_[0] = d.bounds_min.x;
    bounds_[1] = d.bounds_min.y;
    bounds_[2] = d.bounds_min.z;
    bounds_[3] = d.bounds_max.x;
    bounds_[4] = d.bounds_max.y;
    bounds_[5] = d.bounds_max.z;
    float dx = d.bounds_max.x - d.bounds_min.x, dy = d.bounds_max.y - d.bounds_min.y, dz = d.bounds_max.z - d.bounds_min.z;
    extent_ = std::fmax(std::sqrt(dx * dx + dy * dy + dz * dz), 1e-3f);
    if (!std::isfinite(extent_)) extent_ = 1.0f;
    ready_ = true;
}

}  // namespace ptw
