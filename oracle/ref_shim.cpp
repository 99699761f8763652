// Test-infrastructure shim over Photon's own CPU code (the reference build of the oracle).
//
// This file is compiled together with Photon's sources, where they lie, by oracle/Makefile into
// oracle/_ref/libphoton_ref.so. It adds nothing to Photon's algorithms: every entry point converts
// between the C-ABI types of include/photon_wavefront.h and Photon's C++ types, then calls Photon:
//   - Scene::build (src/scene/scene.cpp:212-255) on raw meshes, or make_builtin_scene
//     (src/scene/builtin.cpp:102-186);
//   - the benchmark's procedural scenes: the raw meshes of this repository's seeded generator
//     (photon_b200/csrc/scene_gen.cpp, compiled in by oracle/Makefile: it is the workload's
//     definition, not the renderer) handed to Photon's Scene::build, with Photon's Camera::view;
//   - CpuRenderer::render (src/render/cpu_renderer.cpp:20-39) for images;
//   - render_sample's first steps (src/render/pixel.h:18-24), intersect (src/render/traverse.h:140),
//     surface_at / Bsdf / sample_alias / find_interval (integrator.h, bsdf.h, lights.h) for the
//     discrete decisions that must be bit-exact.
// Only tests, the smoke check and the CPU-baseline leg of the benchmark load the result.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <atomic>
#include <vector>

#include "core/color.h"
#include "render/cpu_renderer.h"
#include "render/pixel.h"
#include "scene/builtin.h"
#include "scene/scene.h"

#include "photon_wavefront.h"
#include "pt_error.h"
#include "scene_build.h"

using namespace photon;

// The C-ABI types must have Photon's layouts exactly (the ABI passes them by pointer cast).
static_assert(sizeof(pt_bvh_node) == sizeof(BvhNode) && sizeof(pt_bvh_node) == 64, "BvhNode layout");
static_assert(offsetof(pt_bvh_node, rcount) == offsetof(BvhNode, rcount), "BvhNode layout");
static_assert(sizeof(pt_tri_geom) == sizeof(TriGeom) && sizeof(pt_tri_geom) == 48, "TriGeom layout");
static_assert(offsetof(pt_tri_geom, flags) == offsetof(TriGeom, flags), "TriGeom layout");
static_assert(sizeof(pt_material) == sizeof(Material) && sizeof(pt_material) == 80, "Material layout");
static_assert(offsetof(pt_material, alpha_cutoff) == offsetof(Material, alpha_cutoff), "Material layout");
static_assert(offsetof(pt_material, occlusion_tex) == offsetof(Material, occlusion_tex), "Material layout");
static_assert(sizeof(pt_texture_info) == sizeof(TextureInfo), "TextureInfo layout");
static_assert(sizeof(pt_emissive_tri) == sizeof(EmissiveTri), "EmissiveTri layout");
static_assert(sizeof(pt_alias_entry) == sizeof(AliasEntry), "AliasEntry layout");
static_assert(sizeof(pt_punctual_light) == sizeof(PunctualLight) && sizeof(pt_punctual_light) == 48, "PunctualLight layout");
static_assert(sizeof(pt_camera) == sizeof(CameraView) && sizeof(pt_camera) == 64, "CameraView layout");
static_assert(offsetof(pt_camera, focus_distance) == offsetof(CameraView, focus_distance), "CameraView layout");

namespace {

struct RefScene {
    Scene scene;
    pt_scene_desc desc{};
    pt_raw_scene raw{};
    std::vector<pt_texture_desc> tex_descs;
};

void fill_desc(RefScene& r) {
    const Scene& s = r.scene;
    pt_scene_desc& d = r.desc;
    d = pt_scene_desc{};
    d.nodes = reinterpret_cast<const pt_bvh_node*>(s.bvh.nodes.data());
    d.num_nodes = int32_t(s.bvh.nodes.size());
    d.tris = reinterpret_cast<const pt_tri_geom*>(s.tris.data());
    d.num_tris = int32_t(s.tris.size());
    d.indices = s.bvh_indices.data();
    d.normals = s.normals.empty() ? nullptr : reinterpret_cast<const pt_vec3*>(s.normals.data());
    d.uvs = s.uvs.empty() ? nullptr : reinterpret_cast<const pt_vec2*>(s.uvs.data());
    d.tangents = s.tangents.empty() ? nullptr : reinterpret_cast<const pt_vec4*>(s.tangents.data());
    d.num_vertices = int32_t(s.positions.size());
    d.materials = reinterpret_cast<const pt_material*>(s.materials.data());
    d.num_materials = int32_t(s.materials.size());
    d.textures = reinterpret_cast<const pt_texture_info*>(s.texture_infos.data());
    d.num_textures = int32_t(s.texture_infos.size());
    d.texels = s.texel_pool.data();
    d.num_texels = s.texel_pool.size();
    d.srgb_lut = s.srgb_lut.data();
    d.emissive = reinterpret_cast<const pt_emissive_tri*>(s.emissive.data());
    d.num_emissive = int32_t(s.emissive.size());
    d.tri_emissive = s.tri_emissive.data();
    d.emissive_alias = reinterpret_cast<const pt_alias_entry*>(s.emissive_alias.data());
    d.emissive_power = s.emissive_power;
    d.punctual = reinterpret_cast<const pt_punctual_light*>(s.punctual.data());
    d.num_punctual = int32_t(s.punctual.size());
    d.env_texels = s.env.texels.empty() ? nullptr : reinterpret_cast<const pt_vec3*>(s.env.texels.data());
    d.env_width = s.env.width;
    d.env_height = s.env.height;
    d.env_marginal = s.env_marginal.empty() ? nullptr : s.env_marginal.data();
    d.env_conditional = s.env_conditional.empty() ? nullptr : s.env_conditional.data();
    d.env_intensity = s.env.intensity;
    d.env_rotation = s.env.rotation;
    d.env_color = {s.env.color.x, s.env.color.y, s.env.color.z};
    d.env_integral = s.env_integral;
    d.p_env = s.p_env;
    d.p_emissive = s.p_emissive;
    d.p_punctual = s.p_punctual;
    d.bounds_min = {s.bvh.bounds.min.x, s.bvh.bounds.min.y, s.bvh.bounds.min.z};
    d.bounds_max = {s.bvh.bounds.max.x, s.bvh.bounds.max.y, s.bvh.bounds.max.z};
}

void fill_raw(RefScene& r) {
    const Scene& s = r.scene;
    pt_raw_scene& w = r.raw;
    w = pt_raw_scene{};
    w.positions = reinterpret_cast<const pt_vec3*>(s.positions.data());
    w.num_positions = int32_t(s.positions.size());
    w.normals = s.normals.empty() ? nullptr : reinterpret_cast<const pt_vec3*>(s.normals.data());
    w.uvs = s.uvs.empty() ? nullptr : reinterpret_cast<const pt_vec2*>(s.uvs.data());
    w.tangents = s.tangents.empty() ? nullptr : reinterpret_cast<const pt_vec4*>(s.tangents.data());
    w.indices = s.indices.data();
    w.num_indices = int32_t(s.indices.size());
    w.tri_material = s.tri_material.data();
    w.materials = reinterpret_cast<const pt_material*>(s.materials.data());
    w.num_materials = int32_t(s.materials.size());
    r.tex_descs.clear();
    for (const Texture& t : s.textures) r.tex_descs.push_back({t.width, t.height, t.texels.data(), t.repeat ? 1 : 0, t.srgb ? 1 : 0});
    w.textures = r.tex_descs.data();
    w.num_textures = int32_t(r.tex_descs.size());
    w.punctual = reinterpret_cast<const pt_punctual_light*>(s.punctual.data());
    w.num_punctual = int32_t(s.punctual.size());
    w.env_texels = s.env.texels.empty() ? nullptr : reinterpret_cast<const pt_vec3*>(s.env.texels.data());
    w.env_width = s.env.width;
    w.env_height = s.env.height;
    w.env_color = {s.env.color.x, s.env.color.y, s.env.color.z};
    w.env_intensity = s.env.intensity;
    w.env_rotation = s.env.rotation;
}

template <typename T, typename U>
std::vector<T> copy_array(const U* p, size_t n) {
    std::vector<T> v(n);
    if (n && p) std::memcpy(v.data(), p, n * sizeof(T));
    static_assert(sizeof(T) == sizeof(U), "element size");
    return v;
}

// A Photon Scene whose built arrays are a copy of a pt_scene_desc (so CpuRenderer can render a
// scene built by any builder; Photon's renderer only reads Scene::view()).
void scene_from_desc(Scene& s, const pt_scene_desc* d) {
    s = Scene();
    s.bvh.nodes = copy_array<BvhNode>(d->nodes, size_t(d->num_nodes));
    s.tris = copy_array<TriGeom>(d->tris, size_t(d->num_tris));
    s.bvh_indices = copy_array<int>(d->indices, size_t(d->num_tris) * 3);
    if (d->normals) s.normals = copy_array<vec3>(d->normals, size_t(d->num_vertices));
    if (d->uvs) s.uvs = copy_array<vec2>(d->uvs, size_t(d->num_vertices));
    if (d->tangents) s.tangents = copy_array<vec4>(d->tangents, size_t(d->num_vertices));
    s.positions.assign(size_t(d->num_vertices), vec3(0));
    s.materials = copy_array<Material>(d->materials, size_t(d->num_materials));
    s.texture_infos = copy_array<TextureInfo>(d->textures, size_t(d->num_textures));
    s.texel_pool = copy_array<uint32_t>(d->texels, size_t(d->num_texels));
    s.srgb_lut = copy_array<float>(d->srgb_lut, 256);
    s.emissive = copy_array<EmissiveTri>(d->emissive, size_t(d->num_emissive));
    s.tri_emissive = copy_array<int>(d->tri_emissive, d->tri_emissive ? size_t(d->num_tris) : 0);
    s.emissive_alias = copy_array<AliasEntry>(d->emissive_alias, size_t(d->num_emissive));
    s.emissive_power = d->emissive_power;
    s.punctual = copy_array<PunctualLight>(d->punctual, size_t(d->num_punctual));
    if (d->env_texels) s.env.texels = copy_array<vec3>(d->env_texels, size_t(d->env_width) * size_t(d->env_height));
    s.env.width = d->env_width;
    s.env.height = d->env_height;
    if (d->env_marginal) s.env_marginal = copy_array<float>(d->env_marginal, size_t(d->env_height) + 1);
    if (d->env_conditional)
        s.env_conditional = copy_array<float>(d->env_conditional, size_t(d->env_height) * size_t(d->env_width + 1));
    s.env.intensity = d->env_intensity;
    s.env.rotation = d->env_rotation;
    s.env.color = vec3(d->env_color.x, d->env_color.y, d->env_color.z);
    s.env_integral = d->env_integral;
    s.p_env = d->p_env;
    s.p_emissive = d->p_emissive;
    s.p_punctual = d->p_punctual;
    s.bvh.bounds.min = vec3(d->bounds_min.x, d->bounds_min.y, d->bounds_min.z);
    s.bvh.bounds.max = vec3(d->bounds_max.x, d->bounds_max.y, d->bounds_max.z);
    s.built = true;
}

CameraView to_view(const pt_camera* c) {
    CameraView v;
    std::memcpy(&v, c, sizeof(v));
    return v;
}

RenderSettings to_settings(const pt_render_settings* s) {
    RenderSettings r;
    r.width = s->width;
    r.height = s->height;
    r.path.max_depth = s->path.max_depth;
    r.path.rr_depth = s->path.rr_depth;
    r.path.clamp = s->path.clamp;
    r.path.nee = s->path.nee;
    r.path.ray_count = nullptr;
    r.exposure = s->exposure;
    r.tonemap = ToneMap(s->tonemap);
    r.seed = s->seed;
    return r;
}

}  // namespace

extern "C" {

// ---- scenes ---------------------------------------------------------------------------------

// Photon's built-in scene `name` ("cornell", "materials", "glass", "furnace"), built by Scene::build.
// flat_normals = 1 clears the vertex normals first (as test_render.cpp:37 does for the furnace).
void* ref_builtin_scene(const char* name, int flat_normals) {
    auto r = std::make_unique<RefScene>();
    if (!make_builtin_scene(name, r->scene)) return nullptr;
    if (flat_normals) r->scene.normals.clear();
    fill_raw(*r);
    r->scene.build();
    fill_desc(*r);
    fill_raw(*r);
    return r.release();
}

}  // extern "C"

namespace {

// Photon's Scene from raw meshes, built by Scene::build (its BVH builder and light tables).
void build_from_raw(RefScene& r, const pt_raw_scene* w, int bins, int max_leaf, int threads) {
    Scene& s = r.scene;
    s.positions = copy_array<vec3>(w->positions, size_t(w->num_positions));
    if (w->normals) s.normals = copy_array<vec3>(w->normals, size_t(w->num_positions));
    if (w->uvs) s.uvs = copy_array<vec2>(w->uvs, size_t(w->num_positions));
    if (w->tangents) s.tangents = copy_array<vec4>(w->tangents, size_t(w->num_positions));
    s.indices = copy_array<int>(w->indices, size_t(w->num_indices));
    s.tri_material = copy_array<int>(w->tri_material, size_t(w->num_indices) / 3);
    s.materials = copy_array<Material>(w->materials, size_t(w->num_materials));
    for (int i = 0; i < w->num_textures; i++) {
        const pt_texture_desc& t = w->textures[i];
        Texture tex;
        tex.width = t.width;
        tex.height = t.height;
        tex.texels.assign(t.texels, t.texels + size_t(t.width) * size_t(t.height));
        tex.repeat = t.repeat != 0;
        tex.srgb = t.srgb != 0;
        s.textures.push_back(std::move(tex));
    }
    s.punctual = copy_array<PunctualLight>(w->punctual, size_t(w->num_punctual));
    if (w->env_texels) s.env.texels = copy_array<vec3>(w->env_texels, size_t(w->env_width) * size_t(w->env_height));
    s.env.width = w->env_width;
    s.env.height = w->env_height;
    s.env.color = vec3(w->env_color.x, w->env_color.y, w->env_color.z);
    s.env.intensity = w->env_intensity;
    s.env.rotation = w->env_rotation;
    BvhBuildOptions opt;
    if (bins > 0) opt.bins = bins;
    if (max_leaf > 0) opt.max_leaf_size = max_leaf;
    opt.threads = threads;
    s.build(opt);
    fill_desc(r);
    fill_raw(r);
}

}  // namespace

extern "C" {

// A raw scene built by Photon's Scene::build (its BVH builder and light tables).
void* ref_scene_from_raw(const pt_raw_scene* w, int bins, int max_leaf, int threads) {
    auto r = std::make_unique<RefScene>();
    build_from_raw(*r, w, bins, max_leaf, threads);
    return r.release();
}

// A procedural scene of the benchmark workloads (kind PT_GEN_BOX or PT_GEN_TERRAIN, triangle count,
// seed): the generator's raw meshes, built by Photon's Scene::build with `threads` builder threads
// (0: all). The scene's camera is the generator's look-at camera, so ref_scene_camera gives Photon's
// Camera::view of it. Returns NULL if the generator rejects the arguments.
void* ref_generated_scene(int kind, int64_t triangles, uint64_t seed, int threads) {
    ptw::GeneratedScene g;
    try {
        ptw::generate_scene(kind, triangles, seed, g);
    } catch (const ptw::Error&) {
        return nullptr;
    }
    auto r = std::make_unique<RefScene>();
    build_from_raw(*r, &g.raw, 0, 0, threads);
    Camera& c = r->scene.camera;
    c.position = vec3(g.cam_pos.x, g.cam_pos.y, g.cam_pos.z);
    c.target = vec3(g.cam_target.x, g.cam_target.y, g.cam_target.z);
    c.up = vec3(g.cam_up.x, g.cam_up.y, g.cam_up.z);
    c.vfov = g.vfov_deg;
    c.aperture = 0.0f;
    c.focus_distance = 0.0f;
    return r.release();
}

// The generator's raw arrays alone (no build), for checking that this library's copy of the
// generator produces what the product library's pt_generate_scene produces. Free with
// ref_generated_raw_free.
void* ref_generated_raw(int kind, int64_t triangles, uint64_t seed, const pt_raw_scene** raw) {
    auto g = std::make_unique<ptw::GeneratedScene>();
    try {
        ptw::generate_scene(kind, triangles, seed, *g);
    } catch (const ptw::Error&) {
        return nullptr;
    }
    *raw = &g->raw;
    return g.release();
}
void ref_generated_raw_free(void* g) { delete static_cast<ptw::GeneratedScene*>(g); }

// A scene whose built arrays are copied from a description (any builder).
void* ref_scene_from_desc(const pt_scene_desc* d) {
    auto r = std::make_unique<RefScene>();
    scene_from_desc(r->scene, d);
    fill_desc(*r);
    return r.release();
}

void ref_scene_free(void* h) { delete static_cast<RefScene*>(h); }
// The photon::Scene object itself (for the GPU shim, which uploads it with GpuRenderer::upload).
const void* ref_scene_object(void* h) { return &static_cast<RefScene*>(h)->scene; }
const pt_scene_desc* ref_scene_desc(void* h) { return &static_cast<RefScene*>(h)->desc; }
const pt_raw_scene* ref_scene_raw(void* h) { return &static_cast<RefScene*>(h)->raw; }

void ref_scene_camera(void* h, float aspect, pt_camera* out) {
    CameraView v = static_cast<RefScene*>(h)->scene.camera.view(aspect);
    std::memcpy(out, &v, sizeof(v));
}

// Camera::view (scene.cpp:13-25) of an arbitrary look-at camera.
void ref_camera_view(const float* position, const float* target, const float* up, float vfov_deg, float aperture,
                     float focus_distance, float aspect, pt_camera* out) {
    Camera c;
    c.position = vec3(position[0], position[1], position[2]);
    c.target = vec3(target[0], target[1], target[2]);
    c.up = vec3(up[0], up[1], up[2]);
    c.vfov = vfov_deg;
    c.aperture = aperture;
    c.focus_distance = focus_distance;
    CameraView v = c.view(aspect);
    std::memcpy(out, &v, sizeof(v));
}

// BvhStats of a scene built by Photon (nodes, leaves, max depth, SAH cost, build ms).
void ref_bvh_stats(void* h, int* nodes, int* leaves, int* depth, float* sah, double* build_ms) {
    const BvhStats& st = static_cast<RefScene*>(h)->scene.bvh.stats;
    *nodes = st.nodes;
    *leaves = st.leaves;
    *depth = st.max_depth;
    *sah = st.sah_cost;
    *build_ms = st.build_ms;
}

// ---- rendering ------------------------------------------------------------------------------

// CpuRenderer::render of `spp` samples starting at sample index 0; writes the average radiance
// (3 floats per pixel). threads = 0 uses every hardware thread. Returns the seconds taken.
double ref_render(void* h, const pt_camera* cam, const pt_render_settings* rs, int spp, int threads, float* rgb) {
    RefScene& r = *static_cast<RefScene*>(h);
    CpuRenderer cpu(r.scene);
    cpu.resize(rs->width, rs->height);
    auto t0 = std::chrono::steady_clock::now();
    cpu.render(to_view(cam), to_settings(rs), spp, threads);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rgb) {
        std::vector<vec3> img = cpu.image();
        std::memcpy(rgb, img.data(), img.size() * sizeof(vec3));
    }
    return secs;
}

// The radiance of single samples: for each of n (x, y, frame) triples, render_sample's result.
void ref_render_samples(void* h, const pt_camera* cam, const pt_render_settings* rs, int n, const int* xyf, float* L3) {
    RefScene& r = *static_cast<RefScene*>(h);
    SceneView v = r.scene.view();
    CameraView c = to_view(cam);
    RenderSettings s = to_settings(rs);
    for (int i = 0; i < n; i++) {
        vec3 L = render_sample(v, c, xyf[3 * i], xyf[3 * i + 1], s.width, s.height, uint32_t(xyf[3 * i + 2]), s.seed, s.path, nullptr);
        L3[3 * i] = L.x;
        L3[3 * i + 1] = L.y;
        L3[3 * i + 2] = L.z;
    }
}

// Rays per sample as `photon bench` measures them (render_cli.cpp:307-318): every 7th pixel,
// sample 0, seed 0, counting camera, extension and shadow rays.
double ref_rays_per_sample(void* h, const pt_camera* cam, const pt_render_settings* rs) {
    RefScene& r = *static_cast<RefScene*>(h);
    SceneView sv = r.scene.view();
    CameraView c = to_view(cam);
    uint32_t rays = 0;
    PathOptions po = to_settings(rs).path;
    po.ray_count = &rays;
    int n = 0;
    for (int y = 0; y < rs->height; y += 7)
        for (int x = (y / 7) % 7; x < rs->width; x += 7, n++) render_sample(sv, c, x, y, rs->width, rs->height, 0, 0, po, nullptr);
    return double(rays) / std::max(n, 1);
}

// Primary closest hits: the camera ray of render_sample (pixel.h:20-24) for sample `frame`,
// intersected by Photon's traversal. Per pixel (t, tri as int bits, u, v).
void ref_trace_primary(void* h, const pt_camera* cam, int w, int hgt, uint32_t frame, uint32_t seed, float* hits4) {
    RefScene& r = *static_cast<RefScene*>(h);
    SceneView s = r.scene.view();
    CameraView c = to_view(cam);
    for (int y = 0; y < hgt; y++)
        for (int x = 0; x < w; x++) {
            uint32_t pixel = uint32_t(y) * uint32_t(w) + uint32_t(x);
            Rng rng(hash_u32(pixel ^ hash_u32(seed)) | (uint64_t(hash_u32(frame + 0x9e3779b9u)) << 32), pixel);
            vec2 jitter = rng.next2();
            vec2 lens = rng.next2();
            Ray ray = camera_ray(c, float(x) + jitter.x, float(y) + jitter.y, w, hgt, lens);
            Hit hit;
            intersect(s, ray, hit);
            float* o = hits4 + 4 * size_t(pixel);
            o[0] = hit.t;
            std::memcpy(&o[1], &hit.tri, 4);
            o[2] = hit.u;
            o[3] = hit.v;
        }
}

// The light pick at the first path vertex (integrator.h:199-209 → lights.h:139-202), recomputed
// with Photon's own sample_alias / find_interval from the same random numbers.
void ref_light_picks_primary(void* h, const pt_camera* cam, const pt_render_settings* rs, uint32_t frame, int* picks4) {
    RefScene& r = *static_cast<RefScene*>(h);
    SceneView s = r.scene.view();
    CameraView c = to_view(cam);
    RenderSettings st = to_settings(rs);
    int w = rs->width, hgt = rs->height;
    bool has_lights = s.p_env + s.p_emissive + s.p_punctual > 0;
    for (int y = 0; y < hgt; y++)
        for (int x = 0; x < w; x++) {
            uint32_t pixel = uint32_t(y) * uint32_t(w) + uint32_t(x);
            int* o = picks4 + 4 * size_t(pixel);
            o[0] = -1;
            o[1] = -1;
            o[2] = -1;
            o[3] = 0;
            Rng rng(hash_u32(pixel ^ hash_u32(st.seed)) | (uint64_t(hash_u32(frame + 0x9e3779b9u)) << 32), pixel);
            vec2 jitter = rng.next2();
            vec2 lens = rng.next2();
            Ray ray = camera_ray(c, float(x) + jitter.x, float(y) + jitter.y, w, hgt, lens);
            Hit hit;
            if (!intersect(s, ray, hit)) continue;
            Interaction it = surface_at(s, ray, hit);
            Bsdf bsdf(it.params);
            if (1 >= st.path.max_depth) continue;
            bool nee = st.path.nee && has_lights && bsdf.samples_lights();
            if (!nee) continue;
            float ug = rng.next();
            vec2 ul = rng.next2();
            float uk = rng.next();
            o[3] = 1;
            if (ug < s.p_emissive && s.num_emissive > 0) {
                float x0 = uk * float(s.num_emissive);
                int bin = int(x0);
                if (bin >= s.num_emissive) bin = s.num_emissive - 1;
                float pmf;
                o[0] = 0;
                o[1] = sample_alias(s.emissive_alias, s.num_emissive, uk, &pmf);
                o[2] = bin;
            } else if (ug < s.p_emissive + s.p_punctual && s.num_punctual > 0) {
                int k = int(uk * float(s.num_punctual));
                if (k >= s.num_punctual) k = s.num_punctual - 1;
                o[0] = 1;
                o[1] = k;
            } else if (s.p_env > 0) {
                o[0] = 2;
                if (s.env.texels) {
                    int yy = find_interval(s.env.marginal_cdf, s.env.height, ul.y);
                    const float* row = s.env.conditional_cdf + yy * (s.env.width + 1);
                    int xx = find_interval(row, s.env.width, ul.x);
                    o[1] = yy * s.env.width + xx;
                }
            }
        }
}

// Photon's any-hit walk (traverse<true>, traverse.h:66-138, as occluded calls it at :144-147) of n
// rays (origin, tmax, direction, unused): (occluded, the accepted triangle or -1, node visits, 0).
void ref_occluded(void* h, const float* rays8, int n, int32_t* out4) {
    RefScene& r = *static_cast<RefScene*>(h);
    SceneView s = r.scene.view();
    for (int i = 0; i < n; i++) {
        const float* q = rays8 + 8 * size_t(i);
        Ray ray;
        ray.o = vec3(q[0], q[1], q[2]);
        ray.tmax = q[3];
        ray.d = vec3(q[4], q[5], q[6]);
        Hit hit;
        int visits = 0;
        const bool occ = traverse<true>(s, ray, hit, &visits);
        out4[4 * i] = occ ? 1 : 0;
        out4[4 * i + 1] = occ ? hit.tri : -1;
        out4[4 * i + 2] = visits;
        out4[4 * i + 3] = 0;
    }
}

// BVH node visits of the primary ray through each pixel centre (gpu_renderer.cu:98-106).
void ref_heatmap(void* h, const pt_camera* cam, int w, int hgt, float* out) {
    RefScene& r = *static_cast<RefScene*>(h);
    SceneView s = r.scene.view();
    CameraView c = to_view(cam);
    for (int y = 0; y < hgt; y++)
        for (int x = 0; x < w; x++) {
            Ray ray = camera_ray(c, float(x) + 0.5f, float(y) + 0.5f, w, hgt, vec2(0.5f, 0.5f));
            Hit hit;
            int visits = 0;
            intersect(s, ray, hit, &visits);
            out[size_t(y) * size_t(w) + size_t(x)] = float(visits);
        }
}

// display_kernel's per-pixel mapping (gpu_renderer.cu:129-175) evaluated on the host with Photon's own
// host-compiled colour functions (color.h:8-41: tone_map, srgb_to_linear, pack_rgba8; math.h:
// luminance, saturate, lerp) and heat_color's ramp (gpu_renderer.cu:108-115): the CPU side of the
// display comparison, against which Photon's --use_fast_math device build and the wavefront's display
// kernel are both measured. Arguments as refgpu_display_buffers (host arrays).
void ref_display_cpu(int w, int h, int mode, float exposure, int tonemap, float samples, float max_depth, float heat_scale, int denoised,
                     const float* accum4, const float* denoised4, const float* albedo4, const float* normal_depth4,
                     const float* variance4, const float* heat, uint32_t* out) {
    const float inv_samples = samples > 0 ? 1.0f / samples : 0.0f;
    auto v4 = [](const float* b, size_t i) { return b ? vec4(b[4 * i], b[4 * i + 1], b[4 * i + 2], b[4 * i + 3]) : vec4(0, 0, 0, 0); };
    auto heat_color = [](float t) {
        t = saturate(t);
        vec3 c0(0.05f, 0.05f, 0.35f), c1(0.0f, 0.6f, 0.4f), c2(0.95f, 0.85f, 0.1f), c3(0.85f, 0.1f, 0.05f);
        if (t < 1.0f / 3) return lerp(c0, c1, t * 3);
        if (t < 2.0f / 3) return lerp(c1, c2, t * 3 - 1);
        return lerp(c2, c3, t * 3 - 2);
    };
    for (size_t i = 0; i < size_t(w) * size_t(h); i++) {
        vec3 c;
        switch (mode) {
            default:
            case 0:
                c = denoised ? v4(denoised4, i).xyz() : v4(accum4, i).xyz() * inv_samples;
                c = tone_map(c, exposure, ToneMap(tonemap));
                break;
            case 1: c = v4(albedo4, i).xyz(); break;
            case 2: {
                vec4 nd = v4(normal_depth4, i);
                c = nd.w > 0 ? nd.xyz() * 0.5f + vec3(0.5f) : vec3(0);
                break;
            }
            case 3: {
                float d = v4(normal_depth4, i).w;
                c = d > 0 ? vec3(1.0f - saturate(d / max_depth)) : vec3(0);
                break;
            }
            case 4: {
                float v;
                if (denoised) {
                    v = v4(variance4, i).w;
                } else {
                    vec4 a = v4(accum4, i);
                    float mean = luminance(a.xyz()) * inv_samples;
                    v = samples > 1 ? std::fmax(0.0f, a.w * inv_samples - mean * mean) / (samples - 1) : 0.0f;
                }
                float t = std::sqrt(v);
                c = vec3(t / (1.0f + t));
                break;
            }
            case 5: c = heat_color((heat ? heat[i] : 0.0f) * heat_scale); break;
        }
        if (mode != 0 && mode != 1) c = vec3(srgb_to_linear(c.x), srgb_to_linear(c.y), srgb_to_linear(c.z));
        out[i] = pack_rgba8(c);
    }
}

// Photon's build_alias_table (scene.cpp:82-111) on a weight list (for known-answer tests).
void ref_alias_table(const float* weights, int n, pt_alias_entry* out) {
    std::vector<float> w(weights, weights + n);
    std::vector<AliasEntry> t = build_alias_table(w);
    std::memcpy(out, t.data(), t.size() * sizeof(AliasEntry));
}

// Photon's PCG32 (sampling.h:9-34): n floats of stream (seed, stream).
void ref_rng_floats(uint64_t seed, uint64_t stream, int n, float* out) {
    Rng rng(seed, stream);
    for (int i = 0; i < n; i++) out[i] = rng.next();
}

// offset_ray (integrator.h:61-69) on n points and normals (3 floats each).
void ref_offset_ray(int n, const float* p, const float* nrm, float* out) {
    for (int i = 0; i < n; i++) {
        vec3 q = offset_ray(vec3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), vec3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]));
        out[3 * i] = q.x;
        out[3 * i + 1] = q.y;
        out[3 * i + 2] = q.z;
    }
}

// Bsdf::sample (bsdf.h:255-281) of one parameter set on n (wo, u_lobe, u.x, u.y, u_sub) rows.
// Output per row: wi (3), f (3), pdf, transmitted, valid.
void ref_bsdf_sample(const float* params7, int n, const float* rows8, float* out9) {
    BsdfParams p;
    p.base = vec3(params7[0], params7[1], params7[2]);
    p.metallic = params7[3];
    p.roughness = params7[4];
    p.transmission = params7[5];
    p.ior = params7[6];
    Bsdf b(p);
    for (int i = 0; i < n; i++) {
        const float* r = rows8 + 8 * i;
        BsdfSample s = b.sample(vec3(r[0], r[1], r[2]), r[3], vec2(r[4], r[5]), r[6]);
        float* o = out9 + 9 * i;
        o[0] = s.wi.x;
        o[1] = s.wi.y;
        o[2] = s.wi.z;
        o[3] = s.f.x;
        o[4] = s.f.y;
        o[5] = s.f.z;
        o[6] = s.pdf;
        o[7] = s.transmitted ? 1.0f : 0.0f;
        o[8] = s.valid ? 1.0f : 0.0f;
    }
}

}  // extern "C"
