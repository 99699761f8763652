// Host-side scene construction: raw meshes -> the arrays of pt_scene_desc, and the procedural
// scenes of the benchmark configurations.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "photon_wavefront.h"

namespace ptw {

struct BvhOptions {
    int bins = 32;             // SAH candidate planes per axis
    int max_leaf = 8;          // leaves never hold more triangles
    float traversal_cost = 1.0f;
    int threads = 0;           // 0: hardware concurrency
    bool gpu = false;          // build on the current CUDA device (the same tree)
};

struct BvhInfo {
    int nodes = 0, leaves = 0, max_depth = 0;
    float sah_cost = 0;
    double build_ms = 0;
};

// Owns the built arrays; `desc` points into them.
struct BuiltScene {
    std::vector<pt_bvh_node> nodes;
    std::vector<pt_tri_geom> tris;
    std::vector<int32_t> indices;
    std::vector<pt_vec3> normals;
    std::vector<pt_vec2> uvs;
    std::vector<pt_vec4> tangents;
    int32_t num_vertices = 0;
    std::vector<pt_material> materials;
    std::vector<pt_texture_info> textures;
    std::vector<uint32_t> texels;
    std::vector<float> srgb_lut;
    std::vector<pt_emissive_tri> emissive;
    std::vector<int32_t> tri_emissive;
    std::vector<pt_alias_entry> alias;
    std::vector<pt_punctual_light> punctual;
    std::vector<pt_vec3> env_texels;
    std::vector<float> env_marginal, env_conditional;
    pt_scene_desc desc{};
    BvhInfo bvh;
};

void build_scene(const pt_raw_scene& raw, const BvhOptions& opt, BuiltScene& out);

// Walker/Vose alias table of a weight list (pmf exact per entry).
std::vector<pt_alias_entry> alias_table(const std::vector<float>& weights);

// A generated raw scene (owning storage) and its camera.
struct GeneratedScene {
    std::vector<pt_vec3> positions, normals;
    std::vector<pt_vec2> uvs;
    std::vector<int32_t> indices, tri_material;
    std::vector<pt_material> materials;
    std::vector<std::vector<uint32_t>> texture_data;
    std::vector<pt_texture_desc> textures;
    std::vector<pt_punctual_light> punctual;
    std::vector<pt_vec3> env;
    int env_w = 0, env_h = 0;
    pt_vec3 env_color{0, 0, 0};
    float env_intensity = 1.0f;
    pt_raw_scene raw{};
    // Look-at camera.
    pt_vec3 cam_pos{0, 0, 5}, cam_target{0, 0, 0}, cam_up{0, 1, 0};
    float vfov_deg = 45.0f;
    pt_camera camera_view(float aspect) const;
    void finalize();
};

void generate_scene(int kind, int64_t triangles, uint64_t seed, GeneratedScene& out);

}  // namespace ptw
