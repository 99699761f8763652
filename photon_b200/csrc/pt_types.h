// Plain structures shared by host and device code (no device functions), so host-only
// translation units can fill them.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ptw {

// Scene arrays on the device. Layouts (all 16-byte aligned):
//   nodes     4 x float4 per node: (lmin, left) (lmax, lcount) (rmin, right) (rmax, rcount)
//   tris      kTriStride (4) x float4 per triangle: (v0, material) (e1, flags) (e2, pad) (the vertex
//             indices as int bits, 0) [BVH order]; 64 bytes each: the intersection test reads the
//             first 48 with a 256-bit and a 128-bit load, the alpha test the indices from the same line
//   tri_idx   int4 per triangle: (vertex 0, vertex 1, vertex 2, emissive entry or -1)
//   normals   float4 per vertex (n, 0);  uvs float2 per vertex;  tangents float4 per vertex
//   materials 5 x float4 per material: Photon's 80-byte Material read as five 16-byte words
//   textures  int4 per texture: (width, height, texel offset, repeat | srgb << 1)
//   env       float4 per texel (rgb, luminance), row_sin per row, rotation cos/sin precomputed
// float4 records per triangle in DevScene::tris (Photon's 48-byte TriGeom padded to 64 bytes).
constexpr int kTriStride = 4;

struct DevScene {
    const float4* nodes;
    const float4* nodes4;     // the 4-wide BVH for any-hit rays (8 float4 per node), or null
    const float4* tris;
    const int4* tri_idx;
    const float4* normals;
    const float2* uvs;
    const float4* tangents;
    const float4* materials;
    const uint8_t* shade_keys;  // per material: its shading class (1..32) for the material-sorted shade
    const int4* textures;
    const uint32_t* texels;
    const float* srgb_lut;
    const int2* emissive;       // (triangle, area bits)
    const float4* alias;        // (prob, alias bits, pmf, 0)
    const float4* punctual;     // 3 x float4: (position, type) (direction, cos_inner) (intensity, cos_outer)
    const float4* env_texels;
    const float* env_marginal;
    const float* env_conditional;
    const float* env_row_sin;
    int num_tris, num_nodes, num_emissive, num_punctual;
    int env_width, env_height;
    float env_intensity, env_integral;
    float env_cos_neg, env_sin_neg, env_cos_pos, env_sin_pos;  // cosf/sinf of -rotation and +rotation
    float env_color_x, env_color_y, env_color_z;
    float p_env, p_emissive, p_punctual;
    int has_lights;
    int bvh_depth;
    float bounds_lo_x, bounds_lo_y, bounds_lo_z;   // scene box (for ray-sort keys)
    float inv_extent_x, inv_extent_y, inv_extent_z;
};

}  // namespace ptw
