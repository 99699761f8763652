// A 4-wide BVH collapsed from Photon's BVH2 (same leaves, same boxes) for any-hit (shadow) rays.
#pragma once

#include <cstdint>
#include <vector>

#include "photon_wavefront.h"

namespace ptw {

// 128 bytes: the four child boxes as SoA rows (x/y/z lows, x/y/z highs), then per child the index
// (a node of this BVH, or the first triangle of a leaf) and the triangle count (0: an interior child;
// an unused slot has index -1).
struct Bvh4Node {
    float lox[4], loy[4], loz[4], hix[4], hiy[4], hiz[4];
    int32_t idx[4], cnt[4];
};
static_assert(sizeof(Bvh4Node) == 128, "Bvh4Node layout");

constexpr int kBvh4StackSize = 96;  // entries per ray; a build deeper than the stack allows is rejected

// Collapses the BVH2 `nodes` (Photon's depth-first layout, root 0): each 4-wide node takes a BVH2 node's
// children, replacing each interior child by its own two children. Every 4-wide child box is a box of
// the BVH2, so a ray reaches exactly the leaves it reaches in the BVH2 (a box test that passes for a
// box also passes for every box containing it: the slab arithmetic is monotone in the bounds).
// Returns false (and leaves `out` empty) when the tree cannot be walked within kBvh4StackSize or a
// leaf does not fit the traversal's leaf encoding (at most 127 triangles, indices below 2^24).
bool build_bvh4(const pt_bvh_node* nodes, int32_t num_nodes, int32_t num_tris, std::vector<Bvh4Node>& out, int* depth_out);

}  // namespace ptw
