// The binned-SAH BVH build of scene_build.cpp on the device: the same decisions (bins, SAH sweeps,
// leaf rule, depth limit) and the same in-place partition, so the tree and the triangle order are
// the host builder's, bit for bit, in a fraction of the time for large scenes.
#pragma once

#include <vector>

namespace ptw {

// One node of the built tree: its box, its range of `order` (leaves) and its children (-1: leaf).
struct FlatBuildNode {
    float lo[3], hi[3];
    int first, count;
    int kid[2];
};

// boxes: 6 floats per primitive (lo xyz, hi xyz); cent: 3 floats per primitive. Fills `order` (the
// primitive permutation) and `nodes` (node 0 is the root). Throws Error on a CUDA failure.
void gpu_build_bvh(int device, const std::vector<float>& boxes, const std::vector<float>& cent, int n, int bins, int max_leaf,
                   float traversal_cost, std::vector<int>& order, std::vector<FlatBuildNode>& nodes);

}  // namespace ptw
