// Collapse of Photon's BVH2 into a 4-wide BVH for any-hit rays (host side).
#include "wide_bvh.h"

#include <algorithm>
#include <limits>

namespace ptw {

namespace {

struct Slot {
    float lo[3], hi[3];
    int32_t idx, cnt;  // BVH2 node index (cnt 0) or leaf
};

void child_slots(const pt_bvh_node& n, Slot out[2], int& k) {
    k = 0;
    const int32_t idx[2] = {n.left, n.right}, cnt[2] = {n.lcount, n.rcount};
    const pt_vec3 lo[2] = {n.lmin, n.rmin}, hi[2] = {n.lmax, n.rmax};
    for (int c = 0; c < 2; c++) {
        if (cnt[c] <= 0 && idx[c] < 0) continue;  // empty child
        Slot s{{lo[c].x, lo[c].y, lo[c].z}, {hi[c].x, hi[c].y, hi[c].z}, idx[c], cnt[c] > 0 ? cnt[c] : 0};
        out[k++] = s;
    }
}

}  // namespace

bool build_bvh4(const pt_bvh_node* nodes, int32_t num_nodes, int32_t num_tris, std::vector<Bvh4Node>& out, int* depth_out) {
    out.clear();
    if (num_nodes < 1 || num_tris >= (1 << 24)) return false;
    // Work list of (BVH2 node, 4-wide node to fill, depth); children get their 4-wide index when queued.
    struct Item {
        int32_t n2, n4, depth;
    };
    std::vector<Item> work{{0, 0, 1}};
    out.emplace_back();
    int max_depth = 1;
    while (!work.empty()) {
        Item it = work.back();
        work.pop_back();
        max_depth = std::max(max_depth, it.depth);
        Slot kids[2];
        int nk = 0;
        child_slots(nodes[it.n2], kids, nk);
        Slot slots[4];
        int ns = 0;
        for (int c = 0; c < nk; c++) {
            if (kids[c].cnt > 0) {
                slots[ns++] = kids[c];
            } else {
                Slot g[2];
                int ng = 0;
                child_slots(nodes[kids[c].idx], g, ng);
                for (int j = 0; j < ng; j++) slots[ns++] = g[j];
            }
        }
        Bvh4Node node;
        const float inf = std::numeric_limits<float>::infinity();
        for (int k = 0; k < 4; k++) {
            node.lox[k] = node.loy[k] = node.loz[k] = inf;
            node.hix[k] = node.hiy[k] = node.hiz[k] = -inf;
            node.idx[k] = -1;
            node.cnt[k] = 0;
        }
        for (int k = 0; k < ns; k++) {
            const Slot& s = slots[k];
            node.lox[k] = s.lo[0];
            node.loy[k] = s.lo[1];
            node.loz[k] = s.lo[2];
            node.hix[k] = s.hi[0];
            node.hiy[k] = s.hi[1];
            node.hiz[k] = s.hi[2];
            if (s.cnt > 0) {
                if (s.cnt > 127) {
                    out.clear();
                    return false;
                }
                node.idx[k] = s.idx;
                node.cnt[k] = s.cnt;
            } else {
                node.idx[k] = int32_t(out.size());
                out.emplace_back();
                work.push_back({s.idx, node.idx[k], it.depth + 1});
            }
        }
        out[size_t(it.n4)] = node;
    }
    // A walk pushes at most four entries per level and pops one.
    if (3 * max_depth + 4 > kBvh4StackSize) {
        out.clear();
        return false;
    }
    if (depth_out) *depth_out = max_depth;
    return true;
}

}  // namespace ptw
