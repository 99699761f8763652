// Scene construction on the host (the role of Photon's Scene::build, src/scene/scene.cpp:212-255):
// a binned-SAH BVH emitted in Photon's 2-child 64-byte node format, triangles re-ordered to BVH
// order, the texel pool, the sRGB table, the emissive-triangle alias table with the light-group
// probabilities, and the environment's 2D sampling distribution. The light tables and the
// environment distribution follow the same definitions as Photon's (scene.cpp:113-210) so that the
// integrator's densities mean the same thing; the BVH is this builder's own (same node semantics,
// its own tree).
#include "scene_build.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <future>
#include <memory>
#include <stdexcept>
#include <condition_variable>
#include <mutex>
#include <thread>

#include "device_scene.h"
#include "gpu_bvh.h"

namespace ptw {

namespace {

constexpr float kPiF = 3.14159265358979323846f;
constexpr float kBig = 1e30f;

struct V3h {
    float x, y, z;
};
inline V3h mk(float x, float y, float z) { return {x, y, z}; }
inline V3h mk(const pt_vec3& v) { return {v.x, v.y, v.z}; }
inline V3h operator+(V3h a, V3h b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3h operator-(V3h a, V3h b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3h operator*(V3h a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3h a, V3h b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3h cross(V3h a, V3h b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float length(V3h a) { return std::sqrt(dot(a, a)); }
inline V3h normalize(V3h a) {
    float l2 = dot(a, a);
    return l2 > 0 ? a * (1.0f / std::sqrt(l2)) : V3h{0, 0, 1};
}
inline pt_vec3 pv(V3h a) { return {a.x, a.y, a.z}; }
inline float lum(V3h c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

struct Box {
    float lo[3] = {kBig, kBig, kBig};
    float hi[3] = {-kBig, -kBig, -kBig};
    void grow(const float* p) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::fmin(lo[k], p[k]);
            hi[k] = std::fmax(hi[k], p[k]);
        }
    }
    void grow(const Box& b) {
        for (int k = 0; k < 3; k++) {
            lo[k] = std::fmin(lo[k], b.lo[k]);
            hi[k] = std::fmax(hi[k], b.hi[k]);
        }
    }
    bool empty() const { return lo[0] > hi[0]; }
    float area() const {
        if (empty()) return 0.0f;
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        return 2.0f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Node {
    Box box;
    int first = 0, count = 0;  // leaf range in `order`
    std::unique_ptr<Node> kid[2];
    bool leaf() const { return !kid[0]; }
};

// A binned-SAH builder (Wald 2007) organised around a task queue: every pending node is a task
// that bins its primitives for all three axes in ONE pass over the range (one bin grid of 3 x B
// cells), picks the cheapest plane from prefix/suffix sweeps, partitions in place and pushes its
// two children as new tasks. Worker threads drain the queue; the tree shape depends only on the
// input (tasks touch disjoint index ranges and write only their own node).
class TaskBvhBuilder {
public:
    TaskBvhBuilder(const std::vector<Box>& boxes, const std::vector<float>& cent, const BvhOptions& opt, std::vector<int>& order)
        : boxes_(boxes), cent_(cent), opt_(opt), order_(order) {
        bins_ = std::max(2, std::min(opt.bins, 64));
        unsigned hc = std::thread::hardware_concurrency();
        workers_ = opt.threads > 0 ? opt.threads : int(hc ? hc : 1);
    }

    std::unique_ptr<Node> run(int n) {
        auto root = std::make_unique<Node>();
        root->first = 0;
        root->count = n;
        push({root.get(), 0});
        std::vector<std::thread> pool;
        int extra = n > 20000 ? workers_ - 1 : 0;
        for (int i = 0; i < extra; i++) pool.emplace_back([this] { drain(); });
        drain();
        for (auto& t : pool) t.join();
        return root;
    }

private:
    struct Task {
        Node* node;
        int depth;
    };
    struct Cell {
        Box box;
        int n = 0;
    };

    void push(Task t) {
        std::lock_guard<std::mutex> g(mu_);
        queue_.push_back(t);
        pending_++;
        cv_.notify_one();
    }

    void drain() {
        for (;;) {
            Task t;
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [this] { return !queue_.empty() || pending_ == 0; });
                if (queue_.empty()) return;
                // Last in, first out: depth-first order keeps the queue short.
                t = queue_.back();
                queue_.pop_back();
            }
            split(t);
            {
                std::lock_guard<std::mutex> g(mu_);
                if (--pending_ == 0) cv_.notify_all();
            }
        }
    }

    void split(Task t) {
        Node* node = t.node;
        const int first = node->first, count = node->count;
        Box cbox;
        for (int i = first; i < first + count; i++) {
            int p = order_[size_t(i)];
            node->box.grow(boxes_[size_t(p)]);
            cbox.grow(&cent_[3 * size_t(p)]);
        }
        if (count <= 1 || t.depth >= 60) return;
        // One pass: bin every primitive on all three axes.
        const int B = bins_;
        Cell grid[3][64];
        float lo[3], scale[3];
        bool usable[3];
        for (int a = 0; a < 3; a++) {
            lo[a] = cbox.lo[a];
            float ext = cbox.hi[a] - cbox.lo[a];
            usable[a] = ext > 1e-12f;
            scale[a] = usable[a] ? float(B) / ext : 0.0f;
        }
        for (int i = first; i < first + count; i++) {
            int p = order_[size_t(i)];
            const float* c = &cent_[3 * size_t(p)];
            for (int a = 0; a < 3; a++) {
                if (!usable[a]) continue;
                int b = std::min(B - 1, int((c[a] - lo[a]) * scale[a]));
                grid[a][b].n++;
                grid[a][b].box.grow(boxes_[size_t(p)]);
            }
        }
        // Suffix sweep (areas and counts right of each plane), then a prefix sweep for the cost.
        const float inv_parent = 1.0f / std::fmax(node->box.area(), 1e-30f);
        float best_cost = kBig;
        int best_axis = -1, best_plane = -1;
        for (int a = 0; a < 3; a++) {
            if (!usable[a]) continue;
            float suffix_area[64];
            int suffix_n[64];
            Box run;
            int cnt = 0;
            for (int b = B - 1; b >= 1; b--) {
                run.grow(grid[a][b].box);
                cnt += grid[a][b].n;
                suffix_area[b] = run.area();
                suffix_n[b] = cnt;
            }
            Box pre;
            int pn = 0;
            for (int plane = 1; plane < B; plane++) {  // plane k splits bins [0, k) | [k, B)
                pre.grow(grid[a][plane - 1].box);
                pn += grid[a][plane - 1].n;
                if (pn == 0 || suffix_n[plane] == 0) continue;
                float c = opt_.traversal_cost + (pre.area() * float(pn) + suffix_area[plane] * float(suffix_n[plane])) * inv_parent;
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_plane = plane;
                }
            }
        }
        const bool forced = count > opt_.max_leaf;
        if (!forced && (best_axis < 0 || best_cost >= float(count))) return;  // a leaf is cheaper
        int mid = first + count / 2;  // degenerate centroids: split the range in half
        if (best_axis >= 0) {
            const int a = best_axis;
            const float l = lo[a], sc = scale[a];
            int* begin = order_.data() + first;
            int* cut = std::partition(begin, begin + count, [&](int p) {
                return std::min(B - 1, int((cent_[3 * size_t(p) + a] - l) * sc)) < best_plane;
            });
            int m = int(cut - order_.data());
            if (m > first && m < first + count) mid = m;
        }
        for (int k = 0; k < 2; k++) {
            node->kid[k] = std::make_unique<Node>();
            node->kid[k]->first = k == 0 ? first : mid;
            node->kid[k]->count = k == 0 ? mid - first : first + count - mid;
        }
        push({node->kid[1].get(), t.depth + 1});
        push({node->kid[0].get(), t.depth + 1});
    }

    const std::vector<Box>& boxes_;
    const std::vector<float>& cent_;
    const BvhOptions& opt_;
    std::vector<int>& order_;
    int bins_ = 32, workers_ = 1;
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<Task> queue_;
    int pending_ = 0;
};

void set_child(pt_bvh_node& n, int side, const Node* c, int out_index) {
    pt_vec3 lo{kBig, kBig, kBig}, hi{-kBig, -kBig, -kBig};
    int idx = -1, cnt = 0;
    if (c) {
        lo = {c->box.lo[0], c->box.lo[1], c->box.lo[2]};
        hi = {c->box.hi[0], c->box.hi[1], c->box.hi[2]};
        idx = c->leaf() ? c->first : out_index;
        cnt = c->leaf() ? c->count : 0;
    }
    if (side == 0) {
        n.lmin = lo;
        n.lmax = hi;
        n.left = idx;
        n.lcount = cnt;
    } else {
        n.rmin = lo;
        n.rmax = hi;
        n.right = idx;
        n.rcount = cnt;
    }
}

// The same flatten over a tree built on the device (gpu_bvh.h).
void set_child_flat(pt_bvh_node& n, int side, const FlatBuildNode* c, int out_index) {
    pt_vec3 lo{kBig, kBig, kBig}, hi{-kBig, -kBig, -kBig};
    int idx = -1, cnt = 0;
    if (c) {
        lo = {c->lo[0], c->lo[1], c->lo[2]};
        hi = {c->hi[0], c->hi[1], c->hi[2]};
        const bool leaf = c->kid[0] < 0;
        idx = leaf ? c->first : out_index;
        cnt = leaf ? c->count : 0;
    }
    if (side == 0) {
        n.lmin = lo;
        n.lmax = hi;
        n.left = idx;
        n.lcount = cnt;
    } else {
        n.rmin = lo;
        n.rmax = hi;
        n.right = idx;
        n.rcount = cnt;
    }
}

float box_area(const float lo[3], const float hi[3]) {
    Box b;
    for (int k = 0; k < 3; k++) {
        b.lo[k] = lo[k];
        b.hi[k] = hi[k];
    }
    return b.area();
}

void flatten_flat(const std::vector<FlatBuildNode>& tree, int n, int out_index, int depth, std::vector<pt_bvh_node>& out, BvhInfo& info,
                  float root_area, float trav) {
    info.nodes++;
    info.max_depth = std::max(info.max_depth, depth);
    for (int side = 0; side < 2; side++) {
        const FlatBuildNode* c = &tree[size_t(tree[size_t(n)].kid[side])];
        const bool leaf = c->kid[0] < 0;
        int child_out = -1;
        if (!leaf) {
            child_out = int(out.size());
            out.push_back(pt_bvh_node{});
            info.sah_cost += trav * box_area(c->lo, c->hi) / root_area;
        } else {
            info.leaves++;
            info.sah_cost += float(c->count) * box_area(c->lo, c->hi) / root_area;
        }
        set_child_flat(out[size_t(out_index)], side, c, child_out);
        if (!leaf) flatten_flat(tree, tree[size_t(n)].kid[side], child_out, depth + 1, out, info, root_area, trav);
    }
}

// Depth-first flatten: each output node holds the two children of an interior build node.
void flatten(const Node* n, int out_index, int depth, std::vector<pt_bvh_node>& out, BvhInfo& info, float root_area, float trav) {
    info.nodes++;
    info.max_depth = std::max(info.max_depth, depth);
    for (int side = 0; side < 2; side++) {
        const Node* c = n->kid[side].get();
        int child_out = -1;
        if (!c->leaf()) {
            child_out = int(out.size());
            out.push_back(pt_bvh_node{});
            info.sah_cost += trav * c->box.area() / root_area;
        } else {
            info.leaves++;
            info.sah_cost += float(c->count) * c->box.area() / root_area;
        }
        set_child(out[size_t(out_index)], side, c, child_out);
        if (!c->leaf()) flatten(c, child_out, depth + 1, out, info, root_area, trav);
    }
}

float srgb_to_linear_host(float c) { return c <= 0.04045f ? c / 12.92f : std::pow((c + 0.055f) / 1.055f, 2.4f); }

// Bilinear RGB lookup on host arrays (for estimating textured emitters).
struct HostTex {
    const pt_texture_info* t;
    const uint32_t* pool;
    const float* lut;
};
V3h host_tex_rgb(const HostTex& h, float u, float v) {
    const pt_texture_info& t = *h.t;
    float x = u * float(t.width) - 0.5f, y = v * float(t.height) - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    if (!(std::fabs(fx) < 1e8f) || !(std::fabs(fy) < 1e8f)) return mk(0, 0, 0);
    int x0 = int(fx), y0 = int(fy);
    float tx = x - fx, ty = y - fy;
    auto wrap = [&](int i, int n) {
        if (t.wrap_repeat) {
            i %= n;
            return i < 0 ? i + n : i;
        }
        return i < 0 ? 0 : (i >= n ? n - 1 : i);
    };
    int xa = wrap(x0, t.width), xb = wrap(x0 + 1, t.width), ya = wrap(y0, t.height), yb = wrap(y0 + 1, t.height);
    auto texel = [&](int xx, int yy) {
        uint32_t p = h.pool[t.offset + uint32_t(yy * t.width + xx)];
        V3h c = t.srgb ? mk(h.lut[p & 0xFF], h.lut[(p >> 8) & 0xFF], h.lut[(p >> 16) & 0xFF])
                       : mk(float(p & 0xFF), float((p >> 8) & 0xFF), float((p >> 16) & 0xFF)) * (1.0f / 255.0f);
        return c;
    };
    V3h top = texel(xa, ya) * (1 - tx) + texel(xb, ya) * tx;
    V3h bot = texel(xa, yb) * (1 - tx) + texel(xb, yb) * tx;
    return top * (1 - ty) + bot * ty;
}

}  // namespace

std::vector<pt_alias_entry> alias_table(const std::vector<float>& weights) {
    // Walker's alias method with Vose's linear-time construction: every bin holds a keep
    // probability and an alias; under-full bins are topped up from over-full ones. Here both
    // worklists are consumed in index order (FIFO). Each entry also stores its exact pmf, which the
    // integrator reads for MIS densities.
    const size_t n = weights.size();
    std::vector<pt_alias_entry> t(n);
    if (n == 0) return t;
    double sum = 0;
    for (float w : weights) sum += w > 0 ? double(w) : 0.0;
    std::vector<double> fill(n);
    std::vector<size_t> under, over;
    under.reserve(n);
    over.reserve(n);
    for (size_t i = 0; i < n; i++) {
        double pmf = sum > 0 ? (weights[i] > 0 ? double(weights[i]) : 0.0) / sum : 1.0 / double(n);
        t[i] = {1.0f, int32_t(i), float(pmf), 0};
        fill[i] = pmf * double(n);
        if (fill[i] < 1.0) under.push_back(i);
        else over.push_back(i);
    }
    size_t u = 0, o = 0;
    while (u < under.size() && o < over.size()) {
        size_t lo = under[u++], hi = over[o];
        t[lo].prob = float(fill[lo]);
        t[lo].alias = int32_t(hi);
        fill[hi] -= 1.0 - fill[lo];
        if (fill[hi] < 1.0) {
            o++;
            under.push_back(hi);
        }
    }
    // Leftovers (rounding) keep themselves with probability 1.
    for (; u < under.size(); u++) t[under[u]].prob = 1.0f;
    for (; o < over.size(); o++) t[over[o]].prob = 1.0f;
    return t;
}

void build_scene(const pt_raw_scene& raw, const BvhOptions& opt, BuiltScene& out) {
    auto t0 = std::chrono::steady_clock::now();
    if (raw.num_indices < 0 || raw.num_indices % 3 || raw.num_positions < 0) throw Error{PT_ERR_INVALID, "raw scene: bad index count"};
    if (raw.num_indices > 0 && (!raw.indices || !raw.positions)) throw Error{PT_ERR_INVALID, "raw scene: missing arrays"};
    for (int32_t i = 0; i < raw.num_indices; i++)
        if (raw.indices[i] < 0 || raw.indices[i] >= raw.num_positions) throw Error{PT_ERR_INVALID, "raw scene: index out of range"};
    out = BuiltScene();
    const int n = raw.num_indices / 3;
    const int nv = raw.num_positions;
    out.num_vertices = nv;
    // Materials (a default one when none are given, as Scene::build does).
    if (raw.num_materials > 0) out.materials.assign(raw.materials, raw.materials + raw.num_materials);
    else {
        pt_material m{};
        m.base_color = {1, 1, 1, 1};
        m.metallic = 1.0f;
        m.roughness = 1.0f;
        m.ior = 1.5f;
        m.normal_scale = 1.0f;
        m.alpha_cutoff = 0.5f;
        m.base_color_tex = m.metallic_roughness_tex = m.normal_tex = m.emissive_tex = m.occlusion_tex = -1;
        out.materials.push_back(m);
    }
    const int nm = int(out.materials.size());
    if (raw.normals) out.normals.assign(raw.normals, raw.normals + nv);
    if (raw.uvs) out.uvs.assign(raw.uvs, raw.uvs + nv);
    if (raw.tangents) out.tangents.assign(raw.tangents, raw.tangents + nv);
    // Tangents from UV derivatives (Lengyel's method) when a normal map needs them.
    bool need_tangents = false;
    for (const pt_material& m : out.materials) need_tangents |= m.normal_tex >= 0;
    if (need_tangents && raw.uvs && !raw.tangents) {
        std::vector<V3h> tan(size_t(nv), mk(0, 0, 0)), bit(size_t(nv), mk(0, 0, 0));
        for (int t = 0; t < n; t++) {
            int a = raw.indices[3 * t], b = raw.indices[3 * t + 1], c = raw.indices[3 * t + 2];
            V3h e1 = mk(raw.positions[b]) - mk(raw.positions[a]), e2 = mk(raw.positions[c]) - mk(raw.positions[a]);
            float d1x = raw.uvs[b].x - raw.uvs[a].x, d1y = raw.uvs[b].y - raw.uvs[a].y;
            float d2x = raw.uvs[c].x - raw.uvs[a].x, d2y = raw.uvs[c].y - raw.uvs[a].y;
            float det = d1x * d2y - d2x * d1y;
            if (std::fabs(det) < 1e-20f) continue;
            float r = 1.0f / det;
            V3h sdir = (e1 * d2y - e2 * d1y) * r, tdir = (e2 * d1x - e1 * d2x) * r;
            for (int v : {a, b, c}) {
                tan[size_t(v)] = tan[size_t(v)] + sdir;
                bit[size_t(v)] = bit[size_t(v)] + tdir;
            }
        }
        out.tangents.resize(size_t(nv));
        for (int v = 0; v < nv; v++) {
            V3h nn = raw.normals ? mk(raw.normals[v]) : mk(0, 0, 1);
            V3h t = tan[size_t(v)] - nn * dot(nn, tan[size_t(v)]);
            if (dot(t, t) < 1e-20f) {
                V3h un = normalize(nn);
                float sign = std::copysign(1.0f, un.z), aa = -1.0f / (sign + un.z);
                t = mk(1.0f + sign * un.x * un.x * aa, sign * un.x * un.y * aa, -sign * un.x);
            }
            t = normalize(t);
            float w = dot(cross(nn, t), bit[size_t(v)]) < 0 ? -1.0f : 1.0f;
            out.tangents[size_t(v)] = {t.x, t.y, t.z, w};
        }
    }

    // BVH.
    std::vector<Box> boxes(static_cast<size_t>(n));
    std::vector<float> cent(3 * size_t(n));
    for (int t = 0; t < n; t++) {
        Box b;
        for (int k = 0; k < 3; k++) {
            const pt_vec3& p = raw.positions[raw.indices[3 * t + k]];
            float q[3] = {p.x, p.y, p.z};
            b.grow(q);
        }
        boxes[size_t(t)] = b;
        for (int k = 0; k < 3; k++) cent[3 * size_t(t) + size_t(k)] = (b.lo[k] + b.hi[k]) * 0.5f;
    }
    std::vector<int> order(static_cast<size_t>(n));
    for (int i = 0; i < n; i++) order[size_t(i)] = i;
    Box root_box;
    if (n == 0) {
        pt_bvh_node r{};
        set_child(r, 0, nullptr, -1);
        set_child(r, 1, nullptr, -1);
        out.nodes.push_back(r);
    } else if (opt.gpu) {
        std::vector<float> flat_boxes(6 * size_t(n));
        for (int t = 0; t < n; t++)
            for (int k = 0; k < 3; k++) {
                flat_boxes[6 * size_t(t) + size_t(k)] = boxes[size_t(t)].lo[k];
                flat_boxes[6 * size_t(t) + 3 + size_t(k)] = boxes[size_t(t)].hi[k];
            }
        int device = 0;
        PTW_CUDA(cudaGetDevice(&device));
        std::vector<FlatBuildNode> tree;
        gpu_build_bvh(device, flat_boxes, cent, n, std::max(2, std::min(opt.bins, 64)), opt.max_leaf, opt.traversal_cost, order, tree);
        const FlatBuildNode& r = tree[0];
        for (int k = 0; k < 3; k++) {
            root_box.lo[k] = r.lo[k];
            root_box.hi[k] = r.hi[k];
        }
        float root_area = std::max(root_box.area(), 1e-20f);
        out.nodes.push_back(pt_bvh_node{});
        if (r.kid[0] < 0) {
            set_child_flat(out.nodes[0], 0, &r, -1);
            set_child_flat(out.nodes[0], 1, nullptr, -1);
            out.bvh.nodes = 1;
            out.bvh.leaves = 1;
            out.bvh.sah_cost = float(r.count);
        } else {
            out.bvh.sah_cost = opt.traversal_cost;
            flatten_flat(tree, 0, 0, 0, out.nodes, out.bvh, root_area, opt.traversal_cost);
        }
    } else {
        TaskBvhBuilder builder(boxes, cent, opt, order);
        std::unique_ptr<Node> root = builder.run(n);
        root_box = root->box;
        float root_area = std::max(root->box.area(), 1e-20f);
        out.nodes.push_back(pt_bvh_node{});
        if (root->leaf()) {
            set_child(out.nodes[0], 0, root.get(), -1);
            set_child(out.nodes[0], 1, nullptr, -1);
            out.bvh.nodes = 1;
            out.bvh.leaves = 1;
            out.bvh.sah_cost = float(root->count);
        } else {
            out.bvh.sah_cost = opt.traversal_cost;
            flatten(root.get(), 0, 0, out.nodes, out.bvh, root_area, opt.traversal_cost);
        }
    }
    // Triangles in BVH order.
    out.tris.resize(size_t(n));
    out.indices.resize(3 * size_t(n));
    for (int i = 0; i < n; i++) {
        int t = order[size_t(i)];
        V3h a = mk(raw.positions[raw.indices[3 * t]]), b = mk(raw.positions[raw.indices[3 * t + 1]]), c = mk(raw.positions[raw.indices[3 * t + 2]]);
        pt_tri_geom g{};
        g.v0 = pv(a);
        g.e1 = pv(b - a);
        g.e2 = pv(c - a);
        int m = raw.tri_material ? raw.tri_material[t] : 0;
        g.material = std::clamp(m, 0, nm - 1);
        g.flags = out.materials[size_t(g.material)].alpha_mode != PT_ALPHA_OPAQUE ? PT_TRI_ALPHA_TESTED : 0;
        out.tris[size_t(i)] = g;
        for (int k = 0; k < 3; k++) out.indices[3 * size_t(i) + size_t(k)] = raw.indices[3 * t + k];
    }
    // Texel pool and sRGB table.
    for (int i = 0; i < raw.num_textures; i++) {
        const pt_texture_desc& t = raw.textures[i];
        if (t.width <= 0 || t.height <= 0 || !t.texels) throw Error{PT_ERR_INVALID, "raw scene: bad texture"};
        pt_texture_info info{};
        info.width = t.width;
        info.height = t.height;
        info.offset = uint32_t(out.texels.size());
        info.wrap_repeat = t.repeat ? 1 : 0;
        info.srgb = t.srgb ? 1 : 0;
        out.texels.insert(out.texels.end(), t.texels, t.texels + size_t(t.width) * size_t(t.height));
        out.textures.push_back(info);
    }
    out.srgb_lut.resize(256);
    for (int i = 0; i < 256; i++) out.srgb_lut[size_t(i)] = srgb_to_linear_host(float(i) / 255.0f);
    out.punctual.assign(raw.punctual, raw.punctual + std::max(0, raw.num_punctual));

    // Emissive triangles by power (the definitions of scene.cpp:113-141).
    out.tri_emissive.assign(size_t(n), -1);
    std::vector<float> power;
    float emissive_power = 0;
    for (int i = 0; i < n; i++) {
        const pt_material& m = out.materials[size_t(out.tris[size_t(i)].material)];
        float l = lum(mk(m.emission));
        if (l <= 0) continue;
        if (m.emissive_tex >= 0 && m.emissive_tex < int(out.textures.size()) && !out.uvs.empty()) {
            static const float pts[7][2] = {{1.f / 3, 1.f / 3}, {0.1f, 0.1f}, {0.8f, 0.1f}, {0.1f, 0.8f}, {0.45f, 0.1f}, {0.45f, 0.45f}, {0.1f, 0.45f}};
            HostTex ht{&out.textures[size_t(m.emissive_tex)], out.texels.data(), out.srgb_lut.data()};
            float sum = 0;
            for (const auto& bb : pts) {
                const int32_t* idx = &out.indices[3 * size_t(i)];
                float w0 = 1 - bb[0] - bb[1];
                float u = out.uvs[size_t(idx[0])].x * w0 + out.uvs[size_t(idx[1])].x * bb[0] + out.uvs[size_t(idx[2])].x * bb[1];
                float v = out.uvs[size_t(idx[0])].y * w0 + out.uvs[size_t(idx[1])].y * bb[0] + out.uvs[size_t(idx[2])].y * bb[1];
                V3h tc = host_tex_rgb(ht, u, v);
                sum += lum(mk(m.emission.x * tc.x, m.emission.y * tc.y, m.emission.z * tc.z));
            }
            l = sum / 7.0f;
            if (l <= 1e-4f) continue;
        }
        float area = 0.5f * length(cross(mk(out.tris[size_t(i)].e1), mk(out.tris[size_t(i)].e2)));
        if (area <= 0) continue;
        out.tri_emissive[size_t(i)] = int32_t(out.emissive.size());
        out.emissive.push_back({int32_t(i), area});
        float p = area * l * kPiF * (m.double_sided ? 2.0f : 1.0f);
        power.push_back(p);
        emissive_power += p;
    }
    out.alias = alias_table(power);

    // Light-group probabilities. The integrator picks a group (emissive, punctual, environment)
    // with these probabilities before picking a light; they estimate each group's power arriving
    // at a sphere bounding the scene (the definition Photon uses, scene.cpp:142-175): a
    // distant source of radiance L over the sphere of radius r delivers L * pi * (pi r^2) * 4, a
    // point source 4 pi I, a directional one E * pi r^2. Every present group keeps >= 5%.
    const float r = root_box.empty()
                        ? 1.0f
                        : 0.5f * length(mk(root_box.hi[0], root_box.hi[1], root_box.hi[2]) - mk(root_box.lo[0], root_box.lo[1], root_box.lo[2]));
    const size_t env_n = size_t(std::max(0, raw.env_width)) * size_t(std::max(0, raw.env_height));
    const bool has_env_image = raw.env_texels && env_n;
    float mean_env = 0;
    if (has_env_image) {
        double s = 0;
        for (size_t i = 0; i < env_n; i++) s += lum(mk(raw.env_texels[i]));
        mean_env = float(s / double(env_n));
    } else {
        mean_env = lum(mk(raw.env_color));
    }
    float group_power[3];  // 0 environment, 1 emissive, 2 punctual
    group_power[0] = mean_env * raw.env_intensity * kPiF * kPiF * r * r * 4.0f;
    group_power[1] = emissive_power;
    group_power[2] = 0;
    for (const pt_punctual_light& l : out.punctual)
        group_power[2] += l.type == PT_LIGHT_DIRECTIONAL ? lum(mk(l.intensity)) * kPiF * r * r : lum(mk(l.intensity)) * 4.0f * kPiF;
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
    const float p_env = prob[0], p_em = prob[1], p_pu = prob[2];

    // The environment's sampling distribution: piecewise constant over the image, proportional to
    // luminance * sin(theta) (the solid-angle Jacobian of the equirectangular map). Rows are
    // chosen by the marginal CDF over row sums, texels by each row's conditional CDF; the mean of
    // the function over the unit square normalises pdf(u, v) = f(u, v) / integral.
    float env_integral = 0;
    if (has_env_image) {
        const int w = raw.env_width, h = raw.env_height;
        out.env_texels.assign(raw.env_texels, raw.env_texels + env_n);
        out.env_conditional.assign(size_t(h) * size_t(w + 1), 0.0f);
        out.env_marginal.assign(size_t(h) + 1, 0.0f);
        std::vector<double> prefix(static_cast<size_t>(w) + 1), row_total(static_cast<size_t>(h));
        for (int y = 0; y < h; y++) {
            const float sin_theta = std::sin((float(y) + 0.5f) / float(h) * kPiF);
            const pt_vec3* row = raw.env_texels + size_t(y) * size_t(w);
            prefix[0] = 0;
            for (int x = 0; x < w; x++) prefix[size_t(x) + 1] = prefix[size_t(x)] + double(lum(mk(row[x]))) * sin_theta;
            const double rs = prefix[size_t(w)];
            row_total[size_t(y)] = rs;
            float* cdf = &out.env_conditional[size_t(y) * size_t(w + 1)];
            for (int x = 1; x <= w; x++) cdf[x] = rs > 0 ? float(double(float(prefix[size_t(x)])) / rs) : float(x) / float(w);
        }
        double all = 0;
        std::vector<double> mprefix(size_t(h) + 1, 0.0);
        for (int y = 0; y < h; y++) mprefix[size_t(y) + 1] = all = all + row_total[size_t(y)];
        for (int y = 1; y <= h; y++) out.env_marginal[size_t(y)] = all > 0 ? float(double(float(mprefix[size_t(y)])) / all) : float(y) / float(h);
        env_integral = float(all / (double(w) * double(h)));
    }

    pt_scene_desc& d = out.desc;
    d = pt_scene_desc{};
    d.nodes = out.nodes.data();
    d.num_nodes = int32_t(out.nodes.size());
    d.tris = out.tris.data();
    d.num_tris = n;
    d.indices = out.indices.data();
    d.normals = out.normals.empty() ? nullptr : out.normals.data();
    d.uvs = out.uvs.empty() ? nullptr : out.uvs.data();
    d.tangents = out.tangents.empty() ? nullptr : out.tangents.data();
    d.num_vertices = nv;
    d.materials = out.materials.data();
    d.num_materials = nm;
    d.textures = out.textures.empty() ? nullptr : out.textures.data();
    d.num_textures = int32_t(out.textures.size());
    d.texels = out.texels.empty() ? nullptr : out.texels.data();
    d.num_texels = out.texels.size();
    d.srgb_lut = out.srgb_lut.data();
    d.emissive = out.emissive.empty() ? nullptr : out.emissive.data();
    d.num_emissive = int32_t(out.emissive.size());
    d.tri_emissive = out.tri_emissive.data();
    d.emissive_alias = out.alias.empty() ? nullptr : out.alias.data();
    d.emissive_power = emissive_power;
    d.punctual = out.punctual.empty() ? nullptr : out.punctual.data();
    d.num_punctual = int32_t(out.punctual.size());
    d.env_texels = out.env_texels.empty() ? nullptr : out.env_texels.data();
    d.env_width = out.env_texels.empty() ? 0 : raw.env_width;
    d.env_height = out.env_texels.empty() ? 0 : raw.env_height;
    d.env_marginal = out.env_marginal.empty() ? nullptr : out.env_marginal.data();
    d.env_conditional = out.env_conditional.empty() ? nullptr : out.env_conditional.data();
    d.env_intensity = raw.env_intensity;
    d.env_rotation = raw.env_rotation;
    d.env_color = raw.env_color;
    d.env_integral = env_integral;
    d.p_env = p_env;
    d.p_emissive = p_em;
    d.p_punctual = p_pu;
    d.bounds_min = {root_box.lo[0], root_box.lo[1], root_box.lo[2]};
    d.bounds_max = {root_box.hi[0], root_box.hi[1], root_box.hi[2]};
    out.bvh.build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace ptw
