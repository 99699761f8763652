// Device build of the binned-SAH BVH (see gpu_bvh.h). Breadth-first: one launch per tree level, one
// block per node of the level. A block reduces its range's box and centroid box, bins the centroids
// on the three axes in shared memory, sweeps the planes exactly as the host builder does (one
// thread, same order of operations), and partitions its range of `order` in place. The host builder
// partitions with the two-pointer exchange (the k-th out-of-place element from the left is swapped
// with the k-th out-of-place element from the right); here the two lists are ranked by block scans
// and the pairs swapped in parallel, which yields the same permutation.
#include "gpu_bvh.h"

#include <cuda_runtime.h>

#include "device_scene.h"

namespace ptw {

namespace {

constexpr float kBig = 1e30f;
constexpr int kMaxBins = 64;
constexpr int kThreads = 256;
constexpr int kMaxDepth = 60;

struct BoxD {
    float lo[3], hi[3];
};

__device__ __forceinline__ float area_of(const float lo[3], const float hi[3]) {
    if (lo[0] > hi[0]) return 0.0f;
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// Float min/max in shared memory (exact; the values are finite).
__device__ __forceinline__ void smem_min(float* a, float v) {
    int* ai = reinterpret_cast<int*>(a);
    int old = *ai;
    while (v < __int_as_float(old)) {
        int prev = atomicCAS(ai, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
}
__device__ __forceinline__ void smem_max(float* a, float v) {
    int* ai = reinterpret_cast<int*>(a);
    int old = *ai;
    while (v > __int_as_float(old)) {
        int prev = atomicCAS(ai, old, __float_as_int(v));
        if (prev == old) break;
        old = prev;
    }
}

struct Task {
    int node, first, count, depth;
};

struct BuildArgs {
    const float* boxes;  // 6 per primitive
    const float* cent;   // 3 per primitive
    int* order;
    int* scratch_l;      // per range: positions of the out-of-place elements
    int* scratch_r;
    FlatBuildNode* nodes;
    int* node_count;
    const Task* tasks;
    Task* next_tasks;
    int* next_count;
    int bins, max_leaf;
    float traversal_cost;
};

// Block-wide exclusive scan of one int per thread; returns the block total.
__device__ __forceinline__ int block_scan(int v, int* smem_warp, int& excl) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kThreads / 32 ? smem_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kThreads / 32) smem_warp[lane] = w;
    }
    __syncthreads();
    int warp_base = warp > 0 ? smem_warp[warp - 1] : 0;
    int total = smem_warp[kThreads / 32 - 1];
    excl = warp_base + x - v;
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(kThreads) k_split(BuildArgs A) {
    __shared__ float s_box[12];  // node lo/hi, centroid lo/hi
    __shared__ int s_n[3][kMaxBins];
    __shared__ float s_bin[3][kMaxBins][6];
    __shared__ int s_warp[kThreads / 32];
    __shared__ int s_decision[4];  // axis, plane, mid, leaf
    __shared__ float s_geom[6];    // lo[3], scale[3]
    __shared__ int s_usable[3];
    __shared__ int s_true;
    const Task t = A.tasks[blockIdx.x];
    const int tid = threadIdx.x, B = A.bins;
    if (tid < 12) s_box[tid] = (tid % 6) < 3 ? kBig : -kBig;
    for (int k = tid; k < 3 * kMaxBins; k += kThreads) {
        s_n[k / kMaxBins][k % kMaxBins] = 0;
        for (int c = 0; c < 6; c++) s_bin[k / kMaxBins][k % kMaxBins][c] = c < 3 ? kBig : -kBig;
    }
    __syncthreads();
    // Node box and centroid box.
    for (int i = t.first + tid; i < t.first + t.count; i += kThreads) {
        const int p = A.order[i];
        const float* b = A.boxes + 6 * size_t(p);
        const float* c = A.cent + 3 * size_t(p);
        for (int k = 0; k < 3; k++) {
            smem_min(&s_box[k], b[k]);
            smem_max(&s_box[3 + k], b[3 + k]);
            smem_min(&s_box[6 + k], c[k]);
            smem_max(&s_box[9 + k], c[k]);
        }
    }
    __syncthreads();
    FlatBuildNode& node = A.nodes[t.node];
    if (tid == 0) {
        for (int k = 0; k < 3; k++) {
            node.lo[k] = s_box[k];
            node.hi[k] = s_box[3 + k];
        }
        node.first = t.first;
        node.count = t.count;
        node.kid[0] = node.kid[1] = -1;
        for (int a = 0; a < 3; a++) {
            s_geom[a] = s_box[6 + a];
            float ext = s_box[9 + a] - s_box[6 + a];
            s_usable[a] = ext > 1e-12f;
            s_geom[3 + a] = s_usable[a] ? float(B) / ext : 0.0f;
        }
    }
    if (t.count <= 1 || t.depth >= kMaxDepth) return;
    __syncthreads();
    // Bin every primitive on the usable axes.
    for (int i = t.first + tid; i < t.first + t.count; i += kThreads) {
        const int p = A.order[i];
        const float* b = A.boxes + 6 * size_t(p);
        const float* c = A.cent + 3 * size_t(p);
        for (int a = 0; a < 3; a++) {
            if (!s_usable[a]) continue;
            int bin = min(B - 1, int((c[a] - s_geom[a]) * s_geom[3 + a]));
            atomicAdd(&s_n[a][bin], 1);
            for (int k = 0; k < 3; k++) {
                smem_min(&s_bin[a][bin][k], b[k]);
                smem_max(&s_bin[a][bin][3 + k], b[3 + k]);
            }
        }
    }
    __syncthreads();
    // The sweeps, in the host builder's order of operations.
    if (tid == 0) {
        const float inv_parent = 1.0f / fmaxf(area_of(s_box, s_box + 3), 1e-30f);
        float best_cost = kBig;
        int best_axis = -1, best_plane = -1;
        for (int a = 0; a < 3; a++) {
            if (!s_usable[a]) continue;
            float suffix_area[kMaxBins];
            int suffix_n[kMaxBins];
            float rlo[3] = {kBig, kBig, kBig}, rhi[3] = {-kBig, -kBig, -kBig};
            int cnt = 0;
            for (int b = B - 1; b >= 1; b--) {
                for (int k = 0; k < 3; k++) {
                    rlo[k] = fminf(rlo[k], s_bin[a][b][k]);
                    rhi[k] = fmaxf(rhi[k], s_bin[a][b][3 + k]);
                }
                cnt += s_n[a][b];
                suffix_area[b] = area_of(rlo, rhi);
                suffix_n[b] = cnt;
            }
            float plo[3] = {kBig, kBig, kBig}, phi[3] = {-kBig, -kBig, -kBig};
            int pn = 0;
            for (int plane = 1; plane < B; plane++) {
                for (int k = 0; k < 3; k++) {
                    plo[k] = fminf(plo[k], s_bin[a][plane - 1][k]);
                    phi[k] = fmaxf(phi[k], s_bin[a][plane - 1][3 + k]);
                }
                pn += s_n[a][plane - 1];
                if (pn == 0 || suffix_n[plane] == 0) continue;
                float c = A.traversal_cost + (area_of(plo, phi) * float(pn) + suffix_area[plane] * float(suffix_n[plane])) * inv_parent;
                if (c < best_cost) {
                    best_cost = c;
                    best_axis = a;
                    best_plane = plane;
                }
            }
        }
        const bool forced = t.count > A.max_leaf;
        s_decision[3] = (!forced && (best_axis < 0 || best_cost >= float(t.count))) ? 1 : 0;
        s_decision[0] = best_axis;
        s_decision[1] = best_plane;
    }
    __syncthreads();
    if (s_decision[3]) return;  // a leaf is cheaper
    const int axis = s_decision[0], plane = s_decision[1];
    int mid = t.first + t.count / 2;
    if (axis >= 0) {
        const float l = s_geom[axis], sc = s_geom[3 + axis];
        auto pred = [&](int p) { return min(B - 1, int((A.cent[3 * size_t(p) + axis] - l) * sc)) < plane; };
        // m = elements on the left side of the plane.
        if (tid == 0) s_true = 0;
        __syncthreads();
        int mine = 0;
        for (int i = t.first + tid; i < t.first + t.count; i += kThreads) mine += pred(A.order[i]) ? 1 : 0;
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
        if ((tid & 31) == 0) atomicAdd(&s_true, mine);
        __syncthreads();
        const int m = s_true;  // relative cut
        // Rank the out-of-place elements: left of the cut and not on the left side (ascending), right of
        // the cut and on the left side (ascending positions; paired from the far end).
        int carry_l = 0, carry_r = 0;
        for (int base = 0; base < t.count; base += kThreads) {
            const int i = base + tid;
            int fl = 0, fr = 0;
            if (i < t.count) {
                bool pv = pred(A.order[t.first + i]);
                fl = (i < m && !pv) ? 1 : 0;
                fr = (i >= m && pv) ? 1 : 0;
            }
            int el, er;
            int tl = block_scan(fl, s_warp, el);
            int tr = block_scan(fr, s_warp, er);
            if (fl) A.scratch_l[t.first + carry_l + el] = t.first + i;
            if (fr) A.scratch_r[t.first + carry_r + er] = t.first + i;
            carry_l += tl;
            carry_r += tr;
        }
        __syncthreads();
        // carry_l == carry_r: swap the k-th from the left with the k-th from the right end.
        const int pairs = carry_l;
        for (int k = tid; k < pairs; k += kThreads) {
            const int a = A.scratch_l[t.first + k], b = A.scratch_r[t.first + pairs - 1 - k];
            const int va = A.order[a];
            A.order[a] = A.order[b];
            A.order[b] = va;
        }
        const int cut = t.first + m;
        if (cut > t.first && cut < t.first + t.count) mid = cut;
    }
    __syncthreads();
    if (tid == 0) {
        int k0 = atomicAdd(A.node_count, 2);
        node.kid[0] = k0;
        node.kid[1] = k0 + 1;
        int q = atomicAdd(A.next_count, 2);
        A.next_tasks[q] = Task{k0, t.first, mid - t.first, t.depth + 1};
        A.next_tasks[q + 1] = Task{k0 + 1, mid, t.first + t.count - mid, t.depth + 1};
    }
}

}  // namespace

void gpu_build_bvh(int device, const std::vector<float>& boxes, const std::vector<float>& cent, int n, int bins, int max_leaf,
                   float traversal_cost, std::vector<int>& order, std::vector<FlatBuildNode>& nodes) {
    bins = bins < 2 ? 2 : (bins > kMaxBins ? kMaxBins : bins);
    int prev = 0;
    PTW_CUDA(cudaGetDevice(&prev));
    PTW_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    PTW_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    try {
        DeviceBuffer<float> d_boxes, d_cent;
        d_boxes.upload(boxes.data(), boxes.size(), s);
        d_cent.upload(cent.data(), cent.size(), s);
        order.resize(size_t(n));
        for (int i = 0; i < n; i++) order[size_t(i)] = i;
        DeviceBuffer<int> d_order, d_l, d_r, d_counts;
        d_order.upload(order.data(), order.size(), s);
        d_l.allocate(size_t(n));
        d_r.allocate(size_t(n));
        d_counts.allocate(2);
        // A binary tree over n primitives has at most 2n - 1 nodes; tasks of one level at most n.
        DeviceBuffer<FlatBuildNode> d_nodes;
        d_nodes.allocate(size_t(2 * n));
        DeviceBuffer<Task> d_tasks[2];
        d_tasks[0].allocate(size_t(n));
        d_tasks[1].allocate(size_t(n));
        Task root{0, 0, n, 0};
        PTW_CUDA(cudaMemcpyAsync(d_tasks[0].ptr, &root, sizeof(Task), cudaMemcpyHostToDevice, s));
        int counts[2] = {1, 0};  // nodes allocated, next level's tasks
        PTW_CUDA(cudaMemcpyAsync(d_counts.ptr, counts, sizeof(counts), cudaMemcpyHostToDevice, s));
        int level_tasks = 1, cur = 0;
        for (int level = 0; level_tasks > 0 && level <= kMaxDepth; level++) {
            BuildArgs a{d_boxes.ptr, d_cent.ptr, d_order.ptr, d_l.ptr, d_r.ptr, d_nodes.ptr, d_counts.ptr, d_tasks[cur].ptr,
                        d_tasks[1 - cur].ptr, d_counts.ptr + 1, bins, max_leaf, traversal_cost};
            k_split<<<level_tasks, kThreads, 0, s>>>(a);
            PTW_CUDA(cudaGetLastError());
            PTW_CUDA(cudaMemcpyAsync(counts, d_counts.ptr, sizeof(counts), cudaMemcpyDeviceToHost, s));
            PTW_CUDA(cudaStreamSynchronize(s));
            level_tasks = counts[1];
            int zero = 0;
            PTW_CUDA(cudaMemcpyAsync(d_counts.ptr + 1, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
            cur = 1 - cur;
        }
        nodes.resize(size_t(counts[0]));
        PTW_CUDA(cudaMemcpyAsync(nodes.data(), d_nodes.ptr, nodes.size() * sizeof(FlatBuildNode), cudaMemcpyDeviceToHost, s));
        PTW_CUDA(cudaMemcpyAsync(order.data(), d_order.ptr, order.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
        PTW_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamDestroy(s);
        cudaSetDevice(prev);
        throw;
    }
    cudaStreamDestroy(s);
    PTW_CUDA(cudaSetDevice(prev));
}

}  // namespace ptw
