// The wavefront kernels of the path tracer (sm_100a).
//
// Photon runs trace_path (src/render/integrator.h:151-263) as one thread per pixel sample. Here the
// same loop is cut at its ray casts into kernels that each advance every live path by one step:
//
//   setup     sizes the iteration from the device counters (no host round trip)
//   generate  refills free path slots with camera paths (render_sample's RNG, jitter, camera ray)
//   trace     closest-hit BVH traversal of every live path's ray
//   shade     emission + MIS, next event estimation (light pick, BSDF eval, shadow ray), BSDF
//             sampling, Russian roulette; continuing paths and shadow rays are appended to
//             compacted queues with one atomic per warp (ballot + popc)
//   shadow    any-hit traversal of the shadow queue; unoccluded contributions are added to their
//             path (or to a finished path's sample) in the same order as Photon adds them
//
// Kernels are persistent: a grid sized to fill the GPU claims 32-path chunks with one atomic per
// warp until the iteration's count (read from device memory) is exhausted. Compiled with
// -fmad=false and IEEE division / square root: see pt_math.cuh.
#include "wavefront.h"
#include "gbuffer.cuh"

#include "pt_traverse.cuh"

namespace ptw {

namespace {

constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ uint32_t warp_fetch(uint32_t* ctr) {
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(ctr, 32u);
    return __shfl_sync(kFull, base, 0);
}

// Appends the lanes with `pred` to a queue: returns each such lane's slot (one atomic per warp).
__device__ __forceinline__ uint32_t warp_append(bool pred, uint32_t* ctr) {
    uint32_t mask = __ballot_sync(kFull, pred);
    if (mask == 0) return 0;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (int(lane_id()) == leader) base = atomicAdd(ctr, uint32_t(__popc(mask)));
    base = __shfl_sync(kFull, base, leader);
    return base + __popc(mask & ((1u << lane_id()) - 1u));
}

__device__ __forceinline__ void warp_add_u64(unsigned long long* ctr, uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if (lane_id() == 0 && v) atomicAdd(ctr, (unsigned long long)v);
}

// Sample slot q of an image -> pixel. Slots run over 8x4 tiles (one warp's camera rays share a
// tile) and then over the right and bottom remainder strips, so the map is a bijection for any size.
__device__ __forceinline__ void tile_pixel(uint32_t q, int W, int H, int& x, int& y) {
    uint32_t tx_n = uint32_t(W) >> 3, ty_n = uint32_t(H) >> 2;
    uint32_t fw = tx_n * 8, fh = ty_n * 4, full = fw * fh;
    if (q < full) {
        uint32_t t = q >> 5, r = q & 31;
        x = int((t % tx_n) * 8 + (r & 7));
        y = int((t / tx_n) * 4 + (r >> 3));
        return;
    }
    uint32_t q2 = q - full, rw = uint32_t(W) - fw, cr = rw * fh;
    if (q2 < cr) {
        x = int(fw + q2 % rw);
        y = int(q2 / rw);
        return;
    }
    uint32_t q3 = q2 - cr;
    x = int(q3 % uint32_t(W));
    y = int(fh + q3 / uint32_t(W));
}

// camera_ray (integrator.h:266-280) from a pt_camera laid out as 16 floats.
__device__ __forceinline__ void camera_ray(const float* c, float px, float py, int width, int height, V2 lens, V3& o, V3& d) {
    V3 pos{c[0], c[1], c[2]}, fwd{c[4], c[5], c[6]}, right{c[8], c[9], c[10]}, up{c[12], c[13], c[14]};
    float tan_half_fov = c[3], aspect = c[7], aperture = c[11], focus = c[15];
    float sx = (2.0f * px / float(width) - 1.0f) * tan_half_fov * aspect;
    float sy = (1.0f - 2.0f * py / float(height)) * tan_half_fov;
    d = normalize(fwd + right * sx + up * sy);
    o = pos;
    if (aperture > 0) {
        V3 focus_p = pos + d * (focus / dot(d, fwd));
        V2 l = concentric_disk(lens) * aperture;
        o = pos + right * l.x + up * l.y;
        d = normalize(focus_p - o);
    }
}

__device__ __forceinline__ const DevScene& scene_for(const WfParams& P, int view) {
    return P.single_scene >= 0 ? P.scenes[P.single_scene] : P.scenes[P.views[view].scene];
}

__device__ __forceinline__ float clamp_contribution(V3& c, int depth, float clamp) {
    if (depth > 0 && clamp > 0) {
        float l = luminance(c);
        if (l > clamp) c = c * (clamp / l);
    }
    return 0;
}

__device__ __forceinline__ int find_view(const DevView* views, int n, unsigned long long w) {
    int lo = 0, hi = n;
    while (lo + 1 < hi) {
        int mid = (lo + hi) >> 1;
        if (views[mid].work_begin <= w) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---- setup ------------------------------------------------------------------------------------------
__global__ void k_setup(const __grid_constant__ WfParams P) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Counters* c = P.ctr;
    const uint32_t capacity = P.pb.capacity, tail_paths = P.tail_paths > 0 ? c->tail_limit : 0u;
    uint32_t p = c->parity ^ 1u;
    c->parity = p;
    uint32_t cnt = c->count[p];
    unsigned long long remaining = c->work_total > c->work_next ? c->work_total - c->work_next : 0ull;
    uint32_t room = capacity > cnt ? capacity - cnt : 0u;
    uint32_t n = remaining < room ? uint32_t(remaining) : room;
    c->gen_base = cnt;
    c->gen_n = n;
    c->work_base = c->work_next;
    // The views are in work order and generation only moves forward: skip those already generated,
    // so that the generate step's search covers the few views ahead (a server appends views for ever).
    uint32_t gv = c->gen_view;
    while (int(gv) + 1 < P.num_views && P.views[gv + 1].work_begin <= c->work_base) gv++;
    c->gen_view = gv;
    c->work_next += n;
    c->count[p] = cnt + n;
    c->count[p ^ 1u] = 0;
    c->shadow_rays += c->shadow_count;
    c->shadow_count = 0;
    c->rays += cnt + n;
    c->tail = (tail_paths > 0 && cnt + n > 0 && cnt + n <= tail_paths && c->work_next >= c->work_total) ? 1u : 0u;
    // Sorting pays for its scan and scatter only on large iterations.
    c->sorting = (P.sort_bits > 0 && !c->tail && cnt + n >= kSortMinPaths) ? 1u : 0u;
    c->shadow_sorting = (P.shadow_sort_bits > 0 && !c->tail && cnt + n >= kSortMinPaths) ? 1u : 0u;
    for (int k = 0; k < 6; k++) c->fetch[k] = 0;
    if (cnt + n > 0) c->iterations++;
}

// ---- generate: render_sample's camera path (pixel.h:18-24) --------------------------------------------
__global__ void __launch_bounds__(256) k_generate(const __grid_constant__ WfParams P) {
    Counters* c = P.ctr;
    const uint32_t p = c->parity, base = c->gen_base, n = c->gen_n;
    const unsigned long long wb = c->work_base;
    // Every path costs the same here, so a static grid-stride split replaces the claim counter: one
    // atomic per warp on one address held this kernel at 1.5 ms per 1080p frame (0.56 ms without).
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        unsigned long long wg = wb + k;
        const int v0 = int(c->gen_view);
        int vi = v0 + find_view(P.views + v0, P.num_views - v0, wg);
        const DevView& v = P.views[vi];
        uint32_t local = uint32_t(v.local_base + (wg - v.work_begin));
        uint32_t npix = uint32_t(v.width) * uint32_t(v.height);
        uint32_t s = local / npix, q = local - s * npix;
        int x, y;
        tile_pixel(q, v.width, v.height, x, y);
        uint32_t pixel = uint32_t(y) * uint32_t(v.width) + uint32_t(x);
        Rng rng = pixel_rng(pixel, v.seed, v.frame0 + s);
        V2 jitter = rng_next2(rng);
        V2 lens = rng_next2(rng);
        V3 o, d;
        camera_ray(v.cam, float(x) + jitter.x, float(y) + jitter.y, v.width, v.height, lens, o, d);
        uint32_t slot = base + k;
        P.pb.o[p][slot] = make_float4(o.x, o.y, o.z, 0.0f);
        P.pb.d[p][slot] = make_float4(d.x, d.y, d.z, __uint_as_float(1u << 16));  // depth 0, prev_delta
        P.pb.beta[p][slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        P.pb.lr[p][slot] = make_float4(0.0f, 0.0f, __uint_as_float(uint32_t(rng.state)), __uint_as_float(uint32_t(rng.state >> 32)));
        P.pb.id[p][slot] = make_uint4(uint32_t(vi), local, pixel, s);
    }
}

// ---- the queue walk shared by trace and shadow -------------------------------------------------------
// Persistent walk over a ray queue with warp-granular refill (dynamic ray fetch, after Aila and Laine,
// "Understanding the Efficiency of Ray Traversal on GPUs", HPG 2009). Each lane advances its ray one
// walk step at a time (a node visit or a triangle test). A warp that claimed 32 rays and walked them to
// the end would idle most lanes behind its longest ray; here, whenever fewer than `refill` lanes hold
// a live ray and the queue is not exhausted, the idle lanes claim the next rays of the queue together
// (one atomic per warp) and start them on the spot. A ray's walk, and so its result and its counts,
// does not depend on the lane or the moment it starts, so every `refill` gives the same results;
// refill = 1 claims only once all lanes have finished (32 consecutive rays at a time).
// The warp looks at its lanes only every `burst` steps: in between, each lane steps on its own, so
// lanes in different phases of their walks (visiting nodes, testing a leaf's triangles) proceed as
// separate groups whose load latencies overlap, instead of meeting at a warp-wide vote every step.
// begin(i, w, ws) initialises walker w from queue entry i (and, unless Single, sets the lane's scene
// arrays ws) and returns the index of the ray's record; end(record, w) consumes the finished walk. Single: every ray walks `uniform`, whose array
// bases stay in registers for the whole loop. Count: tc.steps counts lane steps and warp_steps the
// loop's iterations.
template <typename W, int Overflow, bool Count, bool Single, typename Begin, typename End>
__device__ __forceinline__ void walk_queue(uint32_t n, uint32_t* claim, uint32_t refill, uint32_t burst, int* stack, int stride,
                                           const WalkScene& uniform, TraversalCounters& tc, uint32_t& warp_steps, Begin begin, End end) {
    int overflow[Overflow];
    W w;
    WalkScene ws = uniform;
    uint32_t idx = 0;
    bool live = false, drained = false;
    const uint32_t lane = lane_id(), below = (1u << lane) - 1u;
    for (;;) {
        uint32_t act = __ballot_sync(kFull, live);
        if (!drained && uint32_t(__popc(act)) < refill) {
            const uint32_t idle = ~act, want = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(claim, want);
            base = __shfl_sync(kFull, base, 0);
            drained = base + want >= n;
            if (!live) {
                const uint32_t r = base + uint32_t(__popc(idle & below));
                if (r < n) {
                    idx = begin(r, w, ws);
                    live = true;
                }
            }
            act = __ballot_sync(kFull, live);
        }
        if (act == 0) break;
        uint32_t taken = 0;
        if (live) {
            while (taken < burst) {
                taken++;
                if (!w.step(Single ? uniform : ws, stack, stride, overflow, &tc)) {
                    end(idx, w);
                    live = false;
                    break;
                }
            }
        }
        if (Count) {
            tc.steps += taken;
            warp_steps += __reduce_max_sync(kFull, taken);  // the warp's steps in this burst: its busiest lane's
        }
    }
}

// ---- the pair walk -----------------------------------------------------------------------------------
// A warp's shared memory in the pair walk (2,080 bytes after the block's stacks): each lane's PairLane
// slots, the owners' result slots of a pair pass and a round's owner table.
struct PairSlots {
    float4 ray[32];
    int4 leaves[32];
    float4 hit[32];
    unsigned long long best[32];  // nearest accepted pair: distance bits << 32 | pair (any-hit: pair); ~0 none
    float2 uv[32];                // barycentrics of the pair a lane accepted
    uint8_t head[32];             // a round's segment heads: the lane whose pairs start at base + j
    __device__ __forceinline__ PairLane lane(uint32_t l) { return PairLane{ray[l], leaves[l], hit[l]}; }
};
static_assert(sizeof(PairSlots) == 2080, "PairSlots layout");

// Tests the leaf pairs of a warp's lanes. Lane k, whose last node visit found m_k leaf triangles, owns
// pairs [first_k, first_k + m_k) of the warp's list (an exclusive scan of m). The lanes take the list
// 32 pairs at a time: lane j finds the owner of pair base + j from the round's segment heads (one
// warp-wide OR of their start bits and a shared-memory table; it replaced a binary search of the scan
// by five dependent shuffles: trace 23.8 -> 23.55, shadow 10.92 -> 10.85 ms per 1080p frame),
// takes its origin by shuffles and its direction, tmax and leaf ranges from its slots (`scene`: the
// lane's own scene, in multi-scene launches), tests that triangle against the owner's tmax, and an
// accepted pair enters the owner's slot by a 64-bit atomicMin of (distance bits << 32 | pair index):
// positive distances order as their bits, so the owner gets its least distance, on a tie its earliest
// pair. A sequential leaf walk (traverse.h
// :93-104) accepts a triangle only when it lowers tmax, so it ends on the first pair of least distance
// below the entering tmax: the same triangle, distance and barycentrics. Any-hit keys are the pair
// index alone (the first accepted pair, where the sequential walk stops). An owner whose pairs span two
// rounds enters the second with its lowered tmax (an answered any-hit ray with 0, which accepts
// nothing). Returns whether the lane's own ray got a hit (any-hit: its answer).
template <bool AnyHit, bool Count, bool Single, typename W>
__device__ __forceinline__ bool pair_pass(W& w, uint32_t m, PairSlots& ps, const WalkScene& uniform, const DevScene* scene,
                                          TraversalCounters& tc) {
    const uint32_t lane = lane_id();
    uint32_t incl = m;
#pragma unroll
    for (uint32_t s = 1; s < 32; s <<= 1) {
        const uint32_t x = __shfl_up_sync(kFull, incl, s);
        if (lane >= s) incl += x;
    }
    const uint32_t total = __shfl_sync(kFull, incl, 31), first = incl - m;
    if (m) {
        ps.ray[lane].w = w.tmax;
        ps.leaves[lane].w = int(first);
    }
    __syncwarp();
    const V3 o = w.origin();
    bool answered = false;
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t p = base + lane;
        // The owner of pair p: the lane whose segment starts last at or below p in this round (its
        // start bit in `heads`, its lane in ps.head), else the one whose segment runs in from before.
        const bool starts = m && first >= base && first < base + 32;
        const uint32_t heads = __reduce_or_sync(kFull, starts ? 1u << (first - base) : 0u);
        const uint32_t carry = __ballot_sync(kFull, m && first < base && incl > base);
        if (starts) ps.head[first - base] = uint8_t(lane);
        __syncwarp();
        const uint32_t upto = heads & (lane == 31 ? kFull : ((2u << lane) - 1u));
        const uint32_t k = upto ? uint32_t(ps.head[31 - __clz(upto)]) : uint32_t(__ffs(carry) - 1) & 31u;
        const V3 ko{__shfl_sync(kFull, o.x, k), __shfl_sync(kFull, o.y, k), __shfl_sync(kFull, o.z, k)};
        const DevScene* sc = Single ? uniform.scene : reinterpret_cast<const DevScene*>(__shfl_sync(kFull, reinterpret_cast<unsigned long long>(scene), k));
        if (p < total) {
            const float4 kr = ps.ray[k];
            const int4 lv = ps.leaves[k];
            const int i = pair_triangle(lv, int(p) - lv.w);
            const float4* g = (Single ? uniform.tris : sc->tris) + kTriStride * i;
            float4 g0, g1;
            ldg_pair(g, g0, g1);
            const float4 g2 = __ldg(g + 2);  // the record's fourth float4 is padding
            float t, tu, tv;
            if (Count) tc.tris++;
            if (tri_intersect(g0, g1, g2, ko, xyz(kr), kr.w, t, tu, tv) &&
                !((__float_as_int(g1.w) & 1) && alpha_passes(*sc, g, __float_as_int(g0.w), tu, tv))) {
                const unsigned long long key = AnyHit ? (unsigned long long)p : ((unsigned long long)__float_as_uint(t) << 32 | p);
                atomicMin(&ps.best[k], key);
                if (!AnyHit) ps.uv[lane] = make_float2(tu, tv);
            }
        }
        __syncwarp();
        if (m) {
            const unsigned long long key = ps.best[lane];
            if (key != ~0ull) {
                ps.best[lane] = ~0ull;
                const uint32_t pw = uint32_t(key);
                const int tri = pair_triangle(ps.leaves[lane], int(pw - first));
                const float2 uv = AnyHit ? make_float2(0.0f, 0.0f) : ps.uv[pw - base];
                ps.hit[lane] = make_float4(__int_as_float(tri), uv.x, uv.y, 0.0f);
                if (!AnyHit) w.tmax = __uint_as_float(uint32_t(key >> 32));
                ps.ray[lane].w = AnyHit ? 0.0f : w.tmax;
                answered = true;
            }
        }
        __syncwarp();
    }
    return answered;
}

// Persistent walk over a ray queue in warp steps of the pair walk: in each of `visits` rounds, every
// live lane that has not yet met leaf children visits its next node; then the warp tests all the leaf
// pairs met together (pair_pass) and their owners decide. Every lane is at a node at the start of a
// step, so the node visits run on all live lanes at once, and a leaf's triangles are tested by as many
// lanes as it has triangles, instead of the triangle tests of a few lanes running beside the node
// visits of the others. (A warp-wide vote in the rounds, to end them once enough lanes wait, measured
// slower: the rounds then reconverge the warp after every visit.) Refill, begin and end as in
// walk_queue, checked once per step; begin(i, w, ws, lane slots) and end(record, w, hit slot).
// Count: tc.steps counts node visits and warp_steps the rounds.
template <typename W, int Overflow, bool AnyHit, bool Count, bool Single, typename Begin, typename End>
__device__ __forceinline__ void walk_queue_pairs(uint32_t n, uint32_t* claim, uint32_t refill, uint32_t visits, int* stack, int stride,
                                                 PairSlots& ps, const WalkScene& uniform, TraversalCounters& tc, uint32_t& warp_steps,
                                                 Begin begin, End end) {
    int overflow[Overflow];
    W w;
    WalkScene ws = uniform;
    uint32_t idx = 0;
    bool live = false, drained = false;
    const uint32_t lane = lane_id(), below = (1u << lane) - 1u;
    const PairLane sl = ps.lane(lane);
    ps.best[lane] = ~0ull;
    for (;;) {
        uint32_t act = __ballot_sync(kFull, live);
        if (!drained && uint32_t(__popc(act)) < refill) {
            const uint32_t idle = ~act, want = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(claim, want);
            base = __shfl_sync(kFull, base, 0);
            drained = base + want >= n;
            if (!live) {
                const uint32_t r = base + uint32_t(__popc(idle & below));
                if (r < n) {
                    idx = begin(r, w, ws, sl);
                    live = true;
                }
            }
            act = __ballot_sync(kFull, live);
        }
        if (act == 0) break;
        uint32_t m = 0;
        NodeChoice ch;  // of a visit that waits for its leaf tests
        for (uint32_t it = 0; it < visits; it++) {
            if (live && m == 0) {
                m = w.visit(Single ? uniform.nodes : ws.nodes, sl, ch, &tc);
                if (Count) tc.steps++;
                if (m == 0 && !w.decide(ch, stack, stride, overflow)) {
                    end(idx, w, sl.hit);
                    live = false;
                }
            }
            if (Count) warp_steps++;
        }
        if (__any_sync(kFull, m != 0)) {
            const bool answered = pair_pass<AnyHit, Count, Single>(w, m, ps, uniform, ws.scene, tc);
            if (m && ((AnyHit && answered) || !w.decide(ch, stack, stride, overflow))) {
                end(idx, w, sl.hit);
                live = false;
            }
        }
    }
}

// The any-hit pair walk over the 4-wide BVH (PairWalker4): each round, a live lane without a leaf
// waiting visits its current node and pops the next entry; a leaf entry waits for the step's pair pass,
// after which the lane pops on (or ends: answered, or the stack ran out). Refill, begin and end as in
// walk_queue_pairs; `uniform` carries the single scene's triangles (the 4-wide BVH is built for the
// renderer's single scene only). Count: tc.steps counts node visits and warp_steps the rounds.
template <int Overflow, bool Count, typename Begin, typename End>
__device__ __forceinline__ void walk_queue_pairs4(uint32_t n, uint32_t* claim, uint32_t refill, uint32_t visits, int* stack, int stride,
                                                  PairSlots& ps, const float4* nodes4, const WalkScene& uniform, TraversalCounters& tc,
                                                  uint32_t& warp_steps, Begin begin, End end) {
    int overflow[Overflow];
    PairWalker4<Count> w;
    WalkScene ws = uniform;
    uint32_t idx = 0;
    bool live = false, drained = false;
    const uint32_t lane = lane_id(), below = (1u << lane) - 1u;
    const PairLane sl = ps.lane(lane);
    ps.best[lane] = ~0ull;
    for (;;) {
        uint32_t act = __ballot_sync(kFull, live);
        if (!drained && uint32_t(__popc(act)) < refill) {
            const uint32_t idle = ~act, want = uint32_t(__popc(idle));
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(claim, want);
            base = __shfl_sync(kFull, base, 0);
            drained = base + want >= n;
            if (!live) {
                const uint32_t r = base + uint32_t(__popc(idle & below));
                if (r < n) {
                    idx = begin(r, w, ws, sl);
                    live = true;
                }
            }
            act = __ballot_sync(kFull, live);
        }
        if (act == 0) break;
        uint32_t m = 0;
        for (uint32_t it = 0; it < visits; it++) {
            if (live && m == 0) {
                m = w.leaf_pairs(sl);
                if (m == 0) {
                    if (Count) tc.steps++;
                    if (w.visit(nodes4, stack, stride, overflow, &tc)) {
                        m = w.leaf_pairs(sl);
                    } else {
                        end(idx, w, sl.hit);
                        live = false;
                    }
                }
            }
            if (Count) warp_steps++;
        }
        if (__any_sync(kFull, m != 0)) {
            const bool answered = pair_pass<true, Count, true>(w, m, ps, uniform, uniform.scene, tc);
            if (m && (answered || !w.pop(stack, stride, overflow))) {
                end(idx, w, sl.hit);
                live = false;
            }
        }
    }
}

// The scene arrays of a launch whose views all use one scene (the renderer), or null arrays (the
// server: each ray's scene comes from its view).
__device__ __forceinline__ WalkScene single_walk_scene(const WfParams& P, bool wide) {
    if (P.single_scene < 0) return WalkScene{nullptr, nullptr, nullptr};
    return WalkScene{wide ? P.single_nodes4 : P.single_nodes, P.single_tris, P.scenes + P.single_scene};
}

// ---- trace: closest hit (traverse.h:140-142) -------------------------------------------------------
// Single: every view of the launch uses scene slot P.single_scene (the renderer); otherwise each ray's
// scene comes from its view (the server).
template <bool Count, bool Packed, bool Single>
__global__ void __maxnreg__(56) k_trace(const __grid_constant__ WfParams P) {
    extern __shared__ int smem_stack[];
    int* stack = smem_stack + threadIdx.x;
    Counters* c = P.ctr;
    if (c->tail) return;
    const uint32_t p = c->parity, n = c->count[p];
    TraversalCounters tc{0, 0, 0};
    uint32_t warp_steps = 0;
    using W = Walker<false, Count, Packed>;
    auto end = [&](uint32_t i, const W& w) {
        P.pb.hit[i] = w.tri >= 0 ? make_float4(w.tmax, __int_as_float(w.tri), w.u, w.v) : make_float4(kInf, __int_as_float(-1), 0.0f, 0.0f);
    };
    const WalkScene uni = single_walk_scene(P, false);
    if (Single) {
        walk_queue<W, kStackSize - kSmemStack, Count, true>(
            n, &c->fetch[1], P.trace_refill, P.walk_burst, stack, blockDim.x, uni, tc, warp_steps,
            [&](uint32_t i, W& w, WalkScene&) {
                w.init(xyz(P.pb.o[p][i]), xyz(P.pb.d[p][i]), kInf);
                return i;
            },
            end);
    } else {
        walk_queue<W, kStackSize - kSmemStack, Count, false>(
            n, &c->fetch[1], P.trace_refill, P.walk_burst, stack, blockDim.x, uni, tc, warp_steps,
            [&](uint32_t i, W& w, WalkScene& ws) {
                const DevScene& s = P.scenes[P.views[P.pb.id[p][i].x].scene];
                ws = WalkScene{s.nodes, s.tris, &s};
                w.init(xyz(P.pb.o[p][i]), xyz(P.pb.d[p][i]), kInf);
                return i;
            },
            end);
    }
    if (Count) {
        warp_add_u64(&c->node_visits, tc.nodes);
        warp_add_u64(&c->tri_tests, tc.tris);
        warp_add_u64(&c->trace_lane_steps, tc.steps);
        if (lane_id() == 0) atomicAdd(&c->trace_warp_steps, (unsigned long long)warp_steps);
    }
}

// The closest-hit walk as a pair walk (walk_queue_pairs): the same hits as k_trace. Dynamic shared
// memory: the stacks, then one PairSlots per warp. 56 registers (nine blocks of 128 threads per SM),
// where the single-scene kernels need no spills: spill traffic through L1 evicts node lines (24 MB of
// local stores per 960x540 bounce when the walk kept more state in registers), and 64 or 72 registers
// (eight or seven blocks) measured slower than 56 without spills.
template <bool Count, bool Single>
__global__ void __maxnreg__(56) k_trace_pairs(const __grid_constant__ WfParams P) {
    extern __shared__ int smem_stack[];
    int* stack = smem_stack + threadIdx.x;
    PairSlots& ps = reinterpret_cast<PairSlots*>(smem_stack + kSmemStack * blockDim.x)[threadIdx.x >> 5];
    Counters* c = P.ctr;
    if (c->tail) return;
    const uint32_t p = c->parity, n = c->count[p];
    TraversalCounters tc{0, 0, 0};
    uint32_t warp_steps = 0;
    using W = PairWalker<false, Count>;
    auto end = [&](uint32_t i, const W& w, const float4& h) {
        P.pb.hit[i] = __float_as_int(h.x) >= 0 ? make_float4(w.tmax, h.x, h.y, h.z) : make_float4(kInf, __int_as_float(-1), 0.0f, 0.0f);
    };
    const WalkScene uni = single_walk_scene(P, false);
    walk_queue_pairs<W, kStackSize - kSmemStack, false, Count, Single>(
        n, &c->fetch[1], P.trace_refill, P.pair_visits, stack, blockDim.x, ps, uni, tc, warp_steps,
        [&](uint32_t i, W& w, WalkScene& ws, const PairLane& sl) {
            if (!Single) {
                const DevScene& s = P.scenes[P.views[P.pb.id[p][i].x].scene];
                ws = WalkScene{s.nodes, s.tris, &s};
            }
            w.init(xyz(P.pb.o[p][i]), xyz(P.pb.d[p][i]), kInf, sl);
            return i;
        },
        end);
    if (Count) {
        warp_add_u64(&c->node_visits, tc.nodes);
        warp_add_u64(&c->tri_tests, tc.tris);
        warp_add_u64(&c->trace_lane_steps, tc.steps);
        if (lane_id() == 0) atomicAdd(&c->trace_warp_steps, (unsigned long long)warp_steps);
    }
}

// Sort key of a continuing ray: direction octant, then the Morton code of its origin's cell in the
// scene box (`bits` per axis). Rays in one bucket start close together and head the same way, so
// a warp of them walks similar nodes.
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
    v &= 0x3ff;
    v = (v | (v << 16)) & 0x030000FF;
    v = (v | (v << 8)) & 0x0300F00F;
    v = (v | (v << 4)) & 0x030C30C3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}
__device__ __forceinline__ uint32_t ray_key(const DevScene& s, V3 o, V3 d, int bits) {
    float cells = float(1u << bits);
    auto cell = [&](float x, float lo, float inv) {
        float f = (x - lo) * inv * cells;
        f = fminf(fmaxf(f, 0.0f), cells - 1.0f);
        return uint32_t(f);
    };
    uint32_t m = spread3(cell(o.x, s.bounds_lo_x, s.inv_extent_x)) | (spread3(cell(o.y, s.bounds_lo_y, s.inv_extent_y)) << 1) |
                 (spread3(cell(o.z, s.bounds_lo_z, s.inv_extent_z)) << 2);
    uint32_t oct = (d.x < 0 ? 1u : 0u) | (d.y < 0 ? 2u : 0u) | (d.z < 0 ? 4u : 0u);
    return (oct << (3 * bits)) | m;
}

// ---- shade: one vertex of trace_path (integrator.h:158-262) -----------------------------------------
struct PathState {
    V3 ro, rd, beta, L;
    float prev_pdf;
    uint32_t flags;  // depth | prev_delta << 16
    uint4 id;        // (view, local work index, pixel, sample in pass)
    Rng rng;
};
struct ShadowRay {
    V3 o, d, c;
    float tmax;
};

__device__ __forceinline__ PathState load_path(const WfParams& P, uint32_t p, uint32_t i) {
    PathState st;
    float4 o4 = P.pb.o[p][i], d4 = P.pb.d[p][i], b4 = P.pb.beta[p][i], l4 = P.pb.lr[p][i];
    st.id = P.pb.id[p][i];
    st.ro = xyz(o4);
    st.rd = xyz(d4);
    st.prev_pdf = o4.w;
    st.flags = __float_as_uint(d4.w);
    st.beta = xyz(b4);
    st.L = V3{b4.w, l4.x, l4.y};
    st.rng.state = uint64_t(__float_as_uint(l4.z)) | (uint64_t(__float_as_uint(l4.w)) << 32);
    st.rng.inc = (uint64_t(st.id.z) << 1u) | 1u;
    return st;
}

// One vertex of trace_path for a path whose closest hit is h4 = (t, tri, u, v): adds the emitted
// light it sees to st.L, writes the first vertex's G-buffer, samples the light (a shadow ray in *sh
// when `shadow` comes back true) and the continuation (st's ray, throughput and flags). Returns
// whether the path continues.
__device__ __forceinline__ bool shade_vertex(const WfParams& P, PathState& st, float4 h4, bool& shadow, ShadowRay& sh) {
    const uint4 id = st.id;
    const DevView& v = P.views[id.x];
    const DevScene& s = scene_for(P, id.x);
    V3& ro = st.ro;
    V3& rd = st.rd;
    V3& beta = st.beta;
    V3& L = st.L;
    float& prev_pdf = st.prev_pdf;
    Rng& rng = st.rng;
    bool cont = false;
    shadow = false;
    int depth = int(st.flags & 0xffffu);
    bool prev_delta = (st.flags >> 16) & 1u;
    int tri = __float_as_int(h4.y);
    bool gbuf = v.gbuffer && id.w == 0 && depth == 0;
    if (tri < 0) {
        // Miss: the environment, weighted against light sampling (integrator.h:159-177).
        V3 le = env_radiance(s, rd);
        float w = (prev_delta || s.p_env <= 0) ? 1.0f : power_heuristic(prev_pdf, env_pdf(s, rd));
        V3 cc = beta * le * w;
        clamp_contribution(cc, depth, v.clamp);
        L = L + cc;
        if (gbuf) {
            V3 pos = ro + rd * 1e4f;
            v.g_albedo[id.z] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
            v.g_normal_depth[id.z] = make_float4(-rd.x, -rd.y, -rd.z, 0.0f);
            if (v.g_position) v.g_position[id.z] = make_float4(pos.x, pos.y, pos.z, -1.0f);
            if (v.g_emission) v.g_emission[id.z] = make_float4(le.x, le.y, le.z, 1.0f);
            if (v.g_edge) {
                v.g_edge[id.z] = edge_record(-rd, 0.0f, -1);
                v.g_motion[id.z] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            }
        }
        return false;
    }
    Interaction it = surface_at(s, ro, rd, h4.x, tri, h4.z, h4.w);
    V3 wo_world = -rd;
    if (!is_black(it.emission)) {
        float w = 1.0f;
        if (!prev_delta) w = power_heuristic(prev_pdf, emissive_pdf(s, tri, it.emissive_entry, rd, h4.x));
        V3 cc = beta * it.emission * w;
        clamp_contribution(cc, depth, v.clamp);
        L = L + cc;
    }
    Bsdf bsdf = make_bsdf(it.params);
    if (gbuf) {
        V3 alb = bsdf_albedo(bsdf);
        v.g_albedo[id.z] = make_float4(alb.x, alb.y, alb.z, 1.0f);
        v.g_normal_depth[id.z] = make_float4(it.ns.x, it.ns.y, it.ns.z, h4.x);
        if (v.g_position) v.g_position[id.z] = make_float4(it.p.x, it.p.y, it.p.z, float(it.material));
        if (v.g_emission) v.g_emission[id.z] = make_float4(it.emission.x, it.emission.y, it.emission.z, 1.0f);
        if (v.g_edge) {
            const int px = int(id.z % uint32_t(v.width)), py = int(id.z / uint32_t(v.width));
            v.g_edge[id.z] = edge_record(it.ns, h4.x, it.material);
            v.g_motion[id.z] = motion_record(*reinterpret_cast<const PrevCamera*>(v.prev_cam), v.has_prev != 0, it.p, it.material, px, py,
                                             v.width, v.height);
        }
    }
    if (depth + 1 >= v.max_depth) return false;
    V3 wo = to_local(it.frame, wo_world);
    bool nee = v.nee && s.has_lights && samples_lights(bsdf);
    if (nee) {
        float ug = rng_next(rng);
        V2 ul = rng_next2(rng);
        float uk = rng_next(rng);
        LightSample ls = sample_light(s, it.p, ug, ul, uk, nullptr);
        if (ls.pdf > 0 && !is_black(ls.radiance)) {
            V3 wi = to_local(it.frame, ls.wi);
            float pdf_b;
            V3 f = bsdf_eval_pdf(bsdf, wo, wi, &pdf_b);
            if (!is_black(f)) {
                sh.o = offset_ray(it.p, dot(ls.wi, it.ng) > 0 ? it.ng : -it.ng);
                sh.d = ls.wi;
                sh.tmax = ls.dist == kInf ? kInf : ls.dist * (1.0f - 1e-4f);
                float w = ls.delta ? 1.0f : power_heuristic(ls.pdf, pdf_b);
                sh.c = beta * f * fabsf(wi.z) * ls.radiance * (w / ls.pdf);
                clamp_contribution(sh.c, depth, v.clamp);
                shadow = true;
            }
        }
    }
    float u_lobe = rng_next(rng);
    V2 u = rng_next2(rng);
    float u_sub = rng_next(rng);
    BsdfSample bs = bsdf_sample(bsdf, wo, u_lobe, u, u_sub);
    if (bs.valid) {
        beta = beta * (bs.f * (fabsf(bs.wi.z) / bs.pdf));
        if (is_finite(beta) && !is_black(beta)) {
            V3 wi_world = to_world(it.frame, bs.wi);
            float side = dot(wi_world, it.ng) * dot(wo_world, it.ng);
            if (!(bs.transmitted ? side >= 0 : side <= 0)) {
                prev_pdf = bs.pdf;
                ro = offset_ray(it.p, dot(wi_world, it.ng) > 0 ? it.ng : -it.ng);
                rd = normalize(wi_world);
                cont = true;
                if (depth + 1 >= v.rr_depth) {
                    float qq = fmaxf(0.05f, 1.0f - max_component(beta));
                    if (rng_next(rng) < qq) cont = false;
                    else beta = beta * (1.0f / (1.0f - qq));
                }
                st.flags = uint32_t(depth + 1) | ((nee ? 0u : 1u) << 16);
            }
        }
    }
    return cont;
}

// Shades path `i` of the current queue and appends its continuation and shadow ray to the next
// queues (every lane of the warp calls it; `active` is false for lanes without a path).
__device__ __forceinline__ void shade_path(const WfParams& P, Counters* c, uint32_t p, uint32_t i, bool active) {
    const uint32_t q = p ^ 1u;
    bool cont = false, shadow = false;
    PathState st;
    ShadowRay sh;
    if (active) {
        st = load_path(P, p, i);
        cont = shade_vertex(P, st, P.pb.hit[i], shadow, sh);
    } else {
        st.id = make_uint4(0, 0, 0, 0);
    }
    const uint4 id = st.id;
    // Continuing paths move to the other buffer, compacted.
    uint32_t slot = warp_append(cont, &c->count[q]);
    if (P.sort_bits > 0 && c->sorting) {
        uint32_t key = cont ? ray_key(scene_for(P, id.x), st.ro, st.rd, P.sort_bits) : 0xffffffffu;
        uint32_t peers = __match_any_sync(kFull, key);
        if (cont) {
            P.keys[slot] = key;
            if (int(lane_id()) == __ffs(peers) - 1) atomicAdd(&P.hist[key], uint32_t(__popc(peers)));
        }
    }
    if (cont) {
        P.pb.o[q][slot] = make_float4(st.ro.x, st.ro.y, st.ro.z, st.prev_pdf);
        P.pb.d[q][slot] = make_float4(st.rd.x, st.rd.y, st.rd.z, __uint_as_float(st.flags));
        P.pb.beta[q][slot] = make_float4(st.beta.x, st.beta.y, st.beta.z, st.L.x);
        P.pb.lr[q][slot] =
            make_float4(st.L.y, st.L.z, __uint_as_float(uint32_t(st.rng.state)), __uint_as_float(uint32_t(st.rng.state >> 32)));
        P.pb.id[q][slot] = id;
    } else if (active) {
        P.views[id.x].sample_out[id.y] = make_float4(st.L.x, st.L.y, st.L.z, 0.0f);
    }
    // Shadow rays: target the continuing slot, or the finished sample.
    uint32_t qs = warp_append(shadow, &c->shadow_count);
    if (P.shadow_sort_bits > 0 && c->shadow_sorting) {
        // Their sort key (direction octant, Morton cell of the origin) and bucket count, for the walk order.
        const uint32_t key = shadow ? ray_key(scene_for(P, id.x), sh.o, sh.d, P.shadow_sort_bits) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(kFull, key);
        if (shadow) {
            P.shadow_keys[qs] = key;
            if (int(lane_id()) == __ffs(peers) - 1) atomicAdd(&P.shadow_hist[key], uint32_t(__popc(peers)));
        }
    }
    if (shadow) {
        P.pb.sh0[qs] = make_float4(sh.o.x, sh.o.y, sh.o.z, sh.tmax);
        P.pb.sh1[qs] = make_float4(sh.d.x, sh.d.y, sh.d.z, __uint_as_float(cont ? slot : id.y));
        P.pb.sh2[qs] = make_float4(sh.c.x, sh.c.y, sh.c.z, __uint_as_float(id.x | (cont ? 0u : 0x80000000u)));
    }
    // Progress of views that count finished paths (the request server).
    bool finished = active && !cont;
    if (P.num_views > 1 || P.views[0].done_counter) {
        uint32_t key = finished ? id.x : 0xffffffffu;
        uint32_t peers = __match_any_sync(kFull, key);
        if (finished && int(lane_id()) == __ffs(peers) - 1) {
            unsigned long long* dc = P.views[id.x].done_counter;
            if (dc) atomicAdd(dc, (unsigned long long)__popc(peers));
        }
    }
}

// The shading class of a queued path: 0 for a miss, else the class of the hit triangle's material
// (1..32, precomputed per material at upload from its lobes, textures and emission).
constexpr uint32_t kShadeKeys = 64;
__device__ __forceinline__ uint32_t shade_key(const WfParams& P, uint32_t p, uint32_t i) {
    int tri = __float_as_int(P.pb.hit[i].y);
    if (tri < 0) return 0;
    const DevScene& s = scene_for(P, P.single_scene >= 0 ? 0 : int(P.pb.id[p][i].x));
    return s.shade_keys[__float_as_int(__ldg(s.tris + kTriStride * tri).w)];
}

// Persistent over the queue. Without material sorting each warp claims 32 paths in queue order. With
// it each block claims a window of sort_material x blockDim paths, orders them by shading class in
// shared memory (a counting sort on 64 keys) and shades them in that order, so a warp mostly runs one
// BSDF lobe and one texture pattern. The order in which paths are shaded changes only where their
// outputs are appended, not any path's result.
// On iterations whose continuing rays are sorted afterwards (Counters::sorting), the order of the
// shade output no longer matters to the next trace, so the window grows fourfold (16 x 256 paths)
// for more coherent shading.
constexpr uint32_t kMaxShadeRounds = 16;
constexpr uint32_t kMaxShadeWindow = kMaxShadeRounds * 256;
__global__ void __launch_bounds__(256) k_shade(const __grid_constant__ WfParams P) {
    Counters* c = P.ctr;
    if (c->tail) return;
    const uint32_t p = c->parity, n = c->count[p];
    if (!P.sort_material) {
        for (;;) {
            uint32_t i0 = warp_fetch(&c->fetch[2]);
            if (i0 >= n) break;
            uint32_t i = i0 + lane_id();
            shade_path(P, c, p, i, i < n);
        }
        return;
    }
    __shared__ uint32_t s_base, s_hist[kShadeKeys], s_perm[kMaxShadeWindow], s_kr[kMaxShadeWindow];
    const uint32_t tid = threadIdx.x;
    const uint32_t rounds = min(uint32_t(P.sort_material) * (c->sorting ? 4u : 1u), kMaxShadeRounds);
    const uint32_t window = rounds * blockDim.x;
    for (;;) {
        if (tid == 0) s_base = atomicAdd(&c->fetch[2], window);
        for (uint32_t k = tid; k < kShadeKeys; k += blockDim.x) s_hist[k] = 0;
        __syncthreads();
        const uint32_t i0 = s_base;
        if (i0 >= n) break;
        // Keys four rounds at a time (their dependent loads overlap), kept with their ranks in
        // shared memory as key << 16 | rank.
        for (uint32_t r0 = 0; r0 < rounds; r0 += 4) {
            uint32_t key[4];
#pragma unroll
            for (uint32_t q = 0; q < 4; q++) {
                const uint32_t i = i0 + (r0 + q) * blockDim.x + tid;
                key[q] = (r0 + q < rounds && i < n) ? shade_key(P, p, i) : kShadeKeys - 1;
            }
#pragma unroll
            for (uint32_t q = 0; q < 4; q++) {
                if (r0 + q < rounds) {
                    const uint32_t rank = atomicAdd(&s_hist[key[q]], 1u);
                    s_kr[(r0 + q) * blockDim.x + tid] = (key[q] << 16) | rank;
                }
            }
        }
        __syncthreads();
        if (tid < 32) {  // exclusive scan of the 64 bucket counts, two per lane
            uint32_t a = s_hist[2 * tid], b = s_hist[2 * tid + 1];
            uint32_t incl = a + b;
            for (int off = 1; off < 32; off <<= 1) {
                uint32_t v = __shfl_up_sync(kFull, incl, off);
                if (int(tid) >= off) incl += v;
            }
            uint32_t excl = incl - a - b;
            s_hist[2 * tid] = excl;
            s_hist[2 * tid + 1] = excl + a;
        }
        __syncthreads();
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t slot = r * blockDim.x + tid, kr = s_kr[slot];
            s_perm[s_hist[kr >> 16] + (kr & 0xffffu)] = i0 + slot;
        }
        __syncthreads();
        for (uint32_t r = 0; r < rounds; r++) {
            const uint32_t j = s_perm[r * blockDim.x + tid];
            shade_path(P, c, p, j, j < n);
        }
        __syncthreads();
    }
}

// ---- tail: the last queued paths, each finished by one thread --------------------------------------------
// Once no new paths remain and few are queued, an iteration's kernels have too little work to cover
// the latency of their longest ray, and every remaining bounce would pay that again. k_tail takes the
// whole queue instead: each thread traces, shades and shadow-tests its path bounce after bounce, in
// the order of the queued kernels (emission, then the light sample's contribution, then the next
// bounce), so each path's result is the same as through the queues.
template <bool Count, bool Packed>
__global__ void __launch_bounds__(256) k_tail(const __grid_constant__ WfParams P) {
    Counters* c = P.ctr;
    if (!c->tail) return;
    extern __shared__ int smem_stack[];
    int* stack = smem_stack + threadIdx.x;
    const uint32_t p = c->parity, n = c->count[p];
    TraversalCounters tc{0, 0}, ts{0, 0};
    unsigned long long rays = 0, shadow_rays = 0;
    for (;;) {
        uint32_t i0 = warp_fetch(&c->fetch[5]);
        if (i0 >= n) break;
        uint32_t i = i0 + lane_id();
        if (i >= n) continue;
        PathState st = load_path(P, p, i);
        const DevScene& s = scene_for(P, st.id.x);
        for (bool first = true;; first = false) {
            Hit h{kInf, -1, 0.0f, 0.0f};
            traverse<false, Count, Packed>(s, st.ro, st.rd, kInf, h, stack, blockDim.x, &tc);
            if (!first) rays++;  // the setup counted each queued path's first ray
            bool shadow = false;
            ShadowRay sh;
            bool cont = shade_vertex(P, st, make_float4(h.t, __int_as_float(h.tri), h.u, h.v), shadow, sh);
            if (shadow) {
                Hit hs{kInf, -1, 0.0f, 0.0f};
                shadow_rays++;
                bool occ = (P.wide_shadows && s.nodes4) ? occluded4<Count, Packed>(s, sh.o, sh.d, sh.tmax, stack, blockDim.x, &ts)
                                                        : traverse<true, Count, Packed>(s, sh.o, sh.d, sh.tmax, hs, stack, blockDim.x, &ts);
                if (!occ) st.L = st.L + sh.c;
            }
            if (!cont) break;
        }
        const DevView& v = P.views[st.id.x];
        v.sample_out[st.id.y] = make_float4(st.L.x, st.L.y, st.L.z, 0.0f);
        if (v.done_counter) atomicAdd(v.done_counter, 1ull);
    }
    if (rays) atomicAdd(&c->rays, rays);
    if (shadow_rays) atomicAdd(&c->shadow_rays, shadow_rays);
    if (Count) {
        warp_add_u64(&c->node_visits, tc.nodes);
        warp_add_u64(&c->tri_tests, tc.tris);
        warp_add_u64(&c->shadow_node_visits, ts.nodes);
        warp_add_u64(&c->shadow_tri_tests, ts.tris);
    }
}

// ---- shadow: any hit (traverse.h:144-147) --------------------------------------------------------------
// Capped at 51 registers (five 256-thread blocks per SM): the any-hit walk gains more from the extra
// resident warps than it loses to the tighter allocation (measured; the closest-hit walk does not).
// Wide: the 4-wide BVH, used when every ray of the launch has it (a single scene that carries one);
// otherwise the BVH2.
// The shadow queue of an iteration: the order it is walked in, and the delivery of unoccluded rays.
struct ShadowQueue {
    const WfParams& P;
    uint32_t q;   // parity of the paths the rays contribute to
    bool sorted;
    // Queue position -> record: the sorted order of this iteration's shadow rays, or the queue's own.
    __device__ __forceinline__ uint32_t record(uint32_t i) const { return sorted ? __ldg(P.shadow_perm + i) : i; }
    // Starts walker w on queue position i; returns the record.
    template <typename W>
    __device__ __forceinline__ uint32_t init(uint32_t i, W& w) const {
        const uint32_t j = record(i);
        const float4 a = P.pb.sh0[j];
        w.init(xyz(a), xyz(P.pb.sh1[j]), a.w);
        return j;
    }
    // The scene of record j (multi-scene launches).
    __device__ __forceinline__ const DevScene& scene(uint32_t j) const {
        return P.scenes[P.views[__float_as_uint(P.pb.sh2[j].w) & 0x7fffffffu].scene];
    }
    // An unoccluded shadow ray adds its contribution to its path (or to its finished sample).
    __device__ __forceinline__ void deliver(uint32_t i) const {
        const float4 cc = P.pb.sh2[i];
        const uint32_t tag = __float_as_uint(cc.w), view = tag & 0x7fffffffu, target = __float_as_uint(P.pb.sh1[i].w);
        if (tag & 0x80000000u) {
            float4* so = P.views[view].sample_out + target;
            float4 l = *so;
            *so = make_float4(l.x + cc.x, l.y + cc.y, l.z + cc.z, l.w);
        } else {
            float4 b4 = P.pb.beta[q][target], l4 = P.pb.lr[q][target];
            b4.w = b4.w + cc.x;
            l4.x = l4.x + cc.y;
            l4.y = l4.y + cc.z;
            P.pb.beta[q][target] = b4;
            P.pb.lr[q][target] = l4;
        }
    }
};

template <bool Count, bool Packed, bool Wide, bool Single>
__global__ void __launch_bounds__(256, 5) k_shadow(const __grid_constant__ WfParams P) {
    extern __shared__ int smem_stack[];
    int* stack = smem_stack + threadIdx.x;
    Counters* c = P.ctr;
    if (c->tail) return;
    const uint32_t n = c->shadow_count;
    TraversalCounters tc{0, 0, 0};
    uint32_t warp_steps = 0;
    const ShadowQueue sq{P, c->parity ^ 1u, c->shadow_sorting != 0};
    auto deliver = [&](uint32_t i) { sq.deliver(i); };
    auto init = [&](uint32_t i, auto& w) { return sq.init(i, w); };
    if (Wide && Single && P.single_nodes4) {
        using W4 = AnyWalker4<Count, Packed>;
        walk_queue<W4, kBvh4Stack - kSmemStack, Count, true>(
            n, &c->fetch[3], P.shadow_refill, P.walk_burst, stack, blockDim.x, single_walk_scene(P, true), tc, warp_steps,
            [&](uint32_t i, W4& w, WalkScene&) { return init(i, w); },
            [&](uint32_t i, const W4& w) {
                if (!w.hit) deliver(i);
            });
    } else {
        using W = Walker<true, Count, Packed>;
        auto end = [&](uint32_t i, const W& w) {
            if (w.tri < 0) deliver(i);
        };
        if (Single) {
            walk_queue<W, kStackSize - kSmemStack, Count, true>(n, &c->fetch[3], P.shadow_refill, P.walk_burst, stack, blockDim.x, single_walk_scene(P, false),
                                                                tc, warp_steps, [&](uint32_t i, W& w, WalkScene&) { return init(i, w); }, end);
        } else {
            walk_queue<W, kStackSize - kSmemStack, Count, false>(
                n, &c->fetch[3], P.shadow_refill, P.walk_burst, stack, blockDim.x, WalkScene{nullptr, nullptr, nullptr}, tc, warp_steps,
                [&](uint32_t i, W& w, WalkScene& ws) {
                    const uint32_t j = init(i, w);
                    const DevScene& s = sq.scene(j);
                    ws = WalkScene{s.nodes, s.tris, &s};
                    return j;
                },
                end);
        }
    }
    if (Count) {
        warp_add_u64(&c->shadow_node_visits, tc.nodes);
        warp_add_u64(&c->shadow_tri_tests, tc.tris);
        warp_add_u64(&c->shadow_lane_steps, tc.steps);
        if (lane_id() == 0) atomicAdd(&c->shadow_warp_steps, (unsigned long long)warp_steps);
    }
}

// The any-hit walk as a pair walk (walk_queue_pairs) over the BVH2, or (Wide, where the single scene
// carries one) over the 4-wide BVH (walk_queue_pairs4): the same answers as k_shadow.
template <bool Count, bool Single, bool Wide>
__global__ void __maxnreg__(56) k_shadow_pairs(const __grid_constant__ WfParams P) {
    extern __shared__ int smem_stack[];
    int* stack = smem_stack + threadIdx.x;
    PairSlots& ps = reinterpret_cast<PairSlots*>(smem_stack + kSmemStack * blockDim.x)[threadIdx.x >> 5];
    Counters* c = P.ctr;
    if (c->tail) return;
    const uint32_t n = c->shadow_count;
    TraversalCounters tc{0, 0, 0};
    uint32_t warp_steps = 0;
    const ShadowQueue sq{P, c->parity ^ 1u, c->shadow_sorting != 0};
    auto end = [&](uint32_t i, const auto&, const float4& h) {
        if (__float_as_int(h.x) < 0) sq.deliver(i);
    };
    if (Wide && Single && P.single_nodes4) {
        walk_queue_pairs4<kBvh4Stack - kSmemStack, Count>(
            n, &c->fetch[3], P.shadow_refill, P.pair_visits, stack, blockDim.x, ps, P.single_nodes4, single_walk_scene(P, false), tc,
            warp_steps,
            [&](uint32_t i, PairWalker4<Count>& w, WalkScene&, const PairLane& sl) {
                const uint32_t j = sq.record(i);
                const float4 a = P.pb.sh0[j];
                w.init(xyz(a), xyz(P.pb.sh1[j]), a.w, sl);
                return j;
            },
            end);
    } else {
        using W = PairWalker<true, Count>;
        walk_queue_pairs<W, kStackSize - kSmemStack, true, Count, Single>(
            n, &c->fetch[3], P.shadow_refill, P.pair_visits, stack, blockDim.x, ps, single_walk_scene(P, false), tc, warp_steps,
            [&](uint32_t i, W& w, WalkScene& ws, const PairLane& sl) {
                const uint32_t j = sq.record(i);
                const float4 a = P.pb.sh0[j];
                w.init(xyz(a), xyz(P.pb.sh1[j]), a.w, sl);
                if (!Single) {
                    const DevScene& s = sq.scene(j);
                    ws = WalkScene{s.nodes, s.tris, &s};
                }
                return j;
            },
            end);
    }
    if (Count) {
        warp_add_u64(&c->shadow_node_visits, tc.nodes);
        warp_add_u64(&c->shadow_tri_tests, tc.tris);
        warp_add_u64(&c->shadow_lane_steps, tc.steps);
        if (lane_id() == 0) atomicAdd(&c->shadow_warp_steps, (unsigned long long)warp_steps);
    }
}

// ---- ray sorting: a counting sort of the shade output by ray key ------------------------------------------
// Exclusive scan of the bucket counts into write offsets (one block), then zero the counts. Each warp
// takes a contiguous 32nd of the buckets and reads it 32 consecutive counts at a time (coalesced):
// a first pass sums its part, the 32 part sums are scanned, and a second pass writes the offsets.
// Shadow: the shadow queue's histogram (shadow_hist -> shadow_offsets), when its order is sorted.
template <bool Shadow>
__global__ void __launch_bounds__(1024) k_sort_scan(const __grid_constant__ WfParams P, uint32_t buckets) {
    if (!(Shadow ? P.ctr->shadow_sorting : P.ctr->sorting)) return;
    uint32_t* const hist = Shadow ? P.shadow_hist : P.hist;
    uint32_t* const offsets = Shadow ? P.shadow_offsets : P.offsets;
    __shared__ uint32_t part[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t per = (buckets + 31u) / 32u;
    const uint32_t lo = min(warp * per, buckets), hi = min(lo + per, buckets);
    uint32_t total = 0;
    for (uint32_t base = lo; base < hi; base += 32u) {
        const uint32_t k = base + lane;
        uint32_t v = k < hi ? hist[k] : 0u;
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
        total += v;
    }
    if (lane == 0) part[warp] = total;
    __syncthreads();
    if (warp == 0) {
        const uint32_t t = part[lane];
        uint32_t incl = t;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, off);
            if (int(lane) >= off) incl += v;
        }
        part[lane] = incl - t;
    }
    __syncthreads();
    uint32_t carry = part[warp];
    for (uint32_t base = lo; base < hi; base += 32u) {
        const uint32_t k = base + lane;
        const uint32_t v = k < hi ? hist[k] : 0u;
        uint32_t incl = v;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t u = __shfl_up_sync(kFull, incl, off);
            if (int(lane) >= off) incl += u;
        }
        if (k < hi) {
            offsets[k] = carry + incl - v;
            hist[k] = 0;
        }
        carry += __shfl_sync(kFull, incl, 31);
    }
}

// Moves every continuing path from the shade output into the (now free) input buffer at its
// bucket's next position; the next setup then finds the sorted paths there.
__global__ void __launch_bounds__(256) k_sort_scatter(const __grid_constant__ WfParams P) {
    Counters* c = P.ctr;
    if (!c->sorting) return;
    const uint32_t p = c->parity, q = p ^ 1u, n = c->count[q];
    // Whole warps over consecutive runs of 32 paths, split statically (no claim counter).
    const uint32_t warps = gridDim.x * (blockDim.x / 32u);
    for (uint32_t i0 = (blockIdx.x * (blockDim.x / 32u) + threadIdx.x / 32u) * 32u; i0 < n; i0 += warps * 32u) {
        uint32_t i = i0 + lane_id();
        uint32_t key = i < n ? P.keys[i] : 0xffffffffu;
        uint32_t peers = __match_any_sync(kFull, key);
        int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (i < n && int(lane_id()) == leader) base = atomicAdd(&P.offsets[key], uint32_t(__popc(peers)));
        base = __shfl_sync(kFull, base, leader);
        if (i < n) {
            uint32_t dst = base + __popc(peers & ((1u << lane_id()) - 1u));
            P.pb.o[p][dst] = P.pb.o[q][i];
            P.pb.d[p][dst] = P.pb.d[q][i];
            P.pb.beta[p][dst] = P.pb.beta[q][i];
            P.pb.lr[p][dst] = P.pb.lr[q][i];
            P.pb.id[p][dst] = P.pb.id[q][i];
        }
    }
}

// The walk order of the shadow queue: each ray's queue position lands at its bucket's next place in
// shadow_perm (the records themselves stay where shade wrote them).
__global__ void __launch_bounds__(256) k_shadow_order(const __grid_constant__ WfParams P) {
    Counters* c = P.ctr;
    if (!c->shadow_sorting) return;
    const uint32_t n = c->shadow_count;
    const uint32_t warps = gridDim.x * (blockDim.x / 32u);
    for (uint32_t i0 = (blockIdx.x * (blockDim.x / 32u) + threadIdx.x / 32u) * 32u; i0 < n; i0 += warps * 32u) {
        const uint32_t i = i0 + lane_id();
        const uint32_t key = i < n ? P.shadow_keys[i] : 0xffffffffu;
        const uint32_t peers = __match_any_sync(kFull, key);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (i < n && int(lane_id()) == leader) base = atomicAdd(&P.shadow_offsets[key], uint32_t(__popc(peers)));
        base = __shfl_sync(kFull, base, leader);
        if (i < n) P.shadow_perm[base + __popc(peers & ((1u << lane_id()) - 1u))] = i;
    }
}

// After the scatter: the sorted paths live in the input buffer; make the next setup flip to it.
__global__ void k_sort_finish(Counters* c) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || !c->sorting) return;
    uint32_t p = c->parity, q = p ^ 1u;
    c->count[p] = c->count[q];
    c->count[q] = 0;
    c->parity = q;
}

// ---- accumulate: CpuRenderer's per-pixel sum in sample order (cpu_renderer.cpp:28-31) ------------------
__global__ void k_accumulate(const DevView* vp, int first, int last) {
    const DevView& v = *vp;
    uint32_t npix = uint32_t(v.width) * uint32_t(v.height);
    uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npix) return;
    int x, y;
    tile_pixel(q, v.width, v.height, x, y);
    uint32_t pix = uint32_t(y) * uint32_t(v.width) + uint32_t(x);
    float4 acc = first ? make_float4(0, 0, 0, 0) : v.acc_pass[pix];
    for (int s = 0; s < v.spp; s++) {
        float4 l4 = v.sample_out[size_t(s) * npix + q];
        V3 l = xyz(l4);
        // render_sample's guard (pixel.h:26-27).
        if (!is_finite(l) || l.x < 0 || l.y < 0 || l.z < 0) l = v3(0);
        acc.x = acc.x + l.x;
        acc.y = acc.y + l.y;
        acc.z = acc.z + l.z;
        float lum = luminance(l);
        acc.w = acc.w + lum * lum;
        if (v.realtime && s == 0 && v.g_color) v.g_color[pix] = make_float4(l.x, l.y, l.z, 1.0f);
    }
    if (last) {
        float4 a = v.accum[pix];
        a.x = a.x + acc.x;
        a.y = a.y + acc.y;
        a.z = a.z + acc.z;
        a.w = a.w + acc.w;
        v.accum[pix] = a;
    } else {
        v.acc_pass[pix] = acc;
    }
}

// ---- probes ----------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_trace_primary(const DevScene* sp, CameraArg cam, int w, int h, uint32_t frame, uint32_t seed,
                                                      float4* out) {
    extern __shared__ int smem_stack[];
    int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= w || y >= h) return;
    const DevScene& s = *sp;
    uint32_t pixel = uint32_t(y) * uint32_t(w) + uint32_t(x);
    Rng rng = pixel_rng(pixel, seed, frame);
    V2 jitter = rng_next2(rng);
    V2 lens = rng_next2(rng);
    V3 o, d;
    camera_ray(cam.c, float(x) + jitter.x, float(y) + jitter.y, w, h, lens, o, d);
    Hit hit{kInf, -1, 0.0f, 0.0f};
    TraversalCounters tc{0, 0};
    traverse<false, false>(s, o, d, kInf, hit, smem_stack + threadIdx.x, blockDim.x, &tc);
    out[pixel] = make_float4(hit.t, __int_as_float(hit.tri), hit.u, hit.v);
}

__global__ void __launch_bounds__(128) k_heatmap(const DevScene* sp, CameraArg cam, int w, int h, float* out) {
    extern __shared__ int smem_stack[];
    int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= w || y >= h) return;
    V3 o, d;
    camera_ray(cam.c, float(x) + 0.5f, float(y) + 0.5f, w, h, V2{0.5f, 0.5f}, o, d);
    Hit hit{kInf, -1, 0.0f, 0.0f};
    TraversalCounters tc{0, 0};
    traverse<false, true>(*sp, o, d, kInf, hit, smem_stack + threadIdx.x, blockDim.x, &tc);
    out[size_t(y) * size_t(w) + size_t(x)] = float(tc.nodes);
}

// Any-hit walks of caller rays (occluded, traverse.h:144-147): per ray whether it is occluded, the
// first triangle accepted (-1: none) and the node visits (BVH2 walk; the 4-wide walk's visits are of
// its own nodes). The same walkers as the shadow kernel.
__global__ void __launch_bounds__(128) k_occlusion_probe(const DevScene* sp, const float4* rays, int n, int wide, int4* out) {
    extern __shared__ int smem_stack[];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevScene& s = *sp;
    const float4 a = rays[2 * i], b = rays[2 * i + 1];
    TraversalCounters tc{0, 0, 0};
    if (wide && s.nodes4) {
        const bool occ = occluded4<true>(s, xyz(a), xyz(b), a.w, smem_stack + threadIdx.x, blockDim.x, &tc);
        out[i] = make_int4(occ ? 1 : 0, -1, int(tc.nodes), int(tc.tris));
        return;
    }
    Hit h{kInf, -1, 0.0f, 0.0f};
    const bool occ = traverse<true, true>(s, xyz(a), xyz(b), a.w, h, smem_stack + threadIdx.x, blockDim.x, &tc);
    out[i] = make_int4(occ ? 1 : 0, occ ? h.tri : -1, int(tc.nodes), int(tc.tris));
}

// The probes above through the pair walks (walk_queue_pairs, PairWalker: the code of k_trace_pairs and
// k_shadow_pairs) over a queue of the probe's rays, so that the default walks are pinned ray by ray:
// the camera rays' hits, and per caller ray the occlusion, first accepted triangle and node visits (the
// triangle tests of a pair walk are done by other lanes: reported as -1). `claim` is a zeroed counter.
__global__ void __launch_bounds__(128) k_trace_primary_pairs(const DevScene* sp, CameraArg cam, int w, int h, uint32_t frame, uint32_t seed,
                                                            float4* out, uint32_t* claim, uint32_t visits) {
    extern __shared__ int smem_stack[];
    PairSlots& ps = reinterpret_cast<PairSlots*>(smem_stack + kSmemStack * blockDim.x)[threadIdx.x >> 5];
    const DevScene& s = *sp;
    const WalkScene uni{s.nodes, s.tris, sp};
    TraversalCounters tc{0, 0, 0};
    uint32_t warp_steps = 0;
    using W = PairWalker<false, false>;
    walk_queue_pairs<W, kStackSize - kSmemStack, false, false, true>(
        uint32_t(w) * uint32_t(h), claim, 24u, visits, smem_stack + threadIdx.x, blockDim.x, ps, uni, tc, warp_steps,
        [&](uint32_t pixel, W& wk, WalkScene&, const PairLane& sl) {
            const int x = int(pixel % uint32_t(w)), y = int(pixel / uint32_t(w));
            Rng rng = pixel_rng(pixel, seed, frame);
            V2 jitter = rng_next2(rng);
            V2 lens = rng_next2(rng);
            V3 o, d;
            camera_ray(cam.c, float(x) + jitter.x, float(y) + jitter.y, w, h, lens, o, d);
            wk.init(o, d, kInf, sl);
            return pixel;
        },
        [&](uint32_t pixel, const W& wk, const float4& hh) {
            out[pixel] = __float_as_int(hh.x) >= 0 ? make_float4(wk.tmax, hh.x, hh.y, hh.z) : make_float4(kInf, __int_as_float(-1), 0.0f, 0.0f);
        });
}

__global__ void __launch_bounds__(128) k_occlusion_probe_pairs(const DevScene* sp, const float4* rays, int n, int4* out, uint32_t* claim,
                                                              uint32_t visits) {
    extern __shared__ int smem_stack[];
    PairSlots& ps = reinterpret_cast<PairSlots*>(smem_stack + kSmemStack * blockDim.x)[threadIdx.x >> 5];
    const DevScene& s = *sp;
    const WalkScene uni{s.nodes, s.tris, sp};
    TraversalCounters tc{0, 0, 0};
    uint32_t warp_steps = 0, start = 0;
    using W = PairWalker<true, true>;
    walk_queue_pairs<W, kStackSize - kSmemStack, true, true, true>(
        uint32_t(n), claim, 24u, visits, smem_stack + threadIdx.x, blockDim.x, ps, uni, tc, warp_steps,
        [&](uint32_t i, W& wk, WalkScene&, const PairLane& sl) {
            const float4 a = rays[2 * i], b = rays[2 * i + 1];
            wk.init(xyz(a), xyz(b), a.w, sl);
            start = tc.nodes;
            return i;
        },
        [&](uint32_t i, const W&, const float4& hh) {
            const int tri = __float_as_int(hh.x);
            out[i] = make_int4(tri >= 0 ? 1 : 0, tri, int(tc.nodes - start), -1);
        });
}

// The light pick of the first vertex of each pixel's sample (integrator.h:199-209).
__global__ void __launch_bounds__(128) k_light_picks(const DevScene* sp, const DevView* vp, int4* out) {
    extern __shared__ int smem_stack[];
    const DevView& v = *vp;
    int x = blockIdx.x * 16 + (threadIdx.x & 15), y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= v.width || y >= v.height) return;
    const DevScene& s = *sp;
    uint32_t pixel = uint32_t(y) * uint32_t(v.width) + uint32_t(x);
    int4 res = make_int4(-1, -1, -1, 0);
    Rng rng = pixel_rng(pixel, v.seed, v.frame0);
    V2 jitter = rng_next2(rng);
    V2 lens = rng_next2(rng);
    V3 o, d;
    camera_ray(v.cam, float(x) + jitter.x, float(y) + jitter.y, v.width, v.height, lens, o, d);
    Hit hit{kInf, -1, 0.0f, 0.0f};
    TraversalCounters tc{0, 0};
    if (traverse<false, false>(s, o, d, kInf, hit, smem_stack + threadIdx.x, blockDim.x, &tc) && 1 < v.max_depth) {
        Interaction it = surface_at(s, o, d, hit.t, hit.tri, hit.u, hit.v);
        Bsdf bsdf = make_bsdf(it.params);
        bool nee = v.nee && s.has_lights && samples_lights(bsdf);
        if (nee) {
            float ug = rng_next(rng);
            V2 ul = rng_next2(rng);
            float uk = rng_next(rng);
            LightPick pk;
            sample_light(s, it.p, ug, ul, uk, &pk);
            res = make_int4(pk.group, pk.index, pk.bin, 1);
        }
    }
    out[pixel] = res;
}

// ---- display (gpu_renderer.cu:108-175 semantics; color.h:8-41) ---------------------------------------------
__device__ float srgb_to_linear_d(float c) { return c <= 0.04045f ? c / 12.92f : powf((c + 0.055f) / 1.055f, 2.4f); }
__device__ float linear_to_srgb_d(float c) {
    c = saturate(c);
    return c <= 0.0031308f ? c * 12.92f : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
}
__device__ V3 aces_fitted_d(V3 c) {
    V3 v{0.59719f * c.x + 0.35458f * c.y + 0.04823f * c.z, 0.07600f * c.x + 0.90834f * c.y + 0.01566f * c.z,
         0.02840f * c.x + 0.13383f * c.y + 0.83777f * c.z};
    V3 a = v * (v + v3(0.0245786f)) - v3(0.000090537f);
    V3 b = v * (v * 0.983729f + v3(0.4329510f)) + v3(0.238081f);
    v = V3{a.x / b.x, a.y / b.y, a.z / b.z};
    V3 r{1.60475f * v.x - 0.53108f * v.y - 0.07367f * v.z, -0.10208f * v.x + 1.10813f * v.y - 0.00605f * v.z,
         -0.00327f * v.x - 0.07276f * v.y + 1.07602f * v.z};
    return V3{clampf(r.x, 0.0f, 1.0f), clampf(r.y, 0.0f, 1.0f), clampf(r.z, 0.0f, 1.0f)};
}
__device__ V3 tone_map_d(V3 c, float exposure, int op) {
    c = c * exposure;
    if (op == 1) return aces_fitted_d(c);
    if (op == 2) return V3{c.x / (1.0f + c.x), c.y / (1.0f + c.y), c.z / (1.0f + c.z)};
    return V3{clampf(c.x, 0.0f, 1.0f), clampf(c.y, 0.0f, 1.0f), clampf(c.z, 0.0f, 1.0f)};
}
__device__ uint32_t quantize_d(float v) { return uint32_t(saturate(v) * 255.0f + 0.5f); }
__device__ uint32_t pack_rgba8_d(V3 c) {
    return quantize_d(linear_to_srgb_d(c.x)) | (quantize_d(linear_to_srgb_d(c.y)) << 8) | (quantize_d(linear_to_srgb_d(c.z)) << 16) |
           0xFF000000u;
}
__device__ V3 heat_color_d(float t) {
    t = saturate(t);
    V3 c0{0.05f, 0.05f, 0.35f}, c1{0.0f, 0.6f, 0.4f}, c2{0.95f, 0.85f, 0.1f}, c3{0.85f, 0.1f, 0.05f};
    if (t < 1.0f / 3) return lerp(c0, c1, t * 3);
    if (t < 2.0f / 3) return lerp(c1, c2, t * 3 - 1);
    return lerp(c2, c3, t * 3 - 2);
}
__global__ void k_display(DisplayParams p, const float4* accum, const float4* denoised, const float4* albedo, const float4* normal_depth,
                          const float4* variance, const float* heat, uint32_t* out) {
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= p.w || y >= p.h) return;
    int i = y * p.w + x;
    V3 c;
    switch (p.mode) {
        case 1: c = xyz(albedo[i]); break;
        case 2: {
            float4 nd = normal_depth[i];
            c = nd.w > 0 ? xyz(nd) * 0.5f + v3(0.5f) : v3(0);
            break;
        }
        case 3: {
            float d = normal_depth[i].w;
            c = d > 0 ? v3(1.0f - saturate(d / p.max_depth)) : v3(0);
            break;
        }
        case 4: {
            float var;
            if (p.denoised) {
                var = variance ? variance[i].w : 0.0f;
            } else {
                float4 a = accum[i];
                float mean = luminance(xyz(a)) * p.inv_samples;
                var = p.samples > 1 ? fmaxf(0.0f, a.w * p.inv_samples - mean * mean) / (p.samples - 1) : 0.0f;
            }
            float t = sqrtf(var);
            c = v3(t / (1.0f + t));
            break;
        }
        case 5: c = heat_color_d(heat[i] * p.heat_scale); break;
        default:
            c = p.denoised ? xyz(denoised[i]) : xyz(accum[i]) * p.inv_samples;
            c = tone_map_d(c, p.exposure, p.tonemap);
            break;
    }
    if (p.mode != 0 && p.mode != 1) c = V3{srgb_to_linear_d(c.x), srgb_to_linear_d(c.y), srgb_to_linear_d(c.z)};
    out[i] = pack_rgba8_d(c);
}

}  // namespace

cudaError_t wf_launch_shape(int device, int trace_block, int shade_block, LaunchShape* out) {
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) return e;
    out->sms = prop.multiProcessorCount;
    int nb = 0;
    out->gen_block = 256;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_generate, 256, 0);
    if (e != cudaSuccess) return e;
    out->gen_grid = prop.multiProcessorCount * (nb > 0 ? nb : 1);
    out->trace_block = trace_block;
    size_t smem = size_t(kSmemStack) * trace_block * sizeof(int);
#define PTW_TRACE_KERNELS(S) (const void*)k_trace<false, false, S>, (const void*)k_trace<false, true, S>, \
                             (const void*)k_trace<true, false, S>, (const void*)k_trace<true, true, S>
#define PTW_SHADOW_KERNELS(W, S) (const void*)k_shadow<false, false, W, S>, (const void*)k_shadow<false, true, W, S>, \
                                 (const void*)k_shadow<true, false, W, S>, (const void*)k_shadow<true, true, W, S>
    const void* smem_kernels[] = {PTW_TRACE_KERNELS(false), PTW_TRACE_KERNELS(true), PTW_SHADOW_KERNELS(false, false),
                                  PTW_SHADOW_KERNELS(false, true), PTW_SHADOW_KERNELS(true, false), PTW_SHADOW_KERNELS(true, true)};
#undef PTW_TRACE_KERNELS
#undef PTW_SHADOW_KERNELS
    for (const void* k : smem_kernels) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e != cudaSuccess) return e;
    }
    const size_t pair_smem = smem + size_t(trace_block / 32) * sizeof(PairSlots);
    const void* pair_kernels[] = {(const void*)k_trace_pairs<false, false>,         (const void*)k_trace_pairs<false, true>,
                                  (const void*)k_trace_pairs<true, false>,          (const void*)k_trace_pairs<true, true>,
                                  (const void*)k_shadow_pairs<false, false, false>, (const void*)k_shadow_pairs<false, true, false>,
                                  (const void*)k_shadow_pairs<true, false, false>,  (const void*)k_shadow_pairs<true, true, false>,
                                  (const void*)k_shadow_pairs<false, true, true>,   (const void*)k_shadow_pairs<true, true, true>};
    for (const void* k : pair_kernels) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(pair_smem));
        if (e != cudaSuccess) return e;
    }
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace_pairs<false, false>, trace_block, pair_smem);
    if (e != cudaSuccess) return e;
    out->pair_trace_grid = prop.multiProcessorCount * (nb > 0 ? nb : 1);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shadow_pairs<false, false, false>, trace_block, pair_smem);
    if (e != cudaSuccess) return e;
    out->pair_shadow_grid = prop.multiProcessorCount * (nb > 0 ? nb : 1);
    // Grids are sized for the heavier (multi-scene) variants, so that every variant's grid fits.
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_trace<false, true, false>, trace_block, smem);
    if (e != cudaSuccess) return e;
    out->trace_grid = prop.multiProcessorCount * (nb > 0 ? nb : 1);
    out->shadow_block = trace_block;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shadow<false, true, true, false>, trace_block, smem);
    if (e != cudaSuccess) return e;
    out->shadow_grid = prop.multiProcessorCount * (nb > 0 ? nb : 1);
    out->shade_block = shade_block;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_shade, shade_block, 0);
    if (e != cudaSuccess) return e;
    out->shade_grid = prop.multiProcessorCount * (nb > 0 ? nb : 1);
    return cudaSuccess;
}

template <bool Count, bool Packed, bool Single>
static void launch_traversals(const WfParams& p, const LaunchShape& ls, cudaStream_t stream, size_t smem, bool shadow) {
    if (Packed && p.pair_visits > 0) {
        const size_t pair_smem = smem + size_t(ls.trace_block / 32) * sizeof(PairSlots);
        if (shadow && Single && p.wide_shadows) k_shadow_pairs<Count, true, true><<<ls.pair_shadow_grid, ls.shadow_block, pair_smem, stream>>>(p);
        else if (shadow) k_shadow_pairs<Count, Single, false><<<ls.pair_shadow_grid, ls.shadow_block, pair_smem, stream>>>(p);
        else k_trace_pairs<Count, Single><<<ls.pair_trace_grid, ls.trace_block, pair_smem, stream>>>(p);
        return;
    }
    if (shadow) {
        if (p.wide_shadows) k_shadow<Count, Packed, true, Single><<<ls.shadow_grid, ls.shadow_block, smem, stream>>>(p);
        else k_shadow<Count, Packed, false, Single><<<ls.shadow_grid, ls.shadow_block, smem, stream>>>(p);
    } else {
        k_trace<Count, Packed, Single><<<ls.trace_grid, ls.trace_block, smem, stream>>>(p);
    }
}

template <bool Count, bool Packed>
static void launch_traversals(const WfParams& p, const LaunchShape& ls, cudaStream_t stream, size_t smem, bool shadow) {
    if (p.single_scene >= 0) launch_traversals<Count, Packed, true>(p, ls, stream, smem, shadow);
    else launch_traversals<Count, Packed, false>(p, ls, stream, smem, shadow);
}

static void launch_traversal(const WfParams& p, const LaunchShape& ls, cudaStream_t stream, size_t smem, bool shadow) {
    if (p.count_work) {
        if (p.packed) launch_traversals<true, true>(p, ls, stream, smem, shadow);
        else launch_traversals<true, false>(p, ls, stream, smem, shadow);
    } else {
        if (p.packed) launch_traversals<false, true>(p, ls, stream, smem, shadow);
        else launch_traversals<false, false>(p, ls, stream, smem, shadow);
    }
}

static void launch_tail(const WfParams& p, const LaunchShape& ls, cudaStream_t stream, size_t smem) {
    if (p.count_work) {
        if (p.packed) k_tail<true, true><<<ls.trace_grid, ls.trace_block, smem, stream>>>(p);
        else k_tail<true, false><<<ls.trace_grid, ls.trace_block, smem, stream>>>(p);
    } else {
        if (p.packed) k_tail<false, true><<<ls.trace_grid, ls.trace_block, smem, stream>>>(p);
        else k_tail<false, false><<<ls.trace_grid, ls.trace_block, smem, stream>>>(p);
    }
}

cudaError_t wf_iteration(const WfParams& p, const LaunchShape& ls, cudaStream_t stream, cudaEvent_t* ev) {
    size_t smem = size_t(kSmemStack) * ls.trace_block * sizeof(int);
    // Timing events: inside a stream capture they must be external event nodes to be recorded at
    // all; outside one they are ordinary records.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (ev) cudaStreamIsCapturing(stream, &cap);
    const unsigned flags = cap == cudaStreamCaptureStatusActive ? cudaEventRecordExternal : cudaEventRecordDefault;
    auto mark = [&](int k) {
        if (ev) cudaEventRecordWithFlags(ev[k], stream, flags);
    };
    mark(0);
    k_setup<<<1, 32, 0, stream>>>(p);
    mark(1);
    k_generate<<<ls.gen_grid, ls.gen_block, 0, stream>>>(p);
    mark(2);
    if (p.tail_paths > 0) launch_tail(p, ls, stream, smem);
    launch_traversal(p, ls, stream, smem, false);
    mark(3);
    k_shade<<<ls.shade_grid, ls.shade_block, 0, stream>>>(p);
    mark(4);
    if (p.shadow_sort_bits > 0) {
        k_sort_scan<true><<<1, 1024, 0, stream>>>(p, 8u << (3 * p.shadow_sort_bits));
        k_shadow_order<<<ls.gen_grid, ls.gen_block, 0, stream>>>(p);
    }
    launch_traversal(p, ls, stream, smem, true);
    if (p.sort_bits > 0) {
        k_sort_scan<false><<<1, 1024, 0, stream>>>(p, 8u << (3 * p.sort_bits));
        k_sort_scatter<<<ls.gen_grid, ls.gen_block, 0, stream>>>(p);
        k_sort_finish<<<1, 32, 0, stream>>>(p.ctr);
    }
    mark(5);
    return cudaGetLastError();
}

__global__ void k_resolve(const float4* __restrict__ accum, uint32_t n, float scale, int apply_scale, float* __restrict__ rgb) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = accum[i];
    if (apply_scale) {
        a.x = a.x * scale;
        a.y = a.y * scale;
        a.z = a.z * scale;
    }
    rgb[3 * size_t(i)] = a.x;
    rgb[3 * size_t(i) + 1] = a.y;
    rgb[3 * size_t(i) + 2] = a.z;
}

cudaError_t wf_resolve(const float4* accum, uint32_t n, float scale, bool apply_scale, float* rgb, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    k_resolve<<<(n + 255) / 256, 256, 0, stream>>>(accum, n, scale, apply_scale ? 1 : 0, rgb);
    return cudaGetLastError();
}

cudaError_t wf_accumulate(const DevView* d_view, const DevView& h_view, int first_pass, int last_pass, cudaStream_t stream) {
    uint32_t npix = uint32_t(h_view.width) * uint32_t(h_view.height);
    if (npix == 0) return cudaSuccess;
    void* args[] = {const_cast<DevView**>(&d_view), &first_pass, &last_pass};
    return cudaLaunchKernel(reinterpret_cast<const void*>(&k_accumulate), dim3((npix + 255) / 256), dim3(256), args, 0, stream);
}

cudaError_t wf_trace_primary(const DevScene* scene, const float* cam16, int w, int h, uint32_t frame, uint32_t seed, float4* out,
                             uint32_t* claim, uint32_t pair_visits, cudaStream_t stream) {
    CameraArg c;
    for (int i = 0; i < 16; i++) c.c[i] = cam16[i];
    if (pair_visits > 0) {
        const size_t smem = size_t(kSmemStack) * 128 * sizeof(int) + 4 * sizeof(PairSlots);
        const uint32_t n = uint32_t(w) * uint32_t(h), blocks = std::min<uint32_t>((n + 127) / 128, 148u * 16u);
        cudaError_t e = cudaMemsetAsync(claim, 0, sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
        k_trace_primary_pairs<<<blocks, 128, smem, stream>>>(scene, c, w, h, frame, seed, out, claim, pair_visits);
        return cudaGetLastError();
    }
    dim3 grid((w + 15) / 16, (h + 7) / 8);
    size_t smem = size_t(kSmemStack) * 128 * sizeof(int);
    k_trace_primary<<<grid, 128, smem, stream>>>(scene, c, w, h, frame, seed, out);
    return cudaGetLastError();
}

cudaError_t wf_light_picks(const DevScene* scene, const DevView* view, int4* out, int w, int h, cudaStream_t stream) {
    dim3 grid((w + 15) / 16, (h + 7) / 8);
    size_t smem = size_t(kSmemStack) * 128 * sizeof(int);
    k_light_picks<<<grid, 128, smem, stream>>>(scene, view, out);
    return cudaGetLastError();
}

cudaError_t wf_occlusion_probe(const DevScene* scene, const float4* rays, int n, int wide, int4* out, uint32_t* claim, uint32_t pair_visits,
                               cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    if (pair_visits > 0 && !wide) {
        const size_t smem = size_t(kSmemStack) * 128 * sizeof(int) + 4 * sizeof(PairSlots);
        const uint32_t blocks = std::min<uint32_t>((uint32_t(n) + 127) / 128, 148u * 16u);
        cudaError_t e = cudaMemsetAsync(claim, 0, sizeof(uint32_t), stream);
        if (e != cudaSuccess) return e;
        k_occlusion_probe_pairs<<<blocks, 128, smem, stream>>>(scene, rays, n, out, claim, pair_visits);
        return cudaGetLastError();
    }
    const size_t smem = size_t(kSmemStack) * 128 * sizeof(int);
    k_occlusion_probe<<<(n + 127) / 128, 128, smem, stream>>>(scene, rays, n, wide, out);
    return cudaGetLastError();
}

cudaError_t wf_heatmap(const DevScene* scene, const float* cam16, int w, int h, float* out, cudaStream_t stream) {
    CameraArg c;
    for (int i = 0; i < 16; i++) c.c[i] = cam16[i];
    dim3 grid((w + 15) / 16, (h + 7) / 8);
    size_t smem = size_t(kSmemStack) * 128 * sizeof(int);
    k_heatmap<<<grid, 128, smem, stream>>>(scene, c, w, h, out);
    return cudaGetLastError();
}

cudaError_t wf_display(const DisplayParams& p, const float4* accum, const float4* denoised, const float4* albedo,
                       const float4* normal_depth, const float4* variance, const float* heat, uint32_t* out, cudaStream_t stream) {
    dim3 block(16, 8), grid((p.w + 15) / 16, (p.h + 7) / 8);
    k_display<<<grid, block, 0, stream>>>(p, accum, denoised, albedo, normal_depth, variance, heat, out);
    return cudaGetLastError();
}

}  // namespace ptw
