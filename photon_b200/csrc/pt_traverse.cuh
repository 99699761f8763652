// BVH2 traversal on the device: Photon's nearest-first stack traversal (src/render/traverse.h:66-138)
// with the stack in shared memory.
//
// The visiting order, the in-place leaf tests, the strict t < tmax test, the left-first tie rule and
// the drop-on-overflow of a 64-entry stack are kept exactly, so closest-hit triangle indices equal
// Photon's. The stack holds one entry per tree level at most; its first kSmemStack entries live in
// shared memory (column per thread, so a warp's pushes hit 32 distinct banks) and the rest, only
// reached by trees deeper than kSmemStack, in local memory.
#pragma once

#include "pt_scene.cuh"

namespace ptw {

constexpr int kStackSize = 64;     // Photon's kStackSize (traverse.h:22)
constexpr int kSmemStack = 16;     // entries per thread kept in shared memory

struct Hit {
    float t;
    int tri;
    float u, v;
};

struct TraversalCounters {
    uint32_t nodes, tris;
    uint32_t steps;  // walk steps of the rays (lane steps of a queue walk)
};

// What a walk step reads of its scene: the node array it walks (the BVH2's, or the 4-wide BVH's), the
// triangles, and the scene for the rare alpha test. Kept apart so that a walk loop can hold the two
// array bases in registers instead of reloading them from the scene table at every step.
struct WalkScene {
    const float4* nodes;
    const float4* tris;
    const DevScene* scene;
};

PT_HD float safe_inv(float x) { return fabsf(x) > 1e-20f ? 1.0f / x : copysignf(1e20f, x); }

// Slab test (traverse.h:40-47): entry distance or kInf.
PT_HD float box_entry(float4 bmin, float4 bmax, V3 o, V3 inv_d, float tmax) {
    float tx0 = (bmin.x - o.x) * inv_d.x, tx1 = (bmax.x - o.x) * inv_d.x;
    float ty0 = (bmin.y - o.y) * inv_d.y, ty1 = (bmax.y - o.y) * inv_d.y;
    float tz0 = (bmin.z - o.z) * inv_d.z, tz1 = (bmax.z - o.z) * inv_d.z;
    float tnear = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    return tnear <= tfar ? tnear : kInf;
}

// Moller-Trumbore (traverse.h:24-37).
PT_HD bool tri_intersect(float4 g0, float4 g1, float4 g2, V3 o, V3 d, float tmax, float& t, float& u, float& v) {
    V3 e1 = xyz(g1), e2 = xyz(g2);
    V3 p = cross(d, e2);
    float det = dot(e1, p);
    if (fabsf(det) < 1e-14f) return false;
    float inv = 1.0f / det;
    V3 s = o - xyz(g0);
    u = dot(s, p) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    V3 q = cross(s, e1);
    v = dot(d, q) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, q) * inv;
    return t > 0.0f && t < tmax;
}

// Packed FP32 pairs (sm_100 add/sub/mul.rn.f32x2): two IEEE round-to-nearest operations per
// instruction, each rounded exactly as the scalar operation, so results are bit-identical. A float4
// loaded by one 128-bit load sits in a register quad, so its (x, y) and (z, w) halves are pairs.
typedef unsigned long long f32x2;
PT_HD f32x2 pack2(float a, float b) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
PT_HD void unpack2(f32x2 r, float& a, float& b) { asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r)); }
PT_HD f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
PT_HD f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}

// Three-input min / max (sm_100): one instruction for two of the slab test's reductions. min and max
// are exact and order-free (a NaN operand is ignored, as fminf / fmaxf ignore it), so the results are
// those of the two-input chains.
PT_HD float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
PT_HD float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// 32 bytes (two float4) in one 256-bit load through the read-only path (sm_100); p is 32-byte aligned.
PT_HD void ldg_pair(const float4* p, float4& a, float4& b) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(p));
}

// The slab test of box_entry with the (bmin - o) * inv_d products computed in pairs and the min/max
// reductions with three inputs where two chained ones stood.
struct RayPairs {
    f32x2 oxy, oz0, ixy, iz0;
};
PT_HD RayPairs ray_pairs(V3 o, V3 inv_d) { return {pack2(o.x, o.y), pack2(o.z, 0.0f), pack2(inv_d.x, inv_d.y), pack2(inv_d.z, 0.0f)}; }
PT_HD float box_entry2(float4 bmin, float4 bmax, const RayPairs& r, float tmax) {
    float tx0, ty0, tz0, tx1, ty1, tz1, w0, w1;
    unpack2(mul2(sub2(pack2(bmin.x, bmin.y), r.oxy), r.ixy), tx0, ty0);
    unpack2(mul2(sub2(pack2(bmin.z, bmin.w), r.oz0), r.iz0), tz0, w0);
    unpack2(mul2(sub2(pack2(bmax.x, bmax.y), r.oxy), r.ixy), tx1, ty1);
    unpack2(mul2(sub2(pack2(bmax.z, bmax.w), r.oz0), r.iz0), tz1, w1);
    float tnear = fmax3(fminf(tx0, tx1), fminf(ty0, ty1), fmaxf(fminf(tz0, tz1), 0.0f));
    float tfar = fmin3(fmaxf(tx0, tx1), fmaxf(ty0, ty1), fminf(fmaxf(tz0, tz1), tmax));
    return tnear <= tfar ? tnear : kInf;
}

// Photon's traversal (traverse.h:66-138) as a state machine advanced one unit per step: a node visit
// (both child slabs) or one triangle test. At each node both children are tested against the current
// tmax; leaf children are then tested in place, side 0 first, and only after their triangles (which may
// lower tmax) does the node push its farther interior child (if nearer than tmax and the 64-entry stack
// has room) and descend to the nearer one (if nearer than tmax), or pop. Ties keep side 0 first. So the
// sequence of node visits and triangle tests per ray, and the resulting hit, are Photon's.
// Stepping one triangle at a time lets a lane that walks a leaf test one triangle while its
// neighbours visit nodes, instead of every lane of the warp idling through the longest leaf loop.
template <bool AnyHit, bool Count, bool Packed = true>
struct Walker {
    V3 o, d, inv_d;
    RayPairs rp;
    float tmax;
    int node;        // the node to visit next; -1 once the ray is finished
    int sp;
    int ti, te;      // leaf mode: the next triangle and the end of its range
    int t1, e1;      // the second leaf range waiting behind the first (t1 == e1: none)
    int near, far;   // inner children waiting for the leaf tests (-1: none)
    float tn_near, tn_far;
    bool leaf_mode;
    int tri;         // closest (or first accepted) triangle, -1 for none; its distance is tmax
    float u, v;

    PT_HD void init(V3 o_, V3 d_, float tmax_) {
        o = o_;
        d = d_;
        inv_d = V3{safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)};
        rp = ray_pairs(o, inv_d);
        tmax = tmax_;
        node = 0;
        sp = 0;
        ti = te = t1 = e1 = 0;
        near = far = -1;
        tn_near = tn_far = 0.0f;
        leaf_mode = false;
        tri = -1;
        u = v = 0.0f;
    }

    // Advances one unit; returns false once the ray is finished.
    PT_HD bool step(const WalkScene& ws, int* stack, int stride, int* overflow, TraversalCounters* cnt) {
        bool decide = false;
        if (!leaf_mode) {
            const float4* n = ws.nodes + 4 * node;  // 64-byte nodes: two 256-bit loads
            float4 n0, n1, n2, n3;
            ldg_pair(n, n0, n1);
            ldg_pair(n + 2, n2, n3);
            if (Count) cnt->nodes++;
            float tl = Packed ? box_entry2(n0, n1, rp, tmax) : box_entry(n0, n1, o, inv_d, tmax);
            float tr = Packed ? box_entry2(n2, n3, rp, tmax) : box_entry(n2, n3, o, inv_d, tmax);
            int c0 = __float_as_int(n1.w), i0 = __float_as_int(n0.w), c1 = __float_as_int(n3.w), i1 = __float_as_int(n2.w);
            bool h0 = tl != kInf, h1 = tr != kInf;
            bool leaf0 = h0 && c0 > 0, leaf1 = h1 && c1 > 0;
            bool in0 = h0 && c0 <= 0 && i0 >= 0, in1 = h1 && c1 <= 0 && i1 >= 0;
            // Inner children in side order, then nearest first (a tie keeps side 0 first).
            near = in0 ? i0 : (in1 ? i1 : -1);
            tn_near = in0 ? tl : tr;
            far = (in0 && in1) ? i1 : -1;
            tn_far = tr;
            if (far >= 0 && tn_near > tn_far) {
                int a = near;
                near = far;
                far = a;
                float b = tn_near;
                tn_near = tn_far;
                tn_far = b;
            }
            if (leaf0 || leaf1) {
                ti = leaf0 ? i0 : i1;
                te = leaf0 ? i0 + c0 : i1 + c1;
                bool both = leaf0 && leaf1;
                t1 = both ? i1 : 0;
                e1 = both ? i1 + c1 : 0;
                leaf_mode = true;
            } else {
                decide = true;
            }
        }
        if (leaf_mode) {
            int i = ti;
            const float4* g = ws.tris + kTriStride * i;  // 64-byte records: a 256-bit and a 128-bit load
            float4 g0, g1;
            ldg_pair(g, g0, g1);
            const float4 g2 = __ldg(g + 2);  // the record's fourth float4 is padding
            float t, tu, tv;
            if (Count) cnt->tris++;
            if (tri_intersect(g0, g1, g2, o, d, tmax, t, tu, tv) &&
                !((__float_as_int(g1.w) & 1) && alpha_passes(*ws.scene, g, __float_as_int(g0.w), tu, tv))) {
                tmax = t;
                tri = i;
                u = tu;
                v = tv;
                if (AnyHit) {
                    node = -1;
                    return false;
                }
            }
            if (++ti == te) {
                if (t1 != e1) {
                    ti = t1;
                    te = e1;
                    t1 = e1 = 0;
                } else {
                    leaf_mode = false;
                    decide = true;
                }
            }
        }
        if (decide) {
            if (far >= 0 && tn_far < tmax && sp < kStackSize) {
                if (sp < kSmemStack) stack[sp * stride] = far;
                else overflow[sp - kSmemStack] = far;
                sp++;
            }
            if (near >= 0 && tn_near < tmax) {
                node = near;
            } else if (sp == 0) {
                node = -1;
            } else {
                --sp;
                node = sp < kSmemStack ? stack[sp * stride] : overflow[sp - kSmemStack];
            }
        }
        return node >= 0;
    }
};

// The ray of box_entry with its x and y halves in pairs and z alone: the same operations as
// box_entry2 without the idle second half of the z pairs (two registers fewer per ray).
struct RaySlab {
    f32x2 oxy, ixy;
    float oz, iz;
};
PT_HD RaySlab ray_slab(V3 o, V3 inv_d) { return {pack2(o.x, o.y), pack2(inv_d.x, inv_d.y), o.z, inv_d.z}; }
PT_HD float box_entry3(float4 bmin, float4 bmax, const RaySlab& r, float tmax) {
    float tx0, ty0, tx1, ty1;
    unpack2(mul2(sub2(pack2(bmin.x, bmin.y), r.oxy), r.ixy), tx0, ty0);
    unpack2(mul2(sub2(pack2(bmax.x, bmax.y), r.oxy), r.ixy), tx1, ty1);
    const float tz0 = (bmin.z - r.oz) * r.iz, tz1 = (bmax.z - r.oz) * r.iz;
    float tnear = fmax3(fminf(tx0, tx1), fminf(ty0, ty1), fmaxf(fminf(tz0, tz1), 0.0f));
    float tfar = fmin3(fmaxf(tx0, tx1), fmaxf(ty0, ty1), fminf(fmaxf(tz0, tz1), tmax));
    return tnear <= tfar ? tnear : kInf;
}

// Photon's traversal split for the pair walk: visit() is the node half of Walker::step (both child
// slabs against tmax, the inner children ordered nearest first with side 0 first on a tie), and it
// returns the triangles of the node's leaf children instead of testing them; the warp then tests
// those (ray, triangle) pairs of all its lanes together (pair_pass in the walk kernels), which lowers
// tmax to the nearest accepted triangle of the node's leaves exactly as the in-place tests would, and
// decide() pushes the farther inner child, descends or pops with that tmax. So each ray's node visits
// and its hit are Walker's. What only the pair pass and the ray's end read (the direction, the leaf
// ranges, the hit's triangle and barycentrics) lives in the lane's shared-memory slots, not in
// registers: PairLane refers to them. (The inner children of a visit that waits for its leaf tests
// stay in registers: parked in shared memory too, the walk measured slower.)
struct PairLane {
    float4& ray;    // direction, tmax as of the lane's last pair pass
    int4& leaves;   // the last visit's leaf children in side order: first triangles and count of the
                    // first ([l0, l0 + n0)), first triangle of the second, and the lane's first pair
    float4& hit;    // closest (or first accepted) triangle (bits; -1: none), u, v
};

// The inner children of a visit (-1: none), nearest first, and their entry distances.
struct NodeChoice {
    int near, far;
    float tn_near, tn_far;
};

template <bool AnyHit, bool Count>
struct PairWalker {
    RaySlab rs;      // origin and inverse direction (the origin is rs.oxy, rs.oz)
    float tmax;
    int node;        // the node to visit next; -1 once the ray is finished
    int sp;

    PT_HD void init(V3 o_, V3 d_, float tmax_, const PairLane& sl) {
        rs = ray_slab(o_, V3{safe_inv(d_.x), safe_inv(d_.y), safe_inv(d_.z)});
        tmax = tmax_;
        node = 0;
        sp = 0;
        sl.ray = make_float4(d_.x, d_.y, d_.z, tmax_);
        sl.hit = make_float4(__int_as_float(-1), 0.0f, 0.0f, 0.0f);
    }
    PT_HD V3 origin() const {
        float x, y;
        unpack2(rs.oxy, x, y);
        return V3{x, y, rs.oz};
    }
    // Visits `node`: its inner children into `ch`; returns how many triangles its leaf children hold
    // (0: none), whose ranges it leaves in the lane's slot.
    PT_HD uint32_t visit(const float4* nodes, const PairLane& sl, NodeChoice& ch, TraversalCounters* cnt) {
        const float4* n = nodes + 4 * node;
        float4 n0_, n1_, n2_, n3_;
        ldg_pair(n, n0_, n1_);
        ldg_pair(n + 2, n2_, n3_);
        if (Count) cnt->nodes++;
        const float tl = box_entry3(n0_, n1_, rs, tmax), tr = box_entry3(n2_, n3_, rs, tmax);
        const int c0 = __float_as_int(n1_.w), i0 = __float_as_int(n0_.w), c1 = __float_as_int(n3_.w), i1 = __float_as_int(n2_.w);
        const bool h0 = tl != kInf, h1 = tr != kInf;
        const bool leaf0 = h0 && c0 > 0, leaf1 = h1 && c1 > 0;
        const bool in0 = h0 && c0 <= 0 && i0 >= 0, in1 = h1 && c1 <= 0 && i1 >= 0;
        ch.near = in0 ? i0 : (in1 ? i1 : -1);
        ch.tn_near = in0 ? tl : tr;
        ch.far = (in0 && in1) ? i1 : -1;
        ch.tn_far = tr;
        if (ch.far >= 0 && ch.tn_near > ch.tn_far) {
            const int a = ch.near;
            ch.near = ch.far;
            ch.far = a;
            const float b = ch.tn_near;
            ch.tn_near = ch.tn_far;
            ch.tn_far = b;
        }
        if (!(leaf0 || leaf1)) return 0;
        const int n0 = leaf0 ? c0 : c1, n1 = leaf0 && leaf1 ? c1 : 0;
        sl.leaves = make_int4(leaf0 ? i0 : i1, n0, i1, 0);
        return uint32_t(n0 + n1);
    }
    // After the leaf tests: push the farther inner child, descend to the nearer or pop (traverse.h
    // order); returns whether the ray goes on.
    PT_HD bool decide(const NodeChoice& ch, int* stack, int stride, int* overflow) {
        if (ch.far >= 0 && ch.tn_far < tmax && sp < kStackSize) {
            if (sp < kSmemStack) stack[sp * stride] = ch.far;
            else overflow[sp - kSmemStack] = ch.far;
            sp++;
        }
        if (ch.near >= 0 && ch.tn_near < tmax) {
            node = ch.near;
        } else if (sp == 0) {
            node = -1;
        } else {
            --sp;
            node = sp < kSmemStack ? stack[sp * stride] : overflow[sp - kSmemStack];
        }
        return node >= 0;
    }
};

// The triangle of pair j of a visit whose leaf ranges are lv (PairLane::leaves).
PT_HD int pair_triangle(const int4& lv, int j) { return j < lv.y ? lv.x + j : lv.z + (j - lv.y); }

// The any-hit pair walk over the 4-wide BVH (wide_bvh.h): whether some triangle accepts the ray is
// order-free, and the 4-wide tree reaches the BVH2's leaves (see AnyWalker4), so the answer is the
// BVH2 walk's. A visit tests the four children of the current node, pushes the inner ones it enters and
// then its leaf children (so leaves come off the stack first), and pops the next entry; an entry that
// is a leaf is handed to the warp's pair pass as the lane's one leaf range. Half as many dependent node
// reads as the BVH2 walk, at four slab tests per read.
template <bool Count>
struct PairWalker4 {
    RaySlab rs;
    float tmax;
    int cur;   // the current entry: a node index, or a leaf as 0x80000000 | count << 24 | first triangle
    int sp;    // -1 once the stack ran out (the ray is finished)

    PT_HD void init(V3 o_, V3 d_, float tmax_, const PairLane& sl) {
        rs = ray_slab(o_, V3{safe_inv(d_.x), safe_inv(d_.y), safe_inv(d_.z)});
        tmax = tmax_;
        cur = 0;
        sp = 0;
        sl.ray = make_float4(d_.x, d_.y, d_.z, tmax_);
        sl.hit = make_float4(__int_as_float(-1), 0.0f, 0.0f, 0.0f);
    }
    PT_HD V3 origin() const {
        float x, y;
        unpack2(rs.oxy, x, y);
        return V3{x, y, rs.oz};
    }
    PT_HD void push(int e, int* stack, int stride, int* overflow) {
        if (sp < kSmemStack) stack[sp * stride] = e;
        else overflow[sp - kSmemStack] = e;
        sp++;
    }
    // Pops the next entry into cur; false once the stack is empty.
    PT_HD bool pop(int* stack, int stride, int* overflow) {
        if (sp == 0) {
            sp = -1;
            return false;
        }
        --sp;
        cur = sp < kSmemStack ? stack[sp * stride] : overflow[sp - kSmemStack];
        return true;
    }
    // The current entry's triangles if it is a leaf (its range into the lane's slot), else 0.
    PT_HD uint32_t leaf_pairs(const PairLane& sl) const {
        if (cur >= 0) return 0;
        const int n = (cur >> 24) & 0x7f;
        sl.leaves = make_int4(cur & 0xffffff, n, 0, 0);
        return uint32_t(n);
    }
    // Visits the current node (cur >= 0) and pops the next entry; false once the ray is finished.
    PT_HD bool visit(const float4* nodes4, int* stack, int stride, int* overflow, TraversalCounters* cnt) {
        const float4* n = nodes4 + 8 * cur;  // 128-byte nodes: four 256-bit loads
        float4 lx, ly, lz, hx, hy, hz, id4, ct4;
        ldg_pair(n, lx, ly);
        ldg_pair(n + 2, lz, hx);
        ldg_pair(n + 4, hy, hz);
        ldg_pair(n + 6, id4, ct4);
        if (Count) cnt->nodes++;
        const float lxs[4] = {lx.x, lx.y, lx.z, lx.w}, lys[4] = {ly.x, ly.y, ly.z, ly.w}, lzs[4] = {lz.x, lz.y, lz.z, lz.w};
        const float hxs[4] = {hx.x, hx.y, hx.z, hx.w}, hys[4] = {hy.x, hy.y, hy.z, hy.w}, hzs[4] = {hz.x, hz.y, hz.z, hz.w};
        const int ids[4] = {__float_as_int(id4.x), __float_as_int(id4.y), __float_as_int(id4.z), __float_as_int(id4.w)};
        const int cts[4] = {__float_as_int(ct4.x), __float_as_int(ct4.y), __float_as_int(ct4.z), __float_as_int(ct4.w)};
        int leaves[4];
        int nl = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (ids[k] < 0) continue;
            const float t = box_entry3(make_float4(lxs[k], lys[k], lzs[k], 0.0f), make_float4(hxs[k], hys[k], hzs[k], 0.0f), rs, tmax);
            if (t == kInf) continue;
            if (cts[k] > 0) leaves[nl++] = int(0x80000000u | (uint32_t(cts[k]) << 24) | uint32_t(ids[k]));
            else if (t < tmax) push(ids[k], stack, stride, overflow);
        }
        for (int k = 0; k < nl; k++) push(leaves[k], stack, stride, overflow);
        return pop(stack, stride, overflow);
    }
};

// One ray's traversal: AnyHit stops at the first accepted triangle. `stack` is this thread's column of
// the block's shared stack (entry k at stack[k * stride]).
template <bool AnyHit, bool Count, bool Packed = true>
PT_HD bool traverse(const DevScene& s, V3 o, V3 d, float tmax, Hit& hit, int* stack, int stride, TraversalCounters* cnt) {
    int overflow[kStackSize - kSmemStack];
    Walker<AnyHit, Count, Packed> w;
    w.init(o, d, tmax);
    const WalkScene ws{s.nodes, s.tris, &s};
    while (w.step(ws, stack, stride, overflow, cnt)) {
    }
    if (w.tri >= 0) {
        hit.t = w.tmax;
        hit.tri = w.tri;
        hit.u = w.u;
        hit.v = w.v;
    }
    return w.tri >= 0;
}

// ---- any-hit walk over the 4-wide BVH (wide_bvh.h) -----------------------------------------------------
// Whether some triangle accepts the ray within (0, tmax): the set of leaves a ray reaches is the
// BVH2's (every 4-wide box is a BVH2 box, tested with the same slab arithmetic, and a box test that
// passes also passes for the boxes containing it), and an any-hit answer does not depend on the order
// in which they are visited. The one difference in principle: a leaf reached through an interior
// BVH2 child whose entry distance equals tmax exactly is tested here, and Photon's walk stops at that
// child (its `t < tmax` test); the leaf's own entry is then tmax as well.
// One unit per step: a node visit (four slab tests; interior children pushed, then leaf children,
// so leaves are tested first) or one triangle test. Stack entries: a node index, or a leaf as
// 0x80000000 | count << 24 | first triangle.
constexpr int kBvh4Stack = 96;  // = kBvh4StackSize of the builder

template <bool Count, bool Packed = true>
struct AnyWalker4 {
    V3 o, d, inv_d;
    RayPairs rp;
    float tmax;
    int node;  // the node to visit (node mode)
    int sp;
    int ti, te;
    bool leaf_mode, done, hit;

    PT_HD void init(V3 o_, V3 d_, float tmax_) {
        o = o_;
        d = d_;
        inv_d = V3{safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)};
        rp = ray_pairs(o, inv_d);
        tmax = tmax_;
        node = 0;
        sp = 0;
        ti = te = 0;
        leaf_mode = done = hit = false;
    }
    PT_HD void push(int e, int* stack, int stride, int* overflow) {
        if (sp < kSmemStack) stack[sp * stride] = e;
        else overflow[sp - kSmemStack] = e;
        sp++;
    }
    PT_HD void pop(int* stack, int stride, int* overflow) {
        if (sp == 0) {
            done = true;
            return;
        }
        --sp;
        int e = sp < kSmemStack ? stack[sp * stride] : overflow[sp - kSmemStack];
        if (e < 0) {
            leaf_mode = true;
            ti = e & 0xffffff;
            te = ti + ((e >> 24) & 0x7f);
        } else {
            leaf_mode = false;
            node = e;
        }
    }
    // ws.nodes: the 4-wide BVH (8 float4 per node).
    PT_HD bool step(const WalkScene& ws, int* stack, int stride, int* overflow, TraversalCounters* cnt) {
        if (!leaf_mode) {
            const float4* n = ws.nodes + 8 * node;  // 128-byte nodes: four 256-bit loads
            float4 lx, ly, lz, hx, hy, hz, id4, ct4;
            ldg_pair(n, lx, ly);
            ldg_pair(n + 2, lz, hx);
            ldg_pair(n + 4, hy, hz);
            ldg_pair(n + 6, id4, ct4);
            const int4 id = make_int4(__float_as_int(id4.x), __float_as_int(id4.y), __float_as_int(id4.z), __float_as_int(id4.w));
            const int4 ct = make_int4(__float_as_int(ct4.x), __float_as_int(ct4.y), __float_as_int(ct4.z), __float_as_int(ct4.w));
            if (Count) cnt->nodes++;
            const float lxs[4] = {lx.x, lx.y, lx.z, lx.w}, lys[4] = {ly.x, ly.y, ly.z, ly.w}, lzs[4] = {lz.x, lz.y, lz.z, lz.w};
            const float hxs[4] = {hx.x, hx.y, hx.z, hx.w}, hys[4] = {hy.x, hy.y, hy.z, hy.w}, hzs[4] = {hz.x, hz.y, hz.z, hz.w};
            const int ids[4] = {id.x, id.y, id.z, id.w}, cts[4] = {ct.x, ct.y, ct.z, ct.w};
            int leaves[4];
            int nl = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (ids[k] < 0) continue;
                const float4 bmin = make_float4(lxs[k], lys[k], lzs[k], 0.0f), bmax = make_float4(hxs[k], hys[k], hzs[k], 0.0f);
                const float t = Packed ? box_entry2(bmin, bmax, rp, tmax) : box_entry(bmin, bmax, o, inv_d, tmax);
                if (t == kInf) continue;
                if (cts[k] > 0) leaves[nl++] = int(0x80000000u | (uint32_t(cts[k]) << 24) | uint32_t(ids[k]));
                else if (t < tmax) push(ids[k], stack, stride, overflow);
            }
            for (int k = 0; k < nl; k++) push(leaves[k], stack, stride, overflow);
            pop(stack, stride, overflow);
            if (done) return false;
        }
        if (leaf_mode) {
            const int i = ti;
            const float4* g = ws.tris + kTriStride * i;
            float4 g0, g1;
            ldg_pair(g, g0, g1);
            const float4 g2 = __ldg(g + 2);  // the record's fourth float4 is padding
            float t, tu, tv;
            if (Count) cnt->tris++;
            if (tri_intersect(g0, g1, g2, o, d, tmax, t, tu, tv) &&
                !((__float_as_int(g1.w) & 1) && alpha_passes(*ws.scene, g, __float_as_int(g0.w), tu, tv))) {
                hit = true;
                done = true;
                return false;
            }
            if (++ti == te) {
                pop(stack, stride, overflow);
                if (done) return false;
            }
        }
        return true;
    }
};

template <bool Count, bool Packed = true>
PT_HD bool occluded4(const DevScene& s, V3 o, V3 d, float tmax, int* stack, int stride, TraversalCounters* cnt) {
    int overflow[kBvh4Stack - kSmemStack];
    AnyWalker4<Count, Packed> w;
    w.init(o, d, tmax);
    const WalkScene ws{s.nodes4, s.tris, &s};
    while (w.step(ws, stack, stride, overflow, cnt)) {
    }
    return w.hit;
}

}  // namespace ptw
