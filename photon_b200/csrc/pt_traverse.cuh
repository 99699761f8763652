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
constexpr int kSmemStack = 24;     // entries per thread kept in shared memory

struct Hit {
    float t;
    int tri;
    float u, v;
};

struct TraversalCounters {
    uint32_t nodes, tris;
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

// The slab test of box_entry with the (bmin - o) * inv_d products computed in pairs; the min/max
// reduction is unchanged (there is no packed min/max).
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
    float tnear = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    return tnear <= tfar ? tnear : kInf;
}

// One traversal (traverse.h:66-138): nearest-first, leaves tested in place, `stack` is this thread's
// column of the block's shared stack (entry k at stack[k * stride]). AnyHit stops at the first
// accepted triangle. Packed selects the f32x2 slab test (bit-identical results).
template <bool AnyHit, bool Count, bool Packed = true>
PT_HD bool traverse(const DevScene& s, V3 o, V3 d, float tmax, Hit& hit, int* stack, int stride, TraversalCounters* cnt) {
    V3 inv_d{safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)};
    RayPairs rp = ray_pairs(o, inv_d);
    int overflow[kStackSize - kSmemStack];
    int sp = 0;
    int node = 0;
    bool found = false;
    const float4* nodes = s.nodes;
    const float4* tris = s.tris;
    while (true) {
        const float4* n = nodes + 4 * node;
        float4 n0 = __ldg(n), n1 = __ldg(n + 1), n2 = __ldg(n + 2), n3 = __ldg(n + 3);
        if (Count) cnt->nodes++;
        float tl = Packed ? box_entry2(n0, n1, rp, tmax) : box_entry(n0, n1, o, inv_d, tmax);
        float tr = Packed ? box_entry2(n2, n3, rp, tmax) : box_entry(n2, n3, o, inv_d, tmax);
        int next0 = 0, next1 = 0;
        float tn0 = 0, tn1 = 0;
        int nn = 0;
#pragma unroll
        for (int side = 0; side < 2; side++) {
            float tc = side == 0 ? tl : tr;
            if (tc == kInf) continue;
            int count = __float_as_int(side == 0 ? n1.w : n3.w);
            int idx = __float_as_int(side == 0 ? n0.w : n2.w);
            if (count > 0) {
                for (int i = idx; i < idx + count; i++) {
                    const float4* g = tris + 3 * i;
                    float4 g0 = __ldg(g), g1 = __ldg(g + 1), g2 = __ldg(g + 2);
                    float t, u, v;
                    if (Count) cnt->tris++;
                    if (tri_intersect(g0, g1, g2, o, d, tmax, t, u, v)) {
                        if ((__float_as_int(g1.w) & 1) && alpha_passes(s, i, __float_as_int(g0.w), u, v)) continue;
                        if (AnyHit) {
                            hit.t = t;
                            hit.tri = i;
                            return true;
                        }
                        tmax = t;
                        hit.t = t;
                        hit.tri = i;
                        hit.u = u;
                        hit.v = v;
                        found = true;
                    }
                }
            } else if (idx >= 0) {
                if (nn == 0) {
                    next0 = idx;
                    tn0 = tc;
                } else {
                    next1 = idx;
                    tn1 = tc;
                }
                nn++;
            }
        }
        if (nn == 2) {
            if (tn0 > tn1) {
                int a = next0;
                next0 = next1;
                next1 = a;
                float b = tn0;
                tn0 = tn1;
                tn1 = b;
            }
            if (tn1 < tmax && sp < kStackSize) {
                if (sp < kSmemStack) stack[sp * stride] = next1;
                else overflow[sp - kSmemStack] = next1;
                sp++;
            }
            if (tn0 < tmax) {
                node = next0;
                continue;
            }
        } else if (nn == 1 && tn0 < tmax) {
            node = next0;
            continue;
        }
        if (sp == 0) break;
        --sp;
        node = sp < kSmemStack ? stack[sp * stride] : overflow[sp - kSmemStack];
    }
    return found;
}

}  // namespace ptw
