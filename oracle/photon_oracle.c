/*
 * photon_oracle.c — TEST INFRASTRUCTURE: the C restatement of Photon's path-tracing hot path and
 * SVGF (see photon_oracle.h). Arithmetic is FP32 in exactly the evaluation order of Photon's
 * C++ (left-to-right sums, vec3 / s as a multiply by 1 / s), built without FMA contraction, so that
 * it agrees bit-for-bit with Photon's own CPU build. Citations are Photon source paths.
 */
#define _GNU_SOURCE
#include "photon_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* math.h:21-25 */
#define K_PI 3.14159265358979323846f
#define K_TWO_PI 6.28318530717958647692f
#define K_INV_PI 0.31830988618379067154f
#define K_INV_TWO_PI 0.15915494309189533577f
#define K_INF 1e30f

typedef struct { float x, y; } v2;
typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } v4;

/* ---- core/math.h:51-121 ------------------------------------------------------------------- */
static inline v2 V2(float x, float y) { v2 r = {x, y}; return r; }
static inline v3 V3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v4 V4(float x, float y, float z, float w) { v4 r = {x, y, z, w}; return r; }
static inline v3 v3s(float s) { return V3(s, s, s); }
static inline v3 add(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 neg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline v3 mul(v3 a, v3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 muls(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 divv(v3 a, v3 b) { return V3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline v3 divs(v3 a, float s) { float inv = 1.0f / s; return V3(a.x * inv, a.y * inv, a.z * inv); } /* math.h:65-68 */
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) { return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline float length(v3 a) { return sqrtf(dot(a, a)); }
static inline float length2(v3 a) { return dot(a, a); }
static inline v3 normalize(v3 a) { float l2 = dot(a, a); return l2 > 0 ? muls(a, 1.0f / sqrtf(l2)) : V3(0, 0, 1); }
static inline v3 vmax3(v3 a, v3 b) { return V3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
static inline float max_comp(v3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
static inline float lerpf(float a, float b, float t) { return a + (b - a) * t; }
static inline v3 lerp3(v3 a, v3 b, float t) { return add(a, muls(sub(b, a), t)); }
static inline float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
static inline float saturate(float v) { return clampf(v, 0.0f, 1.0f); }
static inline v3 reflect3(v3 v, v3 n) { return sub(muls(n, 2.0f * dot(v, n)), v); }
static inline float luminance(v3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
static inline int is_black(v3 c) { return c.x <= 0 && c.y <= 0 && c.z <= 0; }
static inline int is_finite3(v3 c) { return isfinite(c.x) && isfinite(c.y) && isfinite(c.z); }
static inline float sqr(float x) { return x * x; }
static inline float safe_sqrt(float x) { return sqrtf(fmaxf(x, 0.0f)); }
static inline v3 ld3(const pt_vec3 p) { return V3(p.x, p.y, p.z); }
static inline v2 v2add(v2 a, v2 b) { return V2(a.x + b.x, a.y + b.y); }
static inline v2 v2muls(v2 a, float s) { return V2(a.x * s, a.y * s); }
static inline v4 v4add(v4 a, v4 b) { return V4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline v4 v4muls(v4 a, float s) { return V4(a.x * s, a.y * s, a.z * s, a.w * s); }

/* Frame, math.h:127-150 (Duff et al. 2017). */
typedef struct { v3 t, b, n; } frame_t;
static inline frame_t frame_of(v3 n) {
    frame_t f;
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    f.n = n;
    f.t = V3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    f.b = V3(bb, sign + n.y * n.y * a, -n.y);
    return f;
}
static inline v3 to_local(const frame_t* f, v3 v) { return V3(dot(v, f->t), dot(v, f->b), dot(v, f->n)); }
static inline v3 to_world(const frame_t* f, v3 v) { return add(add(muls(f->t, v.x), muls(f->b, v.y)), muls(f->n, v.z)); }

/* ---- core/sampling.h ------------------------------------------------------------------------ */
typedef struct { uint64_t state, inc; } rng_t;
static inline uint32_t rng_u32(rng_t* r) { /* sampling.h:23-29 */
    uint64_t old = r->state;
    r->state = old * 6364136223846793005ULL + r->inc;
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
}
static inline rng_t rng_make(uint64_t seed, uint64_t stream) { /* sampling.h:14-20 */
    rng_t r;
    r.state = 0;
    r.inc = (stream << 1u) | 1u;
    rng_u32(&r);
    r.state += seed;
    rng_u32(&r);
    return r;
}
static inline float rng_next(rng_t* r) { return fminf((float)(rng_u32(r) >> 8) * (1.0f / 16777216.0f), 0.99999994f); }
static inline v2 rng_next2(rng_t* r) { float a = rng_next(r); float b = rng_next(r); return V2(a, b); }
uint32_t orc_hash_u32(uint32_t x) { /* sampling.h:37-44 */
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
static inline v2 concentric_disk(v2 u) { /* sampling.h:46-58 */
    float a = 2.0f * u.x - 1.0f, b = 2.0f * u.y - 1.0f;
    if (a == 0 && b == 0) return V2(0, 0);
    float r, phi;
    if (fabsf(a) > fabsf(b)) {
        r = a;
        phi = (K_PI / 4) * (b / a);
    } else {
        r = b;
        phi = (K_PI / 2) - (K_PI / 4) * (a / b);
    }
    return V2(r * cosf(phi), r * sinf(phi));
}
static inline v3 cosine_hemisphere(v2 u) { /* sampling.h:60-64 */
    v2 d = concentric_disk(u);
    float z = safe_sqrt(1.0f - d.x * d.x - d.y * d.y);
    return V3(d.x, d.y, z);
}
static inline float cosine_hemisphere_pdf(float c) { return fmaxf(c, 0.0f) * K_INV_PI; }
static inline v3 uniform_sphere(v2 u) { /* sampling.h:68-73 */
    float z = 1.0f - 2.0f * u.x;
    float r = safe_sqrt(1.0f - z * z);
    float phi = K_TWO_PI * u.y;
    return V3(r * cosf(phi), r * sinf(phi), z);
}
static inline v2 uniform_triangle(v2 u) { float su = sqrtf(u.x); return V2(1.0f - su, u.y * su); } /* :76-79 */
static inline float power_heuristic(float pa, float pb) { /* sampling.h:82-85 */
    float a = pa * pa, b = pb * pb;
    return a + b > 0 ? a / (a + b) : 0.0f;
}
static inline v2 direction_to_equirect(v3 d) { /* sampling.h:88-92 */
    float u = atan2f(d.x, -d.z) * K_INV_TWO_PI + 0.5f;
    float v = acosf(clampf(d.y, -1.0f, 1.0f)) * K_INV_PI;
    return V2(u - floorf(u), v);
}
static inline v3 equirect_to_direction(v2 uv) { /* sampling.h:94-99 */
    float phi = (uv.x - 0.5f) * K_TWO_PI;
    float theta = uv.y * K_PI;
    float s = sinf(theta);
    return V3(s * sinf(phi), cosf(theta), -s * cosf(phi));
}

/* ---- render/texture.h ----------------------------------------------------------------------- */
static inline v4 unpack_texel(uint32_t p, int srgb, const float* lut) { /* texture.h:8-12 */
    float r = (float)(p & 0xFF), g = (float)((p >> 8) & 0xFF), b = (float)((p >> 16) & 0xFF), a = (float)(p >> 24);
    if (srgb) return V4(lut[p & 0xFF], lut[(p >> 8) & 0xFF], lut[(p >> 16) & 0xFF], a * (1.0f / 255.0f));
    return v4muls(V4(r, g, b, a), 1.0f / 255.0f);
}
static inline int wrap_coord(int i, int n, int repeat) { /* texture.h:14-20 */
    if (repeat) {
        i %= n;
        return i < 0 ? i + n : i;
    }
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
static v4 sample_texture(const pt_scene_desc* s, int tex, v2 uv, uint64_t* taps) { /* texture.h:22-44 */
    const pt_texture_info* t = &s->textures[tex];
    float x = uv.x * (float)t->width - 0.5f, y = uv.y * (float)t->height - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    if (!(fabsf(fx) < 1e8f) || !(fabsf(fy) < 1e8f)) return V4(0, 0, 0, 1);
    int x0 = (int)fx, y0 = (int)fy;
    float tx = x - fx, ty = y - fy;
    int rep = t->wrap_repeat != 0;
    int xa = wrap_coord(x0, t->width, rep), xb = wrap_coord(x0 + 1, t->width, rep);
    int ya = wrap_coord(y0, t->height, rep), yb = wrap_coord(y0 + 1, t->height, rep);
    const uint32_t* base = s->texels + t->offset;
    int srgb = t->srgb != 0;
    v4 a = unpack_texel(base[ya * t->width + xa], srgb, s->srgb_lut);
    v4 b = unpack_texel(base[ya * t->width + xb], srgb, s->srgb_lut);
    v4 c = unpack_texel(base[yb * t->width + xa], srgb, s->srgb_lut);
    v4 d = unpack_texel(base[yb * t->width + xb], srgb, s->srgb_lut);
    if (taps) *taps += 4;
    v4 top = v4add(v4muls(a, 1 - tx), v4muls(b, tx));
    v4 bottom = v4add(v4muls(c, 1 - tx), v4muls(d, tx));
    return v4add(v4muls(top, 1 - ty), v4muls(bottom, ty));
}

/* ---- render/traverse.h ---------------------------------------------------------------------- */
typedef struct { v3 o, d; float tmax; } ray_t;
typedef struct { float t; int tri; float u, v; } hit_t;
#define STACK_SIZE 64

typedef struct {
    uint64_t node_visits, tri_tests, alpha_tests, texture_taps;
} trav_count;

static inline int intersect_triangle(const pt_tri_geom* g, v3 o, v3 d, float tmax, float* t, float* u, float* v) {
    /* traverse.h:24-37 */
    v3 e1 = ld3(g->e1), e2 = ld3(g->e2);
    v3 p = cross(d, e2);
    float det = dot(e1, p);
    if (fabsf(det) < 1e-14f) return 0;
    float inv = 1.0f / det;
    v3 s = sub(o, ld3(g->v0));
    *u = dot(s, p) * inv;
    if (*u < 0.0f || *u > 1.0f) return 0;
    v3 q = cross(s, e1);
    *v = dot(d, q) * inv;
    if (*v < 0.0f || *u + *v > 1.0f) return 0;
    *t = dot(e2, q) * inv;
    return *t > 0.0f && *t < tmax;
}
static inline float intersect_box(pt_vec3 bmin, pt_vec3 bmax, v3 o, v3 inv_d, float tmax) { /* traverse.h:40-47 */
    float tx0 = (bmin.x - o.x) * inv_d.x, tx1 = (bmax.x - o.x) * inv_d.x;
    float ty0 = (bmin.y - o.y) * inv_d.y, ty1 = (bmax.y - o.y) * inv_d.y;
    float tz0 = (bmin.z - o.z) * inv_d.z, tz1 = (bmax.z - o.z) * inv_d.z;
    float tnear = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
    float tfar = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    return tnear <= tfar ? tnear : K_INF;
}
static inline float safe_inv(float x) { return fabsf(x) > 1e-20f ? 1.0f / x : copysignf(1e20f, x); } /* :49-52 */

static int alpha_passes(const pt_scene_desc* s, int tri, float u, float v, trav_count* c) { /* traverse.h:55-64 */
    const pt_material* m = &s->materials[s->tris[tri].material];
    float alpha = m->base_color.w;
    if (c) c->alpha_tests++;
    if (m->base_color_tex >= 0 && s->uvs) {
        const int32_t* idx = s->indices + 3 * tri;
        v2 uv0 = V2(s->uvs[idx[0]].x, s->uvs[idx[0]].y), uv1 = V2(s->uvs[idx[1]].x, s->uvs[idx[1]].y),
           uv2 = V2(s->uvs[idx[2]].x, s->uvs[idx[2]].y);
        v2 uv = v2add(v2add(v2muls(uv0, 1 - u - v), v2muls(uv1, u)), v2muls(uv2, v));
        alpha *= sample_texture(s, m->base_color_tex, uv, c ? &c->texture_taps : NULL).w;
    }
    return alpha < m->alpha_cutoff;
}

static int traverse(const pt_scene_desc* s, const ray_t* ray, hit_t* hit, int any_hit, int* node_visits,
                    trav_count* cnt) { /* traverse.h:66-138 */
    v3 inv_d = V3(safe_inv(ray->d.x), safe_inv(ray->d.y), safe_inv(ray->d.z));
    float tmax = ray->tmax;
    int stack[STACK_SIZE];
    int sp = 0, node = 0, found = 0, visits = 0;
    for (;;) {
        const pt_bvh_node* n = &s->nodes[node];
        visits++;
        float tl = intersect_box(n->lmin, n->lmax, ray->o, inv_d, tmax);
        float tr = intersect_box(n->rmin, n->rmax, ray->o, inv_d, tmax);
        int next[2];
        float tn[2];
        int nn = 0;
        for (int side = 0; side < 2; side++) {
            float tc = side == 0 ? tl : tr;
            if (tc == K_INF) continue;
            int count = side == 0 ? n->lcount : n->rcount;
            int idx = side == 0 ? n->left : n->right;
            if (count > 0) {
                for (int i = idx; i < idx + count; i++) {
                    float t, u, v;
                    if (cnt) cnt->tri_tests++;
                    if (intersect_triangle(&s->tris[i], ray->o, ray->d, tmax, &t, &u, &v)) {
                        if ((s->tris[i].flags & PT_TRI_ALPHA_TESTED) && alpha_passes(s, i, u, v, cnt)) continue;
                        if (any_hit) {
                            if (node_visits) *node_visits += visits;
                            if (cnt) cnt->node_visits += (uint64_t)visits;
                            hit->t = t;
                            hit->tri = i;
                            return 1;
                        }
                        tmax = t;
                        hit->t = t;
                        hit->tri = i;
                        hit->u = u;
                        hit->v = v;
                        found = 1;
                    }
                }
            } else if (idx >= 0) {
                next[nn] = idx;
                tn[nn] = tc;
                nn++;
            }
        }
        if (nn == 2) {
            if (tn[0] > tn[1]) {
                int a = next[0];
                next[0] = next[1];
                next[1] = a;
                float b = tn[0];
                tn[0] = tn[1];
                tn[1] = b;
            }
            if (tn[1] < tmax && sp < STACK_SIZE) stack[sp++] = next[1];
            if (tn[0] < tmax) {
                node = next[0];
                continue;
            }
        } else if (nn == 1 && tn[0] < tmax) {
            node = next[0];
            continue;
        }
        if (sp == 0) break;
        node = stack[--sp];
    }
    if (node_visits) *node_visits += visits;
    if (cnt) cnt->node_visits += (uint64_t)visits;
    return found;
}
static inline int intersect(const pt_scene_desc* s, const ray_t* r, hit_t* h, trav_count* c) {
    h->t = K_INF;
    h->tri = -1;
    h->u = h->v = 0;
    return traverse(s, r, h, 0, NULL, c);
}
static inline int occluded(const pt_scene_desc* s, const ray_t* r, trav_count* c) {
    hit_t h = {K_INF, -1, 0, 0};
    return traverse(s, r, &h, 1, NULL, c);
}

/* ---- render/bsdf.h -------------------------------------------------------------------------- */
typedef struct { v3 base; float metallic, roughness, transmission, ior; } bsdf_params;
typedef struct { v3 wi, f; float pdf; int transmitted, valid; } bsdf_sample_t;
typedef struct { v3 base; float alpha, ior, w_metal, w_opaque, w_glass, f0, diffuse_norm; } bsdf_t;

static inline float ggx_d(v3 h, float alpha) { /* bsdf.h:45-50 */
    float a2 = alpha * alpha;
    float c2 = h.z * h.z;
    float d = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / (K_PI * d * d);
}
static inline float ggx_lambda(v3 w, float alpha) { /* bsdf.h:52-57 */
    float c2 = w.z * w.z;
    if (c2 >= 1.0f) return 0.0f;
    float t2 = (1.0f - c2) / fmaxf(c2, 1e-12f);
    return 0.5f * (-1.0f + sqrtf(1.0f + alpha * alpha * t2));
}
static inline float ggx_g1(v3 w, float a) { return 1.0f / (1.0f + ggx_lambda(w, a)); }
static inline float ggx_g2(v3 wo, v3 wi, float a) { return 1.0f / (1.0f + ggx_lambda(wo, a) + ggx_lambda(wi, a)); }
static inline v3 sample_vndf(v3 wo, float alpha, v2 u) { /* bsdf.h:65-78 (Heitz 2018) */
    v3 vh = normalize(V3(alpha * wo.x, alpha * wo.y, wo.z));
    float lensq = vh.x * vh.x + vh.y * vh.y;
    v3 t1 = lensq > 0 ? muls(V3(-vh.y, vh.x, 0), 1.0f / sqrtf(lensq)) : V3(1, 0, 0);
    v3 t2 = cross(vh, t1);
    float r = sqrtf(u.x);
    float phi = K_TWO_PI * u.y;
    float p1 = r * cosf(phi), p2 = r * sinf(phi);
    float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * safe_sqrt(1.0f - p1 * p1) + s * p2;
    v3 nh = add(add(muls(t1, p1), muls(t2, p2)), muls(vh, safe_sqrt(1.0f - p1 * p1 - p2 * p2)));
    return normalize(V3(alpha * nh.x, alpha * nh.y, fmaxf(1e-6f, nh.z)));
}
static inline float vndf_pdf(v3 wo, v3 h, float alpha) { /* bsdf.h:80-83 */
    if (wo.z <= 0) return 0.0f;
    return ggx_g1(wo, alpha) * fmaxf(0.0f, dot(wo, h)) * ggx_d(h, alpha) / wo.z;
}
static inline v3 fresnel_schlick(v3 f0, float cos_theta) { /* bsdf.h:85-89 */
    float m = saturate(1.0f - cos_theta);
    float m5 = m * m * m * m * m;
    return add(f0, muls(sub(v3s(1.0f), f0), m5));
}
static inline float fresnel_dielectric(float cos_i, float eta) { /* bsdf.h:92-105 */
    cos_i = clampf(cos_i, -1.0f, 1.0f);
    if (cos_i < 0) {
        eta = 1.0f / eta;
        cos_i = -cos_i;
    }
    float sin2_t = (1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = safe_sqrt(1.0f - sin2_t);
    float r_parl = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    float r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return 0.5f * (r_parl * r_parl + r_perp * r_perp);
}
static inline float fresnel_avg(float eta) { return (eta - 1.0f) / (4.08567f + 1.00071f * eta); } /* :108 */

static inline bsdf_t bsdf_make(bsdf_params p) { /* bsdf.h:119-130 */
    bsdf_t b;
    b.base = p.base;
    float r = clampf(p.roughness, 0.0f, 1.0f);
    b.alpha = fmaxf(r * r, 0.002f);
    b.ior = fmaxf(p.ior, 1.0001f);
    float m = saturate(p.metallic), t = saturate(p.transmission);
    b.w_metal = m;
    b.w_glass = (1 - m) * t;
    b.w_opaque = (1 - m) * (1 - t);
    b.f0 = sqr((b.ior - 1) / (b.ior + 1));
    b.diffuse_norm = 1.0f / (1.0f - fresnel_avg(b.ior));
    return b;
}
static inline float opaque_spec_prob(const bsdf_t* b, float cos_o) { /* bsdf.h:133-138 */
    if (b->f0 < 1e-6f) return 0.0f;
    float f = fresnel_schlick(v3s(b->f0), cos_o).x;
    float d = (1 - f) * fmaxf(luminance(b->base), 0.01f);
    return clampf(f / (f + d), 0.1f, 0.9f);
}
static inline int bsdf_samples_lights(const bsdf_t* b) { return !(b->alpha <= 0.002f) || b->w_opaque > 0; }
static inline v3 bsdf_albedo(const bsdf_t* b) { return add(muls(b->base, b->w_metal + b->w_opaque), v3s(b->w_glass)); }

static v3 glass_eval(const bsdf_t* b, v3 wo, v3 wi, float* pdf_out) { /* bsdf.h:150-182 */
    int refl = wo.z * wi.z > 0;
    float etap = wo.z > 0 ? b->ior : 1.0f / b->ior;
    v3 wm = refl ? add(wo, wi) : add(muls(wi, etap), wo);
    if (length2(wm) < 1e-20f || wo.z == 0 || wi.z == 0) {
        *pdf_out = 0;
        return v3s(0);
    }
    wm = normalize(wm);
    if (wm.z < 0) wm = neg(wm);
    if (dot(wm, wi) * wi.z < 0 || dot(wm, wo) * wo.z < 0) {
        *pdf_out = 0;
        return v3s(0);
    }
    float F = fresnel_dielectric(dot(wo, wm), b->ior);
    float R = F, T = 1 - F;
    v3 wo_up = wo.z > 0 ? wo : neg(wo);
    float pdf_m = vndf_pdf(wo_up, wm, b->alpha);
    float D = ggx_d(wm, b->alpha), G = ggx_g2(wo, wi, b->alpha);
    if (refl) {
        *pdf_out = pdf_m / (4.0f * fabsf(dot(wo, wm))) * R;
        return v3s(D * G * F / (4.0f * fabsf(wi.z * wo.z)));
    }
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / etap);
    float dwm_dwi = fabsf(dot(wi, wm)) / denom;
    *pdf_out = pdf_m * dwm_dwi * T;
    float ft = T * D * G * fabsf(dot(wi, wm) * dot(wo, wm) / (wi.z * wo.z * denom)) / (etap * etap);
    return muls(b->base, ft);
}
static int glass_sample(const bsdf_t* b, v3 wo, v2 u, float u_lobe, v3* wi) { /* bsdf.h:184-205 */
    v3 wo_up = wo.z > 0 ? wo : neg(wo);
    v3 wm = sample_vndf(wo_up, b->alpha, u);
    float F = fresnel_dielectric(dot(wo, wm), b->ior);
    if (u_lobe < F) {
        *wi = reflect3(wo, wm);
        return wi->z * wo.z > 0;
    }
    float etap = wo.z > 0 ? b->ior : 1.0f / b->ior;
    float cos_i = dot(wo, wm);
    v3 n = wm;
    if (cos_i < 0) {
        n = neg(wm);
        cos_i = -cos_i;
    }
    float sin2_t = (1 - cos_i * cos_i) / (etap * etap);
    if (sin2_t >= 1) return 0;
    float cos_t = safe_sqrt(1 - sin2_t);
    *wi = add(divs(neg(wo), etap), muls(n, cos_i / etap - cos_t));
    return wi->z * wo.z < 0;
}
static v3 bsdf_eval_pdf(const bsdf_t* b, v3 wo, v3 wi, float* pdf_out) { /* bsdf.h:220-252 */
    v3 f = v3s(0);
    float pdf = 0;
    int same = wo.z * wi.z > 0;
    if (same && wo.z > 0 && (b->w_metal > 0 || b->w_opaque > 0)) {
        v3 h = normalize(add(wo, wi));
        float D = ggx_d(h, b->alpha), G = ggx_g2(wo, wi, b->alpha);
        float spec = D * G / (4.0f * wo.z * wi.z);
        float pdf_spec = vndf_pdf(wo, h, b->alpha) / (4.0f * dot(wo, h));
        float voh = dot(wo, h);
        if (b->w_metal > 0) {
            f = add(f, muls(fresnel_schlick(b->base, voh), spec * b->w_metal));
            pdf += b->w_metal * pdf_spec;
        }
        if (b->w_opaque > 0) {
            int matched = b->f0 < 1e-6f;
            float F = matched ? 0.0f : fresnel_dielectric(voh, b->ior);
            float base_layer = matched ? K_INV_PI
                                       : (1 - fresnel_dielectric(wo.z, b->ior)) * (1 - fresnel_dielectric(wi.z, b->ior)) *
                                             b->diffuse_norm * K_INV_PI;
            f = add(f, muls(add(v3s(F * spec), muls(b->base, base_layer)), b->w_opaque));
            float ps = opaque_spec_prob(b, wo.z);
            pdf += b->w_opaque * (ps * pdf_spec + (1 - ps) * cosine_hemisphere_pdf(wi.z));
        }
    }
    if (b->w_glass > 0) {
        float pg;
        f = add(f, muls(glass_eval(b, wo, wi, &pg), b->w_glass));
        pdf += b->w_glass * pg;
    }
    *pdf_out = pdf;
    return f;
}
static bsdf_sample_t bsdf_sample(const bsdf_t* b, v3 wo, float u_lobe, v2 u, float u_sub) { /* bsdf.h:255-281 */
    bsdf_sample_t s;
    memset(&s, 0, sizeof(s));
    v3 wi;
    if (u_lobe < b->w_glass) {
        if (!glass_sample(b, wo, u, u_sub, &wi)) return s;
    } else {
        if (wo.z <= 0) return s;
        float ul = (u_lobe - b->w_glass) / fmaxf(1 - b->w_glass, 1e-6f);
        int spec = 1;
        if (ul >= b->w_metal / fmaxf(b->w_metal + b->w_opaque, 1e-6f)) spec = u_sub < opaque_spec_prob(b, wo.z);
        if (spec) {
            v3 h = sample_vndf(wo, b->alpha, u);
            wi = reflect3(wo, h);
        } else {
            wi = cosine_hemisphere(u);
        }
        if (wi.z <= 0) return s;
    }
    s.wi = wi;
    s.f = bsdf_eval_pdf(b, wo, wi, &s.pdf);
    s.transmitted = wi.z * wo.z < 0;
    s.valid = s.pdf > 0 && is_finite3(s.f);
    return s;
}

/* ---- render/lights.h ------------------------------------------------------------------------ */
typedef struct { v3 wi; float dist; v3 radiance; float pdf; int delta; int tri; v2 bary; } light_sample_t;

int orc_sample_alias(const pt_alias_entry* table, int n, float u, float* pmf) { /* lights.h:22-30 */
    float x = u * (float)n;
    int i = (int)x;
    if (i >= n) i = n - 1;
    float frac = x - (float)i;
    int chosen = frac < table[i].prob ? i : table[i].alias;
    *pmf = table[chosen].pmf;
    return chosen;
}
static inline v3 rotate_y(v3 d, float angle) { /* lights.h:34-37 */
    float c = cosf(angle), s = sinf(angle);
    return V3(c * d.x + s * d.z, d.y, -s * d.x + c * d.z);
}
static v3 env_radiance(const pt_scene_desc* s, v3 dir, uint64_t* lookups) { /* lights.h:39-47 */
    if (!s->env_texels) return muls(ld3(s->env_color), s->env_intensity);
    if (lookups) (*lookups)++;
    v2 uv = direction_to_equirect(rotate_y(dir, -s->env_rotation));
    int x = (int)(uv.x * (float)s->env_width);
    int y = (int)(uv.y * (float)s->env_height);
    x = x < 0 ? 0 : (x >= s->env_width ? s->env_width - 1 : x);
    y = y < 0 ? 0 : (y >= s->env_height ? s->env_height - 1 : y);
    return muls(ld3(s->env_texels[y * s->env_width + x]), s->env_intensity);
}
static inline int find_interval(const float* cdf, int n, float u) { /* lights.h:50-58 */
    int lo = 0, hi = n;
    while (lo + 1 < hi) {
        int mid = (lo + hi) / 2;
        if (cdf[mid] <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}
static float env_pdf_dir(const pt_scene_desc* s, v3 dir) { /* lights.h:61-74 */
    if (!s->env_texels) return 1.0f / (4.0f * K_PI);
    v3 d = rotate_y(dir, -s->env_rotation);
    v2 uv = direction_to_equirect(d);
    float sin_theta = safe_sqrt(1 - d.y * d.y);
    if (sin_theta <= 0 || s->env_integral <= 0) return 0;
    int x = (int)(uv.x * (float)s->env_width), y = (int)(uv.y * (float)s->env_height);
    x = x < 0 ? 0 : (x >= s->env_width ? s->env_width - 1 : x);
    y = y < 0 ? 0 : (y >= s->env_height ? s->env_height - 1 : y);
    float row_sin = sinf(((float)y + 0.5f) / (float)s->env_height * K_PI);
    float f = luminance(ld3(s->env_texels[y * s->env_width + x])) * row_sin;
    float pdf_uv = f / s->env_integral;
    return pdf_uv / (2.0f * K_PI * K_PI * sin_theta);
}
static int sample_env(const pt_scene_desc* s, v2 u, v3* dir, float* pdf) { /* lights.h:76-98 */
    if (!s->env_texels) {
        *dir = uniform_sphere(u);
        *pdf = 1.0f / (4.0f * K_PI);
        return 1;
    }
    int w = s->env_width, h = s->env_height;
    int y = find_interval(s->env_marginal, h, u.y);
    float c0 = s->env_marginal[y], c1 = s->env_marginal[y + 1];
    float dv = c1 > c0 ? (u.y - c0) / (c1 - c0) : 0.5f;
    const float* row = s->env_conditional + y * (w + 1);
    int x = find_interval(row, w, u.x);
    float r0 = row[x], r1 = row[x + 1];
    float du = r1 > r0 ? (u.x - r0) / (r1 - r0) : 0.5f;
    v2 uv = V2(((float)x + du) / (float)w, ((float)y + dv) / (float)h);
    v3 d = equirect_to_direction(uv);
    *dir = rotate_y(d, s->env_rotation);
    float sin_theta = safe_sqrt(1 - d.y * d.y);
    if (sin_theta <= 1e-6f) return 0;
    float row_sin = sinf(((float)y + 0.5f) / (float)h * K_PI);
    float f = luminance(ld3(s->env_texels[y * w + x])) * row_sin;
    *pdf = f / s->env_integral / (2.0f * K_PI * K_PI * sin_theta);
    return *pdf > 0;
}
static v3 emitted(const pt_scene_desc* s, int tri, float u, float v, uint64_t* taps) { /* lights.h:104-113 */
    const pt_material* m = &s->materials[s->tris[tri].material];
    v3 e = ld3(m->emission);
    if (m->emissive_tex >= 0 && s->uvs) {
        const int32_t* idx = s->indices + 3 * tri;
        v2 uv0 = V2(s->uvs[idx[0]].x, s->uvs[idx[0]].y), uv1 = V2(s->uvs[idx[1]].x, s->uvs[idx[1]].y),
           uv2 = V2(s->uvs[idx[2]].x, s->uvs[idx[2]].y);
        v2 uv = v2add(v2add(v2muls(uv0, 1 - u - v), v2muls(uv1, u)), v2muls(uv2, v));
        v4 t = sample_texture(s, m->emissive_tex, uv, taps);
        e = mul(e, V3(t.x, t.y, t.z));
    }
    return e;
}
static int emits_towards(const pt_scene_desc* s, int tri, v3 dir_from_light) { /* lights.h:115-119 */
    const pt_tri_geom* g = &s->tris[tri];
    v3 n = cross(ld3(g->e1), ld3(g->e2));
    return s->materials[g->material].double_sided != 0 || dot(n, dir_from_light) > 0;
}
static float emissive_pdf(const pt_scene_desc* s, int tri, v3 dir, float dist) { /* lights.h:123-133 */
    if (s->num_emissive == 0 || !s->tri_emissive) return 0;
    int k = s->tri_emissive[tri];
    if (k < 0) return 0;
    const pt_emissive_tri* e = &s->emissive[k];
    const pt_tri_geom* g = &s->tris[tri];
    v3 n = normalize(cross(ld3(g->e1), ld3(g->e2)));
    float cos_l = fabsf(dot(n, dir));
    if (cos_l <= 0) return 0;
    return s->p_emissive * s->emissive_alias[k].pmf * dist * dist / (e->area * cos_l);
}
static inline float env_pdf(const pt_scene_desc* s, v3 dir) { return s->p_env * env_pdf_dir(s, dir); }

typedef struct { int group, index, bin; } light_pick;

static light_sample_t sample_light(const pt_scene_desc* s, v3 p, float u_group, v2 u, float u_light, light_pick* pick,
                                   uint64_t* taps) { /* lights.h:139-202 */
    light_sample_t ls;
    memset(&ls, 0, sizeof(ls));
    ls.tri = -1;
    if (pick) pick->group = pick->index = pick->bin = -1;
    if (u_group < s->p_emissive && s->num_emissive > 0) {
        float pmf;
        int k = orc_sample_alias(s->emissive_alias, s->num_emissive, u_light, &pmf);
        if (pick) {
            int bin = (int)(u_light * (float)s->num_emissive);
            pick->group = 0;
            pick->index = k;
            pick->bin = bin >= s->num_emissive ? s->num_emissive - 1 : bin;
        }
        const pt_emissive_tri* e = &s->emissive[k];
        const pt_tri_geom* g = &s->tris[e->tri];
        v2 b = uniform_triangle(u);
        v3 q = add(add(ld3(g->v0), muls(ld3(g->e1), b.x)), muls(ld3(g->e2), b.y));
        v3 d = sub(q, p);
        float dist2 = length2(d);
        if (dist2 <= 0) return ls;
        float dist = sqrtf(dist2);
        v3 wi = divs(d, dist);
        v3 n = normalize(cross(ld3(g->e1), ld3(g->e2)));
        float cos_l = fabsf(dot(n, wi));
        if (cos_l <= 1e-8f || !emits_towards(s, e->tri, neg(wi))) return ls;
        ls.wi = wi;
        ls.dist = dist;
        ls.radiance = emitted(s, e->tri, b.x, b.y, taps);
        ls.pdf = s->p_emissive * pmf * dist2 / (e->area * cos_l);
        ls.tri = e->tri;
        ls.bary = b;
        return ls;
    }
    if (u_group < s->p_emissive + s->p_punctual && s->num_punctual > 0) {
        int k = (int)(u_light * (float)s->num_punctual);
        if (k >= s->num_punctual) k = s->num_punctual - 1;
        if (pick) {
            pick->group = 1;
            pick->index = k;
        }
        const pt_punctual_light* l = &s->punctual[k];
        float pk = s->p_punctual / (float)s->num_punctual;
        ls.delta = 1;
        ls.pdf = pk;
        if (l->type == PT_LIGHT_DIRECTIONAL) {
            ls.wi = neg(ld3(l->direction));
            ls.dist = K_INF;
            ls.radiance = ld3(l->intensity);
            return ls;
        }
        v3 d = sub(ld3(l->position), p);
        float dist2 = length2(d);
        if (dist2 <= 0) {
            memset(&ls, 0, sizeof(ls));
            ls.tri = -1;
            return ls;
        }
        float dist = sqrtf(dist2);
        ls.wi = divs(d, dist);
        ls.dist = dist;
        v3 li = divs(ld3(l->intensity), dist2);
        if (l->type == PT_LIGHT_SPOT) {
            float cd = dot(neg(ls.wi), ld3(l->direction));
            float t = saturate((cd - l->cos_outer) / fmaxf(l->cos_inner - l->cos_outer, 1e-4f));
            li = muls(li, t * t);
        }
        ls.radiance = li;
        return ls;
    }
    if (s->p_env > 0) {
        if (pick) pick->group = 2;
        v3 dir;
        float pdf;
        if (s->env_texels && pick) {
            int y = find_interval(s->env_marginal, s->env_height, u.y);
            const float* row = s->env_conditional + y * (s->env_width + 1);
            pick->index = y * s->env_width + find_interval(row, s->env_width, u.x);
        }
        if (!sample_env(s, u, &dir, &pdf)) return ls;
        ls.wi = dir;
        ls.dist = K_INF;
        ls.radiance = env_radiance(s, dir, NULL);
        ls.pdf = s->p_env * pdf;
    }
    return ls;
}

/* ---- render/integrator.h -------------------------------------------------------------------- */
typedef struct {
    v3 position;
    float depth;
    v3 normal;
    int material;
    v3 albedo;
    v3 emission;
} primary_t;

static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline float offset_comp(float pc, float nc) { /* integrator.h:61-69 (Wachter & Binder 2019) */
    const float origin = 1.0f / 32.0f, float_scale = 1.0f / 65536.0f, int_scale = 256.0f;
    int of = (int)(int_scale * nc);
    float pi = bitsf(fbits(pc) + (uint32_t)(pc < 0 ? -of : of));
    return fabsf(pc) < origin ? pc + float_scale * nc : pi;
}
static inline v3 offset_ray(v3 p, v3 n) { return V3(offset_comp(p.x, n.x), offset_comp(p.y, n.y), offset_comp(p.z, n.z)); }

typedef struct {
    v3 p, ng, ns;
    v2 uv;
    frame_t frame;
    bsdf_params params;
    v3 emission;
    int front, material;
} interaction_t;

static interaction_t surface_at(const pt_scene_desc* s, const ray_t* ray, const hit_t* hit, uint64_t* taps,
                                uint64_t* normal_mapped) { /* integrator.h:83-148 */
    interaction_t it;
    const pt_tri_geom* g = &s->tris[hit->tri];
    const pt_material* m = &s->materials[g->material];
    it.material = g->material;
    float w = 1 - hit->u - hit->v;
    it.p = add(ray->o, muls(ray->d, hit->t));
    v3 ng = normalize(cross(ld3(g->e1), ld3(g->e2)));
    const int32_t* idx = s->indices + 3 * hit->tri;
    v3 ns = ng;
    if (s->normals) {
        v3 n = add(add(muls(ld3(s->normals[idx[0]]), w), muls(ld3(s->normals[idx[1]]), hit->u)),
                   muls(ld3(s->normals[idx[2]]), hit->v));
        if (length2(n) > 1e-12f) ns = normalize(n);
        if (dot(ns, ng) < 0) ns = neg(ns);
    }
    if (s->uvs) {
        v2 uv0 = V2(s->uvs[idx[0]].x, s->uvs[idx[0]].y), uv1 = V2(s->uvs[idx[1]].x, s->uvs[idx[1]].y),
           uv2 = V2(s->uvs[idx[2]].x, s->uvs[idx[2]].y);
        it.uv = v2add(v2add(v2muls(uv0, w), v2muls(uv1, hit->u)), v2muls(uv2, hit->v));
    } else {
        it.uv = V2(0, 0);
    }
    it.front = dot(ray->d, ng) < 0;
    if (m->normal_tex >= 0 && s->tangents) {
        const pt_vec4* T = s->tangents;
        v4 t0 = V4(T[idx[0]].x, T[idx[0]].y, T[idx[0]].z, T[idx[0]].w);
        v4 t1 = V4(T[idx[1]].x, T[idx[1]].y, T[idx[1]].z, T[idx[1]].w);
        v4 t2 = V4(T[idx[2]].x, T[idx[2]].y, T[idx[2]].z, T[idx[2]].w);
        v4 t4 = v4add(v4add(v4muls(t0, w), v4muls(t1, hit->u)), v4muls(t2, hit->v));
        v3 t = V3(t4.x, t4.y, t4.z);
        if (normal_mapped) (*normal_mapped)++;
        if (length2(t) > 1e-12f) {
            t = normalize(sub(t, muls(ns, dot(ns, t))));
            v3 b = muls(cross(ns, t), T[idx[0]].w < 0 ? -1.0f : 1.0f);
            v4 tn = sample_texture(s, m->normal_tex, it.uv, taps);
            v3 nt = V3(tn.x * 2 - 1, tn.y * 2 - 1, tn.z * 2 - 1);
            nt.x *= m->normal_scale;
            nt.y *= m->normal_scale;
            v3 n = normalize(add(add(muls(t, nt.x), muls(b, nt.y)), muls(ns, nt.z)));
            if (dot(n, ng) > 0.01f) ns = n;
        }
    }
    v4 base = V4(m->base_color.x, m->base_color.y, m->base_color.z, m->base_color.w);
    if (m->base_color_tex >= 0) {
        v4 tc = sample_texture(s, m->base_color_tex, it.uv, taps);
        base = V4(base.x * tc.x, base.y * tc.y, base.z * tc.z, base.w * tc.w);
    }
    float metallic = m->metallic, roughness = m->roughness;
    if (m->metallic_roughness_tex >= 0) {
        v4 mr = sample_texture(s, m->metallic_roughness_tex, it.uv, taps);
        roughness *= mr.y;
        metallic *= mr.z;
    }
    it.params.base = V3(base.x, base.y, base.z);
    it.params.metallic = metallic;
    it.params.roughness = roughness;
    it.params.transmission = m->transmission;
    it.params.ior = m->ior;
    it.emission = (it.front || m->double_sided) ? emitted(s, hit->tri, hit->u, hit->v, taps) : v3s(0);
    if (m->transmission <= 0 && !it.front) {
        ng = neg(ng);
        ns = neg(ns);
    }
    v3 wo = neg(ray->d);
    if (m->transmission <= 0 && dot(wo, ns) <= 0) ns = ng;
    it.ng = ng;
    it.ns = ns;
    it.frame = frame_of(ns);
    return it;
}

typedef struct {
    int max_depth, rr_depth, nee;
    float clamp;
} path_opts;

typedef struct {
    trav_count trav;
    uint64_t camera_rays, extension_rays, shadow_rays, shade_events, normal_mapped, nee_e, nee_p, nee_env, env_lookups;
} path_count;

static v3 trace_path(const pt_scene_desc* s, ray_t ray, rng_t* rng, const path_opts* opt, primary_t* primary,
                     light_pick* first_pick, int* first_nee, path_count* pc) { /* integrator.h:151-263 */
    v3 L = v3s(0), beta = v3s(1);
    float prev_pdf = 0;
    int prev_delta = 1;
    int has_lights = s->p_env + s->p_emissive + s->p_punctual > 0;
    trav_count* tc = pc ? &pc->trav : NULL;
    uint64_t* taps = pc ? &pc->trav.texture_taps : NULL;
    for (int depth = 0;; depth++) {
        hit_t hit;
        if (pc) {
            if (depth == 0) pc->camera_rays++;
            else pc->extension_rays++;
        }
        if (!intersect(s, &ray, &hit, tc)) {
            v3 le = env_radiance(s, ray.d, pc ? &pc->env_lookups : NULL);
            float w = (prev_delta || s->p_env <= 0) ? 1.0f : power_heuristic(prev_pdf, env_pdf(s, ray.d));
            v3 c = muls(mul(beta, le), w);
            if (depth > 0 && opt->clamp > 0) {
                float l = luminance(c);
                if (l > opt->clamp) c = muls(c, opt->clamp / l);
            }
            L = add(L, c);
            if (depth == 0 && primary) {
                primary->depth = 0;
                primary->material = -1;
                primary->emission = le;
                primary->albedo = v3s(1);
                primary->normal = neg(ray.d);
                primary->position = add(ray.o, muls(ray.d, 1e4f));
            }
            break;
        }
        if (pc) pc->shade_events++;
        interaction_t it = surface_at(s, &ray, &hit, taps, pc ? &pc->normal_mapped : NULL);
        v3 wo_world = neg(ray.d);
        if (!is_black(it.emission)) {
            float w = 1.0f;
            if (!prev_delta) w = power_heuristic(prev_pdf, emissive_pdf(s, hit.tri, ray.d, hit.t));
            v3 c = muls(mul(beta, it.emission), w);
            if (depth > 0 && opt->clamp > 0) {
                float l = luminance(c);
                if (l > opt->clamp) c = muls(c, opt->clamp / l);
            }
            L = add(L, c);
        }
        bsdf_t bsdf = bsdf_make(it.params);
        if (depth == 0 && primary) {
            primary->position = it.p;
            primary->depth = hit.t;
            primary->normal = it.ns;
            primary->material = it.material;
            primary->albedo = bsdf_albedo(&bsdf);
            primary->emission = it.emission;
        }
        if (depth + 1 >= opt->max_depth) break;
        v3 wo = to_local(&it.frame, wo_world);
        int nee = opt->nee && has_lights && bsdf_samples_lights(&bsdf);
        if (depth == 0 && first_nee) *first_nee = nee;
        if (nee) {
            float ug = rng_next(rng);
            v2 ul = rng_next2(rng);
            float uk = rng_next(rng);
            light_pick pk;
            light_sample_t ls = sample_light(s, it.p, ug, ul, uk, &pk, taps);
            if (depth == 0 && first_pick) *first_pick = pk;
            if (pc) {
                if (pk.group == 0) pc->nee_e++;
                else if (pk.group == 1) pc->nee_p++;
                else if (pk.group == 2) pc->nee_env++;
            }
            if (ls.pdf > 0 && !is_black(ls.radiance)) {
                v3 wi = to_local(&it.frame, ls.wi);
                float pdf_b;
                v3 f = bsdf_eval_pdf(&bsdf, wo, wi, &pdf_b);
                if (!is_black(f)) {
                    v3 origin = offset_ray(it.p, dot(ls.wi, it.ng) > 0 ? it.ng : neg(it.ng));
                    ray_t shadow;
                    shadow.o = origin;
                    shadow.d = ls.wi;
                    shadow.tmax = ls.dist == K_INF ? K_INF : ls.dist * (1.0f - 1e-4f);
                    if (pc) pc->shadow_rays++;
                    if (!occluded(s, &shadow, tc)) {
                        float w = ls.delta ? 1.0f : power_heuristic(ls.pdf, pdf_b);
                        v3 c = muls(mul(muls(mul(beta, f), fabsf(wi.z)), ls.radiance), w / ls.pdf);
                        if (depth > 0 && opt->clamp > 0) {
                            float l = luminance(c);
                            if (l > opt->clamp) c = muls(c, opt->clamp / l);
                        }
                        L = add(L, c);
                    }
                }
            }
        }
        float u_lobe = rng_next(rng);
        v2 u = rng_next2(rng);
        float u_sub = rng_next(rng);
        bsdf_sample_t bs = bsdf_sample(&bsdf, wo, u_lobe, u, u_sub);
        if (!bs.valid) break;
        beta = mul(beta, muls(bs.f, fabsf(bs.wi.z) / bs.pdf));
        if (!is_finite3(beta) || is_black(beta)) break;
        prev_pdf = bs.pdf;
        prev_delta = !nee;
        v3 wi_world = to_world(&it.frame, bs.wi);
        float side = dot(wi_world, it.ng) * dot(wo_world, it.ng);
        if (bs.transmitted ? side >= 0 : side <= 0) break;
        ray.o = offset_ray(it.p, dot(wi_world, it.ng) > 0 ? it.ng : neg(it.ng));
        ray.d = normalize(wi_world);
        ray.tmax = K_INF;
        if (depth + 1 >= opt->rr_depth) {
            float q = fmaxf(0.05f, 1.0f - max_comp(beta));
            if (rng_next(rng) < q) break;
            beta = muls(beta, 1.0f / (1.0f - q));
        }
    }
    return L;
}

static ray_t camera_ray(const pt_camera* c, float px, float py, int width, int height, v2 lens) { /* :266-280 */
    float sx = (2.0f * px / (float)width - 1.0f) * c->tan_half_fov * c->aspect;
    float sy = (1.0f - 2.0f * py / (float)height) * c->tan_half_fov;
    v3 fwd = ld3(c->forward), right = ld3(c->right), up = ld3(c->up), pos = ld3(c->position);
    v3 d = normalize(add(add(fwd, muls(right, sx)), muls(up, sy)));
    ray_t r;
    r.o = pos;
    r.d = d;
    r.tmax = K_INF;
    if (c->aperture > 0) {
        v3 focus = add(pos, muls(d, c->focus_distance / dot(d, fwd)));
        v2 l = v2muls(concentric_disk(lens), c->aperture);
        r.o = add(add(pos, muls(right, l.x)), muls(up, l.y));
        r.d = normalize(sub(focus, r.o));
    }
    return r;
}

static inline rng_t pixel_rng(uint32_t pixel, uint32_t seed, uint32_t frame) { /* pixel.h:20-21 */
    uint64_t s0 = (uint64_t)orc_hash_u32(pixel ^ orc_hash_u32(seed)) | ((uint64_t)orc_hash_u32(frame + 0x9e3779b9u) << 32);
    return rng_make(s0, pixel);
}

static inline path_opts opts_of(const pt_render_settings* rs) {
    path_opts o;
    o.max_depth = rs->path.max_depth;
    o.rr_depth = rs->path.rr_depth;
    o.nee = rs->path.nee;
    o.clamp = rs->path.clamp;
    return o;
}

static v3 render_sample(const pt_scene_desc* s, const pt_camera* cam, int x, int y, int width, int height, uint32_t frame,
                        uint32_t seed, const path_opts* opt, primary_t* primary, light_pick* pick, int* first_nee,
                        path_count* pc) { /* pixel.h:18-29 */
    uint32_t pixel = (uint32_t)y * (uint32_t)width + (uint32_t)x;
    rng_t rng = pixel_rng(pixel, seed, frame);
    v2 jitter = rng_next2(&rng);
    v2 lens = rng_next2(&rng);
    ray_t ray = camera_ray(cam, (float)x + jitter.x, (float)y + jitter.y, width, height, lens);
    v3 L = trace_path(s, ray, &rng, opt, primary, pick, first_nee, pc);
    if (!is_finite3(L) || L.x < 0 || L.y < 0 || L.z < 0) L = v3s(0);
    return L;
}

static void primary_init(primary_t* p) {
    memset(p, 0, sizeof(*p));
    p->material = -1;
    p->albedo = v3s(1);
}

/* ---- threaded rows (cpu_renderer.cpp:20-39) ------------------------------------------------- */
typedef struct {
    const pt_scene_desc* s;
    const pt_camera* cam;
    const pt_render_settings* rs;
    int spp;
    uint32_t frame0;
    float* sum;
    float *color4, *albedo4, *nd4, *pos4, *em4;
    int mode; /* 0 render, 1 gbuffer */
    int next_row;
    pthread_mutex_t lock;
} row_job;

static int take_row(row_job* j) {
    pthread_mutex_lock(&j->lock);
    int y = j->next_row++;
    pthread_mutex_unlock(&j->lock);
    return y;
}

static void* row_worker(void* arg) {
    row_job* j = (row_job*)arg;
    path_opts opt = opts_of(j->rs);
    int w = j->rs->width, h = j->rs->height;
    for (;;) {
        int y = take_row(j);
        if (y >= h) break;
        for (int x = 0; x < w; x++) {
            size_t i = (size_t)y * (size_t)w + (size_t)x;
            if (j->mode == 0) {
                v3 acc = v3s(0);
                for (int k = 0; k < j->spp; k++)
                    acc = add(acc, render_sample(j->s, j->cam, x, y, w, h, j->frame0 + (uint32_t)k, j->rs->seed, &opt, NULL,
                                                 NULL, NULL, NULL));
                j->sum[3 * i] += acc.x;
                j->sum[3 * i + 1] += acc.y;
                j->sum[3 * i + 2] += acc.z;
            } else {
                primary_t pr;
                primary_init(&pr);
                v3 L = render_sample(j->s, j->cam, x, y, w, h, j->frame0, j->rs->seed, &opt, &pr, NULL, NULL, NULL);
                float* c = j->color4 + 4 * i;
                c[0] = L.x; c[1] = L.y; c[2] = L.z; c[3] = 1;
                float* a = j->albedo4 + 4 * i;
                a[0] = pr.albedo.x; a[1] = pr.albedo.y; a[2] = pr.albedo.z; a[3] = 1;
                float* nd = j->nd4 + 4 * i;
                nd[0] = pr.normal.x; nd[1] = pr.normal.y; nd[2] = pr.normal.z; nd[3] = pr.depth;
                float* p = j->pos4 + 4 * i;
                p[0] = pr.position.x; p[1] = pr.position.y; p[2] = pr.position.z; p[3] = (float)pr.material;
                float* e = j->em4 + 4 * i;
                e[0] = pr.emission.x; e[1] = pr.emission.y; e[2] = pr.emission.z; e[3] = 1;
            }
        }
    }
    return NULL;
}

static void run_rows(row_job* j, int threads) {
    int n = threads > 0 ? threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1) n = 1;
    if (n > 256) n = 256;
    pthread_t pool[256];
    pthread_mutex_init(&j->lock, NULL);
    j->next_row = 0;
    for (int i = 0; i < n; i++) pthread_create(&pool[i], NULL, row_worker, j);
    for (int i = 0; i < n; i++) pthread_join(pool[i], NULL);
    pthread_mutex_destroy(&j->lock);
}

void orc_render(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, int spp, uint32_t frame0,
                int threads, float* sum_rgb) {
    row_job j;
    memset(&j, 0, sizeof(j));
    j.s = s;
    j.cam = cam;
    j.rs = rs;
    j.spp = spp;
    j.frame0 = frame0;
    j.sum = sum_rgb;
    j.mode = 0;
    run_rows(&j, threads);
}

void orc_sample_gbuffer(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, uint32_t frame,
                        int threads, float* color4, float* albedo4, float* normal_depth4, float* position4,
                        float* emission4) {
    row_job j;
    memset(&j, 0, sizeof(j));
    j.s = s;
    j.cam = cam;
    j.rs = rs;
    j.frame0 = frame;
    j.color4 = color4;
    j.albedo4 = albedo4;
    j.nd4 = normal_depth4;
    j.pos4 = position4;
    j.em4 = emission4;
    j.mode = 1;
    run_rows(&j, threads);
}

void orc_render_sample(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, int x, int y,
                       uint32_t frame, float* L3, float* primary16) {
    path_opts opt = opts_of(rs);
    primary_t pr;
    primary_init(&pr);
    v3 L = render_sample(s, cam, x, y, rs->width, rs->height, frame, rs->seed, &opt, &pr, NULL, NULL, NULL);
    L3[0] = L.x;
    L3[1] = L.y;
    L3[2] = L.z;
    if (primary16) {
        float* o = primary16;
        o[0] = pr.position.x; o[1] = pr.position.y; o[2] = pr.position.z; o[3] = pr.depth;
        o[4] = pr.normal.x; o[5] = pr.normal.y; o[6] = pr.normal.z; o[7] = (float)pr.material;
        o[8] = pr.albedo.x; o[9] = pr.albedo.y; o[10] = pr.albedo.z;
        o[11] = pr.emission.x; o[12] = pr.emission.y; o[13] = pr.emission.z;
        o[14] = 0; o[15] = 0;
    }
}

void orc_trace_primary(const pt_scene_desc* s, const pt_camera* cam, int w, int h, uint32_t frame, uint32_t seed,
                       float* hits4) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            uint32_t pixel = (uint32_t)y * (uint32_t)w + (uint32_t)x;
            rng_t rng = pixel_rng(pixel, seed, frame);
            v2 jitter = rng_next2(&rng);
            v2 lens = rng_next2(&rng);
            ray_t ray = camera_ray(cam, (float)x + jitter.x, (float)y + jitter.y, w, h, lens);
            hit_t hit;
            intersect(s, &ray, &hit, NULL);
            float* o = hits4 + 4 * (size_t)pixel;
            o[0] = hit.t;
            memcpy(&o[1], &hit.tri, 4);
            o[2] = hit.u;
            o[3] = hit.v;
        }
}

void orc_light_picks_primary(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs,
                             uint32_t frame, int32_t* picks4) {
    path_opts opt = opts_of(rs);
    /* Only the first vertex matters: stop after it by limiting the depth to 2 (the pick happens
     * before the depth test of vertex 1). */
    path_opts first = opt;
    if (first.max_depth > 2) first.max_depth = 2;
    for (int y = 0; y < rs->height; y++)
        for (int x = 0; x < rs->width; x++) {
            size_t i = (size_t)y * (size_t)rs->width + (size_t)x;
            light_pick pk = {-1, -1, -1};
            int nee = 0;
            if (opt.max_depth >= 2) render_sample(s, cam, x, y, rs->width, rs->height, frame, rs->seed, &first, NULL, &pk, &nee, NULL);
            picks4[4 * i] = nee ? pk.group : -1;
            picks4[4 * i + 1] = nee ? pk.index : -1;
            picks4[4 * i + 2] = nee ? pk.bin : -1;
            picks4[4 * i + 3] = nee;
        }
}

void orc_occluded(const pt_scene_desc* s, const float* rays8, int n, int32_t* out4) { /* traverse.h:144-147 */
    for (int i = 0; i < n; i++) {
        const float* q = rays8 + 8 * (size_t)i;
        ray_t r;
        r.o = V3(q[0], q[1], q[2]);
        r.tmax = q[3];
        r.d = V3(q[4], q[5], q[6]);
        hit_t h = {K_INF, -1, 0, 0};
        int visits = 0;
        trav_count c;
        memset(&c, 0, sizeof(c));
        int occ = traverse(s, &r, &h, 1, &visits, &c);
        out4[4 * i] = occ;
        out4[4 * i + 1] = occ ? h.tri : -1;
        out4[4 * i + 2] = visits;
        out4[4 * i + 3] = (int32_t)c.tri_tests;
    }
}

void orc_heatmap(const pt_scene_desc* s, const pt_camera* cam, int w, int h, float* out) {
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            ray_t ray = camera_ray(cam, (float)x + 0.5f, (float)y + 0.5f, w, h, V2(0.5f, 0.5f));
            hit_t hit = {K_INF, -1, 0, 0};
            int visits = 0;
            traverse(s, &ray, &hit, 0, &visits, NULL);
            out[(size_t)y * (size_t)w + (size_t)x] = (float)visits;
        }
}

void orc_count(const pt_scene_desc* s, const pt_camera* cam, const pt_render_settings* rs, int stride, orc_counters* out) {
    path_opts opt = opts_of(rs);
    path_count pc;
    memset(&pc, 0, sizeof(pc));
    uint64_t n = 0;
    int w = rs->width, h = rs->height;
    if (stride < 1) stride = 1;
    for (int y = 0; y < h; y += stride)
        for (int x = (y / stride) % stride; x < w; x += stride, n++)
            render_sample(s, cam, x, y, w, h, 0, rs->seed, &opt, NULL, NULL, NULL, &pc);
    memset(out, 0, sizeof(*out));
    out->samples = n;
    out->camera_rays = pc.camera_rays;
    out->extension_rays = pc.extension_rays;
    out->shadow_rays = pc.shadow_rays;
    out->node_visits = pc.trav.node_visits;
    out->tri_tests = pc.trav.tri_tests;
    out->alpha_tests = pc.trav.alpha_tests;
    out->shade_events = pc.shade_events;
    out->normal_mapped_events = pc.normal_mapped;
    out->nee_emissive = pc.nee_e;
    out->nee_punctual = pc.nee_p;
    out->nee_env = pc.nee_env;
    out->env_lookups = pc.env_lookups;
    out->texture_taps = pc.trav.texture_taps;
}

/* ---- known-answer helpers ------------------------------------------------------------------- */
void orc_rng_floats(uint64_t seed, uint64_t stream, int n, float* out) {
    rng_t r = rng_make(seed, stream);
    for (int i = 0; i < n; i++) out[i] = rng_next(&r);
}
void orc_offset_ray(int n, const float* p, const float* nrm, float* out) {
    for (int i = 0; i < n; i++) {
        v3 q = offset_ray(V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), V3(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]));
        out[3 * i] = q.x;
        out[3 * i + 1] = q.y;
        out[3 * i + 2] = q.z;
    }
}
void orc_bsdf_sample(const float* p7, int n, const float* rows8, float* out9) {
    bsdf_params p;
    p.base = V3(p7[0], p7[1], p7[2]);
    p.metallic = p7[3];
    p.roughness = p7[4];
    p.transmission = p7[5];
    p.ior = p7[6];
    bsdf_t b = bsdf_make(p);
    for (int i = 0; i < n; i++) {
        const float* r = rows8 + 8 * i;
        bsdf_sample_t s = bsdf_sample(&b, V3(r[0], r[1], r[2]), r[3], V2(r[4], r[5]), r[6]);
        float* o = out9 + 9 * i;
        o[0] = s.wi.x; o[1] = s.wi.y; o[2] = s.wi.z;
        o[3] = s.f.x; o[4] = s.f.y; o[5] = s.f.z;
        o[6] = s.pdf;
        o[7] = s.transmitted ? 1.0f : 0.0f;
        o[8] = s.valid ? 1.0f : 0.0f;
    }
}
void orc_sample_light(const pt_scene_desc* s, const float* p3, float u_group, float u0, float u1, float u_light,
                      float* o) {
    light_sample_t ls = sample_light(s, V3(p3[0], p3[1], p3[2]), u_group, V2(u0, u1), u_light, NULL, NULL);
    o[0] = ls.wi.x; o[1] = ls.wi.y; o[2] = ls.wi.z; o[3] = ls.dist;
    o[4] = ls.radiance.x; o[5] = ls.radiance.y; o[6] = ls.radiance.z; o[7] = ls.pdf;
    o[8] = (float)ls.delta; o[9] = (float)ls.tri; o[10] = ls.bary.x; o[11] = ls.bary.y;
}

/* ---- denoise/svgf.cu ------------------------------------------------------------------------ */
struct orc_svgf {
    int w, h, has_history;
    float *prev_illum, *prev_moments, *prev_nd, *prev_pos, *illum, *moments, *filter[2];
};

orc_svgf* orc_svgf_create(int w, int h) { /* Svgf::resize, svgf.cu:225-236 */
    orc_svgf* s = (orc_svgf*)calloc(1, sizeof(orc_svgf));
    s->w = w;
    s->h = h;
    size_t n = (size_t)w * (size_t)h * 4;
    s->prev_illum = (float*)calloc(n, 4);
    s->prev_moments = (float*)calloc(n, 4);
    s->prev_nd = (float*)calloc(n, 4);
    s->prev_pos = (float*)calloc(n, 4);
    s->illum = (float*)calloc(n, 4);
    s->moments = (float*)calloc(n, 4);
    s->filter[0] = (float*)calloc(n, 4);
    s->filter[1] = (float*)calloc(n, 4);
    return s;
}
void orc_svgf_destroy(orc_svgf* s) {
    if (!s) return;
    free(s->prev_illum); free(s->prev_moments); free(s->prev_nd); free(s->prev_pos);
    free(s->illum); free(s->moments); free(s->filter[0]); free(s->filter[1]);
    free(s);
}
void orc_svgf_reset(orc_svgf* s) { s->has_history = 0; }
const float* orc_svgf_variance(const orc_svgf* s) { return s->filter[0]; }

static inline v3 f4xyz(const float* p) { return V3(p[0], p[1], p[2]); }
static inline void st4(float* p, float x, float y, float z, float w) { p[0] = x; p[1] = y; p[2] = z; p[3] = w; }

static int svgf_project(const pt_camera* c, v3 p, int w, int h, float* px, float* py, float* dist) { /* svgf.cu:25-35 */
    v3 d = sub(p, ld3(c->position));
    float z = dot(d, ld3(c->forward));
    if (z <= 1e-4f) return 0;
    float sx = dot(d, ld3(c->right)) / (z * c->tan_half_fov * c->aspect);
    float sy = dot(d, ld3(c->up)) / (z * c->tan_half_fov);
    *px = (sx + 1.0f) * 0.5f * (float)w - 0.5f;
    *py = (1.0f - sy) * 0.5f * (float)h - 0.5f;
    *dist = length(d);
    return 1;
}

void orc_svgf_run(orc_svgf* S, const float* color4, const float* albedo4, const float* nd4, const float* pos4,
                  const float* em4, const pt_camera* prev, const pt_svgf_settings* st, float* out4) {
    int w = S->w, h = S->h;
    /* temporal_kernel, svgf.cu:37-92 */
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int i = y * w + x;
            const float* pos = pos4 + 4 * i;
            v3 col = f4xyz(color4 + 4 * i), em = f4xyz(em4 + 4 * i), alb = f4xyz(albedo4 + 4 * i);
            v3 il = vmax3(sub(col, em), v3s(0));
            v3 cur = V3(il.x / fmaxf(alb.x, 1e-3f), il.y / fmaxf(alb.y, 1e-3f), il.z / fmaxf(alb.z, 1e-3f));
            float lum = luminance(cur);
            v3 hist_c = v3s(0);
            float hm0 = 0, hm1 = 0, hist_len = 0, wsum = 0;
            if (S->has_history && pos[3] >= 0) {
                float px, py, dist;
                if (svgf_project(prev, f4xyz(pos), w, h, &px, &py, &dist)) {
                    v3 n = f4xyz(nd4 + 4 * i);
                    int x0 = (int)floorf(px), y0 = (int)floorf(py);
                    float fx = px - (float)x0, fy = py - (float)y0;
                    for (int k = 0; k < 4; k++) {
                        int xx = x0 + (k & 1), yy = y0 + (k >> 1);
                        if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                        int j = yy * w + xx;
                        const float* pp = S->prev_pos + 4 * j;
                        const float* pn = S->prev_nd + 4 * j;
                        if (pp[3] != pos[3]) continue;
                        if (fabsf(pn[3] - dist) > 0.05f * dist + 0.01f) continue;
                        if (dot(f4xyz(pn), n) < 0.9f) continue;
                        float bw = ((k & 1) ? fx : 1 - fx) * ((k >> 1) ? fy : 1 - fy);
                        const float* pi = S->prev_illum + 4 * j;
                        const float* pm = S->prev_moments + 4 * j;
                        hist_c = add(hist_c, muls(f4xyz(pi), bw));
                        hm0 = hm0 + pm[0] * bw;
                        hm1 = hm1 + pm[1] * bw;
                        hist_len += pi[3] * bw;
                        wsum += bw;
                    }
                }
            }
            v3 c;
            float m0, m1, len;
            if (wsum > 1e-3f) {
                hist_c = divs(hist_c, wsum);
                float inv = 1.0f / wsum;
                hm0 = hm0 * inv;
                hm1 = hm1 * inv;
                len = fminf(hist_len / wsum + 1.0f, 64.0f);
                float ac = fmaxf(st->alpha_color, 1.0f / len), am = fmaxf(st->alpha_moments, 1.0f / len);
                c = lerp3(hist_c, cur, ac);
                m0 = lerpf(hm0, lum, am);
                m1 = lerpf(hm1, lum * lum, am);
            } else {
                len = 1.0f;
                c = cur;
                m0 = lum;
                m1 = lum * lum;
            }
            float variance = fmaxf(0.0f, m1 - m0 * m0);
            st4(S->illum + 4 * i, c.x, c.y, c.z, len);
            st4(S->moments + 4 * i, m0, m1, variance, 0);
        }
    /* variance_kernel, svgf.cu:96-132 */
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int i = y * w + x;
            const float* cc = S->illum + 4 * i;
            v3 c = f4xyz(cc);
            float len = cc[3];
            float variance = S->moments[4 * i + 2];
            if (len < 4.0f && pos4[4 * i + 3] >= 0) {
                v3 n = f4xyz(nd4 + 4 * i);
                float z = nd4[4 * i + 3];
                float wsum = 0, m1 = 0, m2 = 0;
                v3 acc = v3s(0);
                for (int dy = -3; dy <= 3; dy++)
                    for (int dx = -3; dx <= 3; dx++) {
                        int xx = x + dx, yy = y + dy;
                        if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                        int j = yy * w + xx;
                        if (pos4[4 * j + 3] != pos4[4 * i + 3]) continue;
                        const float* nd = nd4 + 4 * j;
                        float wn = powf(fmaxf(0.0f, dot(n, f4xyz(nd))), st->phi_normal);
                        float wz = expf(-fabsf(nd[3] - z) / (0.05f * z + 1e-3f));
                        float wt = wn * wz;
                        const float* m = S->moments + 4 * j;
                        m1 += m[0] * wt;
                        m2 += m[1] * wt;
                        acc = add(acc, muls(f4xyz(S->illum + 4 * j), wt));
                        wsum += wt;
                    }
                if (wsum > 0) {
                    m1 /= wsum;
                    m2 /= wsum;
                    variance = fmaxf(0.0f, m2 - m1 * m1) * (4.0f / len);
                    c = divs(acc, wsum);
                }
            }
            st4(S->filter[0] + 4 * i, c.x, c.y, c.z, variance);
        }
    /* atrous_kernel (svgf.cu:134-186) x iterations; history_kernel (:188-197) after pass 0. */
    int src = 0;
    const float kernel[3] = {3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
    for (int it = 0; it < st->atrous_iterations; it++) {
        int step = 1 << it;
        const float* sbuf = S->filter[src];
        float* dbuf = S->filter[1 - src];
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                int i = y * w + x;
                const float* center = sbuf + 4 * i;
                if (pos4[4 * i + 3] < 0) {
                    memcpy(dbuf + 4 * i, center, 16);
                    continue;
                }
                float var = 0, vw = 0;
                for (int dy = -1; dy <= 1; dy++)
                    for (int dx = -1; dx <= 1; dx++) {
                        int xx = x + dx < 0 ? 0 : (x + dx > w - 1 ? w - 1 : x + dx);
                        int yy = y + dy < 0 ? 0 : (y + dy > h - 1 ? h - 1 : y + dy);
                        float k = (dx == 0 && dy == 0) ? 0.25f : ((dx == 0 || dy == 0) ? 0.125f : 0.0625f);
                        var += sbuf[4 * (yy * w + xx) + 3] * k;
                        vw += k;
                    }
                var /= vw;
                v3 n = f4xyz(nd4 + 4 * i);
                float z = nd4[4 * i + 3];
                int xr = x + 1 < w - 1 ? x + 1 : w - 1, xl = x - 1 > 0 ? x - 1 : 0;
                int yd = y + 1 < h - 1 ? y + 1 : h - 1, yu = y - 1 > 0 ? y - 1 : 0;
                float zx = nd4[4 * (y * w + xr) + 3] - nd4[4 * (y * w + xl) + 3];
                float zy = nd4[4 * (yd * w + x) + 3] - nd4[4 * (yu * w + x) + 3];
                float grad = 0.5f * fmaxf(fabsf(zx), fabsf(zy));
                float lum_c = luminance(f4xyz(center));
                float sigma_l = st->phi_color * sqrtf(fmaxf(var, 0.0f)) + 1e-4f;
                v3 sum = v3s(0);
                float wsum = 0, vsum = 0;
                for (int dy = -2; dy <= 2; dy++)
                    for (int dx = -2; dx <= 2; dx++) {
                        int xx = x + dx * step, yy = y + dy * step;
                        if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                        int j = yy * w + xx;
                        if (pos4[4 * j + 3] != pos4[4 * i + 3]) continue;
                        const float* sv = sbuf + 4 * j;
                        const float* nd = nd4 + 4 * j;
                        float k = kernel[abs(dx)] * kernel[abs(dy)];
                        float wl = expf(-fabsf(luminance(f4xyz(sv)) - lum_c) / sigma_l);
                        float wn = powf(fmaxf(0.0f, dot(n, f4xyz(nd))), st->phi_normal);
                        float dist = sqrtf((float)(dx * dx + dy * dy)) * (float)step;
                        float wz = expf(-fabsf(nd[3] - z) / (st->phi_depth * grad * dist + 1e-3f * z + 1e-4f));
                        float wt = k * wl * wn * wz;
                        sum = add(sum, muls(f4xyz(sv), wt));
                        vsum += wt * wt * sv[3];
                        wsum += wt;
                    }
                if (wsum > 0) {
                    v3 r = divs(sum, wsum);
                    st4(dbuf + 4 * i, r.x, r.y, r.z, vsum / (wsum * wsum));
                } else {
                    memcpy(dbuf + 4 * i, center, 16);
                }
            }
        src = 1 - src;
        if (it == 0) {
            const float* f = S->filter[src];
            for (int i = 0; i < w * h; i++) {
                st4(S->prev_illum + 4 * i, f[4 * i], f[4 * i + 1], f[4 * i + 2], S->illum[4 * i + 3]);
                memcpy(S->prev_moments + 4 * i, S->moments + 4 * i, 16);
                memcpy(S->prev_nd + 4 * i, nd4 + 4 * i, 16);
                memcpy(S->prev_pos + 4 * i, pos4 + 4 * i, 16);
            }
        }
    }
    if (st->atrous_iterations == 0) {
        const float* f = S->filter[src];
        for (int i = 0; i < w * h; i++) {
            st4(S->prev_illum + 4 * i, f[4 * i], f[4 * i + 1], f[4 * i + 2], S->illum[4 * i + 3]);
            memcpy(S->prev_moments + 4 * i, S->moments + 4 * i, 16);
            memcpy(S->prev_nd + 4 * i, nd4 + 4 * i, 16);
            memcpy(S->prev_pos + 4 * i, pos4 + 4 * i, 16);
        }
    }
    /* remodulate_kernel, svgf.cu:199-210 */
    const float* f = S->filter[src];
    for (int i = 0; i < w * h; i++) {
        if (pos4[4 * i + 3] < 0) {
            memcpy(out4 + 4 * i, color4 + 4 * i, 16);
            continue;
        }
        v3 a = f4xyz(albedo4 + 4 * i);
        v3 c = add(mul(f4xyz(f + 4 * i), vmax3(a, v3s(1e-3f))), f4xyz(em4 + 4 * i));
        st4(out4 + 4 * i, c.x, c.y, c.z, 1);
    }
    S->has_history = 1;
}
