// Device vector math for the wavefront path tracer.
//
// The arithmetic mirrors Photon's shared integrator headers (src/core/math.h, src/core/sampling.h)
// operation for operation: sums are evaluated left to right, vec3 / s is a multiply by 1 / s
// (math.h:65-68), and this translation unit is compiled with -fmad=false, IEEE division and square
// root, so that every elementary result rounds exactly as Photon's CPU build does (x86-64 SSE, no
// FMA). Transcendentals (sinf, cosf, atan2f, acosf) are CUDA's precise functions; they may differ
// from glibc in the last bit, which is why image parity is statistical while hit indices and
// light picks are exact.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define PT_HD __device__ __forceinline__

namespace ptw {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kInvTwoPi = 0.15915494309189533577f;
constexpr float kInf = 1e30f;

struct V2 {
    float x, y;
};
struct V3 {
    float x, y, z;
};
struct V4 {
    float x, y, z, w;
};

PT_HD V2 v2(float x, float y) { return {x, y}; }
PT_HD V3 v3(float x, float y, float z) { return {x, y, z}; }
PT_HD V3 v3(float s) { return {s, s, s}; }
PT_HD V4 v4(float x, float y, float z, float w) { return {x, y, z, w}; }
PT_HD V3 xyz(float4 a) { return {a.x, a.y, a.z}; }
PT_HD V3 xyz(V4 a) { return {a.x, a.y, a.z}; }

PT_HD V2 operator+(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
PT_HD V2 operator*(V2 a, float s) { return {a.x * s, a.y * s}; }
PT_HD V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
PT_HD V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
PT_HD V3 operator-(V3 a) { return {-a.x, -a.y, -a.z}; }
PT_HD V3 operator*(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
PT_HD V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
PT_HD V3 operator/(V3 a, float s) {
    float inv = 1.0f / s;
    return {a.x * inv, a.y * inv, a.z * inv};
}
PT_HD V4 operator+(V4 a, V4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
PT_HD V4 operator*(V4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }

PT_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_HD V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
PT_HD float length_sq(V3 a) { return dot(a, a); }
PT_HD float length(V3 a) { return sqrtf(dot(a, a)); }
PT_HD V3 normalize(V3 a) {
    float l2 = dot(a, a);
    return l2 > 0 ? a * (1.0f / sqrtf(l2)) : V3{0, 0, 1};
}
PT_HD V3 vmax(V3 a, V3 b) { return {fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)}; }
PT_HD float max_component(V3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
PT_HD float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
PT_HD float saturate(float v) { return clampf(v, 0.0f, 1.0f); }
PT_HD float lerpf(float a, float b, float t) { return a + (b - a) * t; }
PT_HD V3 lerp(V3 a, V3 b, float t) { return a + (b - a) * t; }
PT_HD V3 reflect(V3 v, V3 n) { return n * (2.0f * dot(v, n)) - v; }
PT_HD float luminance(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
PT_HD bool is_black(V3 c) { return c.x <= 0 && c.y <= 0 && c.z <= 0; }
PT_HD bool is_finite(V3 c) { return isfinite(c.x) && isfinite(c.y) && isfinite(c.z); }
PT_HD float sqr(float x) { return x * x; }
PT_HD float safe_sqrt(float x) { return sqrtf(fmaxf(x, 0.0f)); }

// Orthonormal basis around a unit normal (Duff et al. 2017), as math.h:127-150.
struct Frame {
    V3 t, b, n;
};
PT_HD Frame make_frame(V3 n) {
    Frame f;
    float sign = copysignf(1.0f, n.z);
    float a = -1.0f / (sign + n.z);
    float bb = n.x * n.y * a;
    f.n = n;
    f.t = {1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x};
    f.b = {bb, sign + n.y * n.y * a, -n.y};
    return f;
}
PT_HD V3 to_local(const Frame& f, V3 v) { return {dot(v, f.t), dot(v, f.b), dot(v, f.n)}; }
PT_HD V3 to_world(const Frame& f, V3 v) { return f.t * v.x + f.b * v.y + f.n * v.z; }

// PCG32 (O'Neill 2014) with Photon's seeding and float conversion (sampling.h:9-34). The stream
// increment is 2 * pixel + 1, so a path stores only the 64-bit state and its pixel.
struct Rng {
    uint64_t state, inc;
};
PT_HD uint32_t rng_u32(Rng& r) {
    uint64_t old = r.state;
    r.state = old * 6364136223846793005ULL + r.inc;
    uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((~rot + 1u) & 31));
}
PT_HD Rng rng_seed(uint64_t seed, uint64_t stream) {
    Rng r;
    r.state = 0;
    r.inc = (stream << 1u) | 1u;
    rng_u32(r);
    r.state += seed;
    rng_u32(r);
    return r;
}
PT_HD float rng_next(Rng& r) { return fminf(float(rng_u32(r) >> 8) * (1.0f / 16777216.0f), 0.99999994f); }
PT_HD V2 rng_next2(Rng& r) {
    float a = rng_next(r);
    float b = rng_next(r);
    return {a, b};
}
PT_HD uint32_t hash_u32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
// render_sample's generator for (pixel, sample index, seed), pixel.h:20-21.
PT_HD Rng pixel_rng(uint32_t pixel, uint32_t seed, uint32_t frame) {
    uint64_t s = uint64_t(hash_u32(pixel ^ hash_u32(seed))) | (uint64_t(hash_u32(frame + 0x9e3779b9u)) << 32);
    return rng_seed(s, pixel);
}

// Warps (sampling.h:46-99).
PT_HD V2 concentric_disk(V2 u) {
    float a = 2.0f * u.x - 1.0f, b = 2.0f * u.y - 1.0f;
    if (a == 0 && b == 0) return {0, 0};
    float r, phi;
    if (fabsf(a) > fabsf(b)) {
        r = a;
        phi = (kPi / 4) * (b / a);
    } else {
        r = b;
        phi = (kPi / 2) - (kPi / 4) * (a / b);
    }
    return {r * cosf(phi), r * sinf(phi)};
}
PT_HD V3 cosine_hemisphere(V2 u) {
    V2 d = concentric_disk(u);
    float z = safe_sqrt(1.0f - d.x * d.x - d.y * d.y);
    return {d.x, d.y, z};
}
PT_HD float cosine_hemisphere_pdf(float c) { return fmaxf(c, 0.0f) * kInvPi; }
PT_HD V3 uniform_sphere(V2 u) {
    float z = 1.0f - 2.0f * u.x;
    float r = safe_sqrt(1.0f - z * z);
    float phi = kTwoPi * u.y;
    return {r * cosf(phi), r * sinf(phi), z};
}
PT_HD V2 uniform_triangle(V2 u) {
    float su = sqrtf(u.x);
    return {1.0f - su, u.y * su};
}
PT_HD float power_heuristic(float pa, float pb) {
    float a = pa * pa, b = pb * pb;
    return a + b > 0 ? a / (a + b) : 0.0f;
}
PT_HD V2 direction_to_equirect(V3 d) {
    float u = atan2f(d.x, -d.z) * kInvTwoPi + 0.5f;
    float v = acosf(clampf(d.y, -1.0f, 1.0f)) * kInvPi;
    return {u - floorf(u), v};
}
PT_HD V3 equirect_to_direction(V2 uv) {
    float phi = (uv.x - 0.5f) * kTwoPi;
    float theta = uv.y * kPi;
    float s = sinf(theta);
    return {s * sinf(phi), cosf(theta), -s * cosf(phi)};
}

// Wachter & Binder's ray-origin offset (integrator.h:61-69).
PT_HD float offset_component(float pc, float nc) {
    const float origin = 1.0f / 32.0f, float_scale = 1.0f / 65536.0f, int_scale = 256.0f;
    int of = int(int_scale * nc);
    float pi = __uint_as_float(__float_as_uint(pc) + uint32_t(pc < 0 ? -of : of));
    return fabsf(pc) < origin ? pc + float_scale * nc : pi;
}
PT_HD V3 offset_ray(V3 p, V3 n) { return {offset_component(p.x, n.x), offset_component(p.y, n.y), offset_component(p.z, n.z)}; }

}  // namespace ptw
