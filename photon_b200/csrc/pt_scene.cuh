// The device-resident scene and the shading model: texture fetches, the glTF BSDF, light sampling
// and surface interactions, re-laid for 128-bit loads. Semantics follow Photon's shared integrator
// (src/render/{texture,bsdf,lights,integrator}.h); the evaluation order of every expression is the
// same as there (see pt_math.cuh).
#pragma once

#include "pt_math.cuh"
#include "pt_types.h"

namespace ptw {

// ---- textures (texture.h:8-44) ----------------------------------------------------------------
PT_HD V4 unpack_texel(uint32_t p, bool srgb, const float* lut) {
    float r = float(p & 0xFF), g = float((p >> 8) & 0xFF), b = float((p >> 16) & 0xFF), a = float(p >> 24);
    if (srgb) return {__ldg(lut + (p & 0xFF)), __ldg(lut + ((p >> 8) & 0xFF)), __ldg(lut + ((p >> 16) & 0xFF)), a * (1.0f / 255.0f)};
    return V4{r, g, b, a} * (1.0f / 255.0f);
}
PT_HD int wrap_coord(int i, int n, bool repeat) {
    if (repeat) {
        i %= n;
        return i < 0 ? i + n : i;
    }
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}
PT_HD V4 sample_texture(const DevScene& s, int tex, V2 uv) {
    int4 t = __ldg(s.textures + tex);
    float x = uv.x * float(t.x) - 0.5f, y = uv.y * float(t.y) - 0.5f;
    float fx = floorf(x), fy = floorf(y);
    if (!(fabsf(fx) < 1e8f) || !(fabsf(fy) < 1e8f)) return {0, 0, 0, 1};
    int x0 = int(fx), y0 = int(fy);
    float tx = x - fx, ty = y - fy;
    bool rep = (t.w & 1) != 0, srgb = (t.w & 2) != 0;
    int xa = wrap_coord(x0, t.x, rep), xb = wrap_coord(x0 + 1, t.x, rep);
    int ya = wrap_coord(y0, t.y, rep), yb = wrap_coord(y0 + 1, t.y, rep);
    const uint32_t* base = s.texels + uint32_t(t.z);
    V4 a = unpack_texel(__ldg(base + ya * t.x + xa), srgb, s.srgb_lut);
    V4 b = unpack_texel(__ldg(base + ya * t.x + xb), srgb, s.srgb_lut);
    V4 c = unpack_texel(__ldg(base + yb * t.x + xa), srgb, s.srgb_lut);
    V4 d = unpack_texel(__ldg(base + yb * t.x + xb), srgb, s.srgb_lut);
    V4 top = a * (1 - tx) + b * tx;
    V4 bottom = c * (1 - tx) + d * tx;
    return top * (1 - ty) + bottom * ty;
}

PT_HD V2 load_uv(const DevScene& s, int v) {
    float2 t = __ldg(s.uvs + v);
    return {t.x, t.y};
}
PT_HD V2 interp_uv(const DevScene& s, int4 idx, float u, float v) {
    return load_uv(s, idx.x) * (1 - u - v) + load_uv(s, idx.y) * u + load_uv(s, idx.z) * v;
}

// alpha_passes (traverse.h:55-64): the masked triangle lets the ray through. `g` is the triangle's
// record in DevScene::tris, whose fourth float4 holds its vertex indices: they come from the line the
// intersection test just read instead of a separate tri_idx read, one dependent L2 round trip fewer
// on the way to the texels.
PT_HD bool alpha_passes(const DevScene& s, const float4* g, int material, float u, float v) {
    const float4* m = s.materials + 5 * material;
    float alpha = __ldg(m).w;
    float4 m3 = __ldg(m + 3);
    int base_tex = __float_as_int(m3.w);
    if (base_tex >= 0 && s.uvs) {
        const float4 g3 = __ldg(g + 3);
        V2 uv = interp_uv(s, make_int4(__float_as_int(g3.x), __float_as_int(g3.y), __float_as_int(g3.z), 0), u, v);
        alpha *= sample_texture(s, base_tex, uv).w;
    }
    return alpha < m3.x;
}

// ---- the BSDF (bsdf.h:29-282) --------------------------------------------------------------------
struct BsdfParams {
    V3 base;
    float metallic, roughness, transmission, ior;
};
struct BsdfSample {
    V3 wi, f;
    float pdf;
    bool transmitted, valid;
};

PT_HD float ggx_d(V3 h, float alpha) {
    float a2 = alpha * alpha;
    float c2 = h.z * h.z;
    float d = c2 * (a2 - 1.0f) + 1.0f;
    return a2 / (kPi * d * d);
}
PT_HD float ggx_lambda(V3 w, float alpha) {
    float c2 = w.z * w.z;
    if (c2 >= 1.0f) return 0.0f;
    float t2 = (1.0f - c2) / fmaxf(c2, 1e-12f);
    return 0.5f * (-1.0f + sqrtf(1.0f + alpha * alpha * t2));
}
PT_HD float ggx_g1(V3 w, float a) { return 1.0f / (1.0f + ggx_lambda(w, a)); }
PT_HD float ggx_g2(V3 wo, V3 wi, float a) { return 1.0f / (1.0f + ggx_lambda(wo, a) + ggx_lambda(wi, a)); }
// Visible-normal sampling (Heitz 2018), as bsdf.h:65-78.
PT_HD V3 sample_vndf(V3 wo, float alpha, V2 u) {
    V3 vh = normalize(V3{alpha * wo.x, alpha * wo.y, wo.z});
    float lensq = vh.x * vh.x + vh.y * vh.y;
    V3 t1 = lensq > 0 ? V3{-vh.y, vh.x, 0} * (1.0f / sqrtf(lensq)) : V3{1, 0, 0};
    V3 t2 = cross(vh, t1);
    float r = sqrtf(u.x);
    float phi = kTwoPi * u.y;
    float p1 = r * cosf(phi), p2 = r * sinf(phi);
    float s = 0.5f * (1.0f + vh.z);
    p2 = (1.0f - s) * safe_sqrt(1.0f - p1 * p1) + s * p2;
    V3 nh = t1 * p1 + t2 * p2 + vh * safe_sqrt(1.0f - p1 * p1 - p2 * p2);
    return normalize(V3{alpha * nh.x, alpha * nh.y, fmaxf(1e-6f, nh.z)});
}
PT_HD float vndf_pdf(V3 wo, V3 h, float alpha) {
    if (wo.z <= 0) return 0.0f;
    return ggx_g1(wo, alpha) * fmaxf(0.0f, dot(wo, h)) * ggx_d(h, alpha) / wo.z;
}
PT_HD V3 fresnel_schlick(V3 f0, float cos_theta) {
    float m = saturate(1.0f - cos_theta);
    float m5 = m * m * m * m * m;
    return f0 + (v3(1.0f) - f0) * m5;
}
PT_HD float fresnel_dielectric(float cos_i, float eta) {
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
PT_HD float fresnel_dielectric_average(float eta) { return (eta - 1.0f) / (4.08567f + 1.00071f * eta); }

struct Bsdf {
    V3 base;
    float alpha, ior, w_metal, w_opaque, w_glass, f0, diffuse_norm;
};
PT_HD Bsdf make_bsdf(const BsdfParams& p) {
    Bsdf b;
    b.base = p.base;
    float r = clampf(p.roughness, 0.0f, 1.0f);
    b.alpha = fmaxf(r * r, 0.002f);
    b.ior = fmaxf(p.ior, 1.0001f);
    float m = saturate(p.metallic), t = saturate(p.transmission);
    b.w_metal = m;
    b.w_glass = (1 - m) * t;
    b.w_opaque = (1 - m) * (1 - t);
    b.f0 = sqr((b.ior - 1) / (b.ior + 1));
    b.diffuse_norm = 1.0f / (1.0f - fresnel_dielectric_average(b.ior));
    return b;
}
PT_HD float opaque_spec_prob(const Bsdf& b, float cos_o) {
    if (b.f0 < 1e-6f) return 0.0f;
    float f = fresnel_schlick(v3(b.f0), cos_o).x;
    float d = (1 - f) * fmaxf(luminance(b.base), 0.01f);
    return clampf(f / (f + d), 0.1f, 0.9f);
}
PT_HD bool samples_lights(const Bsdf& b) { return !(b.alpha <= 0.002f) || b.w_opaque > 0; }
PT_HD V3 bsdf_albedo(const Bsdf& b) { return b.base * (b.w_metal + b.w_opaque) + v3(b.w_glass); }

PT_HD V3 glass_eval(const Bsdf& b, V3 wo, V3 wi, float* pdf_out) {
    bool refl = wo.z * wi.z > 0;
    float etap = wo.z > 0 ? b.ior : 1.0f / b.ior;
    V3 wm = refl ? wo + wi : wi * etap + wo;
    if (length_sq(wm) < 1e-20f || wo.z == 0 || wi.z == 0) {
        *pdf_out = 0;
        return v3(0);
    }
    wm = normalize(wm);
    if (wm.z < 0) wm = -wm;
    if (dot(wm, wi) * wi.z < 0 || dot(wm, wo) * wo.z < 0) {
        *pdf_out = 0;
        return v3(0);
    }
    float F = fresnel_dielectric(dot(wo, wm), b.ior);
    float R = F, T = 1 - F;
    V3 wo_up = wo.z > 0 ? wo : -wo;
    float pdf_m = vndf_pdf(wo_up, wm, b.alpha);
    float D = ggx_d(wm, b.alpha), G = ggx_g2(wo, wi, b.alpha);
    if (refl) {
        *pdf_out = pdf_m / (4.0f * fabsf(dot(wo, wm))) * R;
        return v3(D * G * F / (4.0f * fabsf(wi.z * wo.z)));
    }
    float denom = sqr(dot(wi, wm) + dot(wo, wm) / etap);
    float dwm_dwi = fabsf(dot(wi, wm)) / denom;
    *pdf_out = pdf_m * dwm_dwi * T;
    float ft = T * D * G * fabsf(dot(wi, wm) * dot(wo, wm) / (wi.z * wo.z * denom)) / (etap * etap);
    return b.base * ft;
}
PT_HD bool glass_sample(const Bsdf& b, V3 wo, V2 u, float u_lobe, V3& wi) {
    V3 wo_up = wo.z > 0 ? wo : -wo;
    V3 wm = sample_vndf(wo_up, b.alpha, u);
    float F = fresnel_dielectric(dot(wo, wm), b.ior);
    if (u_lobe < F) {
        wi = reflect(wo, wm);
        return wi.z * wo.z > 0;
    }
    float etap = wo.z > 0 ? b.ior : 1.0f / b.ior;
    float cos_i = dot(wo, wm);
    V3 n = wm;
    if (cos_i < 0) {
        n = -wm;
        cos_i = -cos_i;
    }
    float sin2_t = (1 - cos_i * cos_i) / (etap * etap);
    if (sin2_t >= 1) return false;
    float cos_t = safe_sqrt(1 - sin2_t);
    wi = -wo / etap + n * (cos_i / etap - cos_t);
    return wi.z * wo.z < 0;
}
PT_HD V3 bsdf_eval_pdf(const Bsdf& b, V3 wo, V3 wi, float* pdf_out) {
    V3 f = v3(0);
    float pdf = 0;
    bool same = wo.z * wi.z > 0;
    if (same && wo.z > 0 && (b.w_metal > 0 || b.w_opaque > 0)) {
        V3 h = normalize(wo + wi);
        float D = ggx_d(h, b.alpha), G = ggx_g2(wo, wi, b.alpha);
        float spec = D * G / (4.0f * wo.z * wi.z);
        float pdf_spec = vndf_pdf(wo, h, b.alpha) / (4.0f * dot(wo, h));
        float voh = dot(wo, h);
        if (b.w_metal > 0) {
            f = f + fresnel_schlick(b.base, voh) * (spec * b.w_metal);
            pdf += b.w_metal * pdf_spec;
        }
        if (b.w_opaque > 0) {
            bool matched = b.f0 < 1e-6f;
            float F = matched ? 0.0f : fresnel_dielectric(voh, b.ior);
            float base_layer =
                matched ? kInvPi : (1 - fresnel_dielectric(wo.z, b.ior)) * (1 - fresnel_dielectric(wi.z, b.ior)) * b.diffuse_norm * kInvPi;
            f = f + (v3(F * spec) + b.base * base_layer) * b.w_opaque;
            float ps = opaque_spec_prob(b, wo.z);
            pdf += b.w_opaque * (ps * pdf_spec + (1 - ps) * cosine_hemisphere_pdf(wi.z));
        }
    }
    if (b.w_glass > 0) {
        float pg;
        f = f + glass_eval(b, wo, wi, &pg) * b.w_glass;
        pdf += b.w_glass * pg;
    }
    *pdf_out = pdf;
    return f;
}
PT_HD BsdfSample bsdf_sample(const Bsdf& b, V3 wo, float u_lobe, V2 u, float u_sub) {
    BsdfSample s;
    s.pdf = 0;
    s.valid = false;
    s.transmitted = false;
    s.wi = v3(0);
    s.f = v3(0);
    V3 wi;
    if (u_lobe < b.w_glass) {
        if (!glass_sample(b, wo, u, u_sub, wi)) return s;
    } else {
        if (wo.z <= 0) return s;
        float ul = (u_lobe - b.w_glass) / fmaxf(1 - b.w_glass, 1e-6f);
        bool spec = true;
        if (ul >= b.w_metal / fmaxf(b.w_metal + b.w_opaque, 1e-6f)) spec = u_sub < opaque_spec_prob(b, wo.z);
        if (spec) {
            V3 h = sample_vndf(wo, b.alpha, u);
            wi = reflect(wo, h);
        } else {
            wi = cosine_hemisphere(u);
        }
        if (wi.z <= 0) return s;
    }
    s.wi = wi;
    s.f = bsdf_eval_pdf(b, wo, wi, &s.pdf);
    s.transmitted = wi.z * wo.z < 0;
    s.valid = s.pdf > 0 && is_finite(s.f);
    return s;
}

// ---- lights (lights.h:12-202) ----------------------------------------------------------------------
struct LightSample {
    V3 wi;
    float dist;
    V3 radiance;
    float pdf;
    bool delta;
    int tri;
};
struct LightPick {
    int group, index, bin;
};

PT_HD int sample_alias(const float4* table, int n, float u, float* pmf) {
    float x = u * float(n);
    int i = int(x);
    if (i >= n) i = n - 1;
    float frac = x - float(i);
    float4 e = __ldg(table + i);
    int chosen = frac < e.x ? i : __float_as_int(e.y);
    *pmf = __ldg(table + chosen).z;
    return chosen;
}
// rotate_y (lights.h:34-37) with the angle's cosine and sine given.
PT_HD V3 rotate_y(V3 d, float c, float s) { return {c * d.x + s * d.z, d.y, -s * d.x + c * d.z}; }

PT_HD V3 env_color(const DevScene& s) { return V3{s.env_color_x, s.env_color_y, s.env_color_z} * s.env_intensity; }
PT_HD int env_clamp(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
PT_HD V3 env_radiance(const DevScene& s, V3 dir) {
    if (!s.env_texels) return env_color(s);
    V2 uv = direction_to_equirect(rotate_y(dir, s.env_cos_neg, s.env_sin_neg));
    int x = env_clamp(int(uv.x * float(s.env_width)), s.env_width);
    int y = env_clamp(int(uv.y * float(s.env_height)), s.env_height);
    return xyz(__ldg(s.env_texels + y * s.env_width + x)) * s.env_intensity;
}
PT_HD int find_interval(const float* cdf, int n, float u) {
    int lo = 0, hi = n;
    while (lo + 1 < hi) {
        int mid = (lo + hi) / 2;
        if (__ldg(cdf + mid) <= u) lo = mid;
        else hi = mid;
    }
    return lo;
}
PT_HD float env_pdf_dir(const DevScene& s, V3 dir) {
    if (!s.env_texels) return 1.0f / (4.0f * kPi);
    V3 d = rotate_y(dir, s.env_cos_neg, s.env_sin_neg);
    V2 uv = direction_to_equirect(d);
    float sin_theta = safe_sqrt(1 - d.y * d.y);
    if (sin_theta <= 0 || s.env_integral <= 0) return 0;
    int x = env_clamp(int(uv.x * float(s.env_width)), s.env_width);
    int y = env_clamp(int(uv.y * float(s.env_height)), s.env_height);
    float row_sin = __ldg(s.env_row_sin + y);
    float f = __ldg(s.env_texels + y * s.env_width + x).w * row_sin;
    float pdf_uv = f / s.env_integral;
    return pdf_uv / (2.0f * kPi * kPi * sin_theta);
}
PT_HD bool sample_env(const DevScene& s, V2 u, V3& dir, float& pdf, int* cell) {
    if (!s.env_texels) {
        dir = uniform_sphere(u);
        pdf = 1.0f / (4.0f * kPi);
        return true;
    }
    int w = s.env_width, h = s.env_height;
    int y = find_interval(s.env_marginal, h, u.y);
    float c0 = __ldg(s.env_marginal + y), c1 = __ldg(s.env_marginal + y + 1);
    float dv = c1 > c0 ? (u.y - c0) / (c1 - c0) : 0.5f;
    const float* row = s.env_conditional + y * (w + 1);
    int x = find_interval(row, w, u.x);
    if (cell) *cell = y * w + x;
    float r0 = __ldg(row + x), r1 = __ldg(row + x + 1);
    float du = r1 > r0 ? (u.x - r0) / (r1 - r0) : 0.5f;
    V2 uv{(float(x) + du) / float(w), (float(y) + dv) / float(h)};
    V3 d = equirect_to_direction(uv);
    dir = rotate_y(d, s.env_cos_pos, s.env_sin_pos);
    float sin_theta = safe_sqrt(1 - d.y * d.y);
    if (sin_theta <= 1e-6f) return false;
    float row_sin = __ldg(s.env_row_sin + y);
    float f = __ldg(s.env_texels + y * w + x).w * row_sin;
    pdf = f / s.env_integral / (2.0f * kPi * kPi * sin_theta);
    return pdf > 0;
}

PT_HD V3 load_v3(const float4* p) {
    float4 t = __ldg(p);
    return {t.x, t.y, t.z};
}
// emitted (lights.h:104-113).
PT_HD V3 emitted(const DevScene& s, int tri, int material, float u, float v) {
    const float4* m = s.materials + 5 * material;
    V3 e = load_v3(m + 1);
    int emissive_tex = __float_as_int(__ldg(m + 4).z);
    if (emissive_tex >= 0 && s.uvs) {
        V2 uv = interp_uv(s, __ldg(s.tri_idx + tri), u, v);
        V4 t = sample_texture(s, emissive_tex, uv);
        e = e * V3{t.x, t.y, t.z};
    }
    return e;
}
PT_HD int tri_material(const DevScene& s, int tri) { return __float_as_int(__ldg(s.tris + kTriStride * tri).w); }
PT_HD bool mat_double_sided(const DevScene& s, int material) { return __float_as_int(__ldg(s.materials + 5 * material + 3).z) != 0; }

PT_HD float emissive_pdf(const DevScene& s, int tri, int emissive_entry, V3 dir, float dist) {
    if (s.num_emissive == 0) return 0;
    int k = emissive_entry;
    if (k < 0) return 0;
    int2 e = __ldg(s.emissive + k);
    V3 e1 = load_v3(s.tris + kTriStride * tri + 1), e2 = load_v3(s.tris + kTriStride * tri + 2);
    V3 n = normalize(cross(e1, e2));
    float cos_l = fabsf(dot(n, dir));
    if (cos_l <= 0) return 0;
    return s.p_emissive * __ldg(s.alias + k).z * dist * dist / (__int_as_float(e.y) * cos_l);
}
PT_HD float env_pdf(const DevScene& s, V3 dir) { return s.p_env * env_pdf_dir(s, dir); }

// sample_light (lights.h:139-202); `pick` records the discrete choices.
PT_HD LightSample sample_light(const DevScene& s, V3 p, float u_group, V2 u, float u_light, LightPick* pick) {
    LightSample ls;
    ls.wi = v3(0);
    ls.dist = 0;
    ls.radiance = v3(0);
    ls.pdf = 0;
    ls.delta = false;
    ls.tri = -1;
    if (pick) pick->group = pick->index = pick->bin = -1;
    if (u_group < s.p_emissive && s.num_emissive > 0) {
        float pmf;
        int k = sample_alias(s.alias, s.num_emissive, u_light, &pmf);
        if (pick) {
            int bin = int(u_light * float(s.num_emissive));
            pick->group = 0;
            pick->index = k;
            pick->bin = bin >= s.num_emissive ? s.num_emissive - 1 : bin;
        }
        int2 e = __ldg(s.emissive + k);
        const float4* g = s.tris + kTriStride * e.x;
        float4 g0 = __ldg(g);
        V3 v0 = xyz(g0), e1 = load_v3(g + 1), e2 = load_v3(g + 2);
        V2 b = uniform_triangle(u);
        V3 q = v0 + e1 * b.x + e2 * b.y;
        V3 d = q - p;
        float dist2 = length_sq(d);
        if (dist2 <= 0) return ls;
        float dist = sqrtf(dist2);
        V3 wi = d / dist;
        V3 cr = cross(e1, e2);
        V3 n = normalize(cr);
        float cos_l = fabsf(dot(n, wi));
        int material = __float_as_int(g0.w);
        // emits_towards (lights.h:115-119): double-sided or the front faces -wi.
        if (cos_l <= 1e-8f || !(mat_double_sided(s, material) || dot(cr, -wi) > 0)) return ls;
        ls.wi = wi;
        ls.dist = dist;
        ls.radiance = emitted(s, e.x, material, b.x, b.y);
        ls.pdf = s.p_emissive * pmf * dist2 / (__int_as_float(e.y) * cos_l);
        ls.tri = e.x;
        return ls;
    }
    if (u_group < s.p_emissive + s.p_punctual && s.num_punctual > 0) {
        int k = int(u_light * float(s.num_punctual));
        if (k >= s.num_punctual) k = s.num_punctual - 1;
        if (pick) {
            pick->group = 1;
            pick->index = k;
        }
        float4 l0 = __ldg(s.punctual + 3 * k), l1 = __ldg(s.punctual + 3 * k + 1), l2 = __ldg(s.punctual + 3 * k + 2);
        int type = __float_as_int(l0.w);
        float pk = s.p_punctual / float(s.num_punctual);
        ls.delta = true;
        ls.pdf = pk;
        if (type == 2) {  // directional
            ls.wi = -xyz(l1);
            ls.dist = kInf;
            ls.radiance = xyz(l2);
            return ls;
        }
        V3 d = xyz(l0) - p;
        float dist2 = length_sq(d);
        if (dist2 <= 0) {
            ls.delta = false;
            ls.pdf = 0;
            return ls;
        }
        float dist = sqrtf(dist2);
        ls.wi = d / dist;
        ls.dist = dist;
        V3 li = xyz(l2) / dist2;
        if (type == 1) {  // spot
            float cd = dot(-ls.wi, xyz(l1));
            float t = saturate((cd - l2.w) / fmaxf(l1.w - l2.w, 1e-4f));
            li = li * (t * t);
        }
        ls.radiance = li;
        return ls;
    }
    if (s.p_env > 0) {
        if (pick) pick->group = 2;
        V3 dir;
        float pdf;
        int cell = -1;
        bool ok = sample_env(s, u, dir, pdf, &cell);
        if (pick && s.env_texels) pick->index = cell;
        if (!ok) return ls;
        ls.wi = dir;
        ls.dist = kInf;
        ls.radiance = env_radiance(s, dir);
        ls.pdf = s.p_env * pdf;
    }
    return ls;
}

// ---- surface interaction (integrator.h:71-148) ------------------------------------------------------
struct Interaction {
    V3 p, ng, ns;
    Frame frame;
    BsdfParams params;
    V3 emission;
    bool front;
    int material;
    int emissive_entry;
};

PT_HD V3 load_normal(const DevScene& s, int v) { return load_v3(s.normals + v); }

PT_HD Interaction surface_at(const DevScene& s, V3 ro, V3 rd, float t, int tri, float hu, float hv) {
    Interaction it;
    const float4* g = s.tris + kTriStride * tri;
    float4 g0 = __ldg(g);
    V3 e1 = load_v3(g + 1), e2 = load_v3(g + 2);
    int material = __float_as_int(g0.w);
    const float4* m = s.materials + 5 * material;
    float4 m0 = __ldg(m), m1 = __ldg(m + 1), m2 = __ldg(m + 2), m3 = __ldg(m + 3), m4 = __ldg(m + 4);
    it.material = material;
    float w = 1 - hu - hv;
    it.p = ro + rd * t;
    V3 ng = normalize(cross(e1, e2));
    int4 idx = __ldg(s.tri_idx + tri);
    it.emissive_entry = idx.w;
    V3 ns = ng;
    if (s.normals) {
        V3 n = load_normal(s, idx.x) * w + load_normal(s, idx.y) * hu + load_normal(s, idx.z) * hv;
        if (length_sq(n) > 1e-12f) ns = normalize(n);
        if (dot(ns, ng) < 0) ns = -ns;
    }
    V2 uv = s.uvs ? load_uv(s, idx.x) * w + load_uv(s, idx.y) * hu + load_uv(s, idx.z) * hv : V2{0, 0};
    it.front = dot(rd, ng) < 0;
    int base_tex = __float_as_int(m3.w), mr_tex = __float_as_int(m4.x), normal_tex = __float_as_int(m4.y);
    if (normal_tex >= 0 && s.tangents) {
        float4 ta = __ldg(s.tangents + idx.x), tb = __ldg(s.tangents + idx.y), tc = __ldg(s.tangents + idx.z);
        V4 t4 = V4{ta.x, ta.y, ta.z, ta.w} * w + V4{tb.x, tb.y, tb.z, tb.w} * hu + V4{tc.x, tc.y, tc.z, tc.w} * hv;
        V3 tt = xyz(t4);
        if (length_sq(tt) > 1e-12f) {
            tt = normalize(tt - ns * dot(ns, tt));
            V3 b = cross(ns, tt) * (ta.w < 0 ? -1.0f : 1.0f);
            V4 tn = sample_texture(s, normal_tex, uv);
            V3 nt{tn.x * 2 - 1, tn.y * 2 - 1, tn.z * 2 - 1};
            nt.x *= m2.w;
            nt.y *= m2.w;
            V3 n = normalize(tt * nt.x + b * nt.y + ns * nt.z);
            if (dot(n, ng) > 0.01f) ns = n;
        }
    }
    V4 base{m0.x, m0.y, m0.z, m0.w};
    if (base_tex >= 0) {
        V4 tcol = sample_texture(s, base_tex, uv);
        base = V4{base.x * tcol.x, base.y * tcol.y, base.z * tcol.z, base.w * tcol.w};
    }
    float metallic = m1.w, roughness = m2.x;
    if (mr_tex >= 0) {
        V4 mr = sample_texture(s, mr_tex, uv);
        roughness *= mr.y;
        metallic *= mr.z;
    }
    it.params.base = xyz(base);
    it.params.metallic = metallic;
    it.params.roughness = roughness;
    it.params.transmission = m2.z;
    it.params.ior = m2.y;
    bool double_sided = __float_as_int(m3.z) != 0;
    if (it.front || double_sided) {
        V3 e = xyz(m1);
        int emissive_tex = __float_as_int(m4.z);
        if (emissive_tex >= 0 && s.uvs) {
            V4 te = sample_texture(s, emissive_tex, uv);
            e = e * V3{te.x, te.y, te.z};
        }
        it.emission = e;
    } else {
        it.emission = v3(0);
    }
    if (m2.z <= 0 && !it.front) {
        ng = -ng;
        ns = -ns;
    }
    V3 wo = -rd;
    if (m2.z <= 0 && dot(wo, ns) <= 0) ns = ng;
    it.ng = ng;
    it.ns = ns;
    it.frame = make_frame(ns);
    return it;
}

}  // namespace ptw
