// The denoiser's per-pixel records, written by the path tracer's first vertex and by the adapter from
// Photon's SvgfInput layout (src/denoise/svgf.h:24-30).
//   edge   float4: octahedral normal (x, y), depth (hit distance), material id (int32 bits; -1: none)
//   motion float4: offset to the pixel's position in the previous frame (dx, dy), the point's
//                  distance from the previous camera, 1 when it projects into the previous frame
#pragma once

#include "pt_math.cuh"

namespace ptw {

struct PrevCamera {
    float c[16];  // pt_camera
};

PT_HD float sign_nz(float v) { return v < 0.0f ? -1.0f : 1.0f; }

// Octahedral normal encoding (Meyer et al. 2010; Cigolle et al. 2014), FP32.
PT_HD float2 oct_encode(V3 n) {
    float s = fabsf(n.x) + fabsf(n.y) + fabsf(n.z);
    if (!(s > 0.0f)) return make_float2(0.0f, 0.0f);
    float px = n.x / s, py = n.y / s;
    if (n.z < 0.0f) {
        float qx = (1.0f - fabsf(py)) * sign_nz(px), qy = (1.0f - fabsf(px)) * sign_nz(py);
        px = qx;
        py = qy;
    }
    return make_float2(px, py);
}

// project (svgf.cu:25-35): a world position in the previous frame's pixel coordinates.
PT_HD bool project(const PrevCamera& pc, V3 p, int w, int h, float& px, float& py, float& dist) {
    const float* c = pc.c;
    V3 d = p - V3{c[0], c[1], c[2]};
    float z = dot(d, V3{c[4], c[5], c[6]});
    if (z <= 1e-4f) return false;
    float sx = dot(d, V3{c[8], c[9], c[10]}) / (z * c[3] * c[7]);
    float sy = dot(d, V3{c[12], c[13], c[14]}) / (z * c[3]);
    px = (sx + 1.0f) * 0.5f * float(w) - 0.5f;
    py = (1.0f - sy) * 0.5f * float(h) - 0.5f;
    dist = length(d);
    return true;
}

// The edge and motion records of pixel (x, y) whose first hit is p (material >= 0) with shading
// normal n at distance t; a miss passes material -1.
PT_HD float4 edge_record(V3 n, float t, int material) {
    float2 o = oct_encode(n);
    return make_float4(o.x, o.y, t, __int_as_float(material));
}
PT_HD float4 motion_record(const PrevCamera& prev, bool has_prev, V3 p, int material, int x, int y, int w, int h) {
    float px, py, dist;
    if (!has_prev || material < 0 || !project(prev, p, w, h, px, py, dist)) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return make_float4(px - float(x), py - float(y), dist, 1.0f);
}

}  // namespace ptw
