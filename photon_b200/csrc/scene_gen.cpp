// Procedural scenes of the benchmark configurations (seeded, deterministic).
//
//  PT_GEN_BOX      a closed box (5 walls of 2 triangles: grey 0.73, left red, right green), two
//                  boxes rotated about y (12 triangles each, grey 0.73), a ceiling emitter
//                  (2 triangles, radiance (17, 12, 4)); 36 triangles; pinhole camera, 40 deg fov.
//  PT_GEN_TERRAIN  a value-noise height field 512 cells wide (amplitude 0.1 of the extent), 200
//                  instanced spheres / cylinders with random rotation and scale (10% mirrored,
//                  winding flipped), 64 materials (30% metal, 15% glass with IOR 1.5, roughness
//                  U(0,1), base colour U(0.05,0.95)^3, 25% alpha-masked by a 256x256 checker), 64
//                  emissive triangles with log-uniform power over three decades, two point and two
//                  spot lights, and a 1024x512 HDR sky (gradient + three Gaussian lobes, peak 1e3).
//                  The triangle count is exact: the height field takes whatever the shapes and
//                  emitters leave (rows of 512 cells plus one partial row).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "pt_error.h"
#include "scene_build.h"

namespace ptw {

namespace {

constexpr float kPiG = 3.14159265358979323846f;

struct G3 {
    float x, y, z;
};
inline G3 g3(float x, float y, float z) { return {x, y, z}; }
inline G3 operator+(G3 a, G3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline G3 operator-(G3 a, G3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline G3 operator*(G3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float gdot(G3 a, G3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline G3 gcross(G3 a, G3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline G3 gnorm(G3 a) {
    float l = std::sqrt(gdot(a, a));
    return l > 0 ? a * (1.0f / l) : g3(0, 1, 0);
}
inline pt_vec3 P(G3 a) { return {a.x, a.y, a.z}; }

// splitmix64: a small seeded generator for scene construction only.
struct SceneRng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    }
    float uniform() { return float(next() >> 40) * (1.0f / 16777216.0f); }
    float range(float a, float b) { return a + (b - a) * uniform(); }
};

pt_material lambert(float r, float g, float b) {
    pt_material m{};
    m.base_color = {r, g, b, 1};
    m.metallic = 0;
    m.roughness = 1;
    m.ior = 1.5f;
    m.normal_scale = 1;
    m.alpha_cutoff = 0.5f;
    m.base_color_tex = m.metallic_roughness_tex = m.normal_tex = m.emissive_tex = m.occlusion_tex = -1;
    return m;
}

struct MeshOut {
    GeneratedScene& g;
    int add_vertex(G3 p, G3 n, float u, float v) {
        g.positions.push_back(P(p));
        g.normals.push_back(P(n));
        g.uvs.push_back({u, v});
        return int(g.positions.size()) - 1;
    }
    void tri(int a, int b, int c, int material) {
        g.indices.insert(g.indices.end(), {a, b, c});
        g.tri_material.push_back(material);
    }
    // A planar quad corner, corner + eu, corner + eu + ev, corner + ev (front face along eu x ev).
    void quad(G3 corner, G3 eu, G3 ev, int material) {
        G3 n = gnorm(gcross(eu, ev));
        int a = add_vertex(corner, n, 0, 0), b = add_vertex(corner + eu, n, 1, 0), c = add_vertex(corner + eu + ev, n, 1, 1),
            d = add_vertex(corner + ev, n, 0, 1);
        tri(a, b, c, material);
        tri(a, c, d, material);
    }
};

// An axis-aligned box of half extents h rotated by `angle` about y, outward faces.
void rotated_box(MeshOut& m, G3 center, G3 h, float angle, int material) {
    float c = std::cos(angle), s = std::sin(angle);
    auto rot = [&](G3 p) { return g3(c * p.x - s * p.z, p.y, s * p.x + c * p.z); };
    // For each axis a and sign, the face spans the other two axes in right-handed order.
    for (int a = 0; a < 3; a++)
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            float hv[3] = {h.x, h.y, h.z};
            int u = (a + 1) % 3, v = (a + 2) % 3;
            float base[3] = {0, 0, 0}, du[3] = {0, 0, 0}, dv[3] = {0, 0, 0};
            base[a] = float(sgn) * hv[a];
            base[u] = -hv[u];
            base[v] = -hv[v];
            du[u] = 2 * hv[u];
            dv[v] = 2 * hv[v];
            G3 corner = g3(base[0], base[1], base[2]), eu = g3(du[0], du[1], du[2]), ev = g3(dv[0], dv[1], dv[2]);
            if (sgn < 0) std::swap(eu, ev);  // keep the face normal pointing outward
            m.quad(center + rot(corner), rot(eu), rot(ev), material);
        }
}

void make_box_scene(GeneratedScene& g) {
    MeshOut m{g};
    int grey = int(g.materials.size());
    g.materials.push_back(lambert(0.73f, 0.73f, 0.73f));
    int red = int(g.materials.size());
    g.materials.push_back(lambert(0.63f, 0.065f, 0.05f));
    int green = int(g.materials.size());
    g.materials.push_back(lambert(0.14f, 0.45f, 0.09f));
    int lamp = int(g.materials.size());
    pt_material lm = lambert(0.78f, 0.78f, 0.78f);
    lm.emission = {17.0f, 12.0f, 4.0f};
    g.materials.push_back(lm);
    const float S = 5.5f;
    // Floor (up), ceiling (down), back wall (towards the camera at -z), and the side walls. The
    // camera looks along +z, so screen-left is +x: the red wall is at x = S.
    m.quad(g3(0, 0, 0), g3(0, 0, S), g3(S, 0, 0), grey);
    m.quad(g3(0, S, 0), g3(S, 0, 0), g3(0, 0, S), grey);
    m.quad(g3(0, 0, S), g3(0, S, 0), g3(S, 0, 0), grey);
    m.quad(g3(S, 0, 0), g3(0, 0, S), g3(0, S, 0), red);
    m.quad(g3(0, 0, S), g3(0, 0, -S), g3(0, S, 0), green);
    // The emitter just below the ceiling, facing down.
    m.quad(g3(2.13f, S - 0.01f, 2.27f), g3(1.3f, 0, 0), g3(0, 0, 1.05f), lamp);
    rotated_box(m, g3(1.85f, 0.825f, 1.69f), g3(0.825f, 0.825f, 0.825f), -0.29f, grey);
    rotated_box(m, g3(3.68f, 1.65f, 3.51f), g3(0.825f, 1.65f, 0.825f), 0.29f, grey);
    g.cam_pos = {2.78f, 2.73f, -8.0f};
    g.cam_target = {2.78f, 2.73f, 0.0f};
    g.vfov_deg = 40.0f;
}

// ---- the terrain scene --------------------------------------------------------------------------------

float lattice(uint64_t seed, int ix, int iz) {
    uint64_t h = seed ^ (uint64_t(uint32_t(ix)) * 0x9E3779B185EBCA87ULL) ^ (uint64_t(uint32_t(iz)) * 0xC2B2AE3D27D4EB4FULL);
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdULL;
    h ^= h >> 33;
    h *= 0xc4ceb9fe1a85ec53ULL;
    h ^= h >> 33;
    return float(h >> 40) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
}

// Smooth value noise, four octaves, in [-1, 1].
float value_noise(uint64_t seed, float x, float z) {
    float sum = 0, amp = 0.5f, norm = 0;
    for (int o = 0; o < 4; o++) {
        float fx = std::floor(x), fz = std::floor(z);
        int ix = int(fx), iz = int(fz);
        float tx = x - fx, tz = z - fz;
        tx = tx * tx * (3 - 2 * tx);
        tz = tz * tz * (3 - 2 * tz);
        uint64_t s = seed + uint64_t(o) * 0x632BE59BD9B4E019ULL;
        float a = lattice(s, ix, iz), b = lattice(s, ix + 1, iz), c = lattice(s, ix, iz + 1), d = lattice(s, ix + 1, iz + 1);
        float top = a + (b - a) * tx, bot = c + (d - c) * tx;
        sum += amp * (top + (bot - top) * tz);
        norm += amp;
        amp *= 0.5f;
        x *= 2.0f;
        z *= 2.0f;
    }
    return sum / norm;
}

struct Terrain {
    uint64_t seed;
    float x0, z0, cell, amplitude, freq;
    float height(float x, float z) const { return amplitude * value_noise(seed, (x - x0) * freq, (z - z0) * freq); }
};

// Rotation matrix from a random unit quaternion.
void random_rotation(SceneRng& r, float m[9]) {
    float u1 = r.uniform(), u2 = r.uniform(), u3 = r.uniform();
    float a = std::sqrt(1 - u1), b = std::sqrt(u1);
    float qx = a * std::sin(2 * kPiG * u2), qy = a * std::cos(2 * kPiG * u2), qz = b * std::sin(2 * kPiG * u3), qw = b * std::cos(2 * kPiG * u3);
    m[0] = 1 - 2 * (qy * qy + qz * qz);
    m[1] = 2 * (qx * qy - qz * qw);
    m[2] = 2 * (qx * qz + qy * qw);
    m[3] = 2 * (qx * qy + qz * qw);
    m[4] = 1 - 2 * (qx * qx + qz * qz);
    m[5] = 2 * (qy * qz - qx * qw);
    m[6] = 2 * (qx * qz - qy * qw);
    m[7] = 2 * (qy * qz + qx * qw);
    m[8] = 1 - 2 * (qx * qx + qy * qy);
}

// An instance transform: p' = R (S p) + t; normals n' = R (S^-1 n), normalised.
struct Instance {
    float R[9];
    G3 scale, t;
    bool mirrored;
    G3 point(G3 p) const {
        G3 q{p.x * scale.x, p.y * scale.y, p.z * scale.z};
        return g3(R[0] * q.x + R[1] * q.y + R[2] * q.z, R[3] * q.x + R[4] * q.y + R[5] * q.z, R[6] * q.x + R[7] * q.y + R[8] * q.z) + t;
    }
    G3 normal(G3 n) const {
        G3 q{n.x / scale.x, n.y / scale.y, n.z / scale.z};
        return gnorm(g3(R[0] * q.x + R[1] * q.y + R[2] * q.z, R[3] * q.x + R[4] * q.y + R[5] * q.z, R[6] * q.x + R[7] * q.y + R[8] * q.z));
    }
};

void emit_instance_tri(MeshOut& m, const Instance& in, int a, int b, int c, int material) {
    // A mirrored instance flips orientation: swap two vertices so the winding (and the geometric
    // normal cross(e1, e2)) still faces outward.
    if (in.mirrored) m.tri(a, c, b, material);
    else m.tri(a, b, c, material);
}

// UV sphere: `seg` segments, `rings` rings, poles as single triangles: 2 * seg * (rings - 1) tris.
void sphere(MeshOut& m, const Instance& in, int seg, int rings, int material) {
    int base = int(m.g.positions.size());
    for (int r = 0; r <= rings; r++) {
        float th = kPiG * float(r) / float(rings);
        for (int s = 0; s <= seg; s++) {
            float ph = 2 * kPiG * float(s) / float(seg);
            G3 n = g3(std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph));
            m.add_vertex(in.point(n), in.normal(n), float(s) / float(seg), float(r) / float(rings));
        }
    }
    int row = seg + 1;
    for (int r = 0; r < rings; r++)
        for (int s = 0; s < seg; s++) {
            int a = base + r * row + s, b = a + row;
            if (r > 0) emit_instance_tri(m, in, a, a + 1, b, material);
            if (r < rings - 1) emit_instance_tri(m, in, a + 1, b + 1, b, material);
        }
}

// Capped cylinder of radius 1 and height 2 around y: 2n side triangles + 2 (n - 2) cap triangles.
void cylinder(MeshOut& m, const Instance& in, int n, int material) {
    int side = int(m.g.positions.size());
    for (int k = 0; k <= n; k++) {
        float ph = 2 * kPiG * float(k) / float(n);
        G3 d = g3(std::cos(ph), 0, std::sin(ph));
        for (int e = 0; e < 2; e++) m.add_vertex(in.point(g3(d.x, e ? 1.0f : -1.0f, d.z)), in.normal(d), float(k) / float(n), float(e));
    }
    for (int k = 0; k < n; k++) {
        int a = side + 2 * k, b = a + 2;  // bottom vertices; +1 is the top one
        emit_instance_tri(m, in, a, a + 1, b, material);
        emit_instance_tri(m, in, b, a + 1, b + 1, material);
    }
    for (int e = 0; e < 2; e++) {
        int cap = int(m.g.positions.size());
        float y = e ? 1.0f : -1.0f;
        G3 nn = g3(0, y, 0);
        for (int k = 0; k < n; k++) {
            float ph = 2 * kPiG * float(k) / float(n);
            m.add_vertex(in.point(g3(std::cos(ph), y, std::sin(ph))), in.normal(nn), 0.5f + 0.5f * std::cos(ph), 0.5f + 0.5f * std::sin(ph));
        }
        for (int k = 1; k + 1 < n; k++) {
            if (e) emit_instance_tri(m, in, cap, cap + k + 1, cap + k, material);
            else emit_instance_tri(m, in, cap, cap + k, cap + k + 1, material);
        }
    }
}

constexpr int kSphereSeg = 16, kSphereRings = 8, kCylSeg = 26;
constexpr int kSphereTris = 2 * kSphereSeg * (kSphereRings - 1);  // 224
constexpr int kCylTris = 4 * kCylSeg - 4;                          // 100
constexpr int kShapes = 200, kEmitters = 64, kMaterials = 64;

void make_terrain_scene(GeneratedScene& g, int64_t triangles, uint64_t seed) {
    const int64_t shape_tris = int64_t(kShapes / 2) * kSphereTris + int64_t(kShapes / 2) * kCylTris;
    const int64_t hf_tris = triangles - shape_tris - kEmitters;
    int cols = 512 * std::max<int>(1, int(std::lround(std::sqrt(double(triangles) / 262144.0))));
    if (hf_tris < 4LL * cols || hf_tris % 2) throw Error{PT_ERR_INVALID, "terrain scene: the triangle count is too small (or odd)"};
    if (triangles > (int64_t(1) << 30)) throw Error{PT_ERR_INVALID, "terrain scene: too many triangles"};
    const int64_t cells = hf_tris / 2;
    const int rows = int(cells / cols), partial = int(cells % cols);
    SceneRng rng{seed * 0x2545F4914F6CDD1DULL + 0x1234567ULL};
    MeshOut m{g};

    // Materials: 64 slots.
    for (int k = 0; k < kMaterials; k++) {
        pt_material mat = lambert(rng.range(0.05f, 0.95f), rng.range(0.05f, 0.95f), rng.range(0.05f, 0.95f));
        mat.metallic = rng.uniform() < 0.3f ? 1.0f : 0.0f;
        mat.roughness = rng.uniform();
        if (rng.uniform() < 0.15f) {
            mat.transmission = 1.0f;
            mat.ior = 1.5f;
        }
        if (rng.uniform() < 0.25f) {
            mat.alpha_mode = PT_ALPHA_MASK;
            mat.base_color_tex = 0;
            mat.double_sided = 1;
        }
        g.materials.push_back(mat);
    }
    // The checker: white RGB, alpha 0 / 255 in 32-texel squares.
    {
        std::vector<uint32_t> tex(256 * 256);
        for (int y = 0; y < 256; y++)
            for (int x = 0; x < 256; x++) tex[size_t(y) * 256 + size_t(x)] = 0x00FFFFFFu | ((((x >> 5) + (y >> 5)) & 1) ? 0xFF000000u : 0u);
        g.texture_data.push_back(std::move(tex));
        g.textures.push_back({256, 256, nullptr, 1, 1});
    }

    // Height field over x in [-10, 10].
    const float extent = 20.0f;
    Terrain tr{seed ^ 0xA5A5A5A5ULL, -10.0f, 0.0f, extent / float(cols), 0.1f * extent, 4.0f / extent};
    const int vrows = rows + (partial ? 2 : 1);
    const float depth = float(vrows - 1) * tr.cell;
    tr.z0 = -0.5f * depth;
    const int vbase = int(g.positions.size());
    for (int r = 0; r < vrows; r++)
        for (int c = 0; c <= cols; c++) {
            float x = tr.x0 + float(c) * tr.cell, z = tr.z0 + float(r) * tr.cell;
            float e = 0.5f * tr.cell;
            G3 n = gnorm(g3(tr.height(x - e, z) - tr.height(x + e, z), 2 * e, tr.height(x, z - e) - tr.height(x, z + e)));
            m.add_vertex(g3(x, tr.height(x, z), z), n, float(c) / 8.0f, float(r) / 8.0f);
        }
    // Patch materials (32 x 32 cells), drawn from the non-transmissive slots.
    std::vector<int> solid;
    for (int k = 0; k < kMaterials; k++)
        if (g.materials[size_t(k)].transmission <= 0) solid.push_back(k);
    if (solid.empty()) solid.push_back(0);
    const int pcols = (cols + 31) / 32, prows = (vrows + 31) / 32;
    std::vector<int> patch(size_t(pcols) * size_t(prows));
    for (int& p : patch) p = solid[size_t(rng.next() % solid.size())];
    auto cell_tris = [&](int r, int c) {
        int a = vbase + r * (cols + 1) + c, b = a + 1, d = a + (cols + 1), e = d + 1;
        int mat = patch[size_t(r / 32) * size_t(pcols) + size_t(c / 32)];
        // Up-facing winding: cross(e1, e2) points +y.
        m.tri(a, d, b, mat);
        m.tri(b, d, e, mat);
    };
    for (int r = 0; r < rows; r++)
        for (int c = 0; c < cols; c++) cell_tris(r, c);
    for (int c = 0; c < partial; c++) cell_tris(rows, c);

    // Shapes: half spheres, half cylinders, on the terrain.
    const float zmin = tr.z0, zmax = tr.z0 + depth;
    for (int k = 0; k < kShapes; k++) {
        Instance in;
        random_rotation(rng, in.R);
        float s = rng.range(0.2f, 0.6f);
        in.scale = g3(s, s * rng.range(0.7f, 1.4f), s);
        in.mirrored = rng.uniform() < 0.1f;
        if (in.mirrored) in.scale.x = -in.scale.x;
        float x = rng.range(-9.0f, 9.0f), z = rng.range(zmin + 0.5f, zmax - 0.5f);
        in.t = g3(x, tr.height(x, z) + 0.5f * s, z);
        int mat = int(rng.next() % kMaterials);
        if (k % 2 == 0) sphere(m, in, kSphereSeg, kSphereRings, mat);
        else cylinder(m, in, kCylSeg, mat);
    }

    // Emitters: 64 small downward-facing triangles, each with its own material; power log-uniform
    // over three decades.
    for (int k = 0; k < kEmitters; k++) {
        float x = rng.range(-9.5f, 9.5f), z = rng.range(zmin, zmax);
        float y = tr.height(x, z) + rng.range(1.5f, 3.0f);
        float a = rng.range(0.0f, 2 * kPiG), r = rng.range(0.15f, 0.3f);
        pt_material em = lambert(0.8f, 0.8f, 0.8f);
        float power = 0.5f * std::pow(10.0f, rng.range(0.0f, 3.0f));
        float tint = rng.uniform();
        em.emission = {power * (0.9f + 0.1f * tint), power * 0.85f, power * (0.6f + 0.4f * (1 - tint))};
        int mat = int(g.materials.size());
        g.materials.push_back(em);
        G3 c = g3(x, y, z);
        G3 p0 = c + g3(r * std::cos(a), 0, r * std::sin(a));
        G3 p1 = c + g3(r * std::cos(a + 2.0944f), 0, r * std::sin(a + 2.0944f));
        G3 p2 = c + g3(r * std::cos(a + 4.1888f), 0, r * std::sin(a + 4.1888f));
        G3 n = gnorm(gcross(p1 - p0, p2 - p0));
        int i0 = m.add_vertex(p0, n, 0, 0), i1 = m.add_vertex(p1, n, 1, 0), i2 = m.add_vertex(p2, n, 0, 1);
        if (n.y > 0) m.tri(i0, i2, i1, mat);  // face down
        else m.tri(i0, i1, i2, mat);
        if (n.y > 0) {
            G3 fn = n * -1.0f;
            g.normals[size_t(i0)] = P(fn);
            g.normals[size_t(i1)] = P(fn);
            g.normals[size_t(i2)] = P(fn);
        }
    }

    // Two point lights and two spot lights above the terrain.
    for (int k = 0; k < 4; k++) {
        pt_punctual_light l{};
        float x = rng.range(-8.0f, 8.0f), z = rng.range(zmin, zmax);
        l.position = {x, tr.height(x, z) + rng.range(2.0f, 4.0f), z};
        float i = rng.range(20.0f, 120.0f);
        l.intensity = {i, i * 0.9f, i * 0.75f};
        l.direction = {0, -1, 0};
        if (k < 2) {
            l.type = PT_LIGHT_POINT;
            l.cos_inner = 1;
            l.cos_outer = 0;
        } else {
            l.type = PT_LIGHT_SPOT;
            l.cos_inner = std::cos(20.0f * kPiG / 180.0f);
            l.cos_outer = std::cos(35.0f * kPiG / 180.0f);
        }
        g.punctual.push_back(l);
    }

    // The sky: gradient, ground, and three Gaussian lobes (peaks 1000, 300, 100).
    const int ew = 1024, eh = 512;
    g.env_w = ew;
    g.env_h = eh;
    g.env.resize(size_t(ew) * size_t(eh));
    G3 lobe_dir[3];
    float lobe_peak[3] = {1000.0f, 300.0f, 100.0f}, lobe_sigma[3] = {1.5f, 4.0f, 10.0f};
    for (int k = 0; k < 3; k++) {
        float el = rng.range(0.25f, 1.1f), az = rng.range(0.0f, 2 * kPiG);
        lobe_dir[k] = g3(std::cos(el) * std::sin(az), std::sin(el), -std::cos(el) * std::cos(az));
    }
    for (int y = 0; y < eh; y++)
        for (int x = 0; x < ew; x++) {
            float u = (float(x) + 0.5f) / float(ew), v = (float(y) + 0.5f) / float(eh);
            float phi = (u - 0.5f) * 2 * kPiG, theta = v * kPiG;
            G3 d = g3(std::sin(theta) * std::sin(phi), std::cos(theta), -std::sin(theta) * std::cos(phi));
            G3 c;
            if (d.y >= 0) {
                float t = std::pow(d.y, 0.5f);
                c = g3(0.75f, 0.8f, 0.9f) * (1 - t) + g3(0.2f, 0.35f, 0.8f) * t;
            } else {
                c = g3(0.16f, 0.14f, 0.12f) * (0.6f + 0.4f * std::exp(6.0f * d.y));
            }
            for (int k = 0; k < 3; k++) {
                float cosang = std::fmin(1.0f, std::fmax(-1.0f, gdot(d, lobe_dir[k])));
                float ang = std::acos(cosang) * 180.0f / kPiG;
                float w = lobe_peak[k] * std::exp(-0.5f * (ang / lobe_sigma[k]) * (ang / lobe_sigma[k]));
                c = c + g3(1.0f, 0.95f, 0.85f) * w;
            }
            g.env[size_t(y) * size_t(ew) + size_t(x)] = P(c);
        }
    g.env_intensity = 1.0f;
    g.cam_pos = {0.0f, 4.5f, zmin - 6.0f};
    g.cam_target = {0.0f, 0.0f, 0.5f * (zmin + zmax)};
    g.vfov_deg = 45.0f;
}

}  // namespace

pt_camera GeneratedScene::camera_view(float aspect) const {
    // A look-at camera (the convention of Camera::view, scene.cpp:13-25).
    G3 pos = g3(cam_pos.x, cam_pos.y, cam_pos.z), tgt = g3(cam_target.x, cam_target.y, cam_target.z), up = g3(cam_up.x, cam_up.y, cam_up.z);
    G3 dir = tgt - pos;
    float l2 = gdot(dir, dir);
    G3 fwd = l2 > 0 ? dir * (1.0f / std::sqrt(l2)) : g3(0, 0, 1);
    G3 rc = gcross(fwd, up);
    float r2 = gdot(rc, rc);
    G3 right = r2 > 0 ? rc * (1.0f / std::sqrt(r2)) : g3(0, 0, 1);
    if (gdot(right, right) < 1e-12f || r2 < 1e-12f) right = g3(1, 0, 0);
    G3 u = gcross(right, fwd);
    pt_camera c{};
    c.position = P(pos);
    c.forward = P(fwd);
    c.right = P(right);
    c.up = P(u);
    c.tan_half_fov = std::tan(vfov_deg * 0.5f * kPiG / 180.0f);
    c.aspect = aspect;
    c.aperture = 0;
    c.focus_distance = std::sqrt(l2);
    return c;
}

void GeneratedScene::finalize() {
    for (size_t k = 0; k < textures.size(); k++) textures[k].texels = texture_data[k].data();
    raw = pt_raw_scene{};
    raw.positions = positions.data();
    raw.num_positions = int32_t(positions.size());
    raw.normals = normals.empty() ? nullptr : normals.data();
    raw.uvs = uvs.empty() ? nullptr : uvs.data();
    raw.tangents = nullptr;
    raw.indices = indices.data();
    raw.num_indices = int32_t(indices.size());
    raw.tri_material = tri_material.data();
    raw.materials = materials.data();
    raw.num_materials = int32_t(materials.size());
    raw.textures = textures.empty() ? nullptr : textures.data();
    raw.num_textures = int32_t(textures.size());
    raw.punctual = punctual.empty() ? nullptr : punctual.data();
    raw.num_punctual = int32_t(punctual.size());
    raw.env_texels = env.empty() ? nullptr : env.data();
    raw.env_width = env_w;
    raw.env_height = env_h;
    raw.env_color = env_color;
    raw.env_intensity = env_intensity;
    raw.env_rotation = 0;
}

void generate_scene(int kind, int64_t triangles, uint64_t seed, GeneratedScene& out) {
    out = GeneratedScene();
    if (kind == PT_GEN_BOX) make_box_scene(out);
    else if (kind == PT_GEN_TERRAIN) make_terrain_scene(out, triangles, seed);
    else throw Error{PT_ERR_INVALID, "unknown scene kind"};
    out.finalize();
}

}  // namespace ptw
