// Seeded procedural scenes (the synthetic inputs of the benchmark configurations).
//
// Stands in for keepsake's mesh-asset loading (mesh_asset.cpp) with generated geometry:
//   "box_room"   5 axis-aligned wall quads + 2 boxes rotated about y by U[0,90) deg + a 2-triangle
//                area light of radiance (17,12,4); diffuse principled materials, basecolor
//                U[0.1,0.9]^3.
//   "icosphere"  icosphere subdivided `level` times (20*4^level triangles; or, given a frequency f,
//                a geodesic sphere of 20 f^2 triangles) with seeded fBm radial
//                displacement (amplitude 0.05) on a ground quad; one principled material per
//                1024-triangle patch (roughness U[r0,r1], metallic Bernoulli(0.3), basecolor
//                U[0,1]^3); a procedural lat-long HDR sky (gradient + sun lobe of 1e4).
//                options.occluder adds an opaque slab between the sphere and the sun.
//   "instanced"  `prototypes` geodesic spheres of frequency f (20 f^2 triangles each, f = 50 gives
//                50,000) with seeded fBm radial displacement (amplitude 0.05), one principled
//                material each; `instances` instances under random affine transforms (rotation,
//                anisotropic scale U[0.12,0.4], translation over a 16x16 field); `emitters`
//                emissive triangles above the field with radiance log-uniform over 3 decades
//                (one prototype, one identity instance); a ground quad; the sky of "icosphere".
// All randomness comes from a SplitMix64 stream seeded by the caller.
#include "procedural.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>

namespace ksb
{
namespace
{

struct SplitMix
{
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
    uint64_t next()
    {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * 0x1.0p-53; }
    float uniform(float a, float b) { return (float)(a + (b - a) * uniform()); }
};

struct V3
{
    double x, y, z;
};
V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 operator*(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 norm(V3 a)
{
    double n = std::sqrt(dot(a, a));
    return {a.x / n, a.y / n, a.z / n};
}

ks_material_desc default_material()
{
    ks_material_desc m{};
    m.basecolor[0] = m.basecolor[1] = m.basecolor[2] = 0.8f;
    m.roughness = 1.0f;
    m.metallic = 0.0f;
    m.ior = 1.5f;
    m.specular_r0_mul = 0.5f; // remapped x2 by the closure (principled_bsdf.cpp:258)
    m.specular_trans = 0.0f;
    m.diffuse_trans = 0.0f;
    m.diffuse_trans_fwd = 0.5f;
    m.microfacet = 0;
    m.has_emission = 0;
    return m;
}

// Adds a planar quad p0,p1,p2,p3 (counter-clockwise seen from the front) as one mesh.
void add_quad(GeneratedScene &g, V3 p0, V3 p1, V3 p2, V3 p3, uint32_t material)
{
    GeneratedMesh m;
    for (V3 p : {p0, p1, p2, p3}) {
        m.vertices.push_back((float)p.x);
        m.vertices.push_back((float)p.y);
        m.vertices.push_back((float)p.z);
    }
    m.indices = {0, 1, 2, 0, 2, 3};
    m.material = material;
    g.meshes.push_back(std::move(m));
}

void add_box(GeneratedScene &g, V3 center, V3 half, double angle_rad, uint32_t material)
{
    GeneratedMesh m;
    double c = std::cos(angle_rad), s = std::sin(angle_rad);
    for (int k = 0; k < 8; ++k) {
        double lx = (k & 1) ? half.x : -half.x;
        double ly = (k & 2) ? half.y : -half.y;
        double lz = (k & 4) ? half.z : -half.z;
        double wx = c * lx + s * lz, wz = -s * lx + c * lz;
        m.vertices.push_back((float)(center.x + wx));
        m.vertices.push_back((float)(center.y + ly));
        m.vertices.push_back((float)(center.z + wz));
    }
    // 6 faces x 2 triangles, outward winding
    const uint32_t f[12][3] = {{0, 2, 3}, {0, 3, 1}, {4, 5, 7}, {4, 7, 6}, {0, 1, 5}, {0, 5, 4},
                               {2, 6, 7}, {2, 7, 3}, {0, 4, 6}, {0, 6, 2}, {1, 3, 7}, {1, 7, 5}};
    for (auto &t : f)
        for (int i = 0; i < 3; ++i)
            m.indices.push_back(t[i]);
    m.material = material;
    g.meshes.push_back(std::move(m));
}

void look_at(GeneratedScene &g, V3 pos, V3 target, V3 up, double vfov_deg, double aspect)
{
    // look_at (camera.cpp:12-31): columns right, up, back, position
    V3 back = norm(pos - target);
    V3 right = norm(V3{up.y * back.z - up.z * back.y, up.z * back.x - up.x * back.z, up.x * back.y - up.y * back.x});
    V3 u = V3{back.y * right.z - back.z * right.y, back.z * right.x - back.x * right.z,
              back.x * right.y - back.y * right.x};
    float m[16] = {(float)right.x, (float)u.x, (float)back.x, (float)pos.x, (float)right.y, (float)u.y,
                   (float)back.y,  (float)pos.y, (float)right.z, (float)u.z, (float)back.z, (float)pos.z,
                   0.0f,           0.0f,         0.0f,          1.0f};
    std::memcpy(g.camera_to_world, m, sizeof(m));
    g.vfov = (float)(vfov_deg * 3.14159265358979323846 / 180.0);
    g.aspect = (float)aspect;
}

// ---- box room ---------------------------------------------------------------------------
void gen_box_room(GeneratedScene &g, uint64_t seed)
{
    SplitMix rng(seed);
    auto diffuse = [&]() {
        ks_material_desc m = default_material();
        for (int c = 0; c < 3; ++c)
            m.basecolor[c] = rng.uniform(0.1f, 0.9f);
        return m;
    };
    // room [-1,1] x [0,2] x [-1,1], open towards +z
    for (int i = 0; i < 5; ++i)
        g.materials.push_back(diffuse());
    add_quad(g, {-1, 0, -1}, {-1, 0, 1}, {1, 0, 1}, {1, 0, -1}, 0);   // floor
    add_quad(g, {-1, 2, -1}, {1, 2, -1}, {1, 2, 1}, {-1, 2, 1}, 1);   // ceiling
    add_quad(g, {-1, 0, -1}, {1, 0, -1}, {1, 2, -1}, {-1, 2, -1}, 2); // back
    add_quad(g, {-1, 0, -1}, {-1, 2, -1}, {-1, 2, 1}, {-1, 0, 1}, 3); // left
    add_quad(g, {1, 0, -1}, {1, 0, 1}, {1, 2, 1}, {1, 2, -1}, 4);     // right
    g.materials.push_back(diffuse());
    g.materials.push_back(diffuse());
    add_box(g, {-0.35, 0.6, -0.3}, {0.3, 0.6, 0.3}, rng.uniform(0.0f, 90.0f) * 3.14159265358979 / 180.0, 5);
    add_box(g, {0.4, 0.3, 0.35}, {0.3, 0.3, 0.3}, rng.uniform(0.0f, 90.0f) * 3.14159265358979 / 180.0, 6);
    ks_material_desc light = default_material();
    light.basecolor[0] = light.basecolor[1] = light.basecolor[2] = 0.0f;
    light.has_emission = 1;
    light.emission[0] = 17.0f;
    light.emission[1] = 12.0f;
    light.emission[2] = 4.0f;
    g.materials.push_back(light);
    // emitter facing down, slightly below the ceiling
    add_quad(g, {-0.25, 1.98, -0.25}, {0.25, 1.98, -0.25}, {0.25, 1.98, 0.25}, {-0.25, 1.98, 0.25},
             (uint32_t)g.materials.size() - 1);
    g.sky.kind = 0;
    look_at(g, {0, 1, 3.4}, {0, 1, 0}, {0, 1, 0}, 40.0, 1.0);
}

// ---- noise ---------------------------------------------------------------------------------
struct Noise3
{
    int perm[512];
    V3 grad[256];
    explicit Noise3(SplitMix &rng)
    {
        int p[256];
        for (int i = 0; i < 256; ++i)
            p[i] = i;
        for (int i = 255; i > 0; --i)
            std::swap(p[i], p[(int)(rng.next() % (uint64_t)(i + 1))]);
        for (int i = 0; i < 512; ++i)
            perm[i] = p[i & 255];
        for (int i = 0; i < 256; ++i) {
            V3 v;
            do {
                v = {2 * rng.uniform() - 1, 2 * rng.uniform() - 1, 2 * rng.uniform() - 1};
            } while (dot(v, v) > 1.0 || dot(v, v) < 1e-4);
            grad[i] = norm(v);
        }
    }
    static double fade(double t) { return t * t * t * (t * (t * 6 - 15) + 10); }
    double operator()(V3 q) const
    {
        int ix = (int)std::floor(q.x), iy = (int)std::floor(q.y), iz = (int)std::floor(q.z);
        double fx = q.x - ix, fy = q.y - iy, fz = q.z - iz;
        double acc[2][2][2];
        for (int c = 0; c < 8; ++c) {
            int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
            int h = perm[(perm[(perm[(ix + dx) & 255] + iy + dy) & 511] + iz + dz) & 511];
            acc[dx][dy][dz] = dot(grad[h & 255], V3{fx - dx, fy - dy, fz - dz});
        }
        double u = fade(fx), v = fade(fy), w = fade(fz);
        auto L = [](double a, double b, double t) { return a + t * (b - a); };
        return L(L(L(acc[0][0][0], acc[1][0][0], u), L(acc[0][1][0], acc[1][1][0], u), v),
                 L(L(acc[0][0][1], acc[1][0][1], u), L(acc[0][1][1], acc[1][1][1], u), v), w);
    }
    double fbm(V3 q, int octaves) const
    {
        double sum = 0, amp = 0.5, f = 1.0;
        for (int o = 0; o < octaves; ++o) {
            sum += amp * (*this)(f * q);
            amp *= 0.5;
            f *= 2.0;
        }
        return sum;
    }
};

// ---- icosphere -----------------------------------------------------------------------------
void geodesic(uint32_t f, std::vector<V3> &verts, std::vector<uint32_t> &tris);

void icosphere(int level, std::vector<V3> &verts, std::vector<uint32_t> &tris)
{
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    verts = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
             {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto &v : verts)
        v = norm(v);
    tris = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
            3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (int l = 0; l < level; ++l) {
        std::unordered_map<uint64_t, uint32_t> mid;
        mid.reserve(tris.size());
        auto midpoint = [&](uint32_t a, uint32_t b) {
            uint64_t key = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
            auto it = mid.find(key);
            if (it != mid.end())
                return it->second;
            verts.push_back(norm(0.5 * (verts[a] + verts[b])));
            uint32_t id = (uint32_t)verts.size() - 1;
            mid.emplace(key, id);
            return id;
        };
        std::vector<uint32_t> next;
        next.reserve(tris.size() * 4);
        // children of one parent stay consecutive, so runs of 4^k triangles are surface patches
        for (size_t i = 0; i < tris.size(); i += 3) {
            uint32_t a = tris[i], b = tris[i + 1], c = tris[i + 2];
            uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            uint32_t n4[12] = {a, ab, ca, ab, b, bc, ca, bc, c, ab, bc, ca};
            next.insert(next.end(), n4, n4 + 12);
        }
        tris.swap(next);
    }
}

void gen_sky(GeneratedScene &g, uint32_t w, uint32_t h, V3 sun_dir)
{
    g.sky_map.resize((size_t)w * h * 3);
    sun_dir = norm(sun_dir);
    for (uint32_t y = 0; y < h; ++y) {
        double theta = (y + 0.5) / h * 3.14159265358979323846;
        for (uint32_t x = 0; x < w; ++x) {
            double phi = (x + 0.5) / w * 2.0 * 3.14159265358979323846;
            // y-up spherical direction (to_cartesian_yup convention: theta from +y)
            V3 d{std::sin(theta) * std::cos(phi), std::cos(theta), std::sin(theta) * std::sin(phi)};
            double up = std::max(0.0, d.y);
            V3 sky{0.25 + 0.35 * up, 0.35 + 0.45 * up, 0.6 + 0.6 * up};
            if (d.y < 0) {
                double gnd = 0.18 * (1.0 + d.y);
                sky = {gnd, gnd, gnd};
            }
            double cosang = dot(d, sun_dir);
            double ang = std::acos(std::min(1.0, std::max(-1.0, cosang)));
            double lobe = 1e4 * std::exp(-(ang * ang) / (2.0 * 0.0125 * 0.0125));
            float *px = &g.sky_map[((size_t)y * w + x) * 3];
            px[0] = (float)(sky.x + lobe * 1.0);
            px[1] = (float)(sky.y + lobe * 0.92);
            px[2] = (float)(sky.z + lobe * 0.8);
        }
    }
    g.sky.kind = 2;
    g.sky.map_rgb = g.sky_map.data();
    g.sky.width = w;
    g.sky.height = h;
    float id[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
    std::memcpy(g.sky.to_world, id, sizeof(id));
    g.sky.transform_y_up = 1;
    g.sky.strength = 1.0f;
}

void gen_icosphere_scene(GeneratedScene &g, uint64_t seed, const ProceduralOptions &o)
{
    SplitMix rng(seed);
    Noise3 noise(rng);
    std::vector<V3> verts;
    std::vector<uint32_t> tris;
    if (o.geodesic_sphere)
        geodesic(std::max(1u, o.frequency), verts, tris);
    else
        icosphere(o.level, verts, tris);
    for (auto &v : verts) {
        double d = noise.fbm(3.0 * v + V3{17.3, 5.1, 9.7}, 6);
        v = (1.0 + 0.05 * d) * v;
    }
    const uint32_t patch = 1024;
    uint32_t n_tris = (uint32_t)tris.size() / 3;
    // one mesh (and one material) per patch of consecutive triangles; vertices re-indexed locally
    std::vector<uint32_t> remap(verts.size(), ~0u);
    for (uint32_t first = 0; first < n_tris; first += patch) {
        uint32_t last = std::min(n_tris, first + patch);
        GeneratedMesh m;
        std::vector<uint32_t> touched;
        for (uint32_t t = first; t < last; ++t)
            for (int k = 0; k < 3; ++k) {
                uint32_t v = tris[3 * t + k];
                if (remap[v] == ~0u) {
                    remap[v] = (uint32_t)m.vertices.size() / 3;
                    touched.push_back(v);
                    V3 p = verts[v];
                    m.vertices.push_back((float)p.x);
                    m.vertices.push_back((float)(p.y + 1.0));
                    m.vertices.push_back((float)p.z);
                }
                m.indices.push_back(remap[v]);
            }
        for (uint32_t v : touched)
            remap[v] = ~0u;
        ks_material_desc mat = default_material();
        mat.roughness = rng.uniform(o.roughness_min, o.roughness_max);
        mat.metallic = rng.uniform() < 0.3 ? 1.0f : 0.0f;
        for (int c = 0; c < 3; ++c)
            mat.basecolor[c] = rng.uniform(0.0f, 1.0f);
        g.materials.push_back(mat);
        m.material = (uint32_t)g.materials.size() - 1;
        g.meshes.push_back(std::move(m));
    }
    ks_material_desc ground = default_material();
    ground.basecolor[0] = ground.basecolor[1] = ground.basecolor[2] = 0.5f;
    g.materials.push_back(ground);
    const double s = 12.0, gy = -0.06;
    add_quad(g, {-s, gy, -s}, {-s, gy, s}, {s, gy, s}, {s, gy, -s}, (uint32_t)g.materials.size() - 1);
    V3 sun = norm(V3{0.45, 0.6, -0.66});
    if (o.occluder) {
        // slab between the sphere and the sun, casting the sphere into shadow
        ks_material_desc slab = default_material();
        slab.basecolor[0] = slab.basecolor[1] = slab.basecolor[2] = 0.3f;
        g.materials.push_back(slab);
        V3 c = V3{0, 1, 0} + 3.0 * sun;
        V3 a = norm(V3{sun.z, 0, -sun.x});
        V3 b = norm(V3{sun.y * a.z - sun.z * a.y, sun.z * a.x - sun.x * a.z, sun.x * a.y - sun.y * a.x});
        double e = 1.6;
        add_quad(g, c - e * a - e * b, c + e * a - e * b, c + e * a + e * b, c - e * a + e * b,
                 (uint32_t)g.materials.size() - 1);
    }
    gen_sky(g, o.sky_width, o.sky_height, sun);
    look_at(g, {0.0, 1.6, 3.6}, {0, 0.95, 0}, {0, 1, 0}, 38.0, (double)o.width / o.height);
}

} // namespace

namespace
{

// Geodesic sphere: every icosahedron face split into f^2 triangles on a barycentric grid whose
// points are normalised integer-weighted sums of the face corners (points on shared edges come out
// identical from both faces, so the mesh is watertight).
void geodesic(uint32_t f, std::vector<V3> &verts, std::vector<uint32_t> &tris)
{
    std::vector<V3> ico;
    std::vector<uint32_t> faces;
    icosphere(0, ico, faces);
    verts.clear();
    tris.clear();
    for (size_t fi = 0; fi < faces.size(); fi += 3) {
        V3 A = ico[faces[fi]], B = ico[faces[fi + 1]], C = ico[faces[fi + 2]];
        uint32_t base = (uint32_t)verts.size();
        auto id = [&](uint32_t i, uint32_t j) {
            // row i has f + 1 - i points
            return base + i * (f + 1) - i * (i - 1) / 2 + j;
        };
        for (uint32_t i = 0; i <= f; ++i)
            for (uint32_t j = 0; i + j <= f; ++j) {
                double wa = f - i - j, wb = i, wc = j;
                V3 p = (wa * A + wb * B) + wc * C;
                verts.push_back(norm(p));
            }
        for (uint32_t i = 0; i < f; ++i)
            for (uint32_t j = 0; i + j < f; ++j) {
                tris.insert(tris.end(), {id(i, j), id(i + 1, j), id(i, j + 1)});
                if (i + j + 1 < f)
                    tris.insert(tris.end(), {id(i + 1, j), id(i + 1, j + 1), id(i, j + 1)});
            }
    }
}

// Rotation about a unit axis (Rodrigues), row-major 3x3.
void axis_angle(V3 a, double ang, double R[9])
{
    double c = std::cos(ang), s = std::sin(ang), t = 1.0 - c;
    R[0] = t * a.x * a.x + c;
    R[1] = t * a.x * a.y - s * a.z;
    R[2] = t * a.x * a.z + s * a.y;
    R[3] = t * a.x * a.y + s * a.z;
    R[4] = t * a.y * a.y + c;
    R[5] = t * a.y * a.z - s * a.x;
    R[6] = t * a.x * a.z - s * a.y;
    R[7] = t * a.y * a.z + s * a.x;
    R[8] = t * a.z * a.z + c;
}

void gen_instanced_scene(GeneratedScene &g, uint64_t seed, const ProceduralOptions &o)
{
    SplitMix rng(seed);
    const uint32_t f = std::max(1u, o.frequency), n_protos = std::max(1u, o.prototypes);
    std::vector<V3> base_verts;
    std::vector<uint32_t> base_tris;
    geodesic(f, base_verts, base_tris);
    // prototypes 0..n-1: displaced spheres, one mesh and one material each
    for (uint32_t q = 0; q < n_protos; ++q) {
        Noise3 noise(rng);
        GeneratedMesh m;
        V3 off{rng.uniform() * 50.0, rng.uniform() * 50.0, rng.uniform() * 50.0};
        for (const V3 &v : base_verts) {
            double d = noise.fbm(3.0 * v + off, 6);
            V3 p = (1.0 + 0.05 * d) * v;
            m.vertices.insert(m.vertices.end(), {(float)p.x, (float)p.y, (float)p.z});
        }
        m.indices = base_tris;
        ks_material_desc mat = default_material();
        mat.roughness = rng.uniform(0.05f, 1.0f);
        mat.metallic = rng.uniform() < 0.3 ? 1.0f : 0.0f;
        for (int c = 0; c < 3; ++c)
            mat.basecolor[c] = rng.uniform(0.0f, 1.0f);
        g.materials.push_back(mat);
        m.material = (uint32_t)g.materials.size() - 1;
        g.meshes.push_back(std::move(m));
        g.prototypes.push_back(ks_prototype_desc{(uint32_t)g.meshes.size() - 1, 1});
    }
    // instances of the spheres
    const double field = 8.0;
    for (uint32_t i = 0; i < o.instances; ++i) {
        ks_instance_desc inst{};
        inst.prototype = i % n_protos;
        V3 axis = norm(V3{rng.uniform() - 0.5, rng.uniform() - 0.5, rng.uniform() - 0.5});
        double R[9];
        axis_angle(axis, rng.uniform() * 6.283185307179586, R);
        double sc[3];
        for (double &x : sc)
            x = 0.12 + 0.28 * rng.uniform();
        double ty = 0.4 * std::max({sc[0], sc[1], sc[2]}) + 0.6 * rng.uniform() * sc[1];
        double t[3] = {(2.0 * rng.uniform() - 1.0) * field, ty, (2.0 * rng.uniform() - 1.0) * field};
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c)
                inst.to_world[4 * r + c] = (float)(R[3 * r + c] * sc[c]);
            inst.to_world[4 * r + 3] = (float)t[r];
        }
        g.instances.push_back(inst);
    }
    auto identity = [](uint32_t proto) {
        ks_instance_desc d{};
        d.prototype = proto;
        d.to_world[0] = d.to_world[5] = d.to_world[10] = 1.0f;
        return d;
    };
    // emitters: small triangles above the field, radiance log-uniform over 3 decades
    if (o.emitters > 0) {
        uint32_t first = (uint32_t)g.meshes.size();
        for (uint32_t e = 0; e < o.emitters; ++e) {
            V3 c{(2.0 * rng.uniform() - 1.0) * field, 2.5 + 1.5 * rng.uniform(), (2.0 * rng.uniform() - 1.0) * field};
            double r = 0.08 + 0.1 * rng.uniform(), a0 = rng.uniform() * 6.283185307179586;
            GeneratedMesh m;
            for (int k = 0; k < 3; ++k) {
                double a = a0 + k * 2.0943951023931953;
                V3 p{c.x + r * std::cos(a), c.y, c.z - r * std::sin(a)};
                m.vertices.insert(m.vertices.end(), {(float)p.x, (float)p.y, (float)p.z});
            }
            m.indices = {0, 1, 2};
            ks_material_desc mat = default_material();
            double L = std::pow(10.0, 3.0 * rng.uniform());
            mat.has_emission = 1;
            for (int c2 = 0; c2 < 3; ++c2)
                mat.emission[c2] = (float)(L * (0.6 + 0.4 * rng.uniform()));
            g.materials.push_back(mat);
            m.material = (uint32_t)g.materials.size() - 1;
            g.meshes.push_back(std::move(m));
        }
        g.prototypes.push_back(ks_prototype_desc{first, o.emitters});
        g.instances.push_back(identity((uint32_t)g.prototypes.size() - 1));
    }
    // ground
    ks_material_desc ground = default_material();
    ground.basecolor[0] = ground.basecolor[1] = ground.basecolor[2] = 0.5f;
    g.materials.push_back(ground);
    const double s = 20.0;
    add_quad(g, {-s, 0, -s}, {-s, 0, s}, {s, 0, s}, {s, 0, -s}, (uint32_t)g.materials.size() - 1);
    g.prototypes.push_back(ks_prototype_desc{(uint32_t)g.meshes.size() - 1, 1});
    g.instances.push_back(identity((uint32_t)g.prototypes.size() - 1));
    gen_sky(g, o.sky_width, o.sky_height, norm(V3{0.45, 0.6, -0.66}));
    look_at(g, {0.0, 4.5, 12.5}, {0, 0.3, 0}, {0, 1, 0}, 40.0, (double)o.width / o.height);
}

} // namespace

void GeneratedScene::finalize()
{
    mesh_descs.resize(meshes.size());
    for (size_t i = 0; i < meshes.size(); ++i) {
        ks_mesh_desc &d = mesh_descs[i];
        d.vertices = meshes[i].vertices.data();
        d.n_vertices = (uint32_t)meshes[i].vertices.size() / 3;
        d.indices = meshes[i].indices.data();
        d.n_triangles = (uint32_t)meshes[i].indices.size() / 3;
        d.vertex_normals = meshes[i].normals.empty() ? nullptr : meshes[i].normals.data();
        d.texcoords = meshes[i].texcoords.empty() ? nullptr : meshes[i].texcoords.data();
        d.material = meshes[i].material;
        d.twosided = meshes[i].twosided;
        d.use_smooth_normal = meshes[i].use_smooth_normal;
    }
    desc.meshes = mesh_descs.data();
    desc.n_meshes = (uint32_t)mesh_descs.size();
    desc.materials = materials.data();
    desc.n_materials = (uint32_t)materials.size();
    if (sky.kind == 2)
        sky.map_rgb = sky_map.data();
    desc.sky = sky;
    desc.prototypes = prototypes.empty() ? nullptr : prototypes.data();
    desc.n_prototypes = (uint32_t)prototypes.size();
    desc.instances = instances.empty() ? nullptr : instances.data();
    desc.n_instances = (uint32_t)instances.size();
    for (size_t k = 0; k < textures.size(); ++k)
        textures[k].texels = texture_bytes[k].data();
    desc.textures = textures.empty() ? nullptr : textures.data();
    desc.n_textures = (uint32_t)textures.size();
    desc.bindings = bindings.empty() ? nullptr : bindings.data();
    desc.n_bindings = (uint32_t)bindings.size();
}

bool generate_scene(const std::string &kind, uint64_t seed, const ProceduralOptions &opts, GeneratedScene &out)
{
    out = GeneratedScene();
    out.width = opts.width;
    out.height = opts.height;
    if (kind == "box_room") {
        gen_box_room(out, seed);
    } else if (kind == "icosphere") {
        gen_icosphere_scene(out, seed, opts);
    } else if (kind == "instanced") {
        gen_instanced_scene(out, seed, opts);
    } else {
        return false;
    }
    out.finalize();
    return true;
}

} // namespace ksb
