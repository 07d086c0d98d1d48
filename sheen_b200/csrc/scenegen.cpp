// scenegen.cpp -- seeded synthetic scenes for the benchmark workloads.
//
// Every generator is deterministic for a given (config, seed, detail): all
// randomness comes from std::mt19937 (whose sequence the C++ standard fixes)
// converted to floats with explicit 24-bit scaling, and all geometry is built
// with plain float arithmetic in a fixed order.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <unordered_map>
#include <vector>

#include "owned_scene.h"
#include "sheen_c_api.h"

namespace sheen {
void set_error(const char* msg);
}

namespace {

using sheen::OwnedScene;

struct V3 { float x, y, z; };
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline V3 norm(V3 a) { float l = std::sqrt(dot(a, a)); return l > 0.0f ? a * (1.0f / l) : a; }
inline sheen_float3 F(V3 a) { return sheen_float3{a.x, a.y, a.z}; }

struct Rng {
    std::mt19937 g;
    explicit Rng(uint32_t s) : g(s) {}
    float u01() { return (float)(g() >> 8) * (1.0f / 16777216.0f); }
    float uni(float a, float b) { return a + (b - a) * u01(); }
};

// Look-at camera with a horizontal field of view of `hfov_deg` on the wider
// image axis: CameraData's focal_length/sensor_width pair is set so that
// 0.5*sensor/focal = tan(hfov/2) (render_kernel.cu:500-510).
CameraData look_at(V3 pos, V3 target, float hfov_deg) {
    CameraData c;
    std::memset(&c, 0, sizeof(c));
    V3 fwd = norm(target - pos);
    V3 right = norm(cross(fwd, V3{0.0f, 1.0f, 0.0f}));
    V3 up = cross(right, fwd);
    c.position = F(pos);
    c.forward = F(fwd);
    c.right = F(right);
    c.up = F(up);
    c.sensor_width = 36.0f;
    c.focal_length = 18.0f / std::tan(0.5f * hfov_deg * 3.14159265358979f / 180.0f);
    return c;
}

// 3D value noise on an integer lattice with a seeded integer hash, smoothstep
// interpolation; fbm sums `octaves` octaves (lacunarity 2, gain 0.5) and is
// normalised to [0, 1].
inline float lattice(int x, int y, int z, uint32_t seed) {
    uint32_t h = (uint32_t)x * 0x8da6b343u ^ (uint32_t)y * 0xd8163841u ^ (uint32_t)z * 0xcb1ab31fu ^ seed * 0x9e3779b1u;
    h ^= h >> 15; h *= 0x2c1b3c6du; h ^= h >> 12; h *= 0x297a2d39u; h ^= h >> 15;
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

float value_noise(V3 p, uint32_t seed) {
    float fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
    int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
    tx = tx * tx * (3.0f - 2.0f * tx);
    ty = ty * ty * (3.0f - 2.0f * ty);
    tz = tz * tz * (3.0f - 2.0f * tz);
    float c[2][2][2];
    for (int dz = 0; dz < 2; dz++)
        for (int dy = 0; dy < 2; dy++)
            for (int dx = 0; dx < 2; dx++) c[dz][dy][dx] = lattice(ix + dx, iy + dy, iz + dz, seed);
    float x00 = c[0][0][0] + (c[0][0][1] - c[0][0][0]) * tx;
    float x10 = c[0][1][0] + (c[0][1][1] - c[0][1][0]) * tx;
    float x01 = c[1][0][0] + (c[1][0][1] - c[1][0][0]) * tx;
    float x11 = c[1][1][0] + (c[1][1][1] - c[1][1][0]) * tx;
    float y0 = x00 + (x10 - x00) * ty;
    float y1 = x01 + (x11 - x01) * ty;
    return y0 + (y1 - y0) * tz;
}

float fbm(V3 p, int octaves, uint32_t seed) {
    float amp = 0.5f, sum = 0.0f, normz = 0.0f;
    for (int o = 0; o < octaves; o++) {
        sum += amp * value_noise(p, seed + (uint32_t)o * 1013u);
        normz += amp;
        amp *= 0.5f;
        p = p * 2.0f;
    }
    return sum / normz;
}

// Indexed triangle mesh with smooth vertex normals, emitted as Triangles.
struct Mesh {
    std::vector<V3> v;
    std::vector<uint32_t> f;   // 3 per face
    std::vector<V3> n;
    void compute_normals() {
        n.assign(v.size(), V3{0.0f, 0.0f, 0.0f});
        for (size_t i = 0; i < f.size(); i += 3) {
            V3 a = v[f[i]], b = v[f[i + 1]], c = v[f[i + 2]];
            V3 fn = cross(b - a, c - a);   // area weighted
            for (int k = 0; k < 3; k++) n[f[i + (size_t)k]] = n[f[i + (size_t)k]] + fn;
        }
        for (V3& q : n) q = norm(q);
    }
    void emit(OwnedScene& s, int mat) const {
        for (size_t i = 0; i < f.size(); i += 3) {
            float vv[9], nn[9];
            for (int k = 0; k < 3; k++) {
                V3 p = v[f[i + (size_t)k]], q = n[f[i + (size_t)k]];
                vv[3 * k] = p.x; vv[3 * k + 1] = p.y; vv[3 * k + 2] = p.z;
                nn[3 * k] = q.x; nn[3 * k + 1] = q.y; nn[3 * k + 2] = q.z;
            }
            s.add_triangle(vv, nn, nullptr, mat);
        }
    }
};

Mesh icosphere(int level) {
    Mesh m;
    const float t = (1.0f + std::sqrt(5.0f)) * 0.5f;
    const float base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0},
                               {0, -1, t}, {0, 1, t}, {0, -1, -t}, {0, 1, -t},
                               {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& b : base) m.v.push_back(norm(V3{b[0], b[1], b[2]}));
    const uint32_t faces[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                                   {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                   {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                                   {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (auto& f : faces) m.f.insert(m.f.end(), {f[0], f[1], f[2]});
    for (int l = 0; l < level; l++) {
        std::unordered_map<uint64_t, uint32_t> mid;
        mid.reserve(m.f.size() * 2);
        auto midpoint = [&](uint32_t a, uint32_t b) {
            uint64_t key = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            uint32_t id = (uint32_t)m.v.size();
            m.v.push_back(norm((m.v[a] + m.v[b]) * 0.5f));
            mid.emplace(key, id);
            return id;
        };
        std::vector<uint32_t> nf;
        nf.reserve(m.f.size() * 4);
        for (size_t i = 0; i < m.f.size(); i += 3) {
            uint32_t a = m.f[i], b = m.f[i + 1], c = m.f[i + 2];
            uint32_t ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
            nf.insert(nf.end(), {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca});
        }
        m.f.swap(nf);
    }
    return m;
}

Mesh torus(int nu, int nv, float R, float r) {
    Mesh m;
    for (int i = 0; i < nu; i++) {
        float u = 6.28318530718f * (float)i / (float)nu;
        for (int j = 0; j < nv; j++) {
            float w = 6.28318530718f * (float)j / (float)nv;
            m.v.push_back(V3{(R + r * std::cos(w)) * std::cos(u), r * std::sin(w),
                             (R + r * std::cos(w)) * std::sin(u)});
        }
    }
    for (int i = 0; i < nu; i++)
        for (int j = 0; j < nv; j++) {
            uint32_t a = (uint32_t)(i * nv + j), b = (uint32_t)(((i + 1) % nu) * nv + j);
            uint32_t c = (uint32_t)(((i + 1) % nu) * nv + (j + 1) % nv), d = (uint32_t)(i * nv + (j + 1) % nv);
            m.f.insert(m.f.end(), {a, c, b, a, d, c});
        }
    return m;
}

// Displace every vertex along its smooth normal by amp*(2*fbm(p*freq)-1).
void displace(Mesh& m, float amp, float freq, uint32_t seed) {
    m.compute_normals();
    for (size_t i = 0; i < m.v.size(); i++) {
        float h = 2.0f * fbm(m.v[i] * freq, 6, seed) - 1.0f;
        m.v[i] = m.v[i] + m.n[i] * (amp * h);
    }
    m.compute_normals();
}

V3 rotate(V3 p, V3 axis, float ang) {
    float c = std::cos(ang), s = std::sin(ang);
    return p * c + cross(axis, p) * s + axis * (dot(axis, p) * (1.0f - c));
}

// Config 0: 640x480, 1 spp; 64 spheres with centres uniform in [-10,10]^3
// and radii in [0.2,1.0]; ground plane y = -10; one point light at
// (10,20,-10) with power 4*pi*|L|^2 (irradiance 1 at the origin);
// Blinn-Phong, hard shadows, reflect 0.3 on every material.
void gen_spheres(OwnedScene& s, uint32_t seed) {
    Rng rng(seed);
    s.camera = look_at(V3{0.0f, 2.0f, -15.0f}, V3{0.0f, 0.0f, 0.0f}, 60.0f);
    for (int k = 0; k < 8; k++) {
        float r = rng.uni(0.2f, 1.0f), g = rng.uni(0.2f, 1.0f), b = rng.uni(0.2f, 1.0f);
        int m = s.add_material(r, g, b, 0.5f, 32.0f, 0.1f);
        s.materials[(size_t)m].reflect = 0.3f;
    }
    int ground = s.add_material(0.6f, 0.6f, 0.6f, 0.1f, 16.0f, 0.1f);
    s.materials[(size_t)ground].reflect = 0.3f;
    for (int i = 0; i < 64; i++) {
        float cx = rng.uni(-10.0f, 10.0f), cy = rng.uni(-10.0f, 10.0f), cz = rng.uni(-10.0f, 10.0f);
        float r = rng.uni(0.2f, 1.0f);
        s.add_sphere(cx, cy, cz, r, i % 8);
    }
    s.add_plane(0.0f, 1.0f, 0.0f, 10.0f, ground);
    const float L2 = 10.0f * 10.0f + 20.0f * 20.0f + 10.0f * 10.0f;
    s.add_point_light(10.0f, 20.0f, -10.0f, 1.0f, 1.0f, 1.0f, 12.5663706f * L2, 0.0f);
    s.settings.width = 640; s.settings.height = 480; s.settings.aa = 1;
}

// Config 1: a level-`level` icosphere (radius 5; level 8 = 1,310,720
// triangles) displaced by 6-octave fBm (amplitude 0.5) plus 16 copies of a
// displaced 250x100-quad torus (50,000 triangles, R 1.5, r 0.5) on a ring
// with seeded orientations, flattened into one triangle list; 4 point
// lights; every 4th torus is glass (transmission 1, ior 1.5), everything
// else Blinn-Phong with reflect 0.2; a ground plane.
// instanced: the tori as instances of one mesh (scene extension) instead
// of 16 flattened copies; the same draws, so the same scene up to the
// rounding of the transforms.
void gen_mesh(OwnedScene& s, uint32_t seed, int level, bool instanced = false) {
    Rng rng(seed);
    s.camera = look_at(V3{0.0f, 7.0f, -26.0f}, V3{0.0f, 0.0f, 0.0f}, 60.0f);
    int m_sphere = s.add_material(0.75f, 0.55f, 0.4f, 0.4f, 48.0f, 0.05f);
    s.materials[(size_t)m_sphere].reflect = 0.2f;
    int m_glass = s.add_material(0.95f, 0.95f, 0.95f, 0.6f, 96.0f, 0.0f);
    s.materials[(size_t)m_glass].transmission = 1.0f;
    s.materials[(size_t)m_glass].ior = 1.5f;
    int m_torus[4];
    for (int k = 0; k < 4; k++) {
        m_torus[k] = s.add_material(rng.uni(0.2f, 0.9f), rng.uni(0.2f, 0.9f), rng.uni(0.2f, 0.9f),
                                    0.5f, 64.0f, 0.05f);
        s.materials[(size_t)m_torus[k]].reflect = 0.2f;
    }
    int m_ground = s.add_material(0.5f, 0.5f, 0.55f, 0.1f, 16.0f, 0.05f);
    s.materials[(size_t)m_ground].reflect = 0.2f;

    Mesh ico = icosphere(level);
    for (V3& p : ico.v) p = p * 5.0f;
    displace(ico, 0.5f, 0.6f, seed ^ 0x1234567u);
    s.triangles.reserve(ico.f.size() / 3 + 16 * 50000);
    ico.emit(s, m_sphere);

    // Torus grid follows the icosphere detail so small test scenes stay small.
    int nu = 250, nv = 100;
    if (level < 8) { int d = 1 << (8 - level); nu = std::max(10, nu / d); nv = std::max(6, nv / d); }
    Mesh tor = torus(nu, nv, 1.5f, 0.5f);
    displace(tor, 0.06f, 3.0f, seed ^ 0x7654321u);
    if (instanced) {
        const size_t first = s.triangles.size();
        tor.emit(s, m_glass);
        s.mesh_triangles.assign(s.triangles.begin() + (long)first, s.triangles.end());
        s.triangles.resize(first);
        s.meshes.push_back(SheenMesh{0, (int)s.mesh_triangles.size()});
    }
    for (int k = 0; k < 16; k++) {
        float ang = 6.28318530718f * (float)k / 16.0f + rng.uni(-0.08f, 0.08f);
        V3 centre{9.5f * std::cos(ang), rng.uni(-1.5f, 1.5f), 9.5f * std::sin(ang)};
        V3 axis = norm(V3{rng.uni(-1.0f, 1.0f), rng.uni(-1.0f, 1.0f), rng.uni(-1.0f, 1.0f)});
        float rot = rng.uni(0.0f, 3.14159265f);
        if (instanced) {
            // rotate()'s map as a matrix: c I + s [axis]x + (1 - c) axis axis^T
            const double c = std::cos(rot), sn = std::sin(rot), a[3] = {axis.x, axis.y, axis.z};
            const double cx[3][3] = {{0.0, -a[2], a[1]}, {a[2], 0.0, -a[0]}, {-a[1], a[0], 0.0}};
            const double t[3] = {centre.x, centre.y, centre.z};
            SheenInstance in;
            std::memset(&in, 0, sizeof(in));
            for (int r = 0; r < 3; r++) {
                for (int q = 0; q < 3; q++)
                    in.xform[4 * r + q] = (float)((r == q ? c : 0.0) + sn * cx[r][q] + (1.0 - c) * a[r] * a[q]);
                in.xform[4 * r + 3] = (float)t[r];
            }
            in.mesh = 0;
            in.material_id = (k % 4 == 0) ? m_glass : m_torus[k % 4];
            s.instances.push_back(in);
            continue;
        }
        Mesh inst = tor;
        for (size_t i = 0; i < inst.v.size(); i++) {
            inst.v[i] = rotate(tor.v[i], axis, rot) + centre;
            inst.n[i] = rotate(tor.n[i], axis, rot);
        }
        inst.emit(s, (k % 4 == 0) ? m_glass : m_torus[k % 4]);
    }
    s.add_plane(0.0f, 1.0f, 0.0f, 7.0f, m_ground);
    const float lp[4][3] = {{18.0f, 22.0f, -18.0f}, {-18.0f, 22.0f, -18.0f},
                            {18.0f, 22.0f, 18.0f}, {-18.0f, 22.0f, 18.0f}};
    for (auto& p : lp) {
        float L2 = p[0] * p[0] + p[1] * p[1] + p[2] * p[2];
        s.add_point_light(p[0], p[1], p[2], 1.0f, 0.97f, 0.92f, 12.5663706f * L2 * 0.3f, 0.0f);
    }
    s.settings.width = 1920; s.settings.height = 1080; s.settings.aa = 4;
}

// Config 3: glass sphere (ior 1.5, r 2) and a glass lathe (centred on the Y
// axis: the reference's lathe test ignores Lathe.center) over a diffuse
// plane, one spot light; `photons` photons per light, hash cell 0.2
// (gather radius 0.1), caustic gain 1.
void gen_caustics(OwnedScene& s, uint32_t seed, int photons) {
    (void)seed;
    s.camera = look_at(V3{0.0f, 5.0f, -12.0f}, V3{1.2f, 1.0f, 0.0f}, 60.0f);
    int m_floor = s.add_material(0.7f, 0.7f, 0.68f, 0.1f, 16.0f, 0.05f);
    int m_glass = s.add_material(0.95f, 0.95f, 0.95f, 0.6f, 96.0f, 0.0f);
    s.materials[(size_t)m_glass].transmission = 1.0f;
    s.materials[(size_t)m_glass].ior = 1.5f;
    s.add_plane(0.0f, 1.0f, 0.0f, 0.0f, m_floor);
    s.add_sphere(3.5f, 2.0f, 0.5f, 2.0f, m_glass);
    const float prof[][2] = {{0.05f, 0.05f}, {0.2f, 0.9f}, {0.8f, 1.2f}, {1.6f, 1.1f},
                             {2.4f, 0.7f}, {3.0f, 0.6f}, {3.4f, 0.75f}};
    Lathe l;
    std::memset(&l, 0, sizeof(l));
    l.point_offset = (int)s.lathe_points.size();
    l.point_count = (int)(sizeof(prof) / sizeof(prof[0]));
    l.material_id = m_glass;
    for (auto& p : prof) {
        LathePoint q;
        std::memset(&q, 0, sizeof(q));
        q.y = p[0]; q.radius = p[1];
        s.lathe_points.push_back(q);
    }
    s.lathes.push_back(l);
    const float pos[3] = {1.0f, 9.0f, -3.0f}, dir[3] = {0.15f, -1.0f, 0.35f}, col[3] = {1.0f, 0.95f, 0.85f};
    s.add_spot_light(pos, dir, col, 900.0f, 0.55f, 0.2f, 0.0f, 0.0f);
    s.settings.photons = photons;
    s.settings.photon_cell = 0.2f;
    s.settings.caustics = 1.0f;
    s.settings.width = 1920; s.settings.height = 1080; s.settings.aa = 16;
}

}  // namespace

namespace sheen {
void gen_analytic(OwnedScene& s, uint32_t seed, int detail, bool extended);
}

extern "C" int sheen_generate_scene(int config, unsigned int seed, int detail, int photons,
                                    SheenOwnedScene* out) {
    return sheen_generate_scene_ext(config, seed, detail, photons, 0, out);
}

extern "C" int sheen_generate_scene_ext(int config, unsigned int seed, int detail, int photons, int extended,
                                        SheenOwnedScene* out) {
    if (!out) { sheen::set_error("null output handle"); return -1; }
    *out = nullptr;
    if (extended && config != 1 && config != 2) {
        sheen::set_error("extended generator exists for configs 1 and 2 only");
        return -1;
    }
    OwnedScene* s = new OwnedScene();
    switch (config) {
        case 0: gen_spheres(*s, seed); break;
        case 1:
            gen_mesh(*s, seed, detail > 0 ? detail : 8, extended != 0);
            if (extended) s->max_depth = 4;   // reflect + refract recursion to 4 bounces
            break;
        case 2: sheen::gen_analytic(*s, seed, detail, extended != 0); break;
        case 3: gen_caustics(*s, seed, photons > 0 ? photons : 4000000); break;
        default:
            delete s;
            sheen::set_error("unknown scene config");
            return -1;
    }
    s->finalize();
    *out = reinterpret_cast<SheenOwnedScene>(s);
    return 0;
}
