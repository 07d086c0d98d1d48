// scenegen_analytic.cpp -- config 2: analytic primitives and a CSG tree.
//
// 256 superellipsoids (single exponent n = 2/e, e uniform in [0.2, 2], so the
// body stays convex as the reference's sampler assumes), 64 lathes and 64
// prisms whose profiles are 8 seeded cubic-Bezier control points (two cubic
// spans, tessellated 8 pieces per span the way the .sheen lathe_bezier /
// prism_bezier commands do), 32 sphere sweeps along 6-point Catmull-Rom
// paths, one procedural fBm heightfield, and one CSG tree of depth 3 over
// spheres and superellipsoid boxes (n = 12).  Lathes keep center = 0: the
// reference's lathe test ignores Lathe.center, so they share the Y axis.
//
// extended (the workload's extension column, no counterpart in the
// reference): the same scene with two-exponent superellipsoids (both
// exponents 2/e, e uniform in [0.2, 3]), the lathes' and prisms' Bezier
// control points kept as exact surfaces, a 1024 x 1024 FP32 fBm height grid
// for the heightfield, and 128 further CSG trees of depth 3 over spheres,
// boxes and cones.  Its draws come from a second generator stream, so the
// base geometry is the base scene's.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "owned_scene.h"

namespace sheen {

namespace {
struct R {
    std::mt19937 g;
    explicit R(uint32_t s) : g(s) {}
    float u01() { return (float)(g() >> 8) * (1.0f / 16777216.0f); }
    float uni(float a, float b) { return a + (b - a) * u01(); }
};

// Cubic Bezier runs in groups of four control points (the layout of the
// .sheen *_bezier commands): start point, then `sub` samples per span.
std::vector<std::pair<float, float>> bezier_run(const std::vector<std::pair<float, float>>& c, int sub) {
    std::vector<std::pair<float, float>> out;
    if (c.size() < 4) return out;
    out.push_back(c[0]);
    for (size_t s = 0; s + 3 < c.size(); s += 4) {
        for (int k = 1; k <= sub; k++) {
            float t = (float)k / (float)sub, u = 1.0f - t;
            float w0 = u * u * u, w1 = 3.0f * u * u * t, w2 = 3.0f * u * t * t, w3 = t * t * t;
            out.push_back({w0 * c[s].first + w1 * c[s + 1].first + w2 * c[s + 2].first + w3 * c[s + 3].first,
                           w0 * c[s].second + w1 * c[s + 1].second + w2 * c[s + 2].second + w3 * c[s + 3].second});
        }
    }
    return out;
}
}  // namespace

// Seeded value-noise fBm on the unit square, normalised to [0, 1] over the
// grid (the extension's FP32 height grid).
static void fbm_grid(uint32_t seed, int w, int h, std::vector<float>& out) {
    auto hash = [seed](int x, int z) {
        uint32_t v = (uint32_t)x * 0x8da6b343u ^ (uint32_t)z * 0xd8163841u ^ seed * 0xcb1ab31fu;
        v ^= v >> 15; v *= 0x2c1b3c6du; v ^= v >> 12; v *= 0x297a2d39u; v ^= v >> 15;
        return (float)(v >> 8) * (1.0f / 16777216.0f);
    };
    auto noise = [&](float x, float z) {
        const int x0 = (int)std::floor(x), z0 = (int)std::floor(z);
        float tx = x - (float)x0, tz = z - (float)z0;
        tx = tx * tx * (3.0f - 2.0f * tx);
        tz = tz * tz * (3.0f - 2.0f * tz);
        const float a = hash(x0, z0) + (hash(x0 + 1, z0) - hash(x0, z0)) * tx;
        const float b = hash(x0, z0 + 1) + (hash(x0 + 1, z0 + 1) - hash(x0, z0 + 1)) * tx;
        return a + (b - a) * tz;
    };
    out.assign((size_t)w * h, 0.0f);
    float lo = 1e30f, hi = -1e30f;
    for (int v = 0; v < h; v++)
        for (int u = 0; u < w; u++) {
            float fx = 6.0f * (float)u / (float)(w - 1), fz = 6.0f * (float)v / (float)(h - 1);
            float amp = 0.5f, sum = 0.0f;
            for (int o = 0; o < 6; o++) {
                sum += amp * noise(fx + 17.0f * o, fz + 31.0f * o);
                amp *= 0.5f;
                fx *= 2.0f;
                fz *= 2.0f;
            }
            out[(size_t)v * w + u] = sum;
            lo = std::min(lo, sum);
            hi = std::max(hi, sum);
        }
    const float span = hi > lo ? hi - lo : 1.0f;
    for (float& x : out) x = (x - lo) / span;
}

void gen_analytic(OwnedScene& s, uint32_t seed, int detail, bool extended) {
    (void)detail;
    R rng(seed);
    R rng2(seed * 2654435761u ^ 0x5bd1e995u);   // the extensions' stream
    {
        CameraData c;
        std::memset(&c, 0, sizeof(c));
        // look from (0, 9, -30) at (0, 1, 0), 60 degree horizontal field of view
        float px = 0.0f, py = 9.0f, pz = -30.0f, tx = 0.0f, ty = 1.0f, tz = 0.0f;
        float fx = tx - px, fy = ty - py, fz = tz - pz;
        float fl = std::sqrt(fx * fx + fy * fy + fz * fz);
        fx /= fl; fy /= fl; fz /= fl;
        float rx = -fz, rz = fx;   // forward x (0,1,0)
        float rl = std::sqrt(rx * rx + rz * rz);
        rx /= rl; rz /= rl;
        c.position = {px, py, pz};
        c.forward = {fx, fy, fz};
        c.right = {rx, 0.0f, rz};
        c.up = {0.0f * fz - rz * fy, rz * fx - rx * fz, rx * fy - 0.0f * fx};
        c.sensor_width = 36.0f;
        c.focal_length = 18.0f / std::tan(30.0f * 3.14159265358979f / 180.0f);
        s.camera = c;
    }
    for (int k = 0; k < 8; k++) {
        int m = s.add_material(rng.uni(0.2f, 0.9f), rng.uni(0.2f, 0.9f), rng.uni(0.2f, 0.9f),
                               0.4f, 40.0f, 0.08f);
        if (k == 7) s.materials[(size_t)m].reflect = 0.3f;
    }
    const int m_ground = s.add_material(0.55f, 0.6f, 0.5f, 0.05f, 8.0f, 0.1f);

    for (int i = 0; i < 256; i++) {
        Superellipsoid se;
        std::memset(&se, 0, sizeof(se));
        se.center = {rng.uni(-18.0f, 18.0f), rng.uni(0.5f, 6.0f), rng.uni(-6.0f, 18.0f)};
        se.a = rng.uni(0.3f, 0.8f); se.b = rng.uni(0.3f, 0.8f); se.c = rng.uni(0.3f, 0.8f);
        se.n = 2.0f / rng.uni(0.2f, 2.0f);
        se.material_id = i % 7;
        if (extended) {
            se.n = 2.0f / rng2.uni(0.2f, 3.0f);
            s.se_n2.push_back(2.0f / rng2.uni(0.2f, 3.0f));
        }
        s.superellipsoids.push_back(se);
    }
    for (int i = 0; i < 64; i++) {
        std::vector<std::pair<float, float>> ctrl;
        float y = rng.uni(-1.0f, 0.0f);
        for (int k = 0; k < 8; k++) {
            y += rng.uni(0.1f, 0.5f);
            ctrl.push_back({y, rng.uni(0.1f, 1.6f)});
        }
        auto line = bezier_run(ctrl, 8);
        if (extended) {
            s.lathe_bezier.push_back({(int)(s.bezier_ctrl.size() / 2), (int)ctrl.size()});
            for (auto& q : ctrl) { s.bezier_ctrl.push_back(q.first); s.bezier_ctrl.push_back(q.second); }
        }
        Lathe l;
        std::memset(&l, 0, sizeof(l));
        l.point_offset = (int)s.lathe_points.size();
        l.point_count = (int)line.size();
        l.material_id = i % 7;
        for (auto& q : line) {
            LathePoint p;
            std::memset(&p, 0, sizeof(p));
            p.y = q.first; p.radius = q.second;
            s.lathe_points.push_back(p);
        }
        s.lathes.push_back(l);
    }
    for (int i = 0; i < 64; i++) {
        std::vector<std::pair<float, float>> ctrl;
        for (int k = 0; k < 8; k++) {
            float a = 6.2831853f * ((float)k + rng.uni(0.0f, 0.8f)) / 8.0f;
            float r = rng.uni(0.3f, 0.9f);
            ctrl.push_back({r * std::cos(a), r * std::sin(a)});
        }
        auto line = bezier_run(ctrl, 8);
        if (!line.empty()) line.push_back(line.front());   // closed contour
        if (extended) {
            s.prism_bezier.push_back({(int)(s.bezier_ctrl.size() / 2), (int)ctrl.size()});
            for (auto& q : ctrl) { s.bezier_ctrl.push_back(q.first); s.bezier_ctrl.push_back(q.second); }
        }
        Prism p;
        std::memset(&p, 0, sizeof(p));
        p.center = {rng.uni(-18.0f, 18.0f), 0.0f, rng.uni(-4.0f, 16.0f)};
        p.y_min = 0.0f;
        p.y_max = rng.uni(0.3f, 2.5f);
        p.point_offset = (int)s.prism_points.size();
        p.point_count = (int)line.size();
        p.material_id = i % 7;
        for (auto& q : line) {
            PrismPoint pp;
            std::memset(&pp, 0, sizeof(pp));
            pp.x = q.first; pp.z = q.second;
            s.prism_points.push_back(pp);
        }
        s.prisms.push_back(p);
    }
    for (int i = 0; i < 32; i++) {
        std::vector<SweepPoint> ctrl;
        float x = rng.uni(-16.0f, 16.0f), y = rng.uni(0.5f, 3.0f), z = rng.uni(-4.0f, 14.0f);
        for (int k = 0; k < 6; k++) {
            SweepPoint p;
            p.position = {x, y, z};
            p.radius = rng.uni(0.05f, 0.2f);
            ctrl.push_back(p);
            x += rng.uni(-1.0f, 1.0f); y += rng.uni(-0.3f, 0.8f); z += rng.uni(-1.0f, 1.0f);
        }
        s.add_sweep_smooth(ctrl, i % 7, 8);
    }
    {
        HeightField hf;
        std::memset(&hf, 0, sizeof(hf));
        hf.center = {0.0f, -0.5f, 22.0f};
        hf.size_x = 60.0f; hf.size_z = 16.0f; hf.height = 2.0f;
        hf.freq = 6.0f; hf.octaves = 6; hf.seed = (int)(seed & 0xffff);
        hf.material_id = m_ground;
        s.heightfields.push_back(hf);
        s.height_image_of.push_back(-1);
        if (extended) {
            const int gw = 1024, gh = 1024;
            s.hf_grid.push_back({(int)s.hf_heights.size(), gw, gh});
            std::vector<float> g;
            fbm_grid(rng2.g(), gw, gh, g);
            s.hf_heights.insert(s.hf_heights.end(), g.begin(), g.end());
        }
    }
    {
        // Depth-3 tree: difference(intersection(box, sphere), union(sphere, box)).
        auto sphere = [&](float x, float y, float z, float r) {
            s.add_sphere(x, y, z, r, 7);
            return (int)s.objects.size() - 1;
        };
        auto box = [&](float x, float y, float z, float a, float b, float c) {
            Superellipsoid se;
            std::memset(&se, 0, sizeof(se));
            se.center = {x, y, z}; se.a = a; se.b = b; se.c = c; se.n = 12.0f; se.material_id = 7;
            s.superellipsoids.push_back(se);
            // the extension's array has one entry per superellipsoid: the
            // tree's boxes keep the single-exponent body
            if (extended) s.se_n2.push_back(0.0f);
            return (int)s.superellipsoids.size() - 1;
        };
        auto leaf = [&](int kind, int idx) {
            CSGNode n;
            std::memset(&n, 0, sizeof(n));
            n.leaf_kind = kind; n.leaf_index = idx; n.left = n.right = -1;
            s.csg_nodes.push_back(n);
            return (int)s.csg_nodes.size() - 1;
        };
        auto op = [&](int o, int l, int r) {
            CSGNode n;
            std::memset(&n, 0, sizeof(n));
            n.op = o; n.leaf_kind = -1; n.leaf_index = -1; n.left = l; n.right = r;
            s.csg_nodes.push_back(n);
            return (int)s.csg_nodes.size() - 1;
        };
        int a = leaf(1, box(0.0f, 2.0f, -2.0f, 1.6f, 1.6f, 1.6f));
        int b = leaf(0, sphere(0.0f, 2.0f, -2.0f, 2.0f));
        int c = leaf(0, sphere(0.0f, 2.0f, -3.6f, 1.0f));
        int d = leaf(1, box(1.2f, 3.2f, -2.0f, 0.7f, 0.7f, 2.5f));
        int inter = op(1, a, b);
        int uni = op(0, c, d);
        s.csg_root = op(2, inter, uni);
        if (extended) {
            // 128 further trees of depth 3: op(op(leaf, leaf), op(leaf, leaf))
            // over spheres (Objects of type 1: CSG-only, not drawn as spheres),
            // boxes and cones
            auto ext_leaf = [&](float cx, float cy, float cz, float size, int mat) {
                const int kind = (int)(rng2.u01() * 3.0f) % 3;
                const float ox = rng2.uni(-0.5f, 0.5f) * size, oy = rng2.uni(-0.5f, 0.5f) * size;
                const float oz = rng2.uni(-0.5f, 0.5f) * size;
                if (kind == 0) {
                    Object o;
                    std::memset(&o, 0, sizeof(o));
                    o.type = 1;
                    o.material_id = mat;
                    o.param1 = {cx + ox, cy + oy, cz + oz};
                    o.param2 = rng2.uni(0.35f, 0.7f) * size;
                    s.objects.push_back(o);
                    return leaf(0, (int)s.objects.size() - 1);
                }
                if (kind == 1) {
                    SheenCsgBox b;
                    std::memset(&b, 0, sizeof(b));
                    const float hx = rng2.uni(0.25f, 0.6f) * size, hy = rng2.uni(0.25f, 0.6f) * size;
                    const float hz = rng2.uni(0.25f, 0.6f) * size;
                    b.lo = {cx + ox - hx, cy + oy - hy, cz + oz - hz};
                    b.hi = {cx + ox + hx, cy + oy + hy, cz + oz + hz};
                    b.material_id = mat;
                    s.csg_boxes.push_back(b);
                    return leaf(2, (int)s.csg_boxes.size() - 1);
                }
                SheenCsgCone cn;
                std::memset(&cn, 0, sizeof(cn));
                const float hh = rng2.uni(0.4f, 0.9f) * size;
                float ax = rng2.uni(-0.4f, 0.4f), az = rng2.uni(-0.4f, 0.4f);
                cn.p0 = {cx + ox - ax * hh, cy + oy - hh, cz + oz - az * hh};
                cn.p1 = {cx + ox + ax * hh, cy + oy + hh, cz + oz + az * hh};
                cn.r0 = rng2.uni(0.2f, 0.6f) * size;
                cn.r1 = rng2.uni(0.0f, 0.4f) * size;
                cn.material_id = mat;
                s.csg_cones.push_back(cn);
                return leaf(3, (int)s.csg_cones.size() - 1);
            };
            for (int t = 0; t < 128; t++) {
                const float cx = rng2.uni(-17.0f, 17.0f), cy = rng2.uni(0.8f, 5.0f), cz = rng2.uni(-5.0f, 17.0f);
                const float size = rng2.uni(0.5f, 1.1f);
                const int mat = t % 7;
                const int l0 = ext_leaf(cx, cy, cz, size, mat), l1 = ext_leaf(cx, cy, cz, size, mat);
                const int l2 = ext_leaf(cx, cy, cz, size, mat), l3 = ext_leaf(cx, cy, cz, size, mat);
                const int a0 = op((int)(rng2.u01() * 3.0f) % 3, l0, l1);
                const int a1 = op((int)(rng2.u01() * 3.0f) % 3, l2, l3);
                // the top operation keeps some solid: union or intersection-free difference
                s.csg_roots.push_back(op(rng2.u01() < 0.5f ? 0 : 2, a0, a1));
            }
        }
    }
    s.add_plane(0.0f, 1.0f, 0.0f, 0.5f, m_ground);
    for (int k = 0; k < 2; k++) {
        float px = k ? -14.0f : 14.0f, py = 20.0f, pz = -12.0f;
        s.add_point_light(px, py, pz, 1.0f, 1.0f, 1.0f, 12.5663706f * (px * px + py * py + pz * pz) * 0.5f, 0.0f);
    }
    s.settings.width = 1920; s.settings.height = 1080; s.settings.aa = 4;
}

}  // namespace sheen
