// scene_io.cpp -- the .sheen text scene loader behind sheen_load_scene_file.
//
// Same grammar and defaults as the reference loader (api/scene_io.cpp:216-968)
// so existing .sheen files load unchanged: one command per line, '#' starts a
// comment, positional or key=value arguments per command, OBJ / SMESH1 /
// P6 PPM / P5 PGM / strand-file side inputs, procedural hair, cubic-Bezier
// lathe and prism profiles tessellated on the host, and a prefix CSG tree
// (csg_begin / csg_leaf / csg_end).  After the last line every material
// index outside [0, num_materials) is replaced by 0.
//
// Differences: the CSG builder stack is per file (the reference keeps it in
// a static across files), and errors name the failing line in the message
// returned by sheen_get_last_error() instead of printing to stderr.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "owned_scene.h"

namespace sheen {
void set_error(const char* msg);

namespace {

struct Args {
    std::map<std::string, std::string> kv;
    bool has(const std::string& k) const { return kv.count(k) > 0; }
    float f(const std::string& k, float d) const { auto it = kv.find(k); return it == kv.end() ? d : std::stof(it->second); }
    int i(const std::string& k, int d) const { auto it = kv.find(k); return it == kv.end() ? d : std::stoi(it->second); }
    unsigned u(const std::string& k, unsigned d) const {
        auto it = kv.find(k);
        return it == kv.end() ? d : (unsigned)std::stoul(it->second);
    }
    std::string s(const std::string& k) const { auto it = kv.find(k); return it == kv.end() ? std::string() : it->second; }
    sheen_float3 v3(const std::string& k, sheen_float3 d) const {
        auto it = kv.find(k);
        if (it == kv.end()) return d;
        std::string v = it->second;
        std::replace(v.begin(), v.end(), ',', ' ');
        std::istringstream ss(v);
        float x, y, z;
        if (!(ss >> x >> y >> z)) return d;
        return sheen_float3{x, y, z};
    }
    static Args read(std::istream& in) {
        Args a;
        std::string tok;
        while (in >> tok) {
            size_t eq = tok.find('=');
            if (eq != std::string::npos) a.kv[tok.substr(0, eq)] = tok.substr(eq + 1);
        }
        return a;
    }
};

inline sheen_float3 F3(float x, float y, float z) { return sheen_float3{x, y, z}; }

// True when the next token contains '='; the stream position is restored.
bool next_is_named(std::istringstream& in) {
    std::streampos save = in.tellg();
    std::string first;
    in >> first;
    in.clear();
    in.seekg(save);
    return first.find('=') != std::string::npos;
}

struct Loader {
    OwnedScene& s;
    std::vector<int> csg_stack;
    std::vector<int> se_hidden;
    std::string err;

    explicit Loader(OwnedScene& sc) : s(sc) {}

    int material(float r, float g, float b, float spec, float shin, float amb, float aniso = 0.0f, float shift = 0.1f,
                 float sr = 0.0f, float er = 0.0f, float st = 0.0f, float et = 0.0f, float back = 0.0f) {
        int m = s.add_material(r, g, b, spec, shin, amb);
        Material& M = s.materials[(size_t)m];
        M.anisotropy = aniso; M.hair_shift = shift; M.hair_spec_r = sr; M.hair_exp_r = er;
        M.hair_spec_t = st; M.hair_exp_t = et; M.hair_backlight = back;
        return m;
    }

    void tri(sheen_float3 a, sheen_float3 b, sheen_float3 c, sheen_float3 na, sheen_float3 nb, sheen_float3 nc,
             int mat, sheen_float2 ta = {0, 0}, sheen_float2 tb = {0, 0}, sheen_float2 tc = {0, 0}) {
        Triangle t;
        std::memset(&t, 0, sizeof(t));
        t.v0 = a; t.v1 = b; t.v2 = c; t.n0 = na; t.n1 = nb; t.n2 = nc;
        t.uv0 = ta; t.uv1 = tb; t.uv2 = tc;
        t.material_id = mat;
        s.triangles.push_back(t);
    }

    // 12-triangle cube with per-face 0..1 UVs (the layout of scene.h:271-301).
    void cube(sheen_float3 c, float h, int mat) {
        sheen_float3 v[8];
        int k = 0;
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++)
                for (int l = 0; l < 2; l++) v[k++] = F3(c.x + (i ? h : -h), c.y + (j ? h : -h), c.z + (l ? h : -h));
        static const int f[12][3] = {{0, 1, 3}, {0, 3, 2}, {4, 6, 7}, {4, 7, 5}, {0, 4, 5}, {0, 5, 1},
                                     {2, 3, 7}, {2, 7, 6}, {0, 2, 6}, {0, 6, 4}, {1, 5, 7}, {1, 7, 3}};
        static const int axis[6] = {0, 0, 1, 1, 2, 2};
        auto uv = [&](sheen_float3 p, int a) {
            float u = (a == 0) ? (p.z - (c.z - h)) : (p.x - (c.x - h));
            float w = (a == 1) ? (p.z - (c.z - h)) : (p.y - (c.y - h));
            return sheen_float2{u / (2.0f * h), w / (2.0f * h)};
        };
        const sheen_float3 z = F3(0, 0, 0);
        for (int i = 0; i < 12; i++) {
            int ax = axis[i / 2];
            sheen_float3 a = v[f[i][0]], b = v[f[i][1]], d = v[f[i][2]];
            tri(a, b, d, z, z, z, mat, uv(a, ax), uv(b, ax), uv(d, ax));
        }
    }

    void sweep_smooth(const std::vector<SweepPoint>& pts, int mat, int sub) { s.add_sweep_smooth(pts, mat, sub); }

    // Procedural hair on a head sphere (api/scene_io.cpp:104-155).
    void hair(const Args& p) {
        sheen_float3 c = p.v3("center", F3(0.0f, 1.6f, 0.0f));
        float head = p.f("head", 0.55f);
        int count = p.i("count", 500), segs = p.i("segs", 10);
        unsigned seed = p.u("seed", 1u);
        int mat = p.i("mat", 0);
        float rad = p.f("radius", 0.009f), taper = p.f("taper", 0.55f), len = p.f("length", 0.9f);
        float wob = p.f("wobble", 0.012f), curl = p.f("curl", 0.9f), phi0 = p.f("phi0", 0.15f);
        float phi1 = p.f("phi1", 1.20f), spread = p.f("spread", 1.02f);
        std::mt19937 rng(seed);
        std::uniform_real_distribution<float> U(0.0f, 1.0f);
        for (int i = 0; i < count; i++) {
            float theta = 6.2831853f * U(rng);
            float ph = phi0 + (phi1 - phi0) * U(rng);
            float r0 = rad * (0.75f + 0.5f * U(rng));
            float fall = len * head * (0.6f + 0.8f * U(rng));
            std::vector<SweepPoint> pts;
            sheen_float3 pos = c;
            for (int k = 0; k < segs; k++) {
                float t = (float)k / (float)(segs - 1);
                float phi = ph + t * curl;
                sheen_float3 q;
                if (phi < 1.75f) {
                    float rr = head * (spread + 0.10f * t);
                    q = F3(c.x + rr * sinf(phi) * cosf(theta), c.y + rr * cosf(phi), c.z + rr * sinf(phi) * sinf(theta));
                } else {
                    q = pos;
                    q.y -= fall * t;
                    q.x += sinf(t * 6.0f + i) * wob;
                    q.z += cosf(t * 5.0f + i * 0.7f) * wob;
                }
                pos = q;
                SweepPoint sp;
                sp.position = q;
                sp.radius = r0 * (1.0f - taper * t);
                pts.push_back(sp);
            }
            sweep_smooth(pts, mat, 2);
        }
    }

    // Strands grown from mesh vertices (api/scene_io.cpp:158-214).
    bool hair_mesh(const Args& p) {
        int mat = p.i("mat", 1), count = p.i("count", 500), segs = p.i("segs", 10);
        unsigned seed = p.u("seed", 7u);
        float rad = p.f("radius", 0.004f), taper = p.f("taper", 0.6f), len = p.f("length", 0.25f);
        float wob = p.f("wobble", 0.01f), y0 = p.f("y0", 0.0f), y1 = p.f("y1", 1e9f), lift = p.f("lift", 0.5f);
        auto sub3 = [](sheen_float3 a, sheen_float3 b) { return F3(a.x - b.x, a.y - b.y, a.z - b.z); };
        auto nrm = [](sheen_float3 a) {
            float il = 1.0f / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
            return F3(a.x * il, a.y * il, a.z * il);
        };
        std::vector<sheen_float3> roots, norms;
        for (const Triangle& t : s.triangles) {
            sheen_float3 e1 = sub3(t.v1, t.v0), e2 = sub3(t.v2, t.v0);
            sheen_float3 n = nrm(F3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z, e1.x * e2.y - e1.y * e2.x));
            const sheen_float3 vs[3] = {t.v0, t.v1, t.v2};
            for (int k = 0; k < 3; k++)
                if (vs[k].y >= y0 && vs[k].y <= y1) { roots.push_back(vs[k]); norms.push_back(n); }
        }
        if (roots.empty()) return true;   // the reference warns and continues
        std::mt19937 rng(seed);
        std::uniform_int_distribution<size_t> pick(0, roots.size() - 1);
        for (int i = 0; i < count; i++) {
            size_t idx = pick(rng);
            sheen_float3 n = norms[idx];
            sheen_float3 root = F3(roots[idx].x + n.x * 0.002f, roots[idx].y + n.y * 0.002f, roots[idx].z + n.z * 0.002f);
            sheen_float3 dir = nrm(F3(n.x * lift + 0.0f, n.y * lift - 1.0f, n.z * lift + 0.0f));
            float r0 = rad * (0.7f + 0.6f * (float)(rng() % 1000) / 1000.0f);
            std::vector<SweepPoint> pts;
            sheen_float3 pos = root;
            float step = len / (float)(segs - 1);
            for (int k = 0; k < segs; k++) {
                float t = (float)k / (float)(segs - 1);
                SweepPoint sp;
                sp.position = pos;
                sp.radius = r0 * (1.0f - taper * t);
                pts.push_back(sp);
                sheen_float3 w = F3(sinf(t * 9.0f + i * 1.3f) * wob, 0.0f, cosf(t * 7.0f + i * 0.9f) * wob);
                dir = nrm(F3(dir.x + 0.0f + w.x, dir.y + (-0.6f * step) + w.y, dir.z + 0.0f + w.z));
                pos = F3(pos.x + dir.x * step, pos.y + dir.y * step, pos.z + dir.z * step);
            }
            sweep_smooth(pts, mat, 1);
        }
        return true;
    }

    bool obj(const Args& p) {
        std::string file = p.s("file");
        if (file.empty()) { err = "obj: file= is required"; return false; }
        int mat = p.i("mat", 0);
        sheen_float3 off = p.v3("offset", F3(0, 0, 0));
        float sc = p.f("scale", 1.0f);
        bool smooth = p.i("smooth", 1) != 0;
        std::ifstream f(file);
        if (!f) { err = "obj: cannot open " + file; return false; }
        std::vector<sheen_float3> verts, norms;
        std::vector<sheen_float2> uvs;
        std::string line;
        int faces = 0;
        while (std::getline(f, line)) {
            if (line.size() < 2) continue;
            std::istringstream ls(line);
            std::string tag;
            ls >> tag;
            if (tag == "v") {
                float x, y, z; ls >> x >> y >> z;
                verts.push_back(F3(x * sc + off.x, y * sc + off.y, z * sc + off.z));
            } else if (tag == "vn") {
                float x, y, z; ls >> x >> y >> z;
                norms.push_back(F3(x, y, z));
            } else if (tag == "vt") {
                float u, v; ls >> u >> v;
                uvs.push_back(sheen_float2{u, v});
            } else if (tag == "f") {
                std::vector<int> vi, ni, ti;
                std::string tok;
                bool bad = false;
                while (ls >> tok) {
                    int a = 0, b = 0, c = 0;
                    int got = std::sscanf(tok.c_str(), "%d/%d/%d", &a, &b, &c);
                    if (got < 2) b = 0;
                    if (got == 1) {
                        c = 0;
                        if (std::sscanf(tok.c_str(), "%d//%d", &a, &c) != 2) c = 0;
                    }
                    int v = a < 0 ? (int)verts.size() + a : a - 1;
                    int n = c == 0 ? -1 : (c < 0 ? (int)norms.size() + c : c - 1);
                    int t = b == 0 ? -1 : (b < 0 ? (int)uvs.size() + b : b - 1);
                    if (v < 0 || v >= (int)verts.size()) { bad = true; break; }
                    vi.push_back(v); ni.push_back(n); ti.push_back(t);
                }
                if (bad || vi.size() < 3) continue;
                auto nn = [&](int slot) {
                    int k = ni[(size_t)slot];
                    return (smooth && k >= 0 && k < (int)norms.size()) ? norms[(size_t)k] : F3(0, 0, 0);
                };
                auto tt = [&](int slot) {
                    int k = ti[(size_t)slot];
                    return (k >= 0 && k < (int)uvs.size()) ? uvs[(size_t)k] : sheen_float2{0, 0};
                };
                for (size_t k = 2; k < vi.size(); k++) {   // fan triangulation
                    int a = 0, b = (int)k - 1, c = (int)k;
                    tri(verts[(size_t)vi[(size_t)a]], verts[(size_t)vi[(size_t)b]], verts[(size_t)vi[(size_t)c]],
                        nn(a), nn(b), nn(c), mat, tt(a), tt(b), tt(c));
                    faces++;
                }
            }
        }
        if (!faces) { err = "obj: no faces in " + file; return false; }
        return true;
    }

    bool texture(const Args& p) {
        std::string file = p.s("file");
        int max_dim = p.i("max", 2048);
        if (file.empty()) { err = "texture: file= is required"; return false; }
        std::ifstream tf(file, std::ios::binary);
        if (!tf) { err = "texture: cannot open " + file; return false; }
        std::string magic;
        int w = 0, h = 0, maxv = 0;
        tf >> magic >> w >> h >> maxv;
        if (magic != "P6" || w <= 0 || h <= 0 || w > 16384 || h > 16384) { err = "texture: P6 PPM expected"; return false; }
        tf.get();
        std::vector<uint8_t> raw((size_t)w * h * 3);
        tf.read(reinterpret_cast<char*>(raw.data()), (std::streamsize)raw.size());
        if (!tf || tf.gcount() != (std::streamsize)raw.size()) { err = "texture: file shorter than its header"; return false; }
        int step = 1;
        while (w / step > max_dim || h / step > max_dim) step++;
        Texture t;
        if (step > 1) {
            t.w = w / step; t.h = h / step;
            t.rgb.resize((size_t)t.w * t.h * 3);
            for (int y = 0; y < t.h; y++)
                for (int x = 0; x < t.w; x++)
                    for (int c = 0; c < 3; c++)
                        t.rgb[((size_t)y * t.w + x) * 3 + c] = raw[((size_t)(y * step) * w + (size_t)(x * step)) * 3 + c];
        } else {
            t.w = w; t.h = h; t.rgb.swap(raw);
        }
        s.textures.push_back(std::move(t));
        return true;
    }

    bool mesh(const Args& p) {
        std::string file = p.s("file");
        int mat_base = p.i("mat0", 0);
        float sc = p.f("scale", 1.0f);
        if (file.empty()) { err = "mesh: file= is required"; return false; }
        std::ifstream mf(file, std::ios::binary);
        if (!mf) { err = "mesh: cannot open " + file; return false; }
        char magic[8] = {0};
        mf.read(magic, 8);
        if (std::string(magic, 6) != "SMESH1") { err = "mesh: not an SMESH1 file"; return false; }
        uint32_t nv = 0, nn = 0, nu = 0, nt = 0;
        mf.read((char*)&nv, 4); mf.read((char*)&nn, 4); mf.read((char*)&nu, 4); mf.read((char*)&nt, 4);
        mf.seekg(0, std::ios::end);
        uint64_t fsize = (uint64_t)mf.tellg();
        mf.seekg(24, std::ios::beg);
        uint64_t need = 24ull + (uint64_t)nv * 12 + (uint64_t)nn * 12 + (uint64_t)nu * 8 + (uint64_t)nt * 40;
        if (fsize < need || nv > 50000000u || nt > 50000000u) { err = "mesh: corrupt header"; return false; }
        std::vector<sheen_float3> verts(nv), norms(nn);
        std::vector<sheen_float2> uvs(nu);
        mf.read((char*)verts.data(), (std::streamsize)nv * 12);
        mf.read((char*)norms.data(), (std::streamsize)nn * 12);
        mf.read((char*)uvs.data(), (std::streamsize)nu * 8);
        struct Rec { int32_t v[3], n[3], t[3], mat; };
        std::vector<Rec> tris(nt);
        mf.read((char*)tris.data(), (std::streamsize)nt * (std::streamsize)sizeof(Rec));
        std::vector<int> skip;
        if (p.has("skip")) {
            std::string sk = p.s("skip");
            std::replace(sk.begin(), sk.end(), ',', ' ');
            std::istringstream ss(sk);
            int v;
            while (ss >> v) skip.push_back(v);
        }
        for (const Rec& t : tris) {
            if (std::find(skip.begin(), skip.end(), mat_base + t.mat) != skip.end()) continue;
            auto vv = [&](int k) { sheen_float3 q = verts[(size_t)t.v[k]]; return F3(q.x * sc, q.y * sc, q.z * sc); };
            auto nm = [&](int k) { return (t.n[k] >= 0 && t.n[k] < (int)norms.size()) ? norms[(size_t)t.n[k]] : F3(0, 0, 0); };
            auto tc = [&](int k) { return (t.t[k] >= 0 && t.t[k] < (int)uvs.size()) ? uvs[(size_t)t.t[k]] : sheen_float2{0, 0}; };
            tri(vv(0), vv(1), vv(2), nm(0), nm(1), nm(2), mat_base + t.mat, tc(0), tc(1), tc(2));
        }
        return true;
    }

    bool strands(const Args& p) {
        std::string file = p.s("file");
        int mat = p.i("mat", 1);
        float scale = p.f("scale", 1.0f), rad_override = p.f("radius", 0.0f);
        if (file.empty()) { err = "strands: file= is required"; return false; }
        std::ifstream f(file);
        if (!f) { err = "strands: cannot open " + file; return false; }
        std::string line;
        while (std::getline(f, line)) {
            std::istringstream ls(line);
            std::string tag;
            ls >> tag;
            if (tag != "strand") continue;
            float r0, r1;
            int cnt;
            ls >> r0 >> r1 >> cnt;
            if (cnt < 2 || cnt > 100000) continue;
            std::vector<SweepPoint> pts;
            for (int i = 0; i < cnt; i++) {
                float x, y, z;
                if (!(ls >> x >> y >> z)) break;
                float t = (float)i / (float)(cnt - 1);
                SweepPoint sp;
                sp.position = F3(x * scale, y * scale, z * scale);
                sp.radius = rad_override > 0.0f ? rad_override * scale : (r0 + (r1 - r0) * t) * scale;
                pts.push_back(sp);
            }
            if (pts.size() < 2) continue;
            const size_t chunk = 8;   // long strands are cut so their BVH boxes stay tight
            if (pts.size() <= chunk) {
                sweep_smooth(pts, mat, 1);
            } else {
                for (size_t a = 0; a + 1 < pts.size(); a += chunk - 1) {
                    size_t b = std::min(a + chunk, pts.size());
                    std::vector<SweepPoint> part(pts.begin() + (long)a, pts.begin() + (long)b);
                    if (part.size() >= 2) sweep_smooth(part, mat, 1);
                }
            }
        }
        return true;
    }

    // Cubic Bezier runs: groups of 4 control points, `sub` pieces per span.
    static std::vector<std::pair<float, float>> bezier(const std::vector<std::pair<float, float>>& c, int sub) {
        std::vector<std::pair<float, float>> out;
        if (c.size() < 4) return out;
        if (sub < 1) sub = 1;
        out.push_back(c[0]);
        for (size_t s0 = 0; s0 + 3 < c.size(); s0 += 4)
            for (int k = 1; k <= sub; k++) {
                float t = (float)k / (float)sub, u = 1.0f - t;
                float w0 = u * u * u, w1 = 3.0f * u * u * t, w2 = 3.0f * u * t * t, w3 = t * t * t;
                out.push_back({w0 * c[s0].first + w1 * c[s0 + 1].first + w2 * c[s0 + 2].first + w3 * c[s0 + 3].first,
                               w0 * c[s0].second + w1 * c[s0 + 1].second + w2 * c[s0 + 2].second + w3 * c[s0 + 3].second});
            }
        return out;
    }

    void add_lathe(sheen_float3 c, const std::vector<std::pair<float, float>>& prof, int mat) {
        Lathe l;
        std::memset(&l, 0, sizeof(l));
        l.center = c;
        l.point_offset = (int)s.lathe_points.size();
        l.point_count = (int)prof.size();
        l.material_id = mat;
        for (auto& q : prof) {
            LathePoint p;
            std::memset(&p, 0, sizeof(p));
            p.y = q.first; p.radius = q.second;
            s.lathe_points.push_back(p);
        }
        s.lathes.push_back(l);
    }

    void add_prism(sheen_float3 c, const std::vector<std::pair<float, float>>& pts, float y0, float y1, float sweep, int mat) {
        Prism p;
        std::memset(&p, 0, sizeof(p));
        p.center = c; p.y_min = y0; p.y_max = y1; p.sweep = sweep;
        p.point_offset = (int)s.prism_points.size();
        p.point_count = (int)pts.size();
        p.material_id = mat;
        for (auto& q : pts) {
            PrismPoint pp;
            std::memset(&pp, 0, sizeof(pp));
            pp.x = q.first; pp.z = q.second;
            s.prism_points.push_back(pp);
        }
        s.prisms.push_back(p);
    }

    bool line(std::istringstream& in) {
        std::string cmd;
        in >> cmd;
        if (cmd.empty() || cmd[0] == '#') return true;
        SheenSceneSettings& st = s.settings;
        if (cmd == "resolution") {
            if (next_is_named(in)) {
                Args p = Args::read(in);
                st.width = p.i("width", st.width); st.height = p.i("height", st.height); st.aa = p.i("aa", st.aa);
                if (p.has("out")) std::snprintf(st.output, sizeof(st.output), "%s", p.s("out").c_str());
                return true;
            }
            std::string out;
            in >> st.width >> st.height >> st.aa >> out;
            if (!out.empty()) std::snprintf(st.output, sizeof(st.output), "%s", out.c_str());
            return true;
        }
        if (cmd == "camera") {
            CameraData& c = s.camera;
            if (next_is_named(in)) {
                Args p = Args::read(in);
                c.position = p.v3("loc", F3(0.0f, 0.0f, 3.0f));
                c.right = p.v3("right", F3(1.0f, 0.0f, 0.0f));
                c.up = p.v3("up", F3(0.0f, 1.0f, 0.0f));
                c.forward = p.v3("fwd", F3(0.0f, 0.0f, -1.0f));
                c.focal_length = p.f("lens", 50.0f);
                c.sensor_width = p.f("sensor", 36.0f);
                c.shift_x = p.f("shift_x", 0.0f);
                c.shift_y = p.f("shift_y", 0.0f);
                return true;
            }
            float px, py, pz, fx, fy, fz;
            in >> px >> py >> pz >> fx >> fy >> fz;
            c.position = F3(px, py, pz);
            c.forward = F3(fx, fy, fz);
            c.right = F3(1.0f, 0.0f, 0.0f);
            c.up = F3(0.0f, 1.0f, 0.0f);
            c.focal_length = 0.0f;
            return true;
        }
        if (cmd == "material") {
            if (next_is_named(in)) {
                Args p = Args::read(in);
                sheen_float3 col = p.v3("diffuse", F3(0.8f, 0.8f, 0.8f));
                int m = material(col.x, col.y, col.z, p.f("spec", 0.0f), p.f("shin", 32.0f), p.f("amb", 0.1f),
                                 p.f("aniso", 0.0f), p.f("shift", 0.1f), p.f("spec_r", 0.0f), p.f("exp_r", 0.0f),
                                 p.f("spec_t", 0.0f), p.f("exp_t", 0.0f), p.f("back", 0.0f));
                Material& M = s.materials[(size_t)m];
                if (p.has("tex")) M.texture_id = p.i("tex", -1);
                if (p.has("mask")) M.mask_id = p.i("mask", -1);
                if (p.has("normal")) M.normal_id = p.i("normal", -1);
                if (p.has("nstr")) M.normal_strength = p.f("nstr", 1.0f);
                return true;
            }
            float r, g, b, spec, shin, amb;
            in >> r >> g >> b >> spec >> shin >> amb;
            float aniso = 0, shift = 0.1f, sr = 0, er = 0, st2 = 0, et = 0, back = 0;
            if (!(in >> aniso)) { material(r, g, b, spec, shin, amb); return true; }
            in >> shift >> sr >> er >> st2 >> et >> back;
            material(r, g, b, spec, shin, amb, aniso, shift, sr, er, st2, et, back);
            return true;
        }
        if (cmd == "sphere") {
            float x, y, z, r; int m;
            in >> x >> y >> z >> r >> m;
            s.add_sphere(x, y, z, r, m);
            return true;
        }
        if (cmd == "plane") {
            float nx, ny, nz, d; int m;
            in >> nx >> ny >> nz >> d >> m;
            s.add_plane(nx, ny, nz, d, m);
            return true;
        }
        if (cmd == "cube") {
            float x, y, z, h; int m;
            in >> x >> y >> z >> h >> m;
            cube(F3(x, y, z), h, m);
            return true;
        }
        if (cmd == "obj") return obj(Args::read(in));
        if (cmd == "triangle") {
            float a[9]; int m;
            for (float& v : a) in >> v;
            in >> m;
            const sheen_float3 z = F3(0, 0, 0);
            tri(F3(a[0], a[1], a[2]), F3(a[3], a[4], a[5]), F3(a[6], a[7], a[8]), z, z, z, m);
            return true;
        }
        if (cmd == "grid") {
            int nx, nz, matmod;
            float step, y, rad;
            in >> nx >> nz >> step >> y >> rad >> matmod;
            if ((long long)nx * nz > 2000000) { err = "grid: too many spheres"; return false; }
            for (int i = 0; i < nx * nz; i++) {
                float x = (i % nx) * step - nx * step * 0.5f;
                float z = (i / nx) * step - 2.0f;
                s.add_sphere(x, y, z, rad, matmod > 0 ? (i % matmod) : 0);
            }
            return true;
        }
        if (cmd == "hair") {
            Args p;
            if (!next_is_named(in)) {
                float cx, cy, cz, head; int count, segs, mat; unsigned seed;
                in >> cx >> cy >> cz >> head >> count >> segs >> seed >> mat;
                std::stringstream ss;
                ss << "center=" << cx << "," << cy << "," << cz << " head=" << head << " count=" << count
                   << " segs=" << segs << " seed=" << seed << " mat=" << mat;
                std::istringstream rebuilt(ss.str());
                p = Args::read(rebuilt);
            } else {
                p = Args::read(in);
            }
            hair(p);
            return true;
        }
        if (cmd == "hair_mesh") return hair_mesh(Args::read(in));
        if (cmd == "texture") return texture(Args::read(in));
        if (cmd == "mesh") return mesh(Args::read(in));
        if (cmd == "strands") return strands(Args::read(in));
        if (cmd == "light" || cmd == "fill_light") {
            float dx, dy, dz, r, g, b, it;
            in >> dx >> dy >> dz >> r >> g >> b >> it;
            Light l = OwnedScene::default_light();
            l.type = 0;
            float il = 1.0f / std::sqrt(dx * dx + dy * dy + dz * dz);
            l.direction = F3(dx * il, dy * il, dz * il);
            l.color = F3(r, g, b);
            l.intensity = it;
            if (cmd == "fill_light") l.flags = 0;
            s.lights.push_back(l);
            return true;
        }
        if (cmd == "point") {
            float cx, cy, cz, r, g, b, power, radius;
            in >> cx >> cy >> cz >> r >> g >> b >> power >> radius;
            s.add_point_light(cx, cy, cz, r, g, b, power, radius);
            return true;
        }
        if (cmd == "spot") {
            float v[14];
            for (float& x : v) in >> x;
            const float pos[3] = {v[0], v[1], v[2]}, dir[3] = {v[3], v[4], v[5]}, col[3] = {v[6], v[7], v[8]};
            s.add_spot_light(pos, dir, col, v[9], v[10] * 0.5f, v[11], v[12], v[13]);   // full cone angle in the file
            return true;
        }
        if (cmd == "area") {
            float cx, cy, cz, sx, sy, r, g, b, power;
            in >> cx >> cy >> cz >> sx >> sy >> r >> g >> b >> power;
            Light l = OwnedScene::default_light();
            l.type = 2;
            l.position = F3(cx, cy, cz);
            l.u_axis = F3(sx * 0.5f, 0.0f, 0.0f);
            l.v_axis = F3(0.0f, 0.0f, sy * 0.5f);
            l.color = F3(r, g, b);
            l.intensity = power;
            s.lights.push_back(l);
            return true;
        }
        if (cmd == "reflect") {
            int idx; float v;
            in >> idx >> v;
            if (idx >= 0 && idx < (int)s.materials.size()) s.materials[(size_t)idx].reflect = v;
            return true;
        }
        if (cmd == "sun_angle") {
            float a;
            in >> a;
            if (!s.lights.empty()) s.lights.back().angle = a;
            return true;
        }
        if (cmd == "photons") { int n; in >> n; st.photons = n; return true; }
        if (cmd == "caustics") { float v; in >> v; st.caustics = v; return true; }
        if (cmd == "photon_cell") { float v; in >> v; if (v > 0.0f) st.photon_cell = v; return true; }
        if (cmd == "emit") {
            int idx; float r, g, b, k;
            in >> idx >> r >> g >> b >> k;
            if (idx >= 0 && idx < (int)s.materials.size()) {
                s.materials[(size_t)idx].emission_color = F3(r, g, b);
                s.materials[(size_t)idx].emission = k;
            }
            return true;
        }
        if (cmd == "glass") {
            int idx; float t, ior;
            in >> idx >> t >> ior;
            if (idx >= 0 && idx < (int)s.materials.size()) {
                s.materials[(size_t)idx].transmission = t;
                s.materials[(size_t)idx].ior = ior;
            }
            return true;
        }
        if (cmd == "gobo") {
            int li, ti;
            in >> li >> ti;
            if (li >= 0 && li < (int)s.lights.size()) s.lights[(size_t)li].texture_id = ti;
            return true;
        }
        if (cmd == "media") {
            float v[10]; int samples;
            for (float& x : v) in >> x;
            in >> samples;
            Medium m;
            std::memset(&m, 0, sizeof(m));
            m.center = F3(v[0], v[1], v[2]); m.half = F3(v[3], v[4], v[5]); m.sigma_s = F3(v[6], v[7], v[8]);
            m.sigma_t = v[9]; m.samples = samples;
            s.media.push_back(m);
            return true;
        }
        if (cmd == "hf") {
            float cx, cy, cz, sx, sz, h, freq; int oct, seed, mat;
            in >> cx >> cy >> cz >> sx >> sz >> h >> freq >> oct >> seed >> mat;
            HeightField f;
            std::memset(&f, 0, sizeof(f));
            f.center = F3(cx, cy, cz); f.size_x = sx; f.size_z = sz; f.height = h; f.freq = freq;
            f.octaves = oct; f.seed = seed; f.material_id = mat;
            s.heightfields.push_back(f);
            s.height_image_of.push_back(-1);
            return true;
        }
        if (cmd == "hf_image") {
            float cx, cy, cz, sx, sz, h; std::string file; int mat;
            in >> cx >> cy >> cz >> sx >> sz >> h >> file >> mat;
            std::ifstream imf(file, std::ios::binary);
            if (!imf) { err = "hf_image: cannot open " + file; return false; }
            std::string magic;
            int w = 0, hh = 0, maxv = 0;
            imf >> magic >> w >> hh >> maxv;
            if (magic != "P5" || w <= 0 || hh <= 0 || w > 16384 || hh > 16384) { err = "hf_image: P5 PGM expected"; return false; }
            imf.get();
            std::vector<uint8_t> pix((size_t)w * hh);
            imf.read(reinterpret_cast<char*>(pix.data()), (std::streamsize)pix.size());
            if (!imf || imf.gcount() != (std::streamsize)pix.size()) { err = "hf_image: file shorter than its header"; return false; }
            HeightField f;
            std::memset(&f, 0, sizeof(f));
            f.center = F3(cx, cy, cz); f.size_x = sx; f.size_z = sz; f.height = h; f.freq = 1.0f;
            f.octaves = 1; f.seed = -1; f.material_id = mat; f.img_w = w; f.img_h = hh;
            s.heightfields.push_back(f);
            s.height_images.push_back(std::move(pix));
            s.height_image_of.push_back((int)s.height_images.size() - 1);
            return true;
        }
        if (cmd == "se" || cmd == "se_csg") {
            float cx, cy, cz, a, b, c, n; int mat;
            in >> cx >> cy >> cz >> a >> b >> c >> n >> mat;
            Superellipsoid e;
            std::memset(&e, 0, sizeof(e));
            e.center = F3(cx, cy, cz); e.a = a; e.b = b; e.c = c; e.n = n; e.material_id = mat;
            s.superellipsoids.push_back(e);
            if (cmd == "se_csg") se_hidden.push_back((int)s.superellipsoids.size() - 1);
            return true;
        }
        if (cmd == "lathe") {
            float cx, cy, cz; int mat, n;
            in >> cx >> cy >> cz >> mat >> n;
            if (n > 0 && n <= 512) {
                std::vector<std::pair<float, float>> prof;
                for (int i = 0; i < n; i++) { float y, r; in >> y >> r; prof.push_back({y, r}); }
                add_lathe(F3(cx, cy, cz), prof, mat);
            }
            return true;
        }
        if (cmd == "lathe_bezier") {
            float cx, cy, cz; int mat, sub, n;
            in >> cx >> cy >> cz >> mat >> sub >> n;
            if (n > 0 && n <= 2048 && sub >= 1 && sub <= 64) {
                std::vector<std::pair<float, float>> ctrl;
                for (int i = 0; i < n; i++) { float y, r; in >> y >> r; ctrl.push_back({y, r}); }
                ctrl.resize(ctrl.size() / 4 * 4);
                add_lathe(F3(cx, cy, cz), bezier(ctrl, sub), mat);
            }
            return true;
        }
        if (cmd == "prism_bezier" || cmd == "prism") {
            const bool bz = cmd == "prism_bezier";
            float cx, cy, cz, y1, y2, sweep; int mat, sub = 1, n;
            in >> cx >> cy >> cz >> y1 >> y2 >> sweep >> mat;
            if (bz) in >> sub;
            in >> n;
            if (n > 0 && n <= 2048 && (!bz || (sub >= 1 && sub <= 64))) {
                std::vector<std::pair<float, float>> pts;
                for (int i = 0; i < n; i++) { float x, z; in >> x >> z; pts.push_back({x, z}); }
                if (bz) {
                    pts.resize(pts.size() / 4 * 4);
                    pts = bezier(pts, sub);
                    if (!pts.empty()) pts.push_back(pts.front());   // closed contour
                }
                add_prism(F3(cx, cy, cz), pts, y1, y2, sweep, mat);
            }
            return true;
        }
        if (cmd == "csg_begin") {
            int op;
            in >> op;
            CSGNode n;
            std::memset(&n, 0, sizeof(n));
            n.op = op; n.leaf_kind = -1; n.leaf_index = -1; n.left = n.right = -1;
            s.csg_nodes.push_back(n);
            csg_stack.push_back((int)s.csg_nodes.size() - 1);
            return true;
        }
        if (cmd == "csg_leaf") {
            int kind, idx;
            in >> kind >> idx;
            CSGNode n;
            std::memset(&n, 0, sizeof(n));
            n.op = 0; n.leaf_kind = kind; n.leaf_index = idx; n.left = n.right = -1;
            s.csg_nodes.push_back(n);
            if (!csg_stack.empty()) {
                CSGNode& par = s.csg_nodes[(size_t)csg_stack.back()];
                if (par.left < 0) par.left = (int)s.csg_nodes.size() - 1;
                else par.right = (int)s.csg_nodes.size() - 1;
            }
            return true;
        }
        if (cmd == "csg_end") {
            if (!csg_stack.empty()) {
                int cur = csg_stack.back();
                csg_stack.pop_back();
                if (!csg_stack.empty()) {
                    CSGNode& par = s.csg_nodes[(size_t)csg_stack.back()];
                    if (par.left < 0) par.left = cur; else par.right = cur;
                } else {
                    s.csg_root = cur;
                }
            }
            return true;
        }
        if (cmd == "sweep" || cmd == "sweep_smooth") {
            int mat, sub;
            in >> mat >> sub;
            std::vector<SweepPoint> pts;
            float x, y, z, r;
            while (in >> x >> y >> z >> r) {
                SweepPoint p;
                p.position = F3(x, y, z);
                p.radius = r;
                pts.push_back(p);
            }
            if (pts.size() < 2) { err = "sweep: at least two points are required"; return false; }
            if (sub > 0) sweep_smooth(pts, mat, sub);
            else s.add_sweep(pts, mat);
            return true;
        }
        err = "unknown command: " + cmd;
        return false;
    }
};

}  // namespace
}  // namespace sheen

extern "C" int sheen_load_scene_file(const char* path, SheenOwnedScene* out) {
    using namespace sheen;
    if (!out) { set_error("null output handle"); return -1; }
    *out = nullptr;
    if (!path) { set_error("null path"); return -1; }
    std::ifstream f(path);
    if (!f) { set_error((std::string("cannot open scene: ") + path).c_str()); return -1; }
    OwnedScene* s = new OwnedScene();
    Loader L(*s);
    std::string text;
    int line_no = 0;
    while (std::getline(f, text)) {
        line_no++;
        size_t hash = text.find('#');
        if (hash != std::string::npos) text = text.substr(0, hash);
        std::istringstream in(text);
        bool ok;
        try {
            ok = L.line(in);
        } catch (const std::exception& e) {
            L.err = std::string("bad number: ") + e.what();
            ok = false;
        }
        if (!ok) {
            std::string msg = "line " + std::to_string(line_no) + ": " + text + " (" + L.err + ")";
            set_error(msg.c_str());
            delete s;
            return -1;
        }
    }
    const int nm = (int)s->materials.size();
    auto clamp = [&](int& m) { if (nm > 0 && (m < 0 || m >= nm)) m = 0; };
    for (auto& x : s->sweep_strands) clamp(x.material_id);
    for (auto& x : s->triangles) clamp(x.material_id);
    for (auto& x : s->objects) clamp(x.material_id);
    for (auto& x : s->planes) clamp(x.material_id);
    for (auto& x : s->heightfields) clamp(x.material_id);
    for (auto& x : s->superellipsoids) clamp(x.material_id);
    for (auto& x : s->lathes) clamp(x.material_id);
    for (auto& x : s->prisms) clamp(x.material_id);
    s->finalize();
    *out = reinterpret_cast<SheenOwnedScene>(s);
    return 0;
}
