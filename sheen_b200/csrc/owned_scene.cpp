// owned_scene.cpp -- OwnedScene builders and the C view behind SheenOwnedScene.
#include "owned_scene.h"

#include <cmath>
#include <cstring>

namespace sheen {

static sheen_float3 f3(float x, float y, float z) { return sheen_float3{x, y, z}; }

OwnedScene::OwnedScene() {
    settings.width = 800;
    settings.height = 600;
    settings.aa = 4;
    settings.photons = 0;
    settings.photon_cell = 0.25f;
    settings.caustics = 0.0f;
    std::strcpy(settings.output, "scene_output.png");
}

void OwnedScene::finalize() {
    // Height-map images are owned here; point each HF at its copy.
    for (size_t i = 0; i < heightfields.size(); i++) {
        int k = i < height_image_of.size() ? height_image_of[i] : -1;
        if (k >= 0) heightfields[i].image = height_images[(size_t)k].data();
    }
    tex_ptrs.clear(); tex_w.clear(); tex_h.clear();
    for (const Texture& t : textures) {
        tex_ptrs.push_back(t.rgb.empty() ? nullptr : t.rgb.data());
        tex_w.push_back(t.w);
        tex_h.push_back(t.h);
    }
    SheenScene& v = view;
    std::memset(&v, 0, sizeof(v));
    v.camera = camera;
#define SHEEN_VIEW(field) \
    v.field = field.empty() ? nullptr : field.data(); v.num_##field = (int)field.size();
    SHEEN_VIEW(objects)
    SHEEN_VIEW(sweep_points)
    SHEEN_VIEW(sweep_strands)
    SHEEN_VIEW(triangles)
    SHEEN_VIEW(heightfields)
    SHEEN_VIEW(superellipsoids)
    SHEEN_VIEW(lathe_points)
    SHEEN_VIEW(lathes)
    SHEEN_VIEW(prism_points)
    SHEEN_VIEW(prisms)
    SHEEN_VIEW(csg_nodes)
    SHEEN_VIEW(planes)
    SHEEN_VIEW(materials)
    SHEEN_VIEW(lights)
    SHEEN_VIEW(media)
#undef SHEEN_VIEW
    v.csg_root = csg_root;
    {
        SheenSceneExt& x = ext_view;
        std::memset(&x, 0, sizeof(x));
        // per-primitive extension arrays cover every primitive (the library
        // reads one entry per superellipsoid / heightfield / lathe / prism)
        if (!se_n2.empty()) se_n2.resize(superellipsoids.size(), 0.0f);
        if (!hf_grid.empty()) hf_grid.resize(heightfields.size(), SheenHeightGrid{-1, 0, 0});
        if (!lathe_bezier.empty()) lathe_bezier.resize(lathes.size(), SheenBezierRun{0, 0});
        if (!prism_bezier.empty()) prism_bezier.resize(prisms.size(), SheenBezierRun{0, 0});
        auto ptr = [](const auto& vec) { return vec.empty() ? nullptr : vec.data(); };
        x.lathe_bezier = ptr(lathe_bezier);
        x.prism_bezier = ptr(prism_bezier);
        x.bezier_ctrl = ptr(bezier_ctrl);
        x.num_bezier_ctrl = (int)(bezier_ctrl.size() / 2);
        x.se_n2 = ptr(se_n2);
        x.hf_grid = ptr(hf_grid);
        x.hf_heights = ptr(hf_heights);
        x.num_hf_heights = (int)hf_heights.size();
        x.csg_roots = ptr(csg_roots);
        x.num_csg_roots = (int)csg_roots.size();
        x.csg_boxes = ptr(csg_boxes);
        x.num_csg_boxes = (int)csg_boxes.size();
        x.csg_cones = ptr(csg_cones);
        x.num_csg_cones = (int)csg_cones.size();
        x.max_depth = max_depth;
        x.mesh_triangles = ptr(mesh_triangles);
        x.num_mesh_triangles = (int)mesh_triangles.size();
        x.meshes = ptr(meshes);
        x.num_meshes = (int)meshes.size();
        x.instances = ptr(instances);
        x.num_instances = (int)instances.size();
    }
    v.texture_pixels = tex_ptrs.empty() ? nullptr : tex_ptrs.data();
    v.texture_widths = tex_w.empty() ? nullptr : tex_w.data();
    v.texture_heights = tex_h.empty() ? nullptr : tex_h.data();
    v.num_textures = (int)textures.size();
    v.photons = settings.photons;
    v.photon_cell = settings.photon_cell;
    v.caustics = settings.caustics;
}

int OwnedScene::add_material(float r, float g, float b, float spec, float shin, float amb) {
    Material m;
    std::memset(&m, 0, sizeof(m));
    m.diffuse_color = f3(r, g, b);
    m.specular = spec;
    m.shininess = shin;
    m.ambient = amb;
    m.hair_shift = 0.1f;
    m.texture_id = -1;
    m.mask_id = -1;
    m.normal_id = -1;
    m.ior = 1.45f;
    m.normal_strength = 1.0f;
    materials.push_back(m);
    return (int)materials.size() - 1;
}

void OwnedScene::add_sphere(float x, float y, float z, float rad, int mat) {
    Object o;
    std::memset(&o, 0, sizeof(o));
    o.type = 0;
    o.material_id = mat;
    o.param1 = f3(x, y, z);
    o.param2 = rad;
    objects.push_back(o);
}

void OwnedScene::add_plane(float nx, float ny, float nz, float d, int mat) {
    Plane p;
    std::memset(&p, 0, sizeof(p));
    p.normal = f3(nx, ny, nz);
    p.d = d;
    p.material_id = mat;
    planes.push_back(p);
}

void OwnedScene::add_triangle(const float v[9], const float n[9], const float uv[6], int mat) {
    Triangle t;
    std::memset(&t, 0, sizeof(t));
    t.v0 = f3(v[0], v[1], v[2]);
    t.v1 = f3(v[3], v[4], v[5]);
    t.v2 = f3(v[6], v[7], v[8]);
    if (n) {
        t.n0 = f3(n[0], n[1], n[2]);
        t.n1 = f3(n[3], n[4], n[5]);
        t.n2 = f3(n[6], n[7], n[8]);
    }
    if (uv) {
        t.uv0 = sheen_float2{uv[0], uv[1]};
        t.uv1 = sheen_float2{uv[2], uv[3]};
        t.uv2 = sheen_float2{uv[4], uv[5]};
    }
    t.material_id = mat;
    triangles.push_back(t);
}

Light OwnedScene::default_light() {
    Light l;
    std::memset(&l, 0, sizeof(l));
    l.direction = f3(0.0f, 0.0f, -1.0f);
    l.color = f3(1.0f, 1.0f, 1.0f);
    l.intensity = 1.0f;
    l.flags = 1;
    l.texture_id = -1;
    return l;
}

void OwnedScene::add_point_light(float x, float y, float z, float r, float g, float b,
                                 float power, float radius) {
    Light l = default_light();
    l.type = 1;
    l.position = f3(x, y, z);
    l.color = f3(r, g, b);
    l.intensity = power;
    l.radius = radius;
    lights.push_back(l);
}

void OwnedScene::add_spot_light(const float pos[3], const float dir[3], const float col[3],
                                float power, float half_angle, float blend, float radius,
                                float beam) {
    Light l = default_light();
    l.type = 3;
    l.position = f3(pos[0], pos[1], pos[2]);
    float n = 1.0f / std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    l.direction = f3(dir[0] * n, dir[1] * n, dir[2] * n);
    l.color = f3(col[0], col[1], col[2]);
    l.intensity = power;
    l.radius = radius;
    l.angle = half_angle;
    l.blend = blend;
    l.beam = beam;
    lights.push_back(l);
}

void OwnedScene::add_sweep(const std::vector<SweepPoint>& pts, int mat) {
    SweepStrand s;
    std::memset(&s, 0, sizeof(s));
    s.point_offset = (int)sweep_points.size();
    s.point_count = (int)pts.size();
    s.material_id = mat;
    sweep_points.insert(sweep_points.end(), pts.begin(), pts.end());
    sweep_strands.push_back(s);
}

// Uniform Catmull-Rom tessellation of a control polyline with mirrored
// phantom end points (the scheme of scene.h:160-207): the curve passes
// through every control point, each span gets `subdivs` linear pieces, and
// radii follow the same spline, floored at 1e-5.
void OwnedScene::add_sweep_smooth(const std::vector<SweepPoint>& ctrl, int mat, int subdivs) {
    const int nc = (int)ctrl.size();
    if (nc < 2) return;
    std::vector<SweepPoint> p;
    p.reserve((size_t)nc + 2);
    auto mirror = [](const SweepPoint& a, const SweepPoint& b) {
        SweepPoint q = a;
        q.position = f3(a.position.x + (a.position.x - b.position.x),
                        a.position.y + (a.position.y - b.position.y),
                        a.position.z + (a.position.z - b.position.z));
        q.radius = a.radius + (a.radius - b.radius);
        return q;
    };
    p.push_back(mirror(ctrl[0], ctrl[1]));
    p.insert(p.end(), ctrl.begin(), ctrl.end());
    p.push_back(mirror(ctrl[(size_t)nc - 1], ctrl[(size_t)nc - 2]));
    auto cr = [](float a, float b, float c, float d, float u) {
        float u2 = u * u, u3 = u2 * u;
        return 0.5f * ((2.0f * b) + (-a + c) * u + (2.0f * a - 5.0f * b + 4.0f * c - d) * u2 +
                       (-a + 3.0f * b - 3.0f * c + d) * u3);
    };
    std::vector<SweepPoint> out;
    out.push_back(p[1]);
    const int n = (int)p.size();
    for (int i = 1; i < n - 2; i++) {
        const SweepPoint &a = p[(size_t)i - 1], &b = p[(size_t)i], &c = p[(size_t)i + 1], &d = p[(size_t)i + 2];
        for (int j = 1; j <= subdivs; j++) {
            float u = (float)j / (float)subdivs;
            SweepPoint q;
            q.position = f3(cr(a.position.x, b.position.x, c.position.x, d.position.x, u),
                            cr(a.position.y, b.position.y, c.position.y, d.position.y, u),
                            cr(a.position.z, b.position.z, c.position.z, d.position.z, u));
            q.radius = cr(a.radius, b.radius, c.radius, d.radius, u);
            if (q.radius < 1e-5f) q.radius = 1e-5f;
            out.push_back(q);
        }
    }
    add_sweep(out, mat);
}

}  // namespace sheen

extern "C" {

const SheenScene* sheen_owned_view(SheenOwnedScene s) {
    return s ? &reinterpret_cast<sheen::OwnedScene*>(s)->view : nullptr;
}

const SheenSceneExt* sheen_owned_ext(SheenOwnedScene s) {
    return s ? &reinterpret_cast<sheen::OwnedScene*>(s)->ext_view : nullptr;
}

const SheenSceneSettings* sheen_owned_settings(SheenOwnedScene s) {
    return s ? &reinterpret_cast<sheen::OwnedScene*>(s)->settings : nullptr;
}

void sheen_owned_free(SheenOwnedScene s) { delete reinterpret_cast<sheen::OwnedScene*>(s); }

}  // extern "C"
