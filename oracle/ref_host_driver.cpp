// ref_host_driver.cpp -- host driver for the reference renderer compiled for
// the CPU (oracle/_ref/libsheen_ref_host.so).
//
// TEST INFRASTRUCTURE ONLY: used by tests/ as a parity checker and by
// bench.py's reference arm / cpu_baseline leg.  The product never links it.
//
// The reference's per-pixel code (render_kernel.cu:1-926: render_kernel,
// compute_lighting, media_march, photon_kernel and every header they pull in)
// is compiled unchanged from the reference tree with ref_shim.h forced in.
// This file only does what the reference's host side does around it:
//   - scene build: the same steps as build_host_scene
//     (api/sheen_c_api.cu:92-140) -- copy the flat arrays into the
//     reference's Scene, build texture mips and the per-class median BVHs
//     with the reference's own Scene::build_mips / Scene::build_bvh;
//   - photon pass: photon_kernel run once per emission index
//     (render_kernel.cu:928-941 launch, seed 0x5eed1234) with the append slot
//     equal to the emission index, then the hash-grid build of
//     render_kernel.cu:992-1045 (count, prefix sum, scatter) done serially so
//     the photon order inside a cell is the emission order;
//   - the launch: 16x16 blocks over the image (api/sheen_c_api.cu:310-311),
//     each block's 256 threads run in order on one host thread, blocks
//     spread over OpenMP threads.
#include <atomic>
#include <chrono>
#include <cstring>
#include <vector>
#include <omp.h>

#include "render_kernel.h"
#include "scene.h"
#include "sheen_c_api.h"
#include "sampling/aa.h"
#include "integrator/raycast.h"

thread_local uint3 sheen_ref_block_idx;
thread_local uint3 sheen_ref_thread_idx;
thread_local dim3 sheen_ref_block_dim;

// Defined in the reference's render_kernel.cu (compiled with ref_shim.h).
void photon_kernel(PhotonScene s, int per_light, Photon* out, int max_photons,
                   unsigned int* count, unsigned int seed);

namespace {

thread_local unsigned int g_emit_index = 0;
thread_local unsigned char* g_stored_flag = nullptr;

struct RefScene {
    Scene scene;
    std::vector<TextureRef> texrefs;
    std::vector<Photon> photons_sorted;
    std::vector<int> cell_start, cell_count;
    PhotonMap pmap;
    float caustics = 0.0f;
    int photons_stored = 0;
    double build_ms = 0.0, photon_ms = 0.0;
};

void fill_scene(const SheenScene& in, Scene& scene) {
    if (in.objects) scene.objects.assign(in.objects, in.objects + in.num_objects);
    if (in.sweep_points) scene.sweep_points.assign(in.sweep_points, in.sweep_points + in.num_sweep_points);
    if (in.sweep_strands) scene.sweep_strands.assign(in.sweep_strands, in.sweep_strands + in.num_sweep_strands);
    if (in.triangles) scene.triangles.assign(in.triangles, in.triangles + in.num_triangles);
    if (in.heightfields) scene.heightfields.assign(in.heightfields, in.heightfields + in.num_heightfields);
    if (in.superellipsoids) scene.superellipsoids.assign(in.superellipsoids, in.superellipsoids + in.num_superellipsoids);
    if (in.lathe_points) scene.lathe_points.assign(in.lathe_points, in.lathe_points + in.num_lathe_points);
    if (in.lathes) scene.lathes.assign(in.lathes, in.lathes + in.num_lathes);
    if (in.prism_points) scene.prism_points.assign(in.prism_points, in.prism_points + in.num_prism_points);
    if (in.prisms) scene.prisms.assign(in.prisms, in.prisms + in.num_prisms);
    if (in.csg_nodes) scene.csg_nodes.assign(in.csg_nodes, in.csg_nodes + in.num_csg_nodes);
    scene.csg_root = in.csg_root;
    if (in.planes) scene.planes.assign(in.planes, in.planes + in.num_planes);
    if (in.materials) scene.materials.assign(in.materials, in.materials + in.num_materials);
    if (in.lights) scene.lights.assign(in.lights, in.lights + in.num_lights);
    if (in.media) scene.media.assign(in.media, in.media + in.num_media);
    for (int i = 0; i < in.num_textures; i++) {
        Scene::TextureData td;
        td.w = in.texture_widths ? in.texture_widths[i] : 0;
        td.h = in.texture_heights ? in.texture_heights[i] : 0;
        if (in.texture_pixels && in.texture_pixels[i] && td.w > 0 && td.h > 0) {
            td.pixels.assign(in.texture_pixels[i], in.texture_pixels[i] + (size_t)td.w * td.h * 3);
            Scene::build_mips(td);
        }
        scene.textures.push_back(std::move(td));
    }
    scene.camera = in.camera;
    scene.build_bvh();
}

PhotonScene photon_scene(const RefScene& r) {
    const Scene& s = r.scene;
    PhotonScene ps{};
    ps.bvh_nodes = s.bvh_nodes.data(); ps.objects = s.objects.data(); ps.num_objects = (int)s.objects.size();
    ps.strand_bvh_nodes = s.strand_bvh_nodes.data(); ps.strands = s.sweep_strands.data();
    ps.sweep_points = s.sweep_points.data(); ps.num_strands = (int)s.sweep_strands.size();
    ps.mesh_bvh_nodes = s.mesh_bvh_nodes.data(); ps.triangles = s.triangles.data();
    ps.num_triangles = (int)s.triangles.size();
    ps.hf_bvh_nodes = s.hf_bvh_nodes.data(); ps.heightfields = s.heightfields.data();
    ps.num_heightfields = (int)s.heightfields.size();
    ps.se_bvh_nodes = s.se_bvh_nodes.data(); ps.superellipsoids = s.superellipsoids.data();
    ps.num_superellipsoids = (int)s.superellipsoids.size();
    ps.lathe_bvh_nodes = s.lathe_bvh_nodes.data(); ps.lathes = s.lathes.data();
    ps.lathe_points = s.lathe_points.data(); ps.num_lathes = (int)s.lathes.size();
    ps.prism_bvh_nodes = s.prism_bvh_nodes.data(); ps.prisms = s.prisms.data();
    ps.prism_points = s.prism_points.data(); ps.num_prisms = (int)s.prisms.size();
    ps.csg_nodes = s.csg_nodes.data(); ps.csg_root = s.csg_root;
    ps.planes = s.planes.data(); ps.num_planes = (int)s.planes.size();
    ps.materials = s.materials.data(); ps.num_materials = (int)s.materials.size();
    ps.lights = s.lights.data(); ps.num_lights = (int)s.lights.size();
    return ps;
}

void build_photons(RefScene& r, int per_light, float cell, int nthreads) {
    const int nl = (int)r.scene.lights.size();
    long long total = (long long)per_light * nl;
    if (total <= 0) return;
    std::vector<Photon> tmp((size_t)total);
    std::vector<unsigned char> stored((size_t)total, 0);
    PhotonScene ps = photon_scene(r);
    unsigned int dummy = 0;
#pragma omp parallel for schedule(dynamic, 4096) num_threads(nthreads)
    for (long long idx = 0; idx < total; idx++) {
        sheen_ref_block_dim = dim3(128, 1, 1);
        sheen_ref_block_idx = make_uint3((unsigned)(idx / 128), 0, 0);
        sheen_ref_thread_idx = make_uint3((unsigned)(idx % 128), 0, 0);
        g_emit_index = (unsigned)idx;
        g_stored_flag = &stored[(size_t)idx];
        photon_kernel(ps, per_light, tmp.data(), (int)total, &dummy, 0x5eed1234u);
    }
    // The C-API caps the photon buffer at 4M (api/sheen_c_api.cu:276-278).
    std::vector<Photon> list;
    list.reserve((size_t)total);
    for (long long i = 0; i < total && list.size() < 4000000u; i++)
        if (stored[(size_t)i]) list.push_back(tmp[(size_t)i]);
    r.photons_stored = (int)list.size();
    if (list.empty()) return;

    const int num_cells = 1 << 18;
    r.cell_count.assign(num_cells, 0);
    r.cell_start.assign(num_cells + 1, 0);
    std::vector<int> cell_of(list.size());
    for (size_t i = 0; i < list.size(); i++) {
        int ix = (int)floorf(list[i].position.x / cell);
        int iy = (int)floorf(list[i].position.y / cell);
        int iz = (int)floorf(list[i].position.z / cell);
        cell_of[i] = photon_cell_hash(ix, iy, iz, num_cells);
        r.cell_count[cell_of[i]]++;
    }
    int acc = 0;
    for (int c = 0; c < num_cells; c++) { r.cell_start[c] = acc; acc += r.cell_count[c]; }
    r.cell_start[num_cells] = acc;
    std::vector<int> cursor(r.cell_start.begin(), r.cell_start.end() - 1);
    r.photons_sorted.resize(list.size());
    for (size_t i = 0; i < list.size(); i++) r.photons_sorted[cursor[cell_of[i]]++] = list[i];
    r.pmap.photons = r.photons_sorted.data();
    r.pmap.cell_start = r.cell_start.data();
    r.pmap.cell_count = r.cell_count.data();
    r.pmap.num_cells = num_cells;
    r.pmap.cell_size = cell;
}

}  // namespace

unsigned int sheen_ref_atomic_add(unsigned int* p, unsigned int v) {
    (void)p; (void)v;
    if (g_stored_flag) *g_stored_flag = 1;
    return g_emit_index;
}

extern "C" {

void* sheen_ref_scene_create(const SheenScene* in, int nthreads) {
    if (!in) return nullptr;
    RefScene* r = new RefScene();
    auto t0 = std::chrono::steady_clock::now();
    fill_scene(*in, r->scene);
    auto t1 = std::chrono::steady_clock::now();
    r->texrefs.resize(r->scene.textures.size());
    for (size_t i = 0; i < r->scene.textures.size(); i++) {
        const auto& t = r->scene.textures[i];
        TextureRef& ref = r->texrefs[i];
        std::memset(&ref, 0, sizeof(ref));
        if (t.pixels.empty()) continue;
        ref.pixels = t.pixels.data();
        ref.width = t.w; ref.height = t.h; ref.mips = t.mips;
    }
    r->caustics = in->caustics;
    if (in->photons > 0 && in->num_lights > 0)
        build_photons(*r, in->photons, in->photon_cell > 0.0f ? in->photon_cell : 0.25f,
                      nthreads > 0 ? nthreads : omp_get_max_threads());
    auto t2 = std::chrono::steady_clock::now();
    r->build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    r->photon_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    return r;
}

void sheen_ref_scene_destroy(void* h) { delete static_cast<RefScene*>(h); }

int sheen_ref_scene_photons(void* h) { return h ? static_cast<RefScene*>(h)->photons_stored : 0; }

// Copies the stored photons (in emission order after the hash-grid sort) as
// 12 floats each: position, direction, normal, flux.
int sheen_ref_scene_photon_data(void* h, float* out, int max_count) {
    RefScene* r = static_cast<RefScene*>(h);
    int n = (int)r->photons_sorted.size();
    if (n > max_count) n = max_count;
    for (int i = 0; i < n; i++) {
        const Photon& p = r->photons_sorted[i];
        const float v[12] = {p.position.x, p.position.y, p.position.z,
                             p.direction.x, p.direction.y, p.direction.z,
                             p.normal.x, p.normal.y, p.normal.z,
                             p.flux.x, p.flux.y, p.flux.z};
        std::memcpy(out + 12 * (size_t)i, v, sizeof(v));
    }
    return n;
}

double sheen_ref_scene_build_ms(void* h) { return static_cast<RefScene*>(h)->build_ms; }

// Render block rows [by0, by1) of a width x height image (16x16 blocks) into
// `out` (width*height*4 floats, RGBA).  by1 <= 0 means all rows.
int sheen_ref_scene_render(void* h, int width, int height, int aa, float* out,
                           int nthreads, int by0, int by1) {
    RefScene* r = static_cast<RefScene*>(h);
    if (!r || width <= 0 || height <= 0 || !out) return -1;
    const Scene& s = r->scene;
    const int gx = (width + 15) / 16, gy = (height + 15) / 16;
    if (by1 <= 0 || by1 > gy) by1 = gy;
    if (by0 < 0) by0 = 0;
    float4* o = reinterpret_cast<float4*>(out);
    const int nblocks = gx * (by1 - by0);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int b = 0; b < nblocks; b++) {
        sheen_ref_block_dim = dim3(16, 16, 1);
        sheen_ref_block_idx = make_uint3((unsigned)(b % gx), (unsigned)(by0 + b / gx), 0);
        for (int ty = 0; ty < 16; ty++)
            for (int tx = 0; tx < 16; tx++) {
                sheen_ref_thread_idx = make_uint3((unsigned)tx, (unsigned)ty, 0);
                render_kernel(o, width, height, s.camera,
                    s.bvh_nodes.data(), s.objects.data(), (int)s.objects.size(),
                    s.strand_bvh_nodes.data(), s.sweep_strands.data(), s.sweep_points.data(),
                    (int)s.sweep_strands.size(),
                    s.mesh_bvh_nodes.data(), s.triangles.data(), (int)s.triangles.size(),
                    s.hf_bvh_nodes.data(), s.heightfields.data(), (int)s.heightfields.size(),
                    s.se_bvh_nodes.data(), s.superellipsoids.data(), (int)s.superellipsoids.size(),
                    s.lathe_bvh_nodes.data(), s.lathes.data(), s.lathe_points.data(), (int)s.lathes.size(),
                    s.prism_bvh_nodes.data(), s.prisms.data(), s.prism_points.data(), (int)s.prisms.size(),
                    s.csg_nodes.data(), s.csg_root,
                    s.planes.data(), (int)s.planes.size(),
                    s.materials.data(), (int)s.materials.size(),
                    r->texrefs.data(), (int)r->texrefs.size(),
                    s.lights.data(), (int)s.lights.size(),
                    s.media.data(), (int)s.media.size(),
                    aa, r->pmap, r->caustics);
            }
    }
    return 0;
}

// Primary-ray closest hits with the reference's scene_intersect, for every
// pixel and sample: arrays of width*height*ns entries, index (y*width+x)*ns+s.
// The camera ray is the one built in render_kernel.cu:491-518.  obj_id and
// mat_id are -2147483648 on a miss, t is -1.
int sheen_ref_scene_primary_hits(void* h, int width, int height, int aa,
                                 int* obj_id, int* mat_id, float* t_out, int nthreads) {
    RefScene* r = static_cast<RefScene*>(h);
    if (!r) return -1;
    const Scene& s = r->scene;
    const CameraData cam = s.camera;
    const int ns = aa < 1 ? 1 : (aa > SHEEN_AA_MAX ? SHEEN_AA_MAX : aa);
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int y = 0; y < height; y++) {
        for (int x = 0; x < width; x++) {
            for (int si = 0; si < ns; si++) {
                float u, v;
                aa_uv(x, y, width, height, aa_sample_offset_n(si, ns, x, y), u, v);
                float tan_h = 1.0f, tan_x = 1.0f, tan_y = 1.0f;
                if (cam.focal_length > 0.0f) {
                    tan_h = 0.5f * cam.sensor_width / cam.focal_length;
                    if (width >= height) { tan_x = tan_h; tan_y = tan_h * float(height) / float(width); }
                    else { tan_y = tan_h; tan_x = tan_h * float(width) / float(height); }
                }
                Ray ray;
                ray.origin = cam.position;
                ray.direction = normalize(cam.forward
                                          + cam.right * (u * tan_x + cam.shift_x * tan_h)
                                          + cam.up * (v * tan_y + cam.shift_y * tan_h));
                ray.t_min = 0.001f;
                ray.t_max = 1e10f;
                HitRecord rec;
                bool hit = scene_intersect(ray,
                    s.bvh_nodes.data(), s.objects.data(), (int)s.objects.size(),
                    s.strand_bvh_nodes.data(), s.sweep_strands.data(), s.sweep_points.data(),
                    (int)s.sweep_strands.size(),
                    s.mesh_bvh_nodes.data(), s.triangles.data(), (int)s.triangles.size(),
                    s.hf_bvh_nodes.data(), s.heightfields.data(), (int)s.heightfields.size(),
                    s.se_bvh_nodes.data(), s.superellipsoids.data(), (int)s.superellipsoids.size(),
                    s.lathe_bvh_nodes.data(), s.lathes.data(), s.lathe_points.data(), (int)s.lathes.size(),
                    s.prism_bvh_nodes.data(), s.prisms.data(), s.prism_points.data(), (int)s.prisms.size(),
                    s.csg_nodes.data(), s.csg_root,
                    s.planes.data(), (int)s.planes.size(), rec);
                size_t k = ((size_t)y * width + x) * ns + si;
                obj_id[k] = hit ? rec.object_id : (int)0x80000000;
                mat_id[k] = hit ? rec.material_id : (int)0x80000000;
                t_out[k] = hit ? rec.t : -1.0f;
            }
        }
    }
    return 0;
}

int sheen_ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

// ---------------------------------------------------------------------
// The reference's .sheen loader (api/scene_io.cpp:931-968), for loader
// parity: returns a handle whose SheenScene view points into the loaded
// reference Scene.  settings_out: width, height, aa, photons (ints).
// ---------------------------------------------------------------------
#include "api/scene_io.h"

namespace {
struct RefLoaded {
    Scene scene;
    SceneSettings settings;
    SheenScene view;
    std::vector<const unsigned char*> tex_ptrs;
    std::vector<int> tex_w, tex_h;
    std::vector<int> hidden;
};
}  // namespace

extern "C" {

void* sheen_ref_load_scene_file(const char* path) {
    RefLoaded* r = new RefLoaded();
    if (!load_scene_file(path, r->scene, r->settings)) { delete r; return nullptr; }
    Scene& s = r->scene;
    SheenScene& v = r->view;
    std::memset(&v, 0, sizeof(v));
    v.camera = s.camera;
#define V(field, vec) v.field = vec.empty() ? nullptr : vec.data(); v.num_##field = (int)vec.size();
    V(objects, s.objects) V(sweep_points, s.sweep_points) V(sweep_strands, s.sweep_strands)
    V(triangles, s.triangles) V(heightfields, s.heightfields) V(superellipsoids, s.superellipsoids)
    V(lathe_points, s.lathe_points) V(lathes, s.lathes) V(prism_points, s.prism_points) V(prisms, s.prisms)
    V(planes, s.planes) V(materials, s.materials) V(lights, s.lights) V(media, s.media)
#undef V
    v.csg_nodes = s.csg_nodes.empty() ? nullptr : s.csg_nodes.data();
    v.num_csg_nodes = (int)s.csg_nodes.size();
    v.csg_root = s.csg_root;
    for (auto& t : s.textures) {   // level 0 of each mip chain
        r->tex_ptrs.push_back(t.pixels.empty() ? nullptr : t.pixels.data());
        r->tex_w.push_back(t.w);
        r->tex_h.push_back(t.h);
    }
    v.texture_pixels = r->tex_ptrs.empty() ? nullptr : r->tex_ptrs.data();
    v.texture_widths = r->tex_w.empty() ? nullptr : r->tex_w.data();
    v.texture_heights = r->tex_h.empty() ? nullptr : r->tex_h.data();
    v.num_textures = (int)s.textures.size();
    v.photons = r->settings.photons;
    v.photon_cell = r->settings.photon_cell;
    v.caustics = r->settings.caustics;
    r->hidden = s.se_hidden;
    return r;
}

const SheenScene* sheen_ref_loaded_view(void* h) { return &static_cast<RefLoaded*>(h)->view; }

void sheen_ref_loaded_settings(void* h, int* out4) {
    const SceneSettings& st = static_cast<RefLoaded*>(h)->settings;
    out4[0] = st.width; out4[1] = st.height; out4[2] = st.aa; out4[3] = st.photons;
}

void sheen_ref_loaded_free(void* h) { delete static_cast<RefLoaded*>(h); }

}  // extern "C"
