// ref_gpu_driver.cu -- the reference's own CUDA renderer on this GPU
// (oracle/_ref/libsheen_ref_gpu.so), for the comparison column of the
// benchmark.  TEST/MEASUREMENT INFRASTRUCTURE ONLY: the product never links
// it.
//
// render_kernel, launch_photons and build_photon_map are the reference's
// (render_kernel.cu, compiled unchanged for sm_100a by oracle/Makefile);
// this file does what its CLI does around them (tools/render_scene.cu:35-267):
// raise the per-thread stack limit to 16 KB, build the host Scene with the
// reference's Scene::build_bvh, copy every array to the device, run the
// photon pass when asked, and launch render_kernel on 16x16 blocks.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "render_kernel.h"
#include "scene.h"
#include "sheen_c_api.h"

namespace {

template <class T>
T* up(const std::vector<T>& v, std::vector<void*>& owned) {
    if (v.empty()) return nullptr;
    T* d = nullptr;
    if (cudaMalloc(&d, v.size() * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    owned.push_back(d);
    return d;
}

struct RefGpu {
    Scene scene;
    std::vector<void*> owned;
    BVHNode *bvh, *sbvh, *mbvh, *hbvh, *ebvh, *lbvh, *pbvh;
    Object* objects;
    SweepStrand* strands;
    SweepPoint* points;
    Triangle* tris;
    HeightField* hfs;
    Superellipsoid* ses;
    LathePoint* lpts;
    Lathe* lathes;
    PrismPoint* ppts;
    Prism* prisms;
    CSGNode* csg;
    Plane* planes;
    Material* mats;
    Light* lights;
    Medium* media;
    TextureRef* texrefs;
    int ntex = 0;
    PhotonMapBuffers pm;
    Photon* d_photons = nullptr;
    unsigned int* d_count = nullptr;
    float caustics = 0.0f;
};

}  // namespace

extern "C" {

void* sheen_refgpu_scene_create(const SheenScene* in) {
    if (cudaDeviceSetLimit(cudaLimitStackSize, 16384) != cudaSuccess) return nullptr;
    RefGpu* r = new RefGpu();
    Scene& s = r->scene;
    if (in->objects) s.objects.assign(in->objects, in->objects + in->num_objects);
    if (in->sweep_points) s.sweep_points.assign(in->sweep_points, in->sweep_points + in->num_sweep_points);
    if (in->sweep_strands) s.sweep_strands.assign(in->sweep_strands, in->sweep_strands + in->num_sweep_strands);
    if (in->triangles) s.triangles.assign(in->triangles, in->triangles + in->num_triangles);
    if (in->heightfields) s.heightfields.assign(in->heightfields, in->heightfields + in->num_heightfields);
    if (in->superellipsoids) s.superellipsoids.assign(in->superellipsoids, in->superellipsoids + in->num_superellipsoids);
    if (in->lathe_points) s.lathe_points.assign(in->lathe_points, in->lathe_points + in->num_lathe_points);
    if (in->lathes) s.lathes.assign(in->lathes, in->lathes + in->num_lathes);
    if (in->prism_points) s.prism_points.assign(in->prism_points, in->prism_points + in->num_prism_points);
    if (in->prisms) s.prisms.assign(in->prisms, in->prisms + in->num_prisms);
    if (in->csg_nodes) s.csg_nodes.assign(in->csg_nodes, in->csg_nodes + in->num_csg_nodes);
    s.csg_root = in->csg_root;
    if (in->planes) s.planes.assign(in->planes, in->planes + in->num_planes);
    if (in->materials) s.materials.assign(in->materials, in->materials + in->num_materials);
    if (in->lights) s.lights.assign(in->lights, in->lights + in->num_lights);
    if (in->media) s.media.assign(in->media, in->media + in->num_media);
    s.camera = in->camera;
    s.build_bvh();
    auto& o = r->owned;
    r->bvh = up(s.bvh_nodes, o); r->sbvh = up(s.strand_bvh_nodes, o); r->mbvh = up(s.mesh_bvh_nodes, o);
    r->hbvh = up(s.hf_bvh_nodes, o); r->ebvh = up(s.se_bvh_nodes, o); r->lbvh = up(s.lathe_bvh_nodes, o);
    r->pbvh = up(s.prism_bvh_nodes, o);
    r->objects = up(s.objects, o); r->strands = up(s.sweep_strands, o); r->points = up(s.sweep_points, o);
    r->tris = up(s.triangles, o); r->hfs = up(s.heightfields, o); r->ses = up(s.superellipsoids, o);
    r->lpts = up(s.lathe_points, o); r->lathes = up(s.lathes, o); r->ppts = up(s.prism_points, o);
    r->prisms = up(s.prisms, o); r->csg = up(s.csg_nodes, o); r->planes = up(s.planes, o);
    r->mats = up(s.materials, o); r->lights = up(s.lights, o); r->media = up(s.media, o);
    r->texrefs = nullptr;   // the benchmark scenes carry no textures
    r->caustics = in->caustics;
    if (in->photons > 0 && in->num_lights > 0) {
        long long cap = (long long)in->photons * in->num_lights;
        if (cap > 4000000) cap = 4000000;
        cudaMalloc(&r->d_photons, (size_t)cap * sizeof(Photon));
        cudaMalloc(&r->d_count, sizeof(unsigned int));
        PhotonScene ps{};
        ps.bvh_nodes = r->bvh; ps.objects = r->objects; ps.num_objects = (int)s.objects.size();
        ps.strand_bvh_nodes = r->sbvh; ps.strands = r->strands; ps.sweep_points = r->points;
        ps.num_strands = (int)s.sweep_strands.size();
        ps.mesh_bvh_nodes = r->mbvh; ps.triangles = r->tris; ps.num_triangles = (int)s.triangles.size();
        ps.hf_bvh_nodes = r->hbvh; ps.heightfields = r->hfs; ps.num_heightfields = (int)s.heightfields.size();
        ps.se_bvh_nodes = r->ebvh; ps.superellipsoids = r->ses; ps.num_superellipsoids = (int)s.superellipsoids.size();
        ps.lathe_bvh_nodes = r->lbvh; ps.lathes = r->lathes; ps.lathe_points = r->lpts;
        ps.num_lathes = (int)s.lathes.size();
        ps.prism_bvh_nodes = r->pbvh; ps.prisms = r->prisms; ps.prism_points = r->ppts;
        ps.num_prisms = (int)s.prisms.size();
        ps.csg_nodes = r->csg; ps.csg_root = s.csg_root;
        ps.planes = r->planes; ps.num_planes = (int)s.planes.size();
        ps.materials = r->mats; ps.num_materials = (int)s.materials.size();
        ps.lights = r->lights; ps.num_lights = (int)s.lights.size();
        PhotonStats pst = launch_photons(ps, in->photons, r->d_photons, (int)cap, r->d_count);
        if (pst.stored > 0)
            build_photon_map(r->d_photons, pst.stored, in->photon_cell > 0.0f ? in->photon_cell : 0.25f, r->pm);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) { delete r; return nullptr; }
    return r;
}

// Renders `iters` frames into a device buffer, returns the summed device
// time (ms) of the launches and copies the last frame to out_host.
int sheen_refgpu_render(void* h, int W, int H, int aa, float* out_host, int iters, float* ms_out) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r) return -1;
    const Scene& s = r->scene;
    float4* out = nullptr;
    if (cudaMalloc(&out, (size_t)W * H * sizeof(float4)) != cudaSuccess) return -1;
    dim3 block(16, 16), grid((W + 15) / 16, (H + 15) / 16);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float total = 0.0f;
    for (int i = 0; i < iters; i++) {
        cudaEventRecord(e0);
        render_kernel<<<grid, block>>>(out, W, H, s.camera,
            r->bvh, r->objects, (int)s.objects.size(),
            r->sbvh, r->strands, r->points, (int)s.sweep_strands.size(),
            r->mbvh, r->tris, (int)s.triangles.size(),
            r->hbvh, r->hfs, (int)s.heightfields.size(),
            r->ebvh, r->ses, (int)s.superellipsoids.size(),
            r->lbvh, r->lathes, r->lpts, (int)s.lathes.size(),
            r->pbvh, r->prisms, r->ppts, (int)s.prisms.size(),
            r->csg, s.csg_root,
            r->planes, (int)s.planes.size(),
            r->mats, (int)s.materials.size(),
            r->texrefs, r->ntex,
            r->lights, (int)s.lights.size(),
            r->media, (int)s.media.size(),
            aa, photon_map_view(r->pm), r->caustics);
        cudaEventRecord(e1);
        if (cudaEventSynchronize(e1) != cudaSuccess) { cudaFree(out); return -1; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        total += ms;
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && out_host) e = cudaMemcpy(out_host, out, (size_t)W * H * sizeof(float4), cudaMemcpyDeviceToHost);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (ms_out) *ms_out = total;
    return e == cudaSuccess ? 0 : -1;
}

void sheen_refgpu_scene_destroy(void* h) {
    RefGpu* r = static_cast<RefGpu*>(h);
    if (!r) return;
    for (void* p : r->owned) cudaFree(p);
    if (r->pm.photons) free_photon_map(r->pm);
    cudaFree(r->d_photons);
    cudaFree(r->d_count);
    delete r;
}

}  // extern "C"
