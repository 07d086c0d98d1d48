// upload.cu -- SheenScene (host arrays) -> resident DevScene in HBM.
//
// Does what the reference's sheen_render_scene does before its launch
// (api/sheen_c_api.cu:92-266: copy arrays, build texture mips and the
// per-class BVHs, patch height-map pointers) but into ONE device arena sized
// up front (one cudaMalloc, one pinned staging buffer, one H2D copy), and
// keeps it resident until the handle is released.  The wavefront form also
// gets the SAH BVH4 with quantised child boxes over the triangles.
#include <algorithm>
#include <cfloat>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "dev/prims.cuh"
#include "engine.h"

namespace sheen {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

namespace {

// Texture mip chain: 2x2 box filter with edge clamping and rounding, levels
// stored back to back (the layout of scene.h:230-261 that tex_fetch walks).
std::vector<uint8_t> build_mip_chain(const uint8_t* px, int w, int h, int& mips) {
    std::vector<uint8_t> chain(px, px + (size_t)w * h * 3);
    mips = 1;
    if (w < 2 && h < 2) return chain;
    int sw = w, sh = h;
    size_t src = 0;
    while (sw > 1 || sh > 1) {
        const int nw = sw > 1 ? sw / 2 : 1, nh = sh > 1 ? sh / 2 : 1;
        const size_t dst = chain.size();
        chain.resize(dst + (size_t)nw * nh * 3);
        for (int y = 0; y < nh; y++) {
            const int y0 = std::min(2 * y, sh - 1), y1 = std::min(2 * y + 1, sh - 1);
            for (int x = 0; x < nw; x++) {
                const int x0 = std::min(2 * x, sw - 1), x1 = std::min(2 * x + 1, sw - 1);
                for (int c = 0; c < 3; c++) {
                    const int s = chain[src + ((size_t)y0 * sw + x0) * 3 + c] + chain[src + ((size_t)y0 * sw + x1) * 3 + c] +
                                  chain[src + ((size_t)y1 * sw + x0) * 3 + c] + chain[src + ((size_t)y1 * sw + x1) * 3 + c];
                    chain[dst + ((size_t)y * nw + x) * 3 + c] = (uint8_t)((s + 2) / 4);
                }
            }
        }
        src = dst;
        sw = nw;
        sh = nh;
        mips++;
    }
    return chain;
}

// Arena layout builder: records (host source, size) pairs at 256-byte
// aligned offsets; upload_items copies them.
struct Arena {
    struct Item { const void* src; size_t bytes; size_t off; };
    std::vector<Item> items;
    size_t size = 0;
    size_t add(const void* src, size_t bytes) {
        size = (size + 255) & ~(size_t)255;
        items.push_back({src, bytes, size});
        size += bytes;
        return size - bytes;
    }
};

// Host -> device copies through a pinned ring kept for the life of the
// process (per device): kUpWorkers threads each own two kUpSlot-byte pinned
// slots and a stream; a worker copies its chunk into a free slot (waiting on
// the slot's event) and queues the slot's H2D copy, so host copies and DMA
// overlap and several host cores share the memcpy.  Allocating and freeing
// pinned memory per call costs far more than the copy itself.
constexpr int kUpWorkers = 8;
constexpr size_t kUpSlot = 4u << 20;
constexpr int kUpMaxDevices = 64;

struct UploadRing {
    void* slot[2 * kUpWorkers] = {nullptr};
    cudaEvent_t ev[2 * kUpWorkers] = {nullptr};
    cudaStream_t st[kUpWorkers] = {nullptr};
    bool ready = false;
};
std::mutex g_up_mu;
UploadRing g_up[kUpMaxDevices];

cudaError_t ring_init(UploadRing& r) {
    if (r.ready) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 * kUpWorkers && e == cudaSuccess; i++) {
        e = cudaMallocHost(&r.slot[i], kUpSlot);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&r.ev[i], cudaEventDisableTiming);
    }
    for (int w = 0; w < kUpWorkers && e == cudaSuccess; w++) e = cudaStreamCreateWithFlags(&r.st[w], cudaStreamNonBlocking);
    if (e == cudaSuccess) r.ready = true;
    return e;
}

struct Copy { void* dst; const void* src; size_t bytes; };

// Copies every item (src null: zero fill) and waits for completion.
cudaError_t upload_items(const std::vector<Copy>& items) {
    int dev_id = 0;
    cudaError_t e = cudaGetDevice(&dev_id);
    if (e != cudaSuccess) return e;
    if (dev_id < 0 || dev_id >= kUpMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_up_mu);
    UploadRing& r = g_up[dev_id];
    if ((e = ring_init(r)) != cudaSuccess) return e;
    struct Chunk { char* dst; const char* src; size_t bytes; };
    std::vector<Chunk> chunks;
    for (const Copy& c : items) {
        if (!c.bytes) continue;
        if (!c.src) {
            if ((e = cudaMemsetAsync(c.dst, 0, c.bytes, r.st[0])) != cudaSuccess) return e;
            continue;
        }
        for (size_t off = 0; off < c.bytes; off += kUpSlot)
            chunks.push_back({static_cast<char*>(c.dst) + off, static_cast<const char*>(c.src) + off,
                              std::min(kUpSlot, c.bytes - off)});
    }
    const int workers = (int)std::min<size_t>(kUpWorkers, std::max<size_t>(chunks.size(), 1));
    std::vector<cudaError_t> err((size_t)workers, cudaSuccess);
    auto work = [&](int w) {
        cudaSetDevice(dev_id);
        int k = 0;
        for (size_t c = (size_t)w; c < chunks.size(); c += (size_t)workers, k++) {
            const int sl = 2 * w + (k & 1);
            cudaError_t we = cudaEventSynchronize(r.ev[sl]);
            if (we == cudaSuccess) {
                std::memcpy(r.slot[sl], chunks[c].src, chunks[c].bytes);
                we = cudaMemcpyAsync(chunks[c].dst, r.slot[sl], chunks[c].bytes, cudaMemcpyHostToDevice, r.st[w]);
            }
            if (we == cudaSuccess) we = cudaEventRecord(r.ev[sl], r.st[w]);
            if (we != cudaSuccess) { err[(size_t)w] = we; return; }
        }
    };
    if (workers == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int w = 1; w < workers; w++) th.emplace_back(work, w);
        work(0);
        for (auto& t : th) t.join();
    }
    for (int w = 0; w < kUpWorkers; w++) {
        const cudaError_t se = cudaStreamSynchronize(r.st[w]);
        if (e == cudaSuccess) e = se;
    }
    for (cudaError_t we : err)
        if (e == cudaSuccess) e = we;
    return e;
}

}  // namespace

// Device -> host copy into pageable memory through the same pinned ring:
// each worker queues the copy of its next chunk into one of its two slots
// while it copies the previous chunk out of the other, so the DMA overlaps
// the host copies, which several cores share (together with the page faults
// of a freshly allocated destination).  The source must be complete: the
// caller has synchronised the stream that wrote it.
cudaError_t download_to_host(void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    int dev_id = 0;
    cudaError_t e = cudaGetDevice(&dev_id);
    if (e != cudaSuccess) return e;
    if (dev_id < 0 || dev_id >= kUpMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_up_mu);
    UploadRing& r = g_up[dev_id];
    if ((e = ring_init(r)) != cudaSuccess) return e;
    const size_t nchunks = (bytes + kUpSlot - 1) / kUpSlot;
    const int workers = (int)std::min<size_t>(kUpWorkers, nchunks);
    std::vector<cudaError_t> err((size_t)workers, cudaSuccess);
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src);
    auto len = [&](size_t c) { return std::min(kUpSlot, bytes - c * kUpSlot); };
    auto work = [&](int w) {
        cudaSetDevice(dev_id);
        size_t prev = 0;
        int prev_sl = -1, k = 0;
        cudaError_t we = cudaSuccess;
        for (size_t c = (size_t)w; c < nchunks && we == cudaSuccess; c += (size_t)workers, k++) {
            const int sl = 2 * w + (k & 1);
            we = cudaEventSynchronize(r.ev[sl]);
            if (we == cudaSuccess)
                we = cudaMemcpyAsync(r.slot[sl], s + c * kUpSlot, len(c), cudaMemcpyDeviceToHost, r.st[w]);
            if (we == cudaSuccess) we = cudaEventRecord(r.ev[sl], r.st[w]);
            if (we == cudaSuccess && prev_sl >= 0) {
                we = cudaEventSynchronize(r.ev[prev_sl]);
                if (we == cudaSuccess) std::memcpy(d + prev * kUpSlot, r.slot[prev_sl], len(prev));
            }
            prev = c;
            prev_sl = sl;
        }
        if (we == cudaSuccess && prev_sl >= 0) {
            we = cudaEventSynchronize(r.ev[prev_sl]);
            if (we == cudaSuccess) std::memcpy(d + prev * kUpSlot, r.slot[prev_sl], len(prev));
        }
        err[(size_t)w] = we;
    };
    if (workers == 1) {
        work(0);
    } else {
        std::vector<std::thread> th;
        for (int w = 1; w < workers; w++) th.emplace_back(work, w);
        work(0);
        for (auto& t : th) t.join();
    }
    for (cudaError_t we : err)
        if (e == cudaSuccess) e = we;
    return e;
}

namespace {

template <class T>
void push_box(std::vector<float>& lo, std::vector<float>& hi, const T a[3], const T b[3]) {
    for (int k = 0; k < 3; k++) { lo.push_back(a[k]); hi.push_back(b[k]); }
}

}  // namespace

namespace {

// Index checks of a scene before upload.  The device code trusts every index
// it reads (as the reference's does: render_kernel.cu:67 reads
// materials[rec.material_id], integrator/csg.h reads objects / SEs by leaf
// index), so a scene whose indices leave their arrays is refused here
// instead of faulting on the GPU.  Returns null or the first problem.
const char* scene_index_error(const SheenScene* in, const SheenSceneExt* ext) {
    struct Arr { const void* p; int n; const char* what; };
    const Arr arrays[] = {
        {in->objects, in->num_objects, "objects"}, {in->sweep_points, in->num_sweep_points, "sweep points"},
        {in->sweep_strands, in->num_sweep_strands, "sweep strands"}, {in->triangles, in->num_triangles, "triangles"},
        {in->heightfields, in->num_heightfields, "heightfields"},
        {in->superellipsoids, in->num_superellipsoids, "superellipsoids"},
        {in->lathe_points, in->num_lathe_points, "lathe points"}, {in->lathes, in->num_lathes, "lathes"},
        {in->prism_points, in->num_prism_points, "prism points"}, {in->prisms, in->num_prisms, "prisms"},
        {in->planes, in->num_planes, "planes"}, {in->lights, in->num_lights, "lights"},
        {in->media, in->num_media, "media"}};
    for (const Arr& a : arrays) {
        if (a.n < 0) return "negative element count";
        if (a.n > 0 && !a.p) return "null array with a nonzero count";
    }
    const int nm = in->num_materials;
    auto mat_ok = [nm](int m) { return m >= 0 && m < nm; };
    auto range_ok = [](int off, int cnt, int n) { return off >= 0 && cnt >= 0 && (long long)off + cnt <= n; };
    for (int i = 0; i < in->num_objects; i++)
        if (!mat_ok(in->objects[i].material_id)) return "object material_id out of range";
    for (int i = 0; i < in->num_sweep_strands; i++) {
        const SweepStrand& st = in->sweep_strands[i];
        if (!mat_ok(st.material_id)) return "strand material_id out of range";
        if (!range_ok(st.point_offset, st.point_count, in->num_sweep_points)) return "strand points out of range";
    }
    for (int i = 0; i < in->num_heightfields; i++)
        if (!mat_ok(in->heightfields[i].material_id)) return "heightfield material_id out of range";
    for (int i = 0; i < in->num_superellipsoids; i++)
        if (!mat_ok(in->superellipsoids[i].material_id)) return "superellipsoid material_id out of range";
    for (int i = 0; i < in->num_lathes; i++) {
        if (!mat_ok(in->lathes[i].material_id)) return "lathe material_id out of range";
        if (!range_ok(in->lathes[i].point_offset, in->lathes[i].point_count, in->num_lathe_points))
            return "lathe points out of range";
    }
    for (int i = 0; i < in->num_prisms; i++) {
        if (!mat_ok(in->prisms[i].material_id)) return "prism material_id out of range";
        if (!range_ok(in->prisms[i].point_offset, in->prisms[i].point_count, in->num_prism_points))
            return "prism points out of range";
    }
    for (int i = 0; i < in->num_planes; i++)
        if (!mat_ok(in->planes[i].material_id)) return "plane material_id out of range";
    const bool forest = ext && ext->num_csg_roots > 0;
    if (forest) {
        if (!ext->csg_roots) return "null CSG root list with a nonzero count";
        if (!in->csg_nodes || in->num_csg_nodes <= 0) return "CSG roots without CSG nodes";
        for (int i = 0; i < ext->num_csg_roots; i++)
            if (ext->csg_roots[i] < 0 || ext->csg_roots[i] >= in->num_csg_nodes) return "CSG root index out of range";
    }
    if (ext) {
        if (ext->num_csg_boxes < 0 || ext->num_csg_cones < 0 || ext->num_bezier_ctrl < 0 || ext->num_hf_heights < 0 ||
            ext->num_csg_roots < 0)
            return "negative extension count";
        if (ext->max_depth < 0 || ext->max_depth > dev::kMaxDeepBounces) return "max_depth outside 0..8";
        if ((ext->num_csg_boxes > 0 && !ext->csg_boxes) || (ext->num_csg_cones > 0 && !ext->csg_cones) ||
            (ext->num_bezier_ctrl > 0 && !ext->bezier_ctrl) || (ext->num_hf_heights > 0 && !ext->hf_heights))
            return "null extension array with a nonzero count";
        for (int i = 0; i < ext->num_csg_boxes; i++)
            if (!mat_ok(ext->csg_boxes[i].material_id)) return "CSG box material_id out of range";
        for (int i = 0; i < ext->num_csg_cones; i++) {
            if (!mat_ok(ext->csg_cones[i].material_id)) return "CSG cone material_id out of range";
            if (!(ext->csg_cones[i].r0 >= 0.0f && ext->csg_cones[i].r1 >= 0.0f)) return "CSG cone radius negative";
        }
        auto bez_ok = [&](const SheenBezierRun* runs, int n) {
            for (int i = 0; runs && i < n; i++) {
                const SheenBezierRun& r = runs[i];
                if (r.ctrl_count == 0) continue;
                if (r.ctrl_count < 4 || r.ctrl_count % 4 != 0 || !range_ok(r.ctrl_offset, r.ctrl_count, ext->num_bezier_ctrl))
                    return false;
            }
            return true;
        };
        if (!bez_ok(ext->lathe_bezier, in->num_lathes)) return "lathe Bezier run out of range (4k control points)";
        if (!bez_ok(ext->prism_bezier, in->num_prisms)) return "prism Bezier run out of range (4k control points)";
        if (ext->num_mesh_triangles < 0 || ext->num_meshes < 0 || ext->num_instances < 0)
            return "negative instance count";
        if ((ext->num_mesh_triangles > 0 && !ext->mesh_triangles) || (ext->num_meshes > 0 && !ext->meshes) ||
            (ext->num_instances > 0 && !ext->instances))
            return "null instance array with a nonzero count";
        for (int i = 0; i < ext->num_meshes; i++) {
            const SheenMesh& m = ext->meshes[i];
            if (m.tri_count <= 0 || !range_ok(m.tri_offset, m.tri_count, ext->num_mesh_triangles))
                return "mesh triangles out of range";
        }
        long long flat = std::max(in->num_triangles, 0);
        for (int i = 0; i < ext->num_instances; i++) {
            const SheenInstance& x = ext->instances[i];
            if (x.mesh < 0 || x.mesh >= ext->num_meshes) return "instance mesh out of range";
            if (!mat_ok(x.material_id)) return "instance material_id out of range";
            for (float f : x.xform)
                if (!std::isfinite(f)) return "instance transform not finite";
            const float* m = x.xform;
            const double det = (double)m[0] * ((double)m[5] * m[10] - (double)m[6] * m[9]) -
                               (double)m[1] * ((double)m[4] * m[10] - (double)m[6] * m[8]) +
                               (double)m[2] * ((double)m[4] * m[9] - (double)m[5] * m[8]);
            double scale = 0.0;
            for (int k : {0, 1, 2, 4, 5, 6, 8, 9, 10}) scale = std::max(scale, std::fabs((double)m[k]));
            if (!(std::fabs(det) > 1e-9 * scale * scale * scale)) return "instance transform not invertible";
            flat += ext->meshes[x.mesh].tri_count;
            if (flat > 2147483646ll) return "more than 2^31 - 1 triangles with the instances flattened";
        }
        for (int i = 0; ext->hf_grid && i < in->num_heightfields; i++) {
            const SheenHeightGrid& g = ext->hf_grid[i];
            if (g.offset < 0) continue;
            if (g.w < 2 || g.h < 2 || !range_ok(g.offset, (int)std::min<long long>((long long)g.w * g.h, 1ll << 30),
                                                ext->num_hf_heights) || (long long)g.w * g.h > (1ll << 30))
                return "height grid out of range";
        }
    }
    // CSG nodes reachable from the roots in use (the scene's tree, and the
    // extension forest when one is given)
    if (in->csg_nodes && in->num_csg_nodes > 0) {
        std::vector<int> st;
        if (in->csg_root >= 0 && in->csg_root < in->num_csg_nodes) st.push_back(in->csg_root);
        if (forest) st.insert(st.end(), ext->csg_roots, ext->csg_roots + ext->num_csg_roots);
        std::vector<unsigned char> seen((size_t)in->num_csg_nodes, 0);
        while (!st.empty()) {
            const int id = st.back();
            st.pop_back();
            if (seen[(size_t)id]) continue;
            seen[(size_t)id] = 1;
            const CSGNode& c = in->csg_nodes[id];
            if (c.leaf_kind == 2 || c.leaf_kind == 3) {
                const int n = !ext ? 0 : (c.leaf_kind == 2 ? ext->num_csg_boxes : ext->num_csg_cones);
                if (c.leaf_index < 0 || c.leaf_index >= n) return "CSG box / cone leaf index out of range";
            } else if (c.leaf_kind == 0) {
                if (!in->objects || c.leaf_index < 0 || c.leaf_index >= in->num_objects)
                    return "CSG sphere leaf index out of range";
                if (!mat_ok(in->objects[c.leaf_index].material_id)) return "CSG leaf material_id out of range";
            } else if (c.leaf_kind == 1) {
                if (!in->superellipsoids || c.leaf_index < 0 || c.leaf_index >= in->num_superellipsoids)
                    return "CSG superellipsoid leaf index out of range";
            } else if (c.leaf_kind < 0) {
                if (c.left < -1 || c.left >= in->num_csg_nodes || c.right < -1 || c.right >= in->num_csg_nodes)
                    return "CSG child index out of range";
                if (c.left >= 0) st.push_back(c.left);
                if (c.right >= 0) st.push_back(c.right);
            } else {
                return "unknown CSG leaf kind";
            }
        }
    }
    return nullptr;
}

// Triangles' material ids, checked on the device after upload (reading
// 2 M ids on the host would touch the whole 112-byte records).
__global__ void k_check_tri_materials(const Triangle* __restrict__ t, int n, int nm, int* __restrict__ bad) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int m = t[i].material_id;
        if (m < 0 || m >= nm) { atomicExch(bad, 1); return; }
    }
}

}  // namespace

namespace {

// Extension tables (SheenSceneExt) in their device layouts; empty vectors
// when the scene has no such extension.
struct ExtTables {
    std::vector<float> se_n2;           // per superellipsoid
    std::vector<int4> hf_grid;          // per heightfield {offset, w, h, 0}
    std::vector<int4> lathe_bz;         // per lathe {first span, spans, 0, 0}
    std::vector<float4> lathe_bound;    // per lathe {R, y_lo, y_hi, 0}
    std::vector<int4> prism_bz;         // per prism
    std::vector<float4> prism_box;      // per prism {x_lo, z_lo, x_hi, z_hi} about its centre
    std::vector<float4> spans;          // 2 per cubic span
    std::vector<int> csg_roots;
    std::vector<HostNode> csg_root_bvh;
    std::vector<float4> csg_boxes;      // 2 per box
    std::vector<float4> csg_cones;      // 3 per cone
    // instanced meshes
    std::vector<QBvh> meshes;           // per mesh: BVH4 in object space
    std::vector<float4> inst_xf;        // kInstRecord per instance
    std::vector<dev::QNode4> tlas_nodes;  // top-level BVH4 over the instances (and the scene's triangles)
    std::vector<int> tlas_items;        // per top-level leaf slot: instance (num_instances: the scene's triangles)
    int tlas_depth = 0;
    int inst_tri_total = 0;
    int mesh_depth = 0;                 // deepest mesh BVH4
    int inst_flat_leaf = 0;             // the scene's triangles are a top-level leaf
    // tessellated lathes' height buckets (wavefront form)
    std::vector<float4> lathe_grid;
    std::vector<int> lathe_grid_start, lathe_grid_items, lathe_of_point;
};

float4 f4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
float int_bits(int i) { float f; std::memcpy(&f, &i, 4); return f; }

// Box of an extension CSG leaf (kind 2 box, 3 cone).
void csg_ext_leaf_box(const ExtTables& xt, int kind, int idx, float lo[3], float hi[3]) {
    if (kind == 2) {
        const float4 a = xt.csg_boxes[2 * (size_t)idx], b = xt.csg_boxes[2 * (size_t)idx + 1];
        lo[0] = a.x; lo[1] = a.y; lo[2] = a.z;
        hi[0] = b.x; hi[1] = b.y; hi[2] = b.z;
        return;
    }
    const float4 a = xt.csg_cones[3 * (size_t)idx], b = xt.csg_cones[3 * (size_t)idx + 1];
    const float r = std::max(a.w, b.w);
    lo[0] = std::min(a.x, b.x) - r; lo[1] = std::min(a.y, b.y) - r; lo[2] = std::min(a.z, b.z) - r;
    hi[0] = std::max(a.x, b.x) + r; hi[1] = std::max(a.y, b.y) + r; hi[2] = std::max(a.z, b.z) + r;
}

// Box of the CSG tree at `root`: the union of its leaves' boxes (the solid
// lies inside the union of its leaves), widened by 1e-4 relative.
void csg_tree_box(const SheenScene* in, const ExtTables& xt, int root, float lo[3], float hi[3]) {
    for (int k = 0; k < 3; k++) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
    std::vector<int> st{root};
    int guard = 0;
    while (!st.empty() && guard++ <= 4 * in->num_csg_nodes + 4) {
        const int id = st.back();
        st.pop_back();
        if (id < 0 || id >= in->num_csg_nodes) continue;
        const CSGNode& c = in->csg_nodes[id];
        float a[3], b[3];
        if (c.leaf_kind < 0) {
            st.push_back(c.left);
            st.push_back(c.right);
            continue;
        } else if (c.leaf_kind == 0) {
            const Object& o = in->objects[c.leaf_index];
            const float r = std::fabs(o.param2);
            a[0] = o.param1.x - r; a[1] = o.param1.y - r; a[2] = o.param1.z - r;
            b[0] = o.param1.x + r; b[1] = o.param1.y + r; b[2] = o.param1.z + r;
        } else if (c.leaf_kind == 1) {
            const Superellipsoid& e = in->superellipsoids[c.leaf_index];
            a[0] = e.center.x - std::fabs(e.a); a[1] = e.center.y - std::fabs(e.b); a[2] = e.center.z - std::fabs(e.c);
            b[0] = e.center.x + std::fabs(e.a); b[1] = e.center.y + std::fabs(e.b); b[2] = e.center.z + std::fabs(e.c);
        } else {
            csg_ext_leaf_box(xt, c.leaf_kind, c.leaf_index, a, b);
        }
        for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], a[k]); hi[k] = std::max(hi[k], b[k]); }
    }
    if (!(lo[0] <= hi[0])) { for (int k = 0; k < 3; k++) lo[k] = hi[k] = 0.0f; return; }
    float scale = 0.0f;
    for (int k = 0; k < 3; k++) scale = std::max(scale, std::max(std::fabs(lo[k]), std::fabs(hi[k])));
    const float m = 1e-4f * scale + 1e-6f;
    for (int k = 0; k < 3; k++) { lo[k] -= m; hi[k] += m; }
}

// Instanced meshes: a BVH4 per mesh over its object-space triangles (the
// records keep indices into mesh_triangles), one record per instance with
// both maps (the inverse in double, rounded once), and a BVH4 over the
// instances' world boxes (the mesh box's corners through the map, widened
// by 1e-5 of the box's largest coordinate).
void build_instance_tables(const SheenScene* in, const SheenSceneExt* ext, bool flat_leaf, ExtTables& xt) {
    const bool wt = tuning().watertight != 0;
    const int nm = ext->num_meshes;
    xt.meshes.resize((size_t)nm);
    std::vector<std::array<double, 6>> mbox((size_t)nm);
    std::vector<std::thread> workers;
    for (int m = 0; m < nm; m++) {
        workers.emplace_back([&, m] {
            const SheenMesh& me = ext->meshes[m];
            std::vector<int> sub((size_t)me.tri_count);
            std::array<double, 6> b = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
            for (int k = 0; k < me.tri_count; k++) {
                sub[(size_t)k] = me.tri_offset + k;
                const Triangle& t = ext->mesh_triangles[me.tri_offset + k];
                for (const sheen_float3& v : {t.v0, t.v1, t.v2}) {
                    const double c[3] = {v.x, v.y, v.z};
                    for (int a = 0; a < 3; a++) { b[a] = std::min(b[a], c[a]); b[3 + a] = std::max(b[3 + a], c[a]); }
                }
            }
            mbox[(size_t)m] = b;
            build_qbvh4(ext->mesh_triangles, sub, xt.meshes[(size_t)m], wt);
        });
        if (workers.size() == 8 || m == nm - 1) {
            for (auto& w : workers) w.join();
            workers.clear();
        }
    }
    for (const QBvh& q : xt.meshes) xt.mesh_depth = std::max(xt.mesh_depth, q.max_depth);
    std::vector<float> lo, hi;
    std::vector<int> prims;
    int base = 0;
    for (int i = 0; i < ext->num_instances; i++) {
        const SheenInstance& x = ext->instances[i];
        const float* f = x.xform;
        const double M[3][3] = {{f[0], f[1], f[2]}, {f[4], f[5], f[6]}, {f[8], f[9], f[10]}};
        const double T[3] = {f[3], f[7], f[11]};
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) -
                           M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        double I[3][3];
        I[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
        I[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        I[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
        I[1][0] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        I[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
        I[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        I[2][0] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
        I[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        I[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
        for (int r = 0; r < 3; r++) {
            const double ti = -(I[r][0] * T[0] + I[r][1] * T[1] + I[r][2] * T[2]);
            xt.inst_xf.push_back(f4((float)I[r][0], (float)I[r][1], (float)I[r][2], (float)ti));
        }
        for (int r = 0; r < 3; r++) xt.inst_xf.push_back(f4(f[4 * r], f[4 * r + 1], f[4 * r + 2], f[4 * r + 3]));
        const SheenMesh& me = ext->meshes[x.mesh];
        const Material& mat = in->materials[x.material_id];
        const int passable = mat.transmission > 0.5f ? 1 : 0;
        xt.inst_xf.push_back(f4(int_bits(x.mesh), int_bits(x.material_id), int_bits(base - me.tri_offset),
                                int_bits(passable)));
        xt.inst_xf.push_back(f4(int_bits(base), int_bits(me.tri_count), int_bits(me.tri_offset), int_bits(0)));
        // world box
        const std::array<double, 6>& b = mbox[(size_t)x.mesh];
        double wl[3] = {1e300, 1e300, 1e300}, wh[3] = {-1e300, -1e300, -1e300}, big = 0.0;
        for (int corner = 0; corner < 8; corner++) {
            const double p[3] = {b[(corner & 1) ? 3 : 0], b[(corner & 2) ? 4 : 1], b[(corner & 4) ? 5 : 2]};
            for (int r = 0; r < 3; r++) {
                const double w = M[r][0] * p[0] + M[r][1] * p[1] + M[r][2] * p[2] + T[r];
                wl[r] = std::min(wl[r], w);
                wh[r] = std::max(wh[r], w);
                big = std::max(big, std::fabs(w));
            }
        }
        float a[3], c[3];
        for (int r = 0; r < 3; r++) {
            a[r] = (float)(wl[r] - 1e-5 * big - 1e-6);
            c[r] = (float)(wh[r] + 1e-5 * big + 1e-6);
        }
        push_box(lo, hi, a, c);
        prims.push_back(i);
        base += me.tri_count;
    }
    xt.inst_tri_total = base;
    // Wavefront form: the scene's own triangles as one more leaf (index
    // num_instances, identity maps, mesh -1), so that the top-level walk
    // orders them with the instances by entry distance and a hit in either
    // culls the other.
    if (flat_leaf) {
        float a[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, c[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int t = 0; t < in->num_triangles; t++) {
            const Triangle& tr = in->triangles[t];
            for (const sheen_float3& v : {tr.v0, tr.v1, tr.v2}) {
                a[0] = std::min(a[0], v.x); a[1] = std::min(a[1], v.y); a[2] = std::min(a[2], v.z);
                c[0] = std::max(c[0], v.x); c[1] = std::max(c[1], v.y); c[2] = std::max(c[2], v.z);
            }
        }
        for (int r = 0; r < 3; r++) {
            const float pad = 1e-5f * std::max(std::fabs(a[r]), std::fabs(c[r])) + 1e-6f;
            a[r] -= pad;
            c[r] += pad;
        }
        for (int r = 0; r < 3; r++) {
            float4 row = f4(0.0f, 0.0f, 0.0f, 0.0f);
            (&row.x)[r] = 1.0f;
            xt.inst_xf.push_back(row);
        }
        for (int r = 0; r < 3; r++) xt.inst_xf.push_back(xt.inst_xf[xt.inst_xf.size() - 3]);
        xt.inst_xf.push_back(f4(int_bits(-1), int_bits(-1), int_bits(0), int_bits(0)));
        xt.inst_xf.push_back(f4(int_bits(base), int_bits(0), int_bits(0), int_bits(0)));
        push_box(lo, hi, a, c);
        prims.push_back(ext->num_instances);
        xt.inst_flat_leaf = 1;
    }
    // Top level: the BVH4 builder over one stand-in triangle per leaf item
    // whose box is the item's (corners lo and hi, third vertex the centre),
    // so the top level is walked with the same 4-wide quantised nodes; each
    // leaf slot maps to its item.
    const size_t n = prims.size();
    std::vector<Triangle> proxy(n);
    std::vector<int> sub(n);
    for (size_t k = 0; k < n; k++) {
        Triangle& t = proxy[k];
        std::memset(&t, 0, sizeof(t));
        t.v0 = sheen_float3{lo[3 * k], lo[3 * k + 1], lo[3 * k + 2]};
        t.v1 = sheen_float3{hi[3 * k], hi[3 * k + 1], hi[3 * k + 2]};
        t.v2 = sheen_float3{0.5f * (lo[3 * k] + hi[3 * k]), 0.5f * (lo[3 * k + 1] + hi[3 * k + 1]),
                            0.5f * (lo[3 * k + 2] + hi[3 * k + 2])};
        sub[k] = (int)k;
    }
    QBvh top;
    build_qbvh4(proxy.data(), sub, top, false);
    xt.tlas_nodes = std::move(top.nodes);
    xt.tlas_items.resize(top.tris.size() / 3);
    for (size_t slot = 0; slot < xt.tlas_items.size(); slot++) {
        int k;
        std::memcpy(&k, &top.tris[3 * slot].w, 4);
        xt.tlas_items[slot] = prims[(size_t)k];
    }
    xt.tlas_depth = top.max_depth;
}

// Height buckets over the tessellated lathes' profile segments (wavefront
// form; all lathes turn about the world Y axis, so their boxes coincide and
// a per-lathe BVH cannot separate them): each segment is listed in every
// bucket its height range meets, widened by 1e-3 relative -- ten times the
// device's own per-segment margin -- so a segment is listed wherever the
// device test could accept a hit.
void build_lathe_grid(const SheenScene* in, ExtTables& xt) {
    struct SegBox { int p; float ylo, yhi; };
    std::vector<SegBox> segs;
    float Y0 = FLT_MAX, Y1 = -FLT_MAX, R = 0.0f;
    xt.lathe_of_point.assign((size_t)in->num_lathe_points, -1);
    for (int i = 0; i < in->num_lathes; i++) {
        const Lathe& l = in->lathes[i];
        for (int j = 0; j + 1 < l.point_count; j++) {
            const int p = l.point_offset + j;
            xt.lathe_of_point[(size_t)p] = i;
            const LathePoint a = in->lathe_points[p], b = in->lathe_points[p + 1];
            if (a.radius <= 0.0f && b.radius <= 0.0f) continue;
            const float rs = std::max(std::fabs(a.radius), std::fabs(b.radius));
            const float ylo = std::min(a.y, b.y), yhi = std::max(a.y, b.y);
            const float m = 1e-3f * (std::fabs(ylo) + std::fabs(yhi) + rs) + 1e-5f;
            segs.push_back({p, ylo - m, yhi + m});
            Y0 = std::min(Y0, ylo - m);
            Y1 = std::max(Y1, yhi + m);
            R = std::max(R, rs + m);
        }
    }
    if (segs.empty() || !(Y1 > Y0)) { xt.lathe_of_point.clear(); return; }
    const int nb = (int)std::max<size_t>(1, std::min<size_t>(128, segs.size() / 8));
    const float inv_h = (float)nb / (Y1 - Y0);
    auto bucket = [&](float y) { return std::max(0, std::min(nb - 1, (int)std::floor((y - Y0) * inv_h))); };
    std::vector<std::vector<int>> lists((size_t)nb);
    for (const SegBox& sb : segs) {
        const int b0 = bucket(sb.ylo), b1 = bucket(sb.yhi);
        for (int b = b0; b <= b1; b++) lists[(size_t)b].push_back(sb.p | (b0 << 24));
    }
    xt.lathe_grid = {f4(Y0, inv_h, R * 1.001f, int_bits(nb))};
    xt.lathe_grid_start.push_back(0);
    for (const auto& lst : lists) {
        xt.lathe_grid_items.insert(xt.lathe_grid_items.end(), lst.begin(), lst.end());
        xt.lathe_grid_start.push_back((int)xt.lathe_grid_items.size());
    }
}

void build_ext_tables(const SheenScene* in, const SheenSceneExt* ext, int form, ExtTables& xt) {
    if (form == SHEEN_FORM_WAVEFRONT && in->num_lathes > 0 && in->num_lathe_points < (1 << 24) &&
        !(ext && ext->lathe_bezier))
        build_lathe_grid(in, xt);
    if (!ext) return;
    if (ext->se_n2 && in->num_superellipsoids > 0)
        xt.se_n2.assign(ext->se_n2, ext->se_n2 + in->num_superellipsoids);
    if (ext->hf_grid && in->num_heightfields > 0) {
        for (int i = 0; i < in->num_heightfields; i++) {
            const SheenHeightGrid& g = ext->hf_grid[i];
            xt.hf_grid.push_back(g.offset >= 0 ? make_int4(g.offset, g.w, g.h, 0) : make_int4(-1, 0, 0, 0));
        }
    }
    // Bezier runs -> cubic spans, consecutive spans joined (and prism
    // contours closed) by straight spans where their ends differ.
    auto add_run = [&](const SheenBezierRun& r, bool close, float box[4]) -> int4 {
        const float* c = ext->bezier_ctrl + 2 * (size_t)r.ctrl_offset;
        const int first = (int)(xt.spans.size() / 2);
        auto push = [&](float a0, float b0, float a1, float b1, float a2, float b2, float a3, float b3) {
            xt.spans.push_back(f4(a0, b0, a1, b1));
            xt.spans.push_back(f4(a2, b2, a3, b3));
        };
        auto line = [&](float pa, float pb, float qa, float qb) {
            push(pa, pb, pa + (qa - pa) / 3.0f, pb + (qb - pb) / 3.0f, pa + 2.0f * (qa - pa) / 3.0f,
                 pb + 2.0f * (qb - pb) / 3.0f, qa, qb);
        };
        const int ns = r.ctrl_count / 4;
        for (int k = 0; k < ns; k++) {
            const float* q = c + 8 * k;
            if (k > 0 && (q[-2] != q[0] || q[-1] != q[1])) line(q[-2], q[-1], q[0], q[1]);
            push(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]);
        }
        const float* last = c + 8 * (ns - 1) + 6;
        if (close && (last[0] != c[0] || last[1] != c[1])) line(last[0], last[1], c[0], c[1]);
        box[0] = box[2] = c[0];
        box[1] = box[3] = c[1];
        for (int k = 0; k < r.ctrl_count; k++) {
            box[0] = std::min(box[0], c[2 * k]); box[2] = std::max(box[2], c[2 * k]);
            box[1] = std::min(box[1], c[2 * k + 1]); box[3] = std::max(box[3], c[2 * k + 1]);
        }
        return make_int4(first, (int)(xt.spans.size() / 2) - first, 0, 0);
    };
    if (ext->lathe_bezier && in->num_lathes > 0) {
        for (int i = 0; i < in->num_lathes; i++) {
            const SheenBezierRun& r = ext->lathe_bezier[i];
            if (r.ctrl_count < 4) {
                xt.lathe_bz.push_back(make_int4(0, 0, 0, 0));
                xt.lathe_bound.push_back(f4(0, 0, 0, 0));
                continue;
            }
            float box[4];   // {y_lo, r_lo, y_hi, r_hi}
            xt.lathe_bz.push_back(add_run(r, false, box));
            const float R = std::max(std::fabs(box[1]), std::fabs(box[3]));
            const float m = 1e-6f * (std::max(std::fabs(box[0]), std::fabs(box[2])) + R) + 1e-6f;
            xt.lathe_bound.push_back(f4(R + m, box[0] - m, box[2] + m, 0.0f));
        }
    }
    if (ext->prism_bezier && in->num_prisms > 0) {
        for (int i = 0; i < in->num_prisms; i++) {
            const SheenBezierRun& r = ext->prism_bezier[i];
            if (r.ctrl_count < 4) {
                xt.prism_bz.push_back(make_int4(0, 0, 0, 0));
                xt.prism_box.push_back(f4(0, 0, 0, 0));
                continue;
            }
            float box[4];   // {x_lo, z_lo, x_hi, z_hi}
            xt.prism_bz.push_back(add_run(r, true, box));
            const float m = 1e-6f * std::max(std::max(std::fabs(box[0]), std::fabs(box[2])),
                                             std::max(std::fabs(box[1]), std::fabs(box[3]))) + 1e-6f;
            xt.prism_box.push_back(f4(box[0] - m, box[1] - m, box[2] + m, box[3] + m));
        }
    }
    for (int i = 0; i < ext->num_csg_boxes; i++) {
        const SheenCsgBox& b = ext->csg_boxes[i];
        xt.csg_boxes.push_back(f4(b.lo.x, b.lo.y, b.lo.z, int_bits(b.material_id)));
        xt.csg_boxes.push_back(f4(b.hi.x, b.hi.y, b.hi.z, 0.0f));
    }
    for (int i = 0; i < ext->num_csg_cones; i++) {
        const SheenCsgCone& c = ext->csg_cones[i];
        xt.csg_cones.push_back(f4(c.p0.x, c.p0.y, c.p0.z, c.r0));
        xt.csg_cones.push_back(f4(c.p1.x, c.p1.y, c.p1.z, c.r1));
        xt.csg_cones.push_back(f4(int_bits(c.material_id), 0.0f, 0.0f, 0.0f));
    }
    if (ext->num_csg_roots > 0) {
        xt.csg_roots.assign(ext->csg_roots, ext->csg_roots + ext->num_csg_roots);
        std::vector<float> lo, hi;
        std::vector<int> prims;
        for (int k = 0; k < ext->num_csg_roots; k++) {
            float a[3], b[3];
            csg_tree_box(in, xt, ext->csg_roots[k], a, b);
            push_box(lo, hi, a, b);
            prims.push_back(k);
        }
        build_median_bvh(lo, hi, prims, true, xt.csg_root_bvh);
    }
    if (ext->num_instances > 0)
        build_instance_tables(in, ext, form == SHEEN_FORM_WAVEFRONT && in->num_triangles > 0, xt);
}

}  // namespace

int scene_upload(const SheenScene* in, int form, DeviceScene** out) { return scene_upload_ext(in, nullptr, form, out); }

int scene_upload_ext(const SheenScene* in, const SheenSceneExt* ext, int form, DeviceScene** out) {
    *out = nullptr;
    if (!in) { set_error("null scene"); return -1; }
    if (form != SHEEN_FORM_PLAIN && form != SHEEN_FORM_WAVEFRONT) { set_error("unknown renderer form"); return -1; }
    if (in->num_materials <= 0 || !in->materials) { set_error("no materials"); return -1; }
    if (const char* why = scene_index_error(in, ext)) { set_error(why); return -1; }
    ExtTables xt;
    build_ext_tables(in, ext, form, xt);
    DeviceScene* s = new DeviceScene();
    s->form = form;
    cudaGetDevice(&s->device);
    const double t0 = now_ms();

    // ---- host-side derived data -------------------------------------
    std::vector<float> lo, hi;
    std::vector<int> prims;
    std::vector<HostNode> sph_bvh, strand_bvh, mesh_bvh, hf_bvh, se_bvh, lathe_bvh, prism_bvh;

    for (int i = 0; i < in->num_objects; i++) {   // bvh.h:24-35 (type 0 only)
        const Object& o = in->objects[i];
        float a[3] = {0, 0, 0}, b[3] = {0, 0, 0};
        if (o.type == 0) {
            a[0] = o.param1.x - o.param2; a[1] = o.param1.y - o.param2; a[2] = o.param1.z - o.param2;
            b[0] = o.param1.x + o.param2; b[1] = o.param1.y + o.param2; b[2] = o.param1.z + o.param2;
            prims.push_back(i);
        }
        push_box(lo, hi, a, b);
    }
    build_median_bvh(lo, hi, prims, true, sph_bvh);

    lo.clear(); hi.clear(); prims.clear();
    for (int i = 0; i < in->num_sweep_strands; i++) {   // bvh.h:40-62
        const SweepStrand& st = in->sweep_strands[i];
        float a[3] = {1e10f, 1e10f, 1e10f}, b[3] = {-1e10f, -1e10f, -1e10f};
        for (int k = 0; k < st.point_count; k++) {
            const SweepPoint& p = in->sweep_points[st.point_offset + k];
            a[0] = fminf(a[0], p.position.x - p.radius); a[1] = fminf(a[1], p.position.y - p.radius);
            a[2] = fminf(a[2], p.position.z - p.radius);
            b[0] = fmaxf(b[0], p.position.x + p.radius); b[1] = fmaxf(b[1], p.position.y + p.radius);
            b[2] = fmaxf(b[2], p.position.z + p.radius);
        }
        push_box(lo, hi, a, b);
        prims.push_back(i);
    }
    build_median_bvh(lo, hi, prims, true, strand_bvh);

    // Triangles: the plain form walks a median BVH over 48-byte position
    // records; the wavefront form walks only its BVH4s (built below, on the
    // device by default) and needs neither.
    lo.clear(); hi.clear(); prims.clear();
    const bool plain_mesh = form == SHEEN_FORM_PLAIN;
    const bool device_build = form == SHEEN_FORM_WAVEFRONT && tuning().build_device != 0;
    std::vector<float4> tri_verts(plain_mesh ? (size_t)in->num_triangles * 3 : 0);
    if (plain_mesh) {
        lo.reserve((size_t)in->num_triangles * 3);
        hi.reserve((size_t)in->num_triangles * 3);
    }
    for (int i = 0; plain_mesh && i < in->num_triangles; i++) {   // bvh.h:235-242
        const Triangle& t = in->triangles[i];
        float a[3] = {fminf(t.v0.x, fminf(t.v1.x, t.v2.x)), fminf(t.v0.y, fminf(t.v1.y, t.v2.y)),
                      fminf(t.v0.z, fminf(t.v1.z, t.v2.z))};
        float b[3] = {fmaxf(t.v0.x, fmaxf(t.v1.x, t.v2.x)), fmaxf(t.v0.y, fmaxf(t.v1.y, t.v2.y)),
                      fmaxf(t.v0.z, fmaxf(t.v1.z, t.v2.z))};
        push_box(lo, hi, a, b);
        prims.push_back(i);
        tri_verts[3 * (size_t)i] = make_float4(t.v0.x, t.v0.y, t.v0.z, 0.0f);
        tri_verts[3 * (size_t)i + 1] = make_float4(t.v1.x, t.v1.y, t.v1.z, 0.0f);
        tri_verts[3 * (size_t)i + 2] = make_float4(t.v2.x, t.v2.y, t.v2.z, 0.0f);
    }
    if (plain_mesh) build_median_bvh(lo, hi, prims, false, mesh_bvh);

    lo.clear(); hi.clear(); prims.clear();
    for (int i = 0; i < in->num_heightfields; i++) {   // bvh.h:304-309
        const HeightField& f = in->heightfields[i];
        float a[3] = {f.center.x - 0.5f * f.size_x, f.center.y, f.center.z - 0.5f * f.size_z};
        float b[3] = {f.center.x + 0.5f * f.size_x, f.center.y + f.height, f.center.z + 0.5f * f.size_z};
        push_box(lo, hi, a, b);
        prims.push_back(i);
    }
    build_median_bvh(lo, hi, prims, false, hf_bvh);

    lo.clear(); hi.clear(); prims.clear();
    for (int i = 0; i < in->num_superellipsoids; i++) {   // superellipsoid.h:31-36
        const Superellipsoid& e = in->superellipsoids[i];
        float a[3] = {e.center.x - e.a, e.center.y - e.b, e.center.z - e.c};
        float b[3] = {e.center.x + e.a, e.center.y + e.b, e.center.z + e.c};
        push_box(lo, hi, a, b);
        prims.push_back(i);
    }
    build_median_bvh(lo, hi, prims, false, se_bvh);

    lo.clear(); hi.clear(); prims.clear();
    for (int i = 0; i < in->num_lathes; i++) {   // bvh.h:394-407 (x/z start at +-1e30 about the centre)
        const Lathe& l = in->lathes[i];
        if (!xt.lathe_bz.empty() && xt.lathe_bz[(size_t)i].y > 0) {
            // exact surface (extension): its box about the world Y axis
            const float4 b4 = xt.lathe_bound[(size_t)i];
            float a[3] = {-b4.x, b4.y, -b4.x}, b[3] = {b4.x, b4.z, b4.x};
            push_box(lo, hi, a, b);
            prims.push_back(i);
            continue;
        }
        float a[3] = {l.center.x - 1e30f, 1e30f, l.center.z - 1e30f};
        float b[3] = {l.center.x + 1e30f, -1e30f, l.center.z + 1e30f};
        for (int k = 0; k < l.point_count; k++) {
            const LathePoint& p = in->lathe_points[l.point_offset + k];
            if (p.radius < 0.0f) continue;
            a[0] = fminf(a[0], l.center.x - p.radius); a[1] = fminf(a[1], l.center.y + p.y - p.radius);
            a[2] = fminf(a[2], l.center.z - p.radius);
            b[0] = fmaxf(b[0], l.center.x + p.radius); b[1] = fmaxf(b[1], l.center.y + p.y + p.radius);
            b[2] = fmaxf(b[2], l.center.z + p.radius);
        }
        if (a[0] > b[0]) { for (int k = 0; k < 3; k++) a[k] = b[k] = 0.0f; }
        push_box(lo, hi, a, b);
        prims.push_back(i);
    }
    build_median_bvh(lo, hi, prims, false, lathe_bvh);

    lo.clear(); hi.clear(); prims.clear();
    for (int i = 0; i < in->num_prisms; i++) {   // bvh.h:321-332
        const Prism& p = in->prisms[i];
        if (!xt.prism_bz.empty() && xt.prism_bz[(size_t)i].y > 0) {
            // exact contour (extension): the hull of its control points
            const float4 b4 = xt.prism_box[(size_t)i];
            float a[3] = {p.center.x + b4.x, p.center.y + p.y_min, p.center.z + b4.y};
            float b[3] = {p.center.x + b4.z, p.center.y + p.y_max, p.center.z + b4.w};
            push_box(lo, hi, a, b);
            prims.push_back(i);
            continue;
        }
        float a[3] = {1e30f, p.center.y + p.y_min, 1e30f}, b[3] = {-1e30f, p.center.y + p.y_max, -1e30f};
        for (int k = 0; k < p.point_count; k++) {
            const PrismPoint& q = in->prism_points[p.point_offset + k];
            a[0] = fminf(a[0], p.center.x + q.x); b[0] = fmaxf(b[0], p.center.x + q.x);
            a[2] = fminf(a[2], p.center.z + q.z); b[2] = fmaxf(b[2], p.center.z + q.z);
        }
        if (a[0] > b[0]) { a[0] = b[0] = 0.0f; a[1] = b[1] = p.center.y; a[2] = b[2] = 0.0f; }
        push_box(lo, hi, a, b);
        prims.push_back(i);
    }
    build_median_bvh(lo, hi, prims, false, prism_bvh);

    // Wavefront form: BVH4 over all triangles, and -- when some triangles can
    // pass a shadow ray (transmission > 0.5, render_kernel.cu:261-262) -- one
    // over the blocking triangles (derived from the first) and one over the
    // passable ones.
    QBvh q_all, q_block, q_pass;
    if (form == SHEEN_FORM_WAVEFRONT && !device_build && in->num_triangles > 0) {
        std::vector<int> all, pass;
        std::vector<unsigned char> blocking((size_t)in->num_triangles);
        for (int i = 0; i < in->num_triangles; i++) {
            all.push_back(i);
            const int m = in->triangles[i].material_id;
            const bool passable = m >= 0 && m < in->num_materials && in->materials[m].transmission > 0.5f;
            if (passable) pass.push_back(i);
            blocking[(size_t)i] = passable ? 0 : 1;
        }
        const bool wt = tuning().watertight != 0;
        std::thread t2([&] { if (!pass.empty()) build_qbvh4(in->triangles, pass, q_pass, wt); });
        if (!pass.empty()) build_qbvh4_with_kept(in->triangles, in->num_triangles, blocking, q_all, q_block, wt);
        else build_qbvh4(in->triangles, all, q_all, wt);
        t2.join();
        // The traversal stack keeps at most 3 entries per level below the root.
        if (3 * std::max(q_all.max_depth, std::max(q_block.max_depth, q_pass.max_depth)) + 1 > 48) {
            set_error("triangle BVH too deep for the traversal stack");
            delete s;
            return -1;
        }
    }

    // Textures with mips; TextureRef pixel pointers are patched after the
    // arena address is known.
    std::vector<std::vector<uint8_t>> chains((size_t)std::max(in->num_textures, 0));
    std::vector<TextureRef> texrefs((size_t)std::max(in->num_textures, 0));
    for (int i = 0; i < in->num_textures; i++) {
        std::memset(&texrefs[(size_t)i], 0, sizeof(TextureRef));
        const int w = in->texture_widths ? in->texture_widths[i] : 0;
        const int h = in->texture_heights ? in->texture_heights[i] : 0;
        if (!in->texture_pixels || !in->texture_pixels[i] || w <= 0 || h <= 0) continue;
        int mips = 1;
        chains[(size_t)i] = build_mip_chain(in->texture_pixels[i], w, h, mips);
        texrefs[(size_t)i].width = w;
        texrefs[(size_t)i].height = h;
        texrefs[(size_t)i].mips = mips;
    }
    std::vector<HeightField> hfs(in->heightfields, in->heightfields + std::max(in->num_heightfields, 0));
    bool has_glass = false;
    for (int i = 0; i < in->num_materials; i++) {
        has_glass |= in->materials[i].transmission > 0.0f;
        s->wave_fallback |= in->materials[i].shininess < 0.0f;
    }
    for (int i = 0; i < in->num_lights; i++)
        s->wave_fallback |= in->lights[i].type == 3 && in->lights[i].beam > 0.0f;
    const double t1 = now_ms();

    // ---- arena layout -------------------------------------------------
    Arena ar;
    auto add_vec = [&](const auto& v) -> size_t {
        return v.empty() ? (size_t)-1 : ar.add(v.data(), v.size() * sizeof(v[0]));
    };
    auto add_raw = [&](const void* p, int n, size_t elem) -> size_t {
        return (p && n > 0) ? ar.add(p, (size_t)n * elem) : (size_t)-1;
    };
    const size_t o_obj = add_raw(in->objects, in->num_objects, sizeof(Object));
    const size_t o_sphb = add_vec(sph_bvh);
    const size_t o_str = add_raw(in->sweep_strands, in->num_sweep_strands, sizeof(SweepStrand));
    const size_t o_spt = add_raw(in->sweep_points, in->num_sweep_points, sizeof(SweepPoint));
    const size_t o_strb = add_vec(strand_bvh);
    const size_t o_tri = add_raw(in->triangles, in->num_triangles, sizeof(Triangle));
    const size_t o_trv = add_vec(tri_verts);
    const size_t o_meshb = add_vec(mesh_bvh);
    const size_t o_hf = add_vec(hfs);
    const size_t o_hfb = add_vec(hf_bvh);
    const size_t o_se = add_raw(in->superellipsoids, in->num_superellipsoids, sizeof(Superellipsoid));
    const size_t o_seb = add_vec(se_bvh);
    const size_t o_lat = add_raw(in->lathes, in->num_lathes, sizeof(Lathe));
    const size_t o_lpt = add_raw(in->lathe_points, in->num_lathe_points, sizeof(LathePoint));
    const size_t o_latb = add_vec(lathe_bvh);
    const size_t o_pri = add_raw(in->prisms, in->num_prisms, sizeof(Prism));
    const size_t o_ppt = add_raw(in->prism_points, in->num_prism_points, sizeof(PrismPoint));
    const size_t o_prib = add_vec(prism_bvh);
    const size_t o_csg = add_raw(in->csg_nodes, in->num_csg_nodes, sizeof(CSGNode));
    const size_t o_pla = add_raw(in->planes, in->num_planes, sizeof(Plane));
    const size_t o_mat = add_raw(in->materials, in->num_materials, sizeof(Material));
    const size_t o_lig = add_raw(in->lights, in->num_lights, sizeof(Light));
    const size_t o_med = add_raw(in->media, in->num_media, sizeof(Medium));
    const size_t o_qn = add_vec(q_all.nodes);
    const size_t o_qt = add_vec(q_all.tris);
    const size_t o_qbn = add_vec(q_block.nodes);
    const size_t o_qbt = add_vec(q_block.tris);
    const size_t o_qpn = add_vec(q_pass.nodes);
    const size_t o_qpt = add_vec(q_pass.tris);
    std::vector<size_t> o_chain(chains.size(), (size_t)-1);
    for (size_t i = 0; i < chains.size(); i++) o_chain[i] = add_vec(chains[i]);
    std::vector<size_t> o_img(hfs.size(), (size_t)-1);
    for (size_t i = 0; i < hfs.size(); i++)
        if (hfs[i].image && hfs[i].img_w > 0 && hfs[i].img_h > 0)
            o_img[i] = ar.add(hfs[i].image, (size_t)hfs[i].img_w * hfs[i].img_h);
    const size_t o_tex = texrefs.empty() ? (size_t)-1 : ar.add(nullptr, texrefs.size() * sizeof(TextureRef));
    const size_t o_tally = ar.add(nullptr, 8 * sizeof(unsigned long long));
    const size_t o_tricheck = ar.add(nullptr, sizeof(int));   // zero-filled; set by k_check_tri_materials
    const size_t o_lseg = (in->num_lathes > 0 && in->num_lathe_points > 0)
                              ? ar.add(nullptr, 2 * (size_t)in->num_lathe_points * sizeof(float4))
                              : (size_t)-1;   // zero-filled; set by lathe_segments_kernel
    const size_t o_lbnd = (o_lseg != (size_t)-1) ? ar.add(nullptr, (size_t)in->num_lathes * sizeof(float4))
                                                 : (size_t)-1;
    const size_t o_sen2 = add_vec(xt.se_n2);
    const size_t o_hfg = add_vec(xt.hf_grid);
    const size_t o_hfh = (ext && ext->hf_grid && ext->num_hf_heights > 0)
                             ? ar.add(ext->hf_heights, (size_t)ext->num_hf_heights * sizeof(float))
                             : (size_t)-1;
    const size_t o_lbz = add_vec(xt.lathe_bz);
    const size_t o_lbzb = add_vec(xt.lathe_bound);
    const size_t o_pbz = add_vec(xt.prism_bz);
    const size_t o_spans = add_vec(xt.spans);
    const size_t o_croots = add_vec(xt.csg_roots);
    const size_t o_crbvh = add_vec(xt.csg_root_bvh);
    const size_t o_cbox = add_vec(xt.csg_boxes);
    const size_t o_ccone = add_vec(xt.csg_cones);
    // instanced meshes: per-mesh BVH4s, their QMesh descriptors (patched
    // below), the object-space triangles, instance records, the top BVH
    const size_t nmesh = xt.meshes.size();
    std::vector<size_t> o_mnodes(nmesh), o_mtris(nmesh);
    for (size_t m = 0; m < nmesh; m++) {
        o_mnodes[m] = add_vec(xt.meshes[m].nodes);
        o_mtris[m] = add_vec(xt.meshes[m].tris);
    }
    std::vector<dev::QMesh> inst_qm(nmesh);
    const size_t o_iqm = nmesh ? ar.add(nullptr, nmesh * sizeof(dev::QMesh)) : (size_t)-1;
    const size_t o_itri = nmesh ? add_raw(ext->mesh_triangles, ext->num_mesh_triangles, sizeof(Triangle)) : (size_t)-1;
    const size_t o_ixf = add_vec(xt.inst_xf);
    const size_t o_lg = add_vec(xt.lathe_grid);
    const size_t o_lgs = add_vec(xt.lathe_grid_start);
    const size_t o_lgi = add_vec(xt.lathe_grid_items);
    const size_t o_lop = add_vec(xt.lathe_of_point);
    const size_t o_tln = add_vec(xt.tlas_nodes);
    const size_t o_tli = add_vec(xt.tlas_items);
    // the two-level walk's stack (dev/instances.cuh: 72 entries) holds 3 per
    // level of both trees, a marker and a top-level leaf's remainder
    if (3 * xt.mesh_depth + 1 > 48 || 3 * (xt.mesh_depth + xt.tlas_depth) + 2 > 72) {
        set_error("instanced mesh BVH too deep for the traversal stack");
        delete s;
        return -1;
    }
    ar.size = (ar.size + 255) & ~(size_t)255;

    cudaError_t e = dmalloc(&s->arena, ar.size);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); delete s; return -1; }
    s->arena_bytes = ar.size;
    char* base = (char*)s->arena;
    auto dptr = [&](size_t off) -> void* { return off == (size_t)-1 ? nullptr : (void*)(base + off); };

    // Patch device pointers into the host copies that reference other arrays.
    for (size_t i = 0; i < texrefs.size(); i++) texrefs[i].pixels = (const unsigned char*)dptr(o_chain[i]);
    for (size_t i = 0; i < hfs.size(); i++) hfs[i].image = (const unsigned char*)dptr(o_img[i]);
    for (size_t m = 0; m < nmesh; m++) {
        inst_qm[m].nodes = (const dev::QNode4*)dptr(o_mnodes[m]);
        inst_qm[m].tris = (const float4*)dptr(o_mtris[m]);
        inst_qm[m].num_nodes = (int)xt.meshes[m].nodes.size();
        inst_qm[m].num_tris = (int)(xt.meshes[m].tris.size() / 3);
        inst_qm[m].watertight = xt.meshes[m].vertices ? 1 : 0;
    }
    for (auto& it : ar.items) {
        if (it.off == o_tex) it.src = texrefs.data();
        if (it.off == o_hf) it.src = hfs.data();
        if (it.off == o_iqm) it.src = inst_qm.data();
    }

    // Every array straight from its host source through the pinned ring.
    std::vector<Copy> copies;
    for (const auto& it : ar.items) copies.push_back({base + it.off, it.src, it.bytes});
    e = upload_items(copies);
    if (e == cudaSuccess && in->num_triangles > 0) {
        int* bad = reinterpret_cast<int*>(static_cast<char*>(s->arena) + o_tricheck);
        k_check_tri_materials<<<(int)std::min<long long>((in->num_triangles + 255) / 256, 148 * 8), 256>>>(
            reinterpret_cast<const Triangle*>(static_cast<char*>(s->arena) + o_tri), in->num_triangles,
            in->num_materials, bad);
        int bad_h = 0;
        e = cudaMemcpy(&bad_h, bad, sizeof(int), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && bad_h) {
            dfree(s->arena);
            set_error("triangle material_id out of range");
            delete s;
            return -1;
        }
    }
    if (e == cudaSuccess && o_lseg != (size_t)-1) {
        dev::lathe_segments_kernel<<<in->num_lathes, 64>>>((const Lathe*)(base + o_lat), in->num_lathes,
                                                          (const LathePoint*)(base + o_lpt),
                                                          (float4*)(base + o_lseg), (float4*)(base + o_lbnd));
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) { dfree(s->arena); set_error(cudaGetErrorString(e)); delete s; return -1; }
    const double t2 = now_ms();

    dev::DevScene& v = s->view;
    std::memset(&v, 0, sizeof(v));
    v.cam = in->camera;
    v.objects = (const Object*)dptr(o_obj); v.num_objects = in->num_objects; v.sphere_bvh = (const dev::BvhNode*)dptr(o_sphb);
    v.strands = (const SweepStrand*)dptr(o_str); v.sweep_points = (const SweepPoint*)dptr(o_spt);
    v.num_strands = in->num_sweep_strands; v.strand_bvh = (const dev::BvhNode*)dptr(o_strb);
    v.tris = (const Triangle*)dptr(o_tri); v.tri_verts = (const float4*)dptr(o_trv);
    v.num_tris = std::max(in->num_triangles, 0);
    v.mesh_bvh = (const dev::BvhNode*)dptr(o_meshb);
    v.hfs = (const HeightField*)dptr(o_hf); v.num_hfs = in->num_heightfields; v.hf_bvh = (const dev::BvhNode*)dptr(o_hfb);
    v.ses = (const Superellipsoid*)dptr(o_se); v.num_ses = in->num_superellipsoids; v.se_bvh = (const dev::BvhNode*)dptr(o_seb);
    v.lathes = (const Lathe*)dptr(o_lat); v.lathe_points = (const LathePoint*)dptr(o_lpt); v.num_lathes = in->num_lathes;
    v.lathe_seg = (const float4*)dptr(o_lseg);
    v.lathe_bound = (const float4*)dptr(o_lbnd);
    v.lathe_bvh = (const dev::BvhNode*)dptr(o_latb);
    v.prisms = (const Prism*)dptr(o_pri); v.prism_points = (const PrismPoint*)dptr(o_ppt); v.num_prisms = in->num_prisms;
    v.prism_bvh = (const dev::BvhNode*)dptr(o_prib);
    v.csg_nodes = (const CSGNode*)dptr(o_csg);
    v.csg_root = (in->csg_nodes && in->num_csg_nodes > 0 && in->csg_root >= 0 && in->csg_root < in->num_csg_nodes)
                     ? in->csg_root : -1;
    {
        // the box of the tree's leaves (the leaf indices were checked at the
        // start), widened by 1e-4 relative
        float lo3[3], hi3[3];
        if (v.csg_root >= 0) {
            csg_tree_box(in, xt, v.csg_root, lo3, hi3);
        } else {
            for (int k = 0; k < 3; k++) { lo3[k] = FLT_MAX; hi3[k] = -FLT_MAX; }
        }
        for (int k = 0; k < 3; k++) { v.csg_lo[k] = lo3[k]; v.csg_hi[k] = hi3[k]; }
    }
    v.planes = (const Plane*)dptr(o_pla); v.num_planes = in->num_planes;
    v.materials = (const Material*)dptr(o_mat); v.num_materials = in->num_materials;
    v.textures = (const TextureRef*)dptr(o_tex); v.num_textures = in->num_textures;
    v.lights = (const Light*)dptr(o_lig); v.num_lights = in->num_lights;
    v.media = (const Medium*)dptr(o_med); v.num_media = in->num_media;
    v.caustics = in->caustics;
    auto qmesh = [&](const QBvh& q, size_t on, size_t ot) {
        dev::QMesh m;
        m.nodes = (const dev::QNode4*)dptr(on);
        m.tris = (const float4*)dptr(ot);
        m.num_nodes = (int)q.nodes.size();
        m.num_tris = (int)(q.tris.size() / 3);
        m.watertight = q.vertices ? 1 : 0;
        return m;
    };
    v.q_all = qmesh(q_all, o_qn, o_qt);
    v.q_block = qmesh(q_block, o_qbn, o_qbt);
    v.q_pass = qmesh(q_pass, o_qpn, o_qpt);
    v.has_glass = has_glass ? 1 : 0;
    v.aa_centered = tuning().aa_centered;
    v.se_polish = tuning().se_polish;
    v.caustic_knn = tuning().caustic_knn;
    v.se_n2 = (const float*)dptr(o_sen2);
    v.hf_grid = (const int4*)dptr(o_hfg);
    v.hf_heights = (const float*)dptr(o_hfh);
    v.lathe_bz = (const int4*)dptr(o_lbz);
    v.lathe_bz_bound = (const float4*)dptr(o_lbzb);
    v.prism_bz = (const int4*)dptr(o_pbz);
    v.bz_spans = (const float4*)dptr(o_spans);
    v.csg_roots = (const int*)dptr(o_croots);
    v.num_csg_roots = (int)xt.csg_roots.size();
    v.csg_root_bvh = (const dev::BvhNode*)dptr(o_crbvh);
    v.csg_boxes = (const float4*)dptr(o_cbox);
    v.csg_cones = (const float4*)dptr(o_ccone);
    v.bounces = ext && ext->max_depth > 1 ? std::min(ext->max_depth, (int)dev::kMaxDeepBounces) : 0;
    v.inst_tris = (const Triangle*)dptr(o_itri);
    v.inst_mesh = (const dev::QMesh*)dptr(o_iqm);
    v.inst_xf = (const float4*)dptr(o_ixf);
    v.lathe_grid = (const float4*)dptr(o_lg);
    v.lathe_grid_start = (const int*)dptr(o_lgs);
    v.lathe_grid_items = (const int*)dptr(o_lgi);
    v.lathe_of_point = (const int*)dptr(o_lop);
    v.tlas_nodes = (const dev::QNode4*)dptr(o_tln);
    v.tlas_items = (const int*)dptr(o_tli);
    v.num_instances = nmesh ? ext->num_instances : 0;
    v.inst_tri_total = xt.inst_tri_total;
    v.inst_flat_leaf = xt.inst_flat_leaf;
    s->d_tally = (unsigned long long*)dptr(o_tally);
    s->wave_depth = std::max(q_all.max_depth, std::max(q_block.max_depth, q_pass.max_depth));
    s->build_ms = t1 - t0;
    s->upload_ms = t2 - t1;
    if (device_build && v.num_tris > 0) {
        const double tb = now_ms();
        e = build_wave_meshes_device(*s, 0);
        if (e == cudaSuccess) e = cudaStreamSynchronize(0);
        if (e != cudaSuccess) {
            set_error(cudaGetErrorString(e));
            scene_release(s);
            return -1;
        }
        // The traversal stack keeps at most 3 entries per level below the root.
        if (3 * s->wave_depth + 1 > 48) {
            set_error("triangle BVH too deep for the traversal stack");
            scene_release(s);
            return -1;
        }
        s->build_ms += now_ms() - tb;
    }
    if (v.inst_flat_leaf && 3 * (s->wave_depth + xt.tlas_depth) + 2 > 72) {
        set_error("triangle BVH too deep for the instanced walk's stack");
        scene_release(s);
        return -1;
    }
    // the kernels pick their triangle test from q_all's flag: with
    // instances and no triangles of the scene's own, the meshes' flag
    if (!v.q_all.nodes && v.num_instances > 0) v.q_all.watertight = tuning().watertight != 0 ? 1 : 0;

    if (in->photons > 0 && in->num_lights > 0) {
        const double tp = now_ms();
        if (build_photon_map_device(*s, in->photons, in->photon_cell > 0.0f ? in->photon_cell : 0.25f) != 0) {
            scene_release(s);
            return -1;
        }
        s->photon_ms = now_ms() - tp;
    }
    *out = s;
    return 0;
}

// The first render of a process used to pay the pool's growth (hundreds of
// MB mapped by the driver) and the pinned ring's allocation: about 220 ms
// for each of the first two host-array calls of the mesh workload against
// 43 ms after.  sheen_init maps `mb` into the pool (an allocation freed back
// to it; the pool keeps freed memory mapped up to mem.pool_keep_mb) and
// allocates the ring.
cudaError_t prewarm_device(int mb) {
    if (mb > 0) {
        void* p = nullptr;
        cudaError_t e = dmalloc(&p, (size_t)mb << 20);
        if (e != cudaSuccess) {
            cudaGetLastError();   // not enough memory: no warm-up
        } else {
            dfree(p);
        }
    }
    int dev_id = 0;
    cudaError_t e = cudaGetDevice(&dev_id);
    if (e != cudaSuccess || dev_id < 0 || dev_id >= kUpMaxDevices) return e;
    std::lock_guard<std::mutex> lk(g_up_mu);
    return ring_init(g_up[dev_id]);
}

// Frees the pinned upload rings (sheen_cleanup, before the device reset).
void release_upload_rings() {
    std::lock_guard<std::mutex> lk(g_up_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < kUpMaxDevices; d++) {
        UploadRing& r = g_up[d];
        if (!r.ready) continue;
        cudaSetDevice(d);
        for (int i = 0; i < 2 * kUpWorkers; i++) { cudaFreeHost(r.slot[i]); cudaEventDestroy(r.ev[i]); }
        for (int w = 0; w < kUpWorkers; w++) cudaStreamDestroy(r.st[w]);
        r = UploadRing();
    }
    cudaSetDevice(cur);
}

void scene_release(DeviceScene* s) {
    if (!s) return;
    wave_release(*s);
    for (void* p : s->extra) dfree(p);
    dfree(s->arena);
    delete s;
}

}  // namespace sheen
