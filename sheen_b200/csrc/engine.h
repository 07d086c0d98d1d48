// engine.h -- internal interface between the C-ABI layer and the device code.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "sheen_c_api.h"
#include "dev/scene.cuh"

namespace sheen {

void set_error(const char* msg);
void set_errorf(const char* fmt, const char* a);

// Host mirror of dev::BvhNode.
struct HostNode {
    float lo[3];
    int left;
    float hi[3];
    int right;
};
static_assert(sizeof(HostNode) == 32, "BVH node is 32 bytes");

// Median-split BVH with the reference's rules (bvh.h:71-576): object
// median on the largest axis, one primitive per leaf (leaf = ~index in both
// child slots).  `axis_from_centroids` selects the sphere/strand variant
// (axis from the centroid extent) over the mesh/HF/SE/lathe/prism variant
// (axis from the extent of the primitive boxes).
void build_median_bvh(const std::vector<float>& lo, const std::vector<float>& hi,
                      const std::vector<int>& prims, bool axis_from_centroids,
                      std::vector<HostNode>& out);

// Binned-SAH BVH4 over triangles with 8-bit child boxes (bvh4.cpp).
struct QBvh {
    std::vector<dev::QNode4> nodes;
    std::vector<float4> tris;      // 3 float4 per triangle slot in leaf order
    int leaf_size_max = 0;
    int max_depth = 0;            // inner-node levels (the traversal stack holds 3 per level)
    bool vertices = false;        // triangle records hold v1, v2 (watertight test) instead of e1, e2
};
// Builds over the triangles listed in `subset` (indices into `tris`; the
// stored triangle records keep those original indices).  `vertices`
// selects the record layout of the watertight triangle test.
void build_qbvh4(const Triangle* tris, const std::vector<int>& subset, QBvh& out, bool vertices = false);

// The BVH4 over all n triangles, and the one over the triangles with
// keep[i] != 0 derived from it instead of built: the binary tree loses the
// other triangles from its leaves, nodes left with one child are spliced
// out, boxes are refitted to the kept triangles, and the result is collapsed
// like a built tree.  kept_out is empty when nothing is kept.
void build_qbvh4_with_kept(const Triangle* tris, int n, const std::vector<unsigned char>& keep, QBvh& all,
                           QBvh& kept_out, bool vertices = false);

// Every child box of q is exactly the quantised union of the boxes of the
// original triangles (tris) below it; 0 or a negative code (host only).
int check_qbvh4_tight(const QBvh& q, const Triangle* tris);

// The same BVH4 built on the device (bvh4_gpu.cu), byte-identical to
// build_qbvh4's.  nodes/tris are device allocations owned by the caller.
struct DevQBvh {
    dev::QNode4* nodes = nullptr;
    float4* tris = nullptr;
    int num_nodes = 0;
    int num_tris = 0;
    int max_depth = 0;
};
// With keep_dev (one flag per triangle; subset_dev null) it also derives
// build_qbvh4_with_kept's tree over the kept triangles into *kept_out.
cudaError_t build_qbvh4_device(const Triangle* tris_dev, const int* subset_dev, int n, DevQBvh& out,
                               cudaStream_t stream, bool vertices = false, const unsigned char* keep_dev = nullptr,
                               DevQBvh* kept_out = nullptr);

// Result/accounting of one render call.
struct RenderTally {
    unsigned long long primary = 0, shadow = 0, secondary = 0, nodes = 0, prims = 0;
};

// A resident scene (behind SheenDeviceScene).
struct DeviceScene {
    int form = SHEEN_FORM_PLAIN;
    int device = 0;
    dev::DevScene view{};
    void* arena = nullptr;                 // one allocation holding every array
    size_t arena_bytes = 0;
    std::vector<void*> extra;              // photon map buffers
    size_t extra_bytes = 0;
    unsigned long long* d_tally = nullptr; // 8 counters
    double build_ms = 0.0, upload_ms = 0.0, photon_ms = 0.0;
    int photons_stored = 0;
    // Wavefront form state (queues sized for the last render).
    struct Wave* wave = nullptr;
    // Scene features outside the queue pipeline (visible spot beams, the
    // shadow-debug material mode): such frames run on the BVH4 megakernel.
    bool wave_fallback = false;
    int wave_depth = 0;                    // levels of the deepest triangle BVH4
};

// The wavefront form's three triangle BVH4s (all / blocking / passable) of
// a scene whose triangles and materials are already resident, built on the
// device; allocations are added to s.extra.
cudaError_t build_wave_meshes_device(DeviceScene& s, cudaStream_t stream);

int scene_upload(const SheenScene* in, int form, DeviceScene** out);
// With scene extensions (ext may be null).
int scene_upload_ext(const SheenScene* in, const SheenSceneExt* ext, int form, DeviceScene** out);
void release_upload_rings();
// sheen_init's warm-up of the current device: `mb` of device memory mapped
// into the library's pool, and the pinned upload ring.
cudaError_t prewarm_device(int mb);
void scene_release(DeviceScene* s);

// Pixel rectangle [x0, x1) x [y0, y1) of a W x H image; the output buffer
// always holds the whole image (W*H float4), pixels outside are untouched.
struct Region {
    int x0, y0, x1, y1;
};

// Plain form: one thread per pixel.  Asynchronous on `stream`.
// Ray tallies go to `tally` (8 device counters) or, when null, the scene's own.
cudaError_t launch_plain(const DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t stream,
                         bool count_nodes, unsigned long long* tally = nullptr);

// Primary closest hits (object id, material id, t) per pixel sample.
cudaError_t launch_primary_hits_plain(const DeviceScene& s, int W, int H, int ns, int* obj, int* mat, float* t,
                                      cudaStream_t stream);
// Closest hits of arbitrary rays through the scene form's own traversal.
cudaError_t launch_trace_rays(const DeviceScene& s, const float4* rays, int n, int* obj, int* mat, float* t,
                              cudaStream_t stream);
cudaError_t launch_primary_hits_bvh4(const DeviceScene& s, int W, int H, int ns, int* obj, int* mat, float* t,
                                     cudaStream_t stream);

// Megakernel over the BVH4 mesh traversal (wavefront form's queries, one
// thread per pixel); used by the wavefront form for scenes outside its
// queue pipeline and as a measurement point.
cudaError_t launch_mega_bvh4(const DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t stream,
                             bool count_nodes, unsigned long long* tally = nullptr);

// Wavefront form.
cudaError_t launch_wavefront(DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t stream,
                             bool count_nodes);
void wave_release(DeviceScene& s);
// Frees the queue blocks kept from released scenes (render_wave.cu).
void release_parked_waves();
// Forget the cached device address of the allocation-free entry point's
// scratch array (sheen_cleanup resets the device, which invalidates it).
void release_noalloc_scratch();
// Destroy the device BVH builder's cached second streams (one per device).
void release_build_streams();
// Mark the device sRGB threshold tables as not uploaded.
void release_srgb_tables();

// Wavefront form on caller-owned scratch (the request loop: one block per
// in-flight request).  Renders a region with the queue kernels launched
// directly on `stream` (no graph, no synchronisation), its queues carved from
// [scratch, scratch + scratch_bytes) (256-byte aligned, at least
// wave_scratch_bytes(lights, padded region samples)).  Scenes outside the
// queue pipeline (wave_pipeline_used false) run on the BVH4 megakernel and
// need no scratch.  Ray tallies are added to `tally` (device counters
// 0..2) when not null.
cudaError_t launch_wavefront_scratch(DeviceScene& s, void* scratch, size_t scratch_bytes, int W, int H, int aa,
                                     Region rg, float4* out, cudaStream_t stream, unsigned long long* tally);
size_t wave_scratch_bytes(int L, long long nsamples);
bool wave_pipeline_used(const DeviceScene& s);
// Which kernels render a whole W x H frame at aa spp (SHEEN_PATH_*).
int frame_path(const DeviceScene& s, int W, int H, int aa);

// One job of a multi-job wavefront launch: region rg of a W x H frame of
// scene s at aa samples per pixel into the device image `out` (W*H float4).
struct BatchItem {
    DeviceScene* s;
    int W, H, aa;
    Region rg;
    float4* out;
};
// Every job in one pass of the queue kernels (scenes must be wavefront-form
// scenes whose frames run on the queue pipeline).  Ray tallies are added to
// `tally` (device counters 0..2) when not null.
cudaError_t launch_wavefront_batch(const std::vector<BatchItem>& items, cudaStream_t stream,
                                   unsigned long long* tally);
cudaError_t profile_wavefront(DeviceScene& s, int W, int H, int aa, float4* out, cudaStream_t stream,
                              SheenStageProfile* prof);

// Device -> host copy into pageable memory through the library's pinned
// ring, several host threads sharing the copies (upload.cu).  The source
// must be complete.
cudaError_t download_to_host(void* dst, const void* src, size_t bytes);

// Launch parameters of the wavefront form (tuning.cpp).
struct Tuning {
    int shadow_kernel = 1;          // 0: 32-ray batches per warp; 1: per-lane refill
    int refill_min = 16;            // idle lanes that trigger a refill (shadow_kernel 1)
    int inner_min = 10;             // refill shadow stage: descending lanes below which the node phase ends
    int node_cost = 4;              // triangle BVH4 build: a node visit's SAH cost, in quarters of a triangle test
    int shadow_blocks_per_sm = 0;   // 128-thread blocks per SM for the shadow stage; 0: occupancy limit
    int shadow_stack = 0;           // refill shadow stage: traversal stack nodes in 0 local / 1 shared memory
    int build_device = 1;           // wavefront triangle BVH4s: 1 built on the device, 0 on the host
    int build_concurrent = 1;       // device build: the subset trees beside the full tree (2 host threads)
    int pool_keep_mb = 16384;       // freed device memory the library's pool keeps for reuse
    int prewarm_mb = 2048;          // device memory sheen_init maps into the pool up front (0: none)
    int watertight = 0;             // wavefront triangle test: 0 Moller-Trumbore (the reference's), 1 watertight
    int aa_centered = 0;            // camera samples: 0 the reference's jitter, 1 cell centres
    int se_polish = 0;              // superellipsoid entries: 0 on a sample (reference), 1 FP64 Newton polish
    int caustic_knn = 0;            // caustic gather: 0 the reference's, k in 1..64 the k nearest photons
    int tile_w = 16;                // wavefront sample order: width of the 128-pixel tiles (8, 16 or 32)
    int mega_samples = 327680;      // wavefront frames of at most this many samples (tile-padded pixels x spp;
                                    // a quarter of it for scenes with triangles) run on the BVH4 megakernel
                                    // (one launch) instead of the queue stages; 0: never
};
Tuning tuning();
int tuning_generation();
int tuning_set(const char* name, int value);
int tuning_get(const char* name, int* value);

// Photon pass on the device (emission + hash-grid build), called by
// scene_upload when the scene asks for photons.
int build_photon_map_device(DeviceScene& s, int per_light, float cell);

double now_ms();

// PNG path (png.cpp, png_pack.cu): the float4 image packed into PNG raw rows
// (h rows of 1 + 3w bytes) on the device, and a PNG written from such rows.
cudaError_t pack_srgb_rows(const float4* img, int W, int H, unsigned char* rows, cudaStream_t stream);
int write_png_rows(const char* path, const unsigned char* rows, int w, int h);

// Device memory of the library (mem.cpp): a stream-ordered pool per device
// that keeps freed blocks mapped for reuse.  dmalloc's block is usable on
// every stream when it returns; dfree waits for the device (as cudaFree
// does) before returning the block.  The _async forms are ordered on
// `stream` only.
cudaError_t dmalloc(void** ptr, size_t bytes);
cudaError_t dmalloc_async(void** ptr, size_t bytes, cudaStream_t stream);
void dfree(void* ptr);
void dfree_async(void* ptr, cudaStream_t stream);
void release_pools();
void trim_pool();
template <class T>
cudaError_t dmalloc(T** ptr, size_t bytes) { return dmalloc(reinterpret_cast<void**>(ptr), bytes); }
template <class T>
cudaError_t dmalloc_async(T** ptr, size_t bytes, cudaStream_t stream) {
    return dmalloc_async(reinterpret_cast<void**>(ptr), bytes, stream);
}

}  // namespace sheen
