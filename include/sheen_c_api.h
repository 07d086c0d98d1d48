/*
 * sheen_c_api.h -- C-ABI of the B200 renderer core (libsheen_c_api.so).
 *
 * The first four entry points and the SheenScene struct are the drop-in
 * boundary: same names, argument meaning, return codes and struct layout as
 * the reference's sheen_c_api.h (sheen_c_api.h:18-107), so the Blender
 * add-on's ctypes path (addon_sheen/sheen_render/engine.py:88-147) and the
 * native module (api/sheen_py_module.cpp:57-87) load this library unchanged.
 *
 * Everything after them is new and stands beside the drop-in: an RGBA (float)
 * output path for parity checks, device-resident scene handles with a choice
 * of renderer form, the .sheen loader and synthetic scene generators behind a
 * C view, and a continuous-batching request loop.
 *
 * Conventions for the new entry points: return 0 on success and -1 on error
 * (message via sheen_get_last_error(), which is per thread for them); no
 * torch or CUDA types in the signatures; pointers documented as host or
 * device.
 */
#ifndef SHEEN_C_API_H
#define SHEEN_C_API_H

#include <stddef.h>
#include "sheen_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sheen_c_api.h:18-87 -- flat scene description, 352 bytes.  Pointers are
 * host pointers owned by the caller for the duration of a call; NULL when the
 * matching count is 0. */
typedef struct SheenScene {
    CameraData camera;

    const Object* objects;
    int num_objects;

    const SweepPoint* sweep_points;
    int num_sweep_points;
    const SweepStrand* sweep_strands;
    int num_sweep_strands;

    const Triangle* triangles;
    int num_triangles;

    const HeightField* heightfields;
    int num_heightfields;

    const Superellipsoid* superellipsoids;
    int num_superellipsoids;

    const LathePoint* lathe_points;
    int num_lathe_points;
    const Lathe* lathes;
    int num_lathes;

    const PrismPoint* prism_points;
    int num_prism_points;
    const Prism* prisms;
    int num_prisms;

    const CSGNode* csg_nodes;
    int csg_root;               /* -1: no CSG tree */
    int num_csg_nodes;

    const Plane* planes;
    int num_planes;

    const Material* materials;
    int num_materials;

    const unsigned char* const* texture_pixels;   /* [num_textures], RGB8 */
    const int* texture_widths;
    const int* texture_heights;
    int num_textures;

    const Light* lights;
    int num_lights;

    int photons;                /* photons emitted per light; 0 disables the caustic pass */
    float photon_cell;          /* hash-grid cell size (<= 0: 0.25) */
    float caustics;             /* caustic gain; 0 disables the gather */

    const Medium* media;
    int num_media;
} SheenScene;

/* ------------------------------------------------------------------ */
/* Drop-in entry points                                                */
/* ------------------------------------------------------------------ */

/* Replaces sheen_init (sheen_c_api.h:91-93, api/sheen_c_api.cu:160-180).
 * Selects the CUDA device.  cuda_arch is accepted and ignored: the library is
 * built for sm_100a only.  Unlike the reference no 16 KB per-thread stack
 * reservation is needed (no kernel here recurses).  0 / -1. */
int sheen_init(int device_id, int cuda_arch);

/* Replaces sheen_cleanup (sheen_c_api.h:95-96, api/sheen_c_api.cu:182-185).
 * Frees every resident scene, server and pooled buffer, then resets this
 * process's context on the device. */
void sheen_cleanup(void);

/* Replaces sheen_render_scene (sheen_c_api.h:98-105, api/sheen_c_api.cu:187-361).
 * Renders with the plain FP32 form and writes an 8-bit sRGB PNG.  Parameter
 * checks and messages follow the reference: w, h > 0, 1 <= aa <= 64,
 * output_path != NULL, num_materials > 0.  0 / -1. */
int sheen_render_scene(const SheenScene* scene, int width, int height,
                       int aa_samples, const char* output_path);

/* Replaces sheen_get_last_error (sheen_c_api.h:107, api/sheen_c_api.cu:363-365). */
const char* sheen_get_last_error(void);

/* ------------------------------------------------------------------ */
/* Additions                                                           */
/* ------------------------------------------------------------------ */

/* Renderer forms. */
enum {
    SHEEN_FORM_PLAIN = 0,      /* one thread per pixel megakernel, FP32 32-byte nodes, median BVH */
    SHEEN_FORM_WAVEFRONT = 1   /* persistent wavefront integrator, SAH BVH4 with 8-bit child boxes */
};

/* Render flags. */
enum {
    SHEEN_RENDER_COUNT_RAYS = 1,  /* fill SheenRenderStats ray counters */
    SHEEN_RENDER_COUNT_NODES = 2  /* also count box and primitive tests (instrumented
                                     megakernel of the form's traversal; slower) */
};

typedef struct SheenRenderStats {
    unsigned long long primary_rays;     /* W*H*spp */
    unsigned long long shadow_rays;      /* each glass pass counts */
    unsigned long long secondary_rays;   /* reflection + refraction + photon-gather-free bounces */
    unsigned long long total_rays;
    unsigned long long node_visits;      /* box tests issued (counting builds only) */
    unsigned long long prim_tests;       /* primitive tests issued (counting builds only) */
    double build_ms;                     /* BVH builds: host, plus the wavefront form's
                                            triangle BVH4s on the device */
    double upload_ms;                    /* host -> device copies */
    double photon_ms;                    /* photon emission + map build */
    double render_ms;                    /* device time of the render launches */
    unsigned long long device_bytes;     /* resident scene footprint */
    unsigned long long upload_bytes;     /* bytes copied host -> device for the scene */
    unsigned long long shadow_node_visits; /* part of node_visits spent on glass-aware shadow
                                              queries (the wavefront shadow stage) */
    unsigned long long shadow_prim_tests;  /* part of prim_tests spent on them */
} SheenRenderStats;

/* Render into a caller-owned HOST buffer of width*height float4 (RGBA, linear,
 * alpha = 1), the same values the reference kernel writes into its float4
 * output before the sRGB conversion.  Uploads, renders and frees like
 * sheen_render_scene.  stats may be NULL. */
int sheen_render_scene_rgba(const SheenScene* scene, int width, int height,
                            int aa_samples, int form, float* out_rgba_host,
                            SheenRenderStats* stats);

/* Device-resident scenes.  create copies and packs every array to the device
 * (BVH build included) and keeps it until destroy. */
typedef struct SheenDeviceScene_* SheenDeviceScene;
int  sheen_scene_create(const SheenScene* scene, int form, SheenDeviceScene* out);
void sheen_scene_destroy(SheenDeviceScene scene);

/* ------------------------------------------------------------------ */
/* Scene extensions.  No counterpart in the reference: shapes its       */
/* renderer does not have (the benchmark workloads' extension columns:  */
/* exact Bezier surfaces, two-exponent superellipsoids, FP32 height     */
/* grids, forests of CSG trees with box and cone leaves).  Every field  */
/* is optional: a zero-filled SheenSceneExt renders exactly what        */
/* sheen_scene_create renders.                                          */
/* ------------------------------------------------------------------ */

/* ctrl_count control points starting at ctrl_offset, cubic Bezier spans of
 * four points each (the layout of the .sheen lathe_bezier / prism_bezier
 * commands, api/scene_io.cpp:86-102, 791-819); 0 points: no extension. */
typedef struct SheenBezierRun {
    int ctrl_offset;
    int ctrl_count;
} SheenBezierRun;

/* Solid leaves of extension CSG trees (CSGNode.leaf_kind 2 and 3). */
typedef struct SheenCsgBox {        /* axis-aligned box */
    sheen_float3 lo;
    sheen_float3 hi;
    int material_id;
    int _pad0;
} SheenCsgBox;

typedef struct SheenCsgCone {       /* capped cone (frustum) from p0 (radius r0) to p1 (radius r1) */
    sheen_float3 p0;
    float r0;
    sheen_float3 p1;
    float r1;
    int material_id;
    int _pad0, _pad1, _pad2;
} SheenCsgCone;

typedef struct SheenHeightGrid {    /* w x h FP32 heights in [0, 1], row-major, rows along z */
    int offset;                     /* first value in SheenSceneExt.hf_heights; < 0: none */
    int w, h;
} SheenHeightGrid;

/* One mesh of the instanced geometry: a run of SheenSceneExt.mesh_triangles. */
typedef struct SheenMesh {
    int tri_offset;
    int tri_count;
} SheenMesh;

/* One placement of a mesh: xform is the 3x4 affine map from the mesh's
 * object space to the world, row-major (world = xform[:, 0:3] p +
 * xform[:, 3]); it must be invertible.  The instance draws every triangle
 * of the mesh with material_id. */
typedef struct SheenInstance {
    float xform[12];
    int mesh;
    int material_id;
} SheenInstance;

typedef struct SheenSceneExt {
    /* Exact cubic-Bezier surfaces, replacing the tessellation the reference
     * renders (its loader turns Bezier profiles into polylines on the
     * host).  lathe_bezier[i] (num_lathes entries, or NULL): lathe i's
     * profile as control points (y, radius), turned about the world Y axis
     * like the tessellated lathe (whose test ignores Lathe.center).
     * prism_bezier[i] (num_prisms entries, or NULL): prism i's closed
     * contour as control points (x, z) about the prism's centre, extruded
     * over [y_min, y_max].  Control points are (a, b) pairs in bezier_ctrl.
     * The ray-surface roots (a sextic per lathe span, cubics for prism walls
     * and cap contours) are isolated in FP64 on the GPU; everything else
     * stays FP32. */
    const SheenBezierRun* lathe_bezier;
    const SheenBezierRun* prism_bezier;
    const float* bezier_ctrl;
    int num_bezier_ctrl;               /* pairs */
    /* Two-exponent superellipsoids: se_n2[i] > 0 (num_superellipsoids
     * entries, or NULL) gives superellipsoid i the surface
     * (|x/a|^n + |z/c|^n)^(n2/n) + |y/b|^n2 = 1 (n = Superellipsoid.n: the
     * east-west exponent, n2 the north-south one; n2 == n is the
     * reference's single-exponent body), tested with the reference's march
     * and bisection. */
    const float* se_n2;
    /* FP32 height grids: hf_grid[i] (num_heightfields entries, or NULL)
     * replaces heightfield i's procedural or 8-bit height with a bilinear
     * FP32 grid spanning its size_x x size_z footprint, scaled by
     * HeightField.height. */
    const SheenHeightGrid* hf_grid;
    const float* hf_heights;
    int num_hf_heights;
    /* CSG forest: further tree roots beside SheenScene.csg_root (closest
     * hit over all trees), and the box / cone leaves their CSGNode records
     * name with leaf_kind 2 / 3 (leaf_index into these arrays).  A tree
     * keeps the reference's rules (8 intervals per node). */
    const int* csg_roots;
    int num_csg_roots;
    const SheenCsgBox* csg_boxes;
    int num_csg_boxes;
    const SheenCsgCone* csg_cones;
    int num_csg_cones;
    /* Reflect + refract recursion to max_depth bounces (2..8; 0 or 1: the
     * reference's depth-1 mirror ray and up-to-three-face refraction;
     * outside 0..8 the create fails).  Every hit below the limit blends as
     * the reference's primary hit does (lighting x (1 - wr)(1 - wt), a
     * mirror ray x wr (1 - wt), a refracted ray x the face's transmission;
     * wr = min(reflect, 1), wt = min(transmission, 1)); a hit at the limit
     * contributes its lighting alone.  Media act on every segment, beams on
     * the primary ray only.  Such scenes render on the BVH4 megakernel
     * (wavefront form) or the plain kernel. */
    int max_depth;
    /* Instanced meshes in a two-level BVH: mesh_triangles hold every mesh's
     * object-space triangles (their material_id is not used), meshes[i] a
     * run of them, instances[j] one placement.  A BVH4 is built per mesh
     * in object space and a BVH over the instances' world boxes; a query
     * enters a mesh through the instance's inverse map (t is the same in
     * both spaces).  Instanced triangles belong to the mesh category like
     * the scene's own (a query's mesh hit is the closest over both), and a
     * hit on triangle k of instance j reports the object id
     * -(num_triangles + 1 + base_j + k), base_j the triangles of the
     * instances before j: the index it would have with the instances
     * flattened after the scene's triangles.  At most 2^31 - 1 triangles
     * flattened. */
    const Triangle* mesh_triangles;
    int num_mesh_triangles;
    const SheenMesh* meshes;
    int num_meshes;
    const SheenInstance* instances;
    int num_instances;
} SheenSceneExt;

/* sheen_scene_create with extensions (ext may be NULL).  Fails with a
 * message when an extension array names something out of range. */
int  sheen_scene_create_ext(const SheenScene* scene, const SheenSceneExt* ext, int form, SheenDeviceScene* out);
unsigned long long sheen_scene_device_bytes(SheenDeviceScene scene);
int  sheen_scene_form(SheenDeviceScene scene);

/* Which kernels render a whole width x height frame of the scene at
 * aa_samples spp: SHEEN_PATH_PLAIN (a SHEEN_FORM_PLAIN scene: the
 * reference-order kernel), SHEEN_PATH_QUEUES (the wavefront queue stages)
 * or SHEEN_PATH_MEGAKERNEL (the BVH4 megakernel: frames at most
 * wave.mega_samples samples, and scenes outside the queue pipeline --
 * beams, media, shadow-debug materials, more than 16 lights, reflect +
 * refract recursion).  Follows the current tuning; -1 on a null handle or
 * bad sizes.  No counterpart in the reference (one megakernel). */
#define SHEEN_PATH_PLAIN 0
#define SHEEN_PATH_QUEUES 1
#define SHEEN_PATH_MEGAKERNEL 2
int  sheen_scene_frame_path(SheenDeviceScene scene, int width, int height, int aa_samples);

/* Render a resident scene into a DEVICE buffer (width*height float4) on the
 * given CUDA stream (cudaStream_t passed as void*, NULL = legacy default
 * stream).  Asynchronous unless flags has SHEEN_RENDER_COUNT_RAYS or stats
 * is non-NULL, in which case it synchronises the stream before returning. */
int sheen_scene_render_device(SheenDeviceScene scene, int width, int height,
                              int aa_samples, float* out_rgba_device,
                              void* stream, int flags, SheenRenderStats* stats);

/* Render only the pixel rectangle [x0, x1) x [y0, y1) of a width x height
 * image (tiles, progressive refinement, bounded samples).  The DEVICE buffer
 * holds the whole image; pixels outside the rectangle are left unchanged.
 * Same synchronisation rules as sheen_scene_render_device. */
int sheen_scene_render_region(SheenDeviceScene scene, int width, int height, int aa_samples,
                              int x0, int y0, int x1, int y1, float* out_rgba_device,
                              void* stream, int flags, SheenRenderStats* stats);

/* Allocation-free variant of sheen_scene_render_region.  No counterpart in
 * the reference (its C-ABI only renders whole frames to a PNG).
 *
 * For callers that must not have the library allocate GPU memory during a
 * render: a real-time loop that reserves all of its device memory at
 * start-up and treats any later allocation as a fault, or an application
 * whose own memory manager must own every byte on the device.  It renders
 * the pixel rectangle [x0, x1) x [y0, y1) of a width x height image of a
 * SHEEN_FORM_WAVEFRONT scene into the caller's DEVICE buffer (whole image,
 * width*height float4) on `stream`, with the same queue kernels as the
 * regular entry points and their scratch in a fixed array in the library's
 * device globals (about 13 MB, held on every GPU that loads the library
 * until exit).  Nothing is allocated and nothing is synchronised.
 *
 * Limits: at most 16384 samples per call (the rectangle's pixels rounded up
 * to whole tiles of 128 pixels, 16x8 unless "wave.tile_w" says otherwise,
 * times aa_samples -- e.g. 128x128 at 1 spp or 64x64 at 4 spp) and at most
 * 8 lights; larger requests fail with -1 and a message.
 * The first call on each device (and the first after sheen_cleanup) looks up
 * the array's device address; make that call before any stream capture.
 * Each call clears the queue counters it starts from; the rest of the array
 * keeps the last call's contents.  Every call shares the array: calls that
 * can overlap on the GPU race, so serialise them (one stream). */
int sheen_scene_render_region_noalloc(SheenDeviceScene scene, int width, int height, int aa_samples,
                                      int x0, int y0, int x1, int y1, float* out_rgba_device, void* stream);

/* Same, into a HOST buffer; includes the device -> host copy. */
int sheen_scene_render_host(SheenDeviceScene scene, int width, int height,
                            int aa_samples, float* out_rgba_host, int flags,
                            SheenRenderStats* stats);

/* Primary-ray closest hits of a resident scene, for hit-identity checks:
 * for every pixel (x, y) and sample s of clamp(aa, 1, 64) samples, at index
 * (y*width + x)*ns + s of the HOST arrays: the hit's object_id and
 * material_id as the reference's scene_intersect sets them
 * (integrator/raycast.h:14-70; 0x80000000 on a miss) and its t (-1 on a
 * miss).  Uses the scene's form's own traversal. */
int sheen_scene_primary_hits(SheenDeviceScene scene, int width, int height, int aa_samples,
                             int* obj_id_host, int* mat_id_host, float* t_host);

/* Closest hits of arbitrary rays through a resident scene's own traversal.
 * rays_host: n records of 8 floats {origin.xyz, t_min, direction.xyz, t_max}
 * (the direction is used as given); per ray, in HOST arrays: object_id and
 * material_id as scene_intersect sets them (integrator/raycast.h:14-70;
 * 0x80000000 on a miss) and t (-1 on a miss).  No counterpart in the
 * reference (its queries are internal to render_kernel).  0 / -1. */
int sheen_scene_trace(SheenDeviceScene scene, const float* rays_host, int n, int* obj_id_host, int* mat_id_host,
                      float* t_host);

/* Host-side structural check of the wavefront form's triangle BVH (4-wide,
 * 8-bit child boxes) for a scene: every triangle in exactly one leaf, every
 * decoded child box containing all triangles below it.  Returns the tree
 * depth, or a negative code on a violation.  No device work. */
int sheen_selfcheck_bvh4(const SheenScene* scene);

/* Host-side check of the blocking triangles' BVH4 (material transmission
 * <= 0.5), which the wavefront form derives from the tree over all
 * triangles instead of building it: drops the passable triangles from the
 * leaves, splices out nodes left with one child and refits every box.
 * Checks that the tree over all equals the plainly built one byte for byte,
 * that both trees are structurally valid with every child box exactly the
 * quantised union of the triangles below it, and that the derived tree
 * holds each blocking triangle once.  Returns the derived tree's depth (0
 * when nothing blocks) or a negative code.  No device work. */
int sheen_selfcheck_bvh4_kept(const SheenScene* scene);

/* Builds the wavefront form's three triangle BVH4s (all / blocking /
 * passable triangles) of a scene with the host builder and with the device
 * builder and compares them byte for byte.  No counterpart in the reference
 * (its BVH is built on the host, Scene::build_bvh, scene.h:410-481).
 * Returns 0 when identical; 1 + 10*set (node count), 2 + 10*set (node
 * bytes), 3 + 10*set (triangle records) or 4 (depth) for the first
 * difference, set 0 = all, 1 = blocking, 2 = passable; -1 on error.
 * times_ms (may be NULL) receives {host build ms, device build ms}. */
int sheen_bvh4_compare_builders(const SheenScene* scene, double* times_ms);

/* One job of sheen_render_batch: the pixel rectangle [x0, x1) x [y0, y1) of
 * a width x height frame of `scene` (x1 <= x0 or y1 <= y0: the whole frame)
 * at aa_samples per pixel, written into the DEVICE image out_rgba_device
 * (width*height float4; pixels outside the rectangle are left unchanged). */
typedef struct SheenBatchJob {
    SheenDeviceScene scene;
    int width, height, aa_samples;
    int x0, y0, x1, y1;
    float* out_rgba_device;
} SheenBatchJob;

/* Renders every job in one pass of the wavefront queue kernels (one pass per
 * kernel variant: scenes of triangles, spheres and planes only or of every
 * category, with the Moller-Trumbore or the watertight triangle test, so
 * that batching never changes which code renders a job): each stage is
 * one persistent launch over the samples of all jobs (tiles of one frame,
 * several frames, several scenes, of uneven cost), claimed dynamically by
 * the blocks from shared queues.  Each job's pixels are exactly those of
 * rendering it alone.  Jobs on SHEEN_FORM_PLAIN scenes, or whose frames run
 * on the megakernel (beams, media, shadow-debug materials, more than 16
 * lights, reflect + refract recursion), are rendered one by one on the same
 * stream first.  Asynchronous on
 * `stream` unless stats is non-NULL (then it synchronises and fills the ray
 * counts and render_ms).  No counterpart in the reference (one frame per
 * launch, render_kernel.cu:438-814).  0 / -1. */
int sheen_render_batch(const SheenBatchJob* jobs, int num_jobs, void* stream, SheenRenderStats* stats);

/* Stage profile of one wavefront frame (sheen_scene_profile_stages): device
 * times of the queue kernels, measured with CUDA events at the stage
 * boundaries of a frame launched directly (not from the captured graph), and
 * the rays each kernel issued.  No counterpart in the reference (one
 * megakernel, render_kernel.cu:438-814). */
typedef struct SheenStageProfile {
    double primary_ms, shadow_ms[3], reflect_ms, refract_ms, resolve_ms, total_ms;
    unsigned long long primary_rays, shadow_rays[3], reflect_rays, refract_rays;
} SheenStageProfile;

/* One full frame of a SHEEN_FORM_WAVEFRONT scene into a DEVICE buffer
 * (width*height float4) with the stage profile above; synchronous.  Scenes
 * whose frames run on the megakernel (beams, media, shadow-debug materials,
 * more than 16 lights, reflect + refract recursion) have no stages: -1. */
int sheen_scene_profile_stages(SheenDeviceScene scene, int width, int height, int aa_samples,
                               float* out_rgba_device, void* stream, SheenStageProfile* out);

/* Launch parameters of the wavefront form, by name (process-wide; frames
 * captured under older values are re-captured).  No counterpart in the
 * reference (its launch shape is fixed at 16x16 threads per block,
 * api/sheen_c_api.cu:309-312).  Keys and ranges:
 *   "wave.shadow_kernel"         0: every warp takes 32 shadow rays and
 *                                   finishes them together; 1 (default):
 *                                   lanes take new rays as theirs finish
 *   "wave.refill_min"            1..32 (default 16): idle lanes that make a
 *                                   warp take new rays (shadow_kernel 1)
 *   "wave.inner_min"             0..32 (default 10): the refill shadow
 *                                   stage ends a warp's inner-node phase
 *                                   once fewer lanes than this still
 *                                   descend while one waits at a leaf
 *                                   (0: when none descends)
 *   "wave.shadow_blocks_per_sm"  0..16 (default 0 = as many as fit)
 *   "wave.shadow_stack"          0 (default): traversal stack of the refill
 *                                   shadow stage in local memory; 1: node
 *                                   entries in shared memory (24 KB/block)
 *   "build.concurrent"           1 (default): the subset BVH4s are built
 *                                   beside the full one (two host threads)
 *   "mem.pool_keep_mb"           0..1048576 (default 16384): freed device
 *                                   memory the library keeps for reuse
 *   "mem.prewarm_mb"             0..1048576 (default 2048): device memory
 *                                   sheen_init maps into that pool up front
 *                                   (set before sheen_init; 0: none)
 *   "trace.watertight"           0 (default): the wavefront form tests
 *                                   triangles with the reference's
 *                                   Moller-Trumbore; 1: a watertight
 *                                   edge-function test (no ray passes
 *                                   between triangles sharing an edge or
 *                                   a vertex; hits may differ from the
 *                                   reference's on edges).  Read at
 *                                   sheen_scene_create.
 *   "build.node_cost"            1..64 (default 4): the SAH cost of a node
 *                                   visit in quarters of a triangle test,
 *                                   against which the triangle BVH4
 *                                   builders weigh a leaf of <= 8
 *                                   triangles (larger: bigger leaves,
 *                                   fewer nodes).  Read at
 *                                   sheen_scene_create.
 *   "build.device"               1 (default): the wavefront form's triangle
 *                                   BVH4s are built on the GPU; 0: on the
 *                                   host.  Both builders give byte-identical
 *                                   trees; read at sheen_scene_create.
 *   "camera.centered"            0 (default): the reference's sample
 *                                   positions, jittered even at 1 spp
 *                                   (sampling/aa.h:45-58); 1: no jitter --
 *                                   the pixel centre at 1 spp, cell centres
 *                                   otherwise.  Read at sheen_scene_create.
 *   "trace.se_polish"            0 (default): a superellipsoid entry lies on
 *                                   the sample where the reference's 32-step
 *                                   march finds it (superellipsoid.h:100-
 *                                   112); 1: refined in FP64 (safeguarded
 *                                   Newton) onto the surface.  Read at
 *                                   sheen_scene_create.
 *   "caustic.knn"                0 (default): the reference's caustic gather
 *                                   (the first <= 128 photons within
 *                                   cell / 2, render_kernel.h:68-111);
 *                                   k = 1..64: the k nearest photons within
 *                                   r_max = cell / 2, the estimate's radius
 *                                   the k-th distance.  Read at
 *                                   sheen_scene_create.
 * Every other setting gives the same image (watertight, centered, se_polish
 * and knn change it on purpose); only the speed differs.  0 / -1. */
int sheen_tune_set(const char* key, int value);
int sheen_tune_get(const char* key, int* value);

typedef struct SheenTuneResult {
    int shadow_kernel, refill_min, shadow_blocks_per_sm;   /* the setting kept */
    int candidates;                                        /* settings timed */
    double best_ms;                                        /* frame time with it */
    double default_ms;                                     /* frame time with the setting in force before */
    int shadow_stack;                                      /* the setting kept: wave.shadow_stack */
    int inner_min;                                         /* the setting kept: wave.inner_min */
    int tile_w;                                            /* the setting kept: wave.tile_w */
    int mega_samples;                                      /* the setting kept: wave.mega_samples */
} SheenTuneResult;

/* Autotuner: times candidate launch parameters on a resident
 * SHEEN_FORM_WAVEFRONT scene for one frame shape -- per candidate one
 * warm-up frame, then `reps` frames timed with CUDA events -- and keeps the
 * fastest (process-wide, as sheen_tune_set).  First the shadow stage (both
 * variants, refill thresholds 8/16/24, inner-phase thresholds 0/6/10/14,
 * shadow blocks per SM, traversal stack in local or shared memory), then,
 * with the best of those, the pixel tile of the sample order (8x16, 16x8,
 * 32x4) and the small-frame switch (queue stages or the BVH4 megakernel for
 * this frame).  Renders into a device buffer it allocates and frees;
 * synchronous.  0 / -1. */
int sheen_autotune(SheenDeviceScene scene, int width, int height, int aa_samples, int reps,
                   SheenTuneResult* out);

/* Owned host scenes: the .sheen loader and the synthetic generators return
 * one.  sheen_owned_view points into storage owned by the handle. */
typedef struct SheenOwnedScene_* SheenOwnedScene;

typedef struct SheenSceneSettings {
    int width;
    int height;
    int aa;
    int photons;
    float photon_cell;
    float caustics;
    char output[512];
} SheenSceneSettings;

/* Replaces load_scene_file (api/scene_io.h:20, api/scene_io.cpp:931-968):
 * parses a .sheen text file with the reference's grammar.  On a parse error
 * returns -1 with "line N: <text>" in the error message. */
int  sheen_load_scene_file(const char* path, SheenOwnedScene* out);
const SheenScene* sheen_owned_view(SheenOwnedScene scene);
const SheenSceneSettings* sheen_owned_settings(SheenOwnedScene scene);
void sheen_owned_free(SheenOwnedScene scene);

/* Seeded synthetic scene generators for the benchmark workloads.
 *   0: 64 spheres + ground plane + 1 point light, reflect 0.3
 *   1: displaced level-`level` icosphere + 16 displaced 50k-triangle tori,
 *      4 point lights, 4 glass tori (ior 1.5), reflect 0.2 elsewhere
 *   2: analytic primitives + one CSG tree (superellipsoids, lathes, prisms,
 *      sweeps, procedural heightfield)
 *   3: glass sphere + glass lathe over a diffuse plane, one spot light,
 *      caustics on (photons per light = `photons`)
 * `detail` scales the geometry: for config 1 it is the icosphere subdivision
 * level (8 = 1,310,720 triangles) and the torus grid is scaled with it; for
 * the others it is ignored unless > 0 where noted. */
int sheen_generate_scene(int config, unsigned int seed, int detail, int photons,
                         SheenOwnedScene* out);

/* The workload generators with their extension column (no counterpart in
 * the reference).  extended != 0, config 1: the same scene with its 16 tori
 * as instances of one 50,000-triangle mesh (SheenSceneExt.instances) and
 * reflect + refract recursion to 4 bounces (SheenSceneExt.max_depth).  Config 2: the
 * same scene with
 * two-exponent superellipsoids (both exponents 2/e, e uniform in [0.2, 3]),
 * the lathes' and prisms' Bezier control points as exact surfaces, a
 * 1024 x 1024 FP32 height grid (heights in [0, 2]) for the heightfield, and
 * 128 further CSG trees of depth 3 over spheres, boxes and cones.  The
 * extensions are read with sheen_owned_ext() and passed to
 * sheen_scene_create_ext(); the SheenScene view alone is the reference's
 * scene.  Configs 0 and 3: extended must be 0. */
int sheen_generate_scene_ext(int config, unsigned int seed, int detail, int photons, int extended,
                             SheenOwnedScene* out);

/* The extension arrays of an owned scene (zero-filled when it has none). */
const SheenSceneExt* sheen_owned_ext(SheenOwnedScene scene);

/* 8-bit sRGB PNG writer used by sheen_render_scene (png_color.h:11-20 conversion). */
int sheen_write_png_srgb(const char* path, const float* rgba, int width, int height);

/* The conversion's byte steps: out[b - 1] = the smallest non-negative float
 * whose sRGB byte is >= b, b = 1..255 (255 floats).  sheen_render_scene packs
 * on the device by searching these, which gives the host conversion's bytes
 * exactly.  No counterpart in the reference (it converts on the host). */
void sheen_srgb_thresholds(float* out);

/* ------------------------------------------------------------------ */
/* Request loop (continuous batching).  No counterpart in the reference, */
/* whose C-ABI renders one frame per call and rebuilds and re-uploads   */
/* the scene every time (api/sheen_c_api.cu:187-361).                   */
/* ------------------------------------------------------------------ */

/* A server owns resident scenes and renders requests against them.  Each
 * request (scene, width, height, spp, caller's host buffer) is queued on
 * submit and admitted onto the GPU when one of max_inflight slots (one CUDA
 * stream each) is free and its device footprint -- wavefront queues for one
 * band of rows plus the band's output -- fits in the HBM budget beside the
 * resident scenes; requests that arrive while others run overlap with them
 * on the device.  A request behind one that does not fit may be admitted
 * first, until the blocked one has been passed 16 times.  Images do not
 * depend on what else runs: a request's result is the same alone and in a
 * mix.  All functions are thread-safe. */
typedef struct SheenServer_* SheenServer;

typedef struct SheenServerConfig {
    int form;                        /* SHEEN_FORM_WAVEFRONT or SHEEN_FORM_PLAIN for the server's scenes */
    int max_inflight;                /* requests on the GPU at once (1..64); <= 0: 4 */
    unsigned long long hbm_budget;   /* device bytes for scenes + in-flight requests; 0: 90% of free memory */
    long long tile_samples;          /* samples per band of rows; <= 0: 4194304 */
} SheenServerConfig;

enum {
    SHEEN_REQ_PENDING = 0,   /* queued, not admitted */
    SHEEN_REQ_RUNNING = 1,   /* admitted, on the GPU */
    SHEEN_REQ_DONE = 2,      /* image in the caller's buffer */
    SHEEN_REQ_FAILED = 3     /* see SheenRequestInfo.error */
};

typedef struct SheenRequestInfo {
    int status;
    int scene_id, width, height, aa_samples;
    int tiles;                       /* bands of rows the request was rendered in */
    unsigned long long rays;         /* primary + shadow + secondary rays traced */
    unsigned long long hbm_bytes;    /* device footprint while in flight */
    double queue_ms;                 /* submit -> admitted */
    double run_ms;                   /* admitted -> image in the caller's buffer */
    double latency_ms;               /* submit -> image in the caller's buffer */
    char error[128];
} SheenRequestInfo;

typedef struct SheenServerStats {
    unsigned long long submitted, completed, failed;
    unsigned long long rays;         /* over completed requests */
    double p50_ms, p99_ms, mean_ms, max_ms;   /* latency of completed requests (nearest rank) */
    double busy_ms;                  /* first submit -> last completion */
    unsigned long long hbm_budget, hbm_used, hbm_peak, scene_bytes;
    int inflight_peak, inflight, pending;
} SheenServerStats;

/* cfg may be NULL (defaults).  The server uses the current CUDA device. */
int  sheen_server_create(const SheenServerConfig* cfg, SheenServer* out);
/* Cancels pending requests (status FAILED), waits for in-flight ones, frees
 * every scene and buffer of the server. */
void sheen_server_destroy(SheenServer server);
/* Builds and uploads a scene (host BVH build included) and keeps it resident;
 * fails when it does not fit in the budget. */
int  sheen_server_add_scene(SheenServer server, const SheenScene* scene, int* scene_id);
/* Frees the scene once no queued or running request uses it; new submits
 * naming it fail at once. */
int  sheen_server_remove_scene(SheenServer server, int scene_id);
/* Queues a request.  out_rgba_host: width*height float4, written when the
 * request completes (RGBA, linear, as sheen_render_scene_rgba writes it); it
 * must stay valid until then.  Fails at once on bad parameters, an unknown
 * scene, or a footprint that could never fit. */
int  sheen_server_submit(SheenServer server, int scene_id, int width, int height, int aa_samples,
                         float* out_rgba_host, unsigned long long* request_id);
/* Status of a request (SHEEN_REQ_*), or -1 for an unknown id. */
int  sheen_server_poll(SheenServer server, unsigned long long request_id);
/* Waits up to timeout_ms (< 0: no limit).  Returns 1 when the request has
 * finished (info filled, the id is released), 0 on timeout (info filled with
 * the current state), -1 for an unknown id.  info may be NULL. */
int  sheen_server_wait(SheenServer server, unsigned long long request_id, double timeout_ms,
                       SheenRequestInfo* info);
int  sheen_server_stats(SheenServer server, SheenServerStats* out);

#ifdef __cplusplus
}
#endif

#endif /* SHEEN_C_API_H */
