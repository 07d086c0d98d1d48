// scene.cuh -- device view of a resident scene, shared by every renderer form.
//
// All arrays live in HBM for the lifetime of a SheenDeviceScene.  The ABI
// records (Material, Light, Object, ...) are uploaded unchanged; what the
// traversal reads in its inner loops is repacked into 16-byte-aligned
// records loaded with 128-bit loads:
//   BvhNode   32 B  {lo.xyz, left}, {hi.xyz, right}   (plain form, one per
//                   box, leaf: left = right = ~primitive, the reference
//                   encoding of bvh.h:14-19)
//   TriVerts  48 B  {v0.xyz, -}, {v1.xyz, -}, {v2.xyz, -} positions only;
//                   normals/UVs stay in the 112-byte Triangle record that is
//                   read once per shaded hit.
#pragma once
#include <cuda_runtime.h>

#include <vector_types.h>

#include "sheen_c_api.h"

namespace sheen {
namespace dev {

struct __align__(16) BvhNode {
    float4 a;   // lo.xyz, left child (or ~prim)
    float4 b;   // hi.xyz, right child (or ~prim)
};

struct PhotonMapView {
    const float4* pos;      // xyz position, w unused        (stored by cell)
    const float4* nrm;      // xyz normal
    const float4* flux;     // xyz flux
    const int* cell_start;  // [num_cells + 1]
    const int* cell_count;  // [num_cells]
    int num_cells;          // 2^18, or 0 when there is no map
    float cell_size;
};

// Wide BVH of the wavefront form: 4 children with 8-bit boxes quantised in
// a per-node frame (see bvh4.h for the encoding).
struct __align__(16) QNode4 {
    float4 origin_exp;      // origin.xyz, exponents packed in w (3 x int8 + child count)
    uint4 child;            // child index / leaf (offset<<4 | count) per slot
    uint4 qbox;             // 4 x {qlo.x, qhi.x, qlo.y, qhi.y}
    uint2 qz;               // 4 x {qlo.z, qhi.z}
    uint2 pad;
};

// One BVH4 over a set of triangles: nodes and 3 float4 per triangle slot in
// leaf order.  watertight selects the triangle test and the record layout:
// 0 the reference's Moller-Trumbore on {v0, original index}, {e1, 0},
// {e2, 0}; 1 the watertight edge-function test on {v0, index}, {v1, 0},
// {v2, 0}.
struct QMesh {
    const QNode4* nodes;
    const float4* tris;
    int num_nodes;
    int num_tris;
    int watertight;
};

// float4 per instance record: world-to-object rows (3), object-to-world
// rows (3), {mesh, material, base - first triangle of the mesh, passable},
// {base, triangles, first triangle of the mesh, 0} (ints); base = the
// triangles of the instances before it.
constexpr int kInstRecord = 8;

// Reflect + refract recursion depth limit of the extension scenes.
constexpr int kMaxDeepBounces = 8;

struct DevScene {
    CameraData cam;

    const Object* objects; int num_objects;  const BvhNode* sphere_bvh;
    const SweepStrand* strands; const SweepPoint* sweep_points; int num_strands; const BvhNode* strand_bvh;
    const Triangle* tris; const float4* tri_verts; int num_tris; const BvhNode* mesh_bvh;
    const HeightField* hfs; int num_hfs; const BvhNode* hf_bvh;
    const Superellipsoid* ses; int num_ses; const BvhNode* se_bvh;
    const Lathe* lathes; const LathePoint* lathe_points; int num_lathes; const BvhNode* lathe_bvh;
    // Per lathe point p (the segment from p to p + 1): cone_test's profile
    // constants, {y0, r0, k, L} and {axis y, 0, 0, 1 when the segment is
    // tested}, computed on the device by lathe_segments_kernel with
    // cone_test's own expressions.
    const float4* lathe_seg;
    // Per lathe: {R, y_lo, y_hi, valid}, a box about the world Y axis that
    // holds the lathe's surface (|x|, |z| <= R, y in [y_lo, y_hi]) with a
    // margin of 1e-4 relative; a ray that misses it cannot hit the lathe.
    const float4* lathe_bound;
    const Prism* prisms; const PrismPoint* prism_points; int num_prisms; const BvhNode* prism_bvh;
    const CSGNode* csg_nodes; int csg_root;
    // Box holding every CSG leaf solid (sphere: centre +- radius;
    // superellipsoid: centre +- (a, b, c)), widened by 1e-4 relative: the
    // tree's solid lies inside the union of its leaves, so a ray that misses
    // the box has no CSG hit.  Empty (lo > hi) without a tree.
    float csg_lo[3], csg_hi[3];
    const Plane* planes; int num_planes;
    const Material* materials; int num_materials;
    const TextureRef* textures; int num_textures;
    const Light* lights; int num_lights;
    const Medium* media; int num_media;
    PhotonMapView pmap;
    float caustics;

    // Wavefront form: BVH4 meshes (root at node 0; nodes == null when empty).
    //   q_all     every triangle (closest-hit queries)
    //   q_block   triangles whose material can never pass a shadow ray
    //             (transmission <= 0.5): any-hit shadow queries
    //   q_pass    the others (transmission > 0.5, possibly through a mask):
    //             closest-hit shadow queries, usually a small set
    QMesh q_all, q_block, q_pass;
    int has_glass;                 // any material with transmission > 0
    int aa_centered;               // camera samples without jitter (extension; 0: the reference's jitter)
    int se_polish;                 // FP64 Newton polish of superellipsoid entries (extension; 0: off)
    int caustic_knn;               // k-nearest-photon gather (extension; 0: the reference's gather)

    // Scene extensions (SheenSceneExt; no counterpart in the reference).
    // Null / 0 when the scene has none.
    const float* se_n2;            // per superellipsoid: north-south exponent (> 0: two-exponent body)
    const int4* hf_grid;           // per heightfield: {offset into hf_heights (< 0: none), w, h, -}
    const float* hf_heights;
    const int4* lathe_bz;          // per lathe: {first span, spans, -, -} (spans 0: tessellated)
    const float4* lathe_bz_bound;  // per lathe: {R, y_lo, y_hi, -} of its exact surface
    const int4* prism_bz;          // per prism: {first span, spans, -, -}
    const float4* bz_spans;        // 2 float4 per cubic span: {a0, b0, a1, b1}, {a2, b2, a3, b3}
    const int* csg_roots;          // further CSG tree roots (closest hit over all trees)
    int num_csg_roots;
    const BvhNode* csg_root_bvh;   // median BVH over the further roots' leaf boxes
    const float4* csg_boxes;       // leaf_kind 2: {lo, material as int}, {hi, 0}
    const float4* csg_cones;       // leaf_kind 3: {p0, r0}, {p1, r1}, {material as int, 0, 0, 0}
    int bounces;                   // reflect + refract bounces (> 1: the recursion of render_sample_deep)
    // Wavefront form, tessellated lathes: their profile segments bucketed by
    // height over the union of the lathes (all turn about the world Y axis):
    // {y0, 1 / bucket height, radius bound, buckets as int}; bucket b's items
    // in [start[b], start[b + 1]), each a profile point p (low 24 bits) with
    // the first bucket listing it (high 8 bits); the lathe of each point.
    // Null without lathes or with exact Bezier ones.
    const float4* lathe_grid;
    const int* lathe_grid_start;
    const int* lathe_grid_items;
    const int* lathe_of_point;
    // Instanced meshes (two-level BVH); num_instances 0 without.
    const Triangle* inst_tris;     // every mesh's object-space triangles
    const QMesh* inst_mesh;        // per mesh: its BVH4 in object space
    const float4* inst_xf;         // per instance kInstRecord float4 (dev/instances.cuh)
    const QNode4* tlas_nodes;      // BVH4 over the instances' world boxes (root node 0)
    const int* tlas_items;         // per top-level leaf slot: instance (num_instances: the scene's triangles)
    int num_instances;
    int inst_tri_total;            // triangles of all instances (flattened count)
    int inst_flat_leaf;            // 1: top-level leaf num_instances is the scene's own triangles
};

struct Ray {
    float3 o, d;
    float tmin, tmax;
};

// Closest hit: the reference's HitRecord fields (types.h:34-44).
struct Hit {
    float t;
    int mat;
    int obj;
    float3 p, n, tan;
    float2 uv;
};

}  // namespace dev
}  // namespace sheen
