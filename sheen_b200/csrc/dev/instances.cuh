// instances.cuh -- instanced meshes in a two-level BVH (scene extension, no
// counterpart in the reference, whose loader flattens every copy).
//
// Top level: a BVH4 over the instances' world boxes.  Bottom level: one
// BVH4 per mesh in object space.  Both are walked in one loop (inst_walk).  A ray enters an instance through the instance's
// world-to-object map applied to origin and direction, the direction left
// unnormalised, so a hit's t is the same in both spaces and the closest hit
// over instances and the scene's own triangles compares plain t values.
//
// Instanced triangles belong to the mesh category: the mesh hit of a query
// is the closest over the scene's triangles and the instances (in the
// wavefront form the scene's triangles are one more top-level leaf, walked
// in the same loop; in the plain form they are walked first and a tie keeps
// them), and a shadow query classifies that hit like the scene's
// own (an instance passes a shadow ray when its material's transmission is
// above 0.5).  A hit reports the triangle's flattened index (the scene's
// triangles, then instance by instance), so shading reads the same triangle
// a flattened copy of the scene would.
#pragma once
#include "trace_bvh4.cuh"

namespace sheen {
namespace dev {

__device__ __forceinline__ float3 xf_point(float4 a, float4 b, float4 c, float3 p) {
    return f3(fmaf(a.x, p.x, fmaf(a.y, p.y, fmaf(a.z, p.z, a.w))), fmaf(b.x, p.x, fmaf(b.y, p.y, fmaf(b.z, p.z, b.w))),
              fmaf(c.x, p.x, fmaf(c.y, p.y, fmaf(c.z, p.z, c.w))));
}
__device__ __forceinline__ float3 xf_dir(float4 a, float4 b, float4 c, float3 d) {
    return f3(fmaf(a.x, d.x, fmaf(a.y, d.y, a.z * d.z)), fmaf(b.x, d.x, fmaf(b.y, d.y, b.z * d.z)),
              fmaf(c.x, d.x, fmaf(c.y, d.y, c.z * d.z)));
}

// The ray in instance i's object space (same tmin / tmax).
__device__ __forceinline__ Ray inst_ray(const DevScene& S, int i, const Ray& r) {
    const float4* xf = S.inst_xf + (size_t)kInstRecord * i;
    const float4 a = __ldg(&xf[0]), b = __ldg(&xf[1]), c = __ldg(&xf[2]);
    Ray o;
    o.o = xf_point(a, b, c, r.o);
    o.d = xf_dir(a, b, c, r.d);
    o.tmin = r.tmin;
    o.tmax = r.tmax;
    return o;
}

__device__ __forceinline__ int4 inst_meta(const DevScene& S, int i) {
    return __ldg(reinterpret_cast<const int4*>(S.inst_xf + (size_t)kInstRecord * i + 6));
}

// Children of a BVH4 node onto a walk's stack: qmesh_trace's order (any
// order for ANY walks; near to far for closest-hit walks, the nearer pushed
// last) and entry distances.  Returns the child to visit next and its entry
// distance in `next_t`.
template <bool ANY, int CAP = kQStack>
__device__ __forceinline__ uint32_t qnode_push(int mask, const float tn[4], const uint4& ch, uint32_t* stack_e,
                                               float* stack_t, int& sp, float& next_t) {
    const uint32_t cid[4] = {ch.x, ch.y, ch.z, ch.w};
    if constexpr (ANY) {
        int first = -1;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!(mask & (1 << k))) continue;
            if (first < 0) first = k;
            else if (sp < CAP) stack_e[sp++] = cid[k];
        }
        next_t = tn[first];
        return cid[first];
    } else {
        uint32_t key[4];
        int n = 0;
#pragma unroll
        for (int k = 0; k < 4; k++)
            if (mask & (1 << k)) key[n++] = (__float_as_uint(fmaxf(tn[k], 0.0f)) & ~3u) | (uint32_t)k;
#define CSWAP(a, b) if (key[a] > key[b]) { uint32_t t_ = key[a]; key[a] = key[b]; key[b] = t_; }
        if (n == 2) { CSWAP(0, 1) }
        else if (n == 3) { CSWAP(0, 1) CSWAP(1, 2) CSWAP(0, 1) }
        else if (n == 4) { CSWAP(0, 1) CSWAP(2, 3) CSWAP(0, 2) CSWAP(1, 3) CSWAP(1, 2) }
#undef CSWAP
        for (int k = n - 1; k >= 1; k--) {
            if (sp < CAP) {
                stack_e[sp] = cid[key[k] & 3u];
                stack_t[sp] = tn[key[k] & 3u];
                sp++;
            }
        }
        next_t = tn[key[0] & 3u];
        return cid[key[0] & 3u];
    }
}

// Stack entries of the two-level walk: at most 3 per level of either tree,
// the marker between them, and a top-level leaf's remainder.
constexpr int kInstStack = 72;
constexpr uint32_t kInstMarker = 0x7fffffffu;   // never an inner node id

// Closest instanced triangle strictly below `best` (in/out) among the
// instances WANT selects (0 all, 1 passable, 2 blocking; the scene's own
// triangles, when they are a top-level leaf: q_all, q_pass, or q_block --
// q_all when nothing passes); ANY: the first such hit.  Returns the
// instance (num_instances: the scene's triangles; -1: no hit) with the
// triangle and its barycentrics.
//
// One loop and one stack walk both levels, one BVH4 node per iteration:
// the inner-node step is the same code for the top level (the instances'
// world boxes, world ray) and a mesh (object-space ray), so the lanes of a
// warp stay together whichever level each is in.  Entering an item pushes
// a marker; popping the marker restores the world ray and the top level.
// A top-level leaf of several items visits the first and pushes the rest.
// Child order, culling and the triangle test are qmesh_trace's.
template <bool ANY, bool COUNT, int TRI, int WANT>
__device__ __forceinline__ int inst_walk(const DevScene& S, const Ray& r, float& best, int& tri, float& bu,
                                         float& bv, Counters& c) {
    constexpr uint32_t kLeaf = 0x80000000u;
    uint32_t stack_e[kInstStack];
    float stack_t[ANY ? 1 : kInstStack];
    int sp = 0;
    int found = -1;
    int item = -1;                   // item whose mesh is being walked (-1: the top level)
    QRay q = make_qray(r);           // the current level's ray
    const QNode4* nodes = S.tlas_nodes;
    const float4* tris = nullptr;
    int wt = 0;
    uint32_t e = 0;                  // top-level root (inner)
    float et = 0.0f;                 // entry distance of e
    while (true) {
        if (!(e & kLeaf)) {
            float tn[4];
            uint4 ch;
            if (COUNT) c.nodes++;
            const int mask = qnode_children(nodes, (int)e, q, best, tn, ch);
            if (mask != 0) {
                e = qnode_push<ANY, kInstStack>(mask, tn, ch, stack_e, stack_t, sp, et);
                continue;
            }
        } else if (item < 0) {
            // top-level leaf: enter its first item
            const int first = (int)((e & 0x7fffffffu) >> 3);
            const int count = (int)(e & 7u) + 1;
            const int i = __ldg(&S.tlas_items[first]);
            if (count > 1 && sp < kInstStack) {      // the leaf's other items, same entry distance
                stack_e[sp] = kLeaf | ((uint32_t)(first + 1) << 3) | (uint32_t)(count - 2);
                if (!ANY) stack_t[sp] = et;
                sp++;
            }
            const int4 meta = inst_meta(S, i);
            QMesh m;
            m.nodes = nullptr;
            if (meta.x < 0) m = WANT == 0 ? S.q_all : (WANT == 1 ? S.q_pass : (S.q_pass.nodes ? S.q_block : S.q_all));
            else if (!((WANT == 1 && !meta.w) || (WANT == 2 && meta.w))) m = S.inst_mesh[meta.x];
            if (m.nodes && sp < kInstStack) {
                if (COUNT) c.prims++;
                stack_e[sp] = kInstMarker;
                if (!ANY) stack_t[sp] = -INFINITY;
                sp++;
                if (meta.x >= 0) q = make_qray(inst_ray(S, i, r));
                nodes = m.nodes; tris = m.tris; wt = m.watertight;
                item = i; e = 0;
                continue;
            }
        } else {
            const int first = (int)((e & 0x7fffffffu) >> 3);
            const int count = (int)(e & 7u) + 1;
            for (int k = 0; k < count; k++) {
                const int slot = first + k;
                const float4 a = __ldg(&tris[3 * slot]);
                const float4 b = __ldg(&tris[3 * slot + 1]);
                const float4 cc = __ldg(&tris[3 * slot + 2]);
                if (COUNT) c.prims++;
                float t, u, v;
                if (qtri_test<TRI>(q, a, b, cc, q.tmin, r.tmax, t, u, v, wt) && t < best) {
                    best = t; bu = u; bv = v;
                    tri = __float_as_int(a.w);
                    found = item;
                    if (ANY) return found;
                }
            }
        }
        // next entry; the marker returns to the top level
        while (true) {
            if (sp == 0) return found;
            --sp;
            if (stack_e[sp] == kInstMarker) {
                item = -1;
                q = make_qray(r);
                nodes = S.tlas_nodes;
                continue;
            }
            if (ANY || stack_t[sp] <= best) {
                e = stack_e[sp];
                if (!ANY) et = stack_t[sp];
                break;
            }
        }
    }
}

// Hit record of triangle `tri` of instance i at t: position on the world
// ray, normal through the inverse transpose, tangent through the forward
// map, the instance's material, the flattened triangle index.
static __device__ __noinline__ void inst_finish(const DevScene& S, int i, int tri, const Ray& r, float t, float u,
                                                float v, Hit& h) {
    const Ray ro = inst_ray(S, i, r);
    tri_finish(ro, S.inst_tris[tri], t, u, v, h);
    const float4* xf = S.inst_xf + (size_t)kInstRecord * i;
    const float4 a = __ldg(&xf[0]), b = __ldg(&xf[1]), c = __ldg(&xf[2]);
    const float4 fa = __ldg(&xf[3]), fb = __ldg(&xf[4]), fc = __ldg(&xf[5]);
    const int4 meta = inst_meta(S, i);
    const float3 n = h.n, tg = h.tan;
    h.n = normalize(f3(a.x * n.x + b.x * n.y + c.x * n.z, a.y * n.x + b.y * n.y + c.y * n.z,
                       a.z * n.x + b.z * n.y + c.z * n.z));
    h.tan = normalize(xf_dir(fa, fb, fc, tg));
    h.p = r.o + t * r.d;
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    h.mat = meta.y;
    h.obj = -(S.num_tris + 1 + meta.z + tri);
}

// ---- the mesh category with instances (the hooks of mesh_q, mesh_ref,
// mesh_shadow_q and mesh_any_q) --------------------------------------------

template <bool COUNT, int TRI>
__device__ __noinline__ bool mesh_q_inst(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.inst_flat_leaf) {
        // one walk over the scene's triangles and the instances together
        float best = r.tmax, u = 0.0f, v = 0.0f;
        int tri = -1;
        const int found = inst_walk<false, COUNT, TRI, 0>(S, r, best, tri, u, v, c);
        if (found < 0) return false;
        if (found < S.num_instances) {
            inst_finish(S, found, tri, r, best, u, v, h);
        } else {
            tri_finish(r, S.tris[tri], best, u, v, h);
            h.obj = -(tri + 1);
        }
        return true;
    }
    float best = r.tmax, u = 0.0f, v = 0.0f;
    int flat = -1;
    if (S.q_all.nodes) {
        const QRay q = make_qray(r);
        flat = qmesh_trace<false, COUNT, TRI>(S.q_all, q, r.tmax, best, u, v, c);
    }
    int tri = -1;
    float iu = 0.0f, iv = 0.0f;
    const int inst = inst_walk<false, COUNT, TRI, 0>(S, r, best, tri, iu, iv, c);
    if (inst >= 0) {
        inst_finish(S, inst, tri, r, best, iu, iv, h);
        return true;
    }
    if (flat < 0) return false;
    tri_finish(r, S.tris[flat], best, u, v, h);
    h.obj = -(flat + 1);
    return true;
}

template <bool COUNT>
__device__ __noinline__ bool mesh_ref_inst(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    Hit flat;
    const bool hf = mesh_ref_flat<COUNT>(S, r, flat, c);
    float best = hf ? flat.t : r.tmax;
    int tri = -1;
    float u = 0.0f, v = 0.0f;
    const int inst = inst_walk<false, COUNT, 0, 0>(S, r, best, tri, u, v, c);
    if (inst >= 0) {
        inst_finish(S, inst, tri, r, best, u, v, h);
        return true;
    }
    if (hf) h = flat;
    return hf;
}

// Shadow query of the mesh category: the closest passable hit over both
// levels, any blocking hit strictly before it blocks, else the passable hit
// is classified (kClear when neither level has a hit).
template <bool COUNT, int TRI>
__device__ __noinline__ int mesh_shadow_q_inst(const DevScene& S, const Ray& r, bool mask_aware, ShadowHit& sh,
                                               Counters& c) {
    if (S.inst_flat_leaf) {
        // passable set (the scene's q_pass and the passable instances), then
        // the blocking set strictly before its closest hit, each in one walk
        float tp = r.tmax, up = 0.0f, vp = 0.0f;
        int ptri = -1;
        const int pfound = inst_walk<false, COUNT, TRI, 1>(S, r, tp, ptri, up, vp, c);
        float tb = tp, ub, vb;
        int bt;
        if (inst_walk<true, COUNT, TRI, 2>(S, r, tb, bt, ub, vb, c) >= 0) return kBlocked;
        if (pfound < 0) return kClear;
        Hit h;
        if (pfound < S.num_instances) inst_finish(S, pfound, ptri, r, tp, up, vp, h);
        else tri_finish(r, S.tris[ptri], tp, up, vp, h);
        return classify_shadow_hit(S, h, mask_aware, sh);
    }
    const QRay q = make_qray(r);
    float tp = r.tmax, up = 0.0f, vp = 0.0f;
    int pass_flat = -1;
    if (S.q_pass.nodes) pass_flat = qmesh_trace<false, COUNT, TRI>(S.q_pass, q, r.tmax, tp, up, vp, c);
    int ptri = -1;
    float iu = 0.0f, iv = 0.0f;
    const int pinst = inst_walk<false, COUNT, TRI, 1>(S, r, tp, ptri, iu, iv, c);
    // blocking triangles of the scene: q_block, or every triangle when none passes
    const QMesh& blk = S.q_pass.nodes ? S.q_block : S.q_all;
    if (blk.nodes) {
        float tb = tp, ub, vb;
        if (qmesh_trace<true, COUNT, TRI>(blk, q, r.tmax, tb, ub, vb, c) >= 0) return kBlocked;
    }
    {
        float tb = tp, ub, vb;
        int bt;
        if (inst_walk<true, COUNT, TRI, 2>(S, r, tb, bt, ub, vb, c) >= 0) return kBlocked;
    }
    Hit h;
    if (pinst >= 0) inst_finish(S, pinst, ptri, r, tp, iu, iv, h);
    else if (pass_flat >= 0) tri_finish(r, S.tris[pass_flat], tp, up, vp, h);
    else return kClear;
    return classify_shadow_hit(S, h, mask_aware, sh);
}

template <bool COUNT, int TRI>
__device__ __noinline__ bool mesh_any_q_inst(const DevScene& S, const Ray& r, Counters& c) {
    float t = r.tmax, u, v;
    if (S.inst_flat_leaf) {
        int tri;
        return inst_walk<true, COUNT, TRI, 0>(S, r, t, tri, u, v, c) >= 0;
    }
    if (S.q_all.nodes) {
        const QRay q = make_qray(r);
        if (qmesh_trace<true, COUNT, TRI>(S.q_all, q, r.tmax, t, u, v, c) >= 0) return true;
    }
    int tri;
    t = r.tmax;
    return inst_walk<true, COUNT, TRI, 0>(S, r, t, tri, u, v, c) >= 0;
}

}  // namespace dev
}  // namespace sheen
