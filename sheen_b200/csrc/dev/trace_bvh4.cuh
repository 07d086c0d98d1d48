// trace_bvh4.cuh -- triangle queries of the wavefront form over the 4-wide
// BVH with 8-bit child boxes (bvh4.cpp), plus the query policy FastTracer.
//
// Closest hit: nearest-child-first traversal with culling against the
// closest hit found so far; stack entries carry their entry distance and are
// dropped when popped behind the current hit.  Any hit: the same walk,
// returning at the first accepted triangle.  The triangle test is the
// reference's Moller-Trumbore (primitives/triangle.h:8-36) on the stored
// v0/e1/e2, so a triangle answers exactly as in the plain form; only the
// order of visits differs, which changes the result only for exact ties.
//
// Child-box test: each child interval is decoded as t = fmaf(q, s * 1/d,
// (origin - o) * 1/d) per plane (one FMA), and the entry/exit distances are
// widened by 2^-20 relative before the range test, more than the rounding of
// the folded arithmetic, so a box is never culled where its triangles hit.
#pragma once
#include "trace_ref.cuh"

namespace sheen {
namespace dev {

constexpr int kQStack = 48;

struct QRay {
    float3 o, d;
    float ox, oy, oz;      // origin
    float ix, iy, iz;      // 1 / direction, zero components nudged to +-1e-30
    float tmin;
    uint32_t octant;       // bit k set when inverse direction component k is negative
};

__device__ __forceinline__ float safe_inv(float d) {
    return 1.0f / (fabsf(d) > 1e-30f ? d : copysignf(1e-30f, d));
}

__device__ __forceinline__ QRay make_qray(const Ray& r) {
    QRay q;
    q.o = r.o; q.d = r.d;
    q.ox = r.o.x; q.oy = r.o.y; q.oz = r.o.z;
    q.ix = safe_inv(r.d.x); q.iy = safe_inv(r.d.y); q.iz = safe_inv(r.d.z);
    q.tmin = r.tmin;
    q.octant = (q.ix < 0.0f ? 1u : 0u) | (q.iy < 0.0f ? 2u : 0u) | (q.iz < 0.0f ? 4u : 0u);
    return q;
}

// Three-input maximum / minimum (one instruction on sm_100).  Exact, so
// identical to two nested fmaxf / fminf on non-NaN operands.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Byte i of w as a float: one byte permute builds the float 2^23 + byte
// (exponent bits 0x4B in the top byte), one add removes 2^23.  Exact for
// every byte value.
__device__ __forceinline__ float byte_as_float(uint32_t w, int i) {
    // selector nibbles pick result bytes (low to high): byte i of w, then
    // zero, zero, 0x4B from the second operand (bytes 4..7 = 00 00 00 4B)
    const uint32_t sel = (uint32_t)i | 0x7440u;
    return __uint_as_float(__byte_perm(w, 0x4B000000u, sel)) - 8388608.0f;
}

// Tests the up-to-4 children of `node`; returns a bit mask of hit children
// and their entry distances.
//
// With a = s / d >= 0 the decoded plane distance fmaf(q, a, b) grows with q
// (fmaf is monotone in q), so the low byte gives the entry plane and the
// high byte the exit plane; with a < 0 the other way round.  The ray's
// octant picks the entry and exit words once per node, which gives exactly
// the min / max of the two plane distances without computing both orders.
// All four slots are evaluated and the unused ones masked off by the child
// count, so lanes on nodes with different counts do not diverge.
__device__ __forceinline__ int qnode_children(const QNode4* __restrict__ nodes, int id, const QRay& r, float tfar,
                                              float tn[4], uint4& child) {
    const float4 oe = __ldg(&nodes[id].origin_exp);
    child = __ldg(&nodes[id].child);
    const uint4 qb = __ldg(&nodes[id].qbox);
    const uint2 qz = __ldg(&nodes[id].qz);
    const uint32_t packed = __float_as_uint(oe.w);
    const int count = (int)(packed >> 24);
    const float sx = __uint_as_float((packed & 0xffu) << 23);
    const float sy = __uint_as_float(((packed >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((packed >> 16) & 0xffu) << 23);
    // t(q) = q * (s / d) + (origin - o) / d
    const float ax = sx * r.ix, bx = (oe.x - r.ox) * r.ix;
    const float ay = sy * r.iy, by = (oe.y - r.oy) * r.iy;
    const float az = sz * r.iz, bz = (oe.z - r.oz) * r.iz;
    const uint32_t xn = (r.octant & 1u) ? qb.y : qb.x, xf = (r.octant & 1u) ? qb.x : qb.y;
    const uint32_t yn = (r.octant & 2u) ? qb.w : qb.z, yf = (r.octant & 2u) ? qb.z : qb.w;
    const uint32_t zn = (r.octant & 4u) ? qz.y : qz.x, zf = (r.octant & 4u) ? qz.x : qz.y;
    int mask = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float x0 = fmaf(byte_as_float(xn, i), ax, bx), x1 = fmaf(byte_as_float(xf, i), ax, bx);
        const float y0 = fmaf(byte_as_float(yn, i), ay, by), y1 = fmaf(byte_as_float(yf, i), ay, by);
        const float z0 = fmaf(byte_as_float(zn, i), az, bz), z1 = fmaf(byte_as_float(zf, i), az, bz);
        const float tnear = fmax3(x0, y0, fmaxf(z0, r.tmin));
        const float texit = fmin3(x1, y1, fminf(z1, tfar));
        // widen by 2^-20 relative (texit grows, tnear shrinks)
        const float lo = tnear - fabsf(tnear) * 9.5367431640625e-7f;
        const float hi = texit + fabsf(texit) * 9.5367431640625e-7f;
        tn[i] = lo;
        if (lo <= hi && i < count) mask |= 1 << i;
    }
    return mask;
}

// Moller-Trumbore on stored {v0, e1, e2} (primitives/triangle.h:8-36).
__device__ __forceinline__ bool qtri_test_mt(const QRay& r, float4 a, float4 b, float4 c, float tmin, float tmax,
                                             float& t, float& u, float& v) {
    const float3 e1 = f3(b.x, b.y, b.z), e2 = f3(c.x, c.y, c.z);
    const float3 pv = cross(r.d, e2);
    const float det = dot(e1, pv);
    if (fabsf(det) < 1e-8f) return false;
    const float inv = 1.0f / det;
    const float3 tv = r.o - f3(a.x, a.y, a.z);
    u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    const float3 qv = cross(tv, e1);
    v = dot(r.d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, qv) * inv;
    return !(t < tmin || t > tmax);
}

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Watertight ray / triangle test (Woop, Benthin and Wald, "Watertight
// Ray/Triangle Intersection", JCGT 2013, restated).  The ray is sheared so
// that its direction becomes +z; the three 2D edge functions of the sheared
// triangle then decide the hit, each computed from the vertices alone, so
// two triangles sharing an edge evaluate that edge with the same operands
// and a ray through the edge (or a shared vertex) cannot pass between them.
// An edge function that rounds to exactly 0 is recomputed in double (the
// paper's fallback).  Same outputs as the Moller-Trumbore test: t and the
// weights u of v1, v of v2.
__device__ __forceinline__ bool qtri_test_wt(const QRay& r, float4 a, float4 b, float4 c, float tmin, float tmax,
                                             float& t, float& u, float& v) {
    const float ax = fabsf(r.d.x), ay = fabsf(r.d.y), az = fabsf(r.d.z);
    const int kz = ax > ay ? (ax > az ? 0 : 2) : (ay > az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    const float dz = comp(r.d, kz);
    if (dz < 0.0f) { const int k = kx; kx = ky; ky = k; }   // keep the winding
    const float sx = comp(r.d, kx) / dz, sy = comp(r.d, ky) / dz, sz = 1.0f / dz;
    const float3 A = f3(a.x, a.y, a.z) - r.o, B = f3(b.x, b.y, b.z) - r.o, C = f3(c.x, c.y, c.z) - r.o;
    const float Ax = comp(A, kx) - sx * comp(A, kz), Ay = comp(A, ky) - sy * comp(A, kz);
    const float Bx = comp(B, kx) - sx * comp(B, kz), By = comp(B, ky) - sy * comp(B, kz);
    const float Cx = comp(C, kx) - sx * comp(C, kz), Cy = comp(C, ky) - sy * comp(C, kz);
    // Products rounded separately (no fused multiply-add): a neighbour
    // evaluates the shared edge with the operands swapped, and only then is
    // its value exactly the negation of this one.
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
        V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
        W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float T = U * (sz * comp(A, kz)) + V * (sz * comp(B, kz)) + W * (sz * comp(C, kz));
    const float inv = 1.0f / det;
    t = T * inv;
    if (t < tmin || t > tmax) return false;
    u = V * inv;
    v = W * inv;
    return true;
}

// Triangle test selection: TRI 1 Moller-Trumbore, 2 watertight, 0 by the
// mesh's own flag at run time.  The hot queue kernels are compiled per test
// (TRI 1 or 2): the watertight code inlined beside the default one, even
// untaken, costs the default scenes 3% of their frame time.
template <int TRI>
__device__ __forceinline__ bool qtri_test(const QRay& r, float4 a, float4 b, float4 c, float tmin, float tmax,
                                          float& t, float& u, float& v, int watertight) {
    if constexpr (TRI == 1) return qtri_test_mt(r, a, b, c, tmin, tmax, t, u, v);
    else if constexpr (TRI == 2) return qtri_test_wt(r, a, b, c, tmin, tmax, t, u, v);
    else return watertight ? qtri_test_wt(r, a, b, c, tmin, tmax, t, u, v)
                           : qtri_test_mt(r, a, b, c, tmin, tmax, t, u, v);
}

// Closest (ANY = false) or any (ANY = true) triangle hit with t in
// [r.tmin, tmax] and strictly below `t_best` (in/out).  Returns the original
// triangle index or -1.
template <bool ANY, bool COUNT, int TRI>
__device__ __forceinline__ int qmesh_trace(const QMesh& m, const QRay& r, float tmax, float& t_best, float& bu,
                                           float& bv, Counters& c) {
    if (!m.nodes) return -1;
    // Any-hit walks need no visiting order: their stack holds entries only.
    // Closest-hit walks visit children near to far and keep each pushed
    // entry's distance so that entries behind the current hit are dropped.
    uint32_t stack_e[kQStack];
    float stack_t[ANY ? 1 : kQStack];
    int sp = 0;
    uint32_t entry = 0;   // root (inner)
    int best = -1;
    while (true) {
        if (!(entry & 0x80000000u)) {
            float tn[4];
            uint4 ch;
            if (COUNT) c.nodes++;
            const int mask = qnode_children(m.nodes, (int)entry, r, t_best, tn, ch);
            const uint32_t cid[4] = {ch.x, ch.y, ch.z, ch.w};
            if (mask == 0) goto pop;
            if constexpr (ANY) {
                int first = -1;
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (!(mask & (1 << i))) continue;
                    if (first < 0) first = i;
                    else if (sp < kQStack) stack_e[sp++] = cid[i];
                }
                entry = cid[first];
                continue;
            } else {
                // keys = distance bits with the slot in the low 2 bits (entry
                // distances are >= 0 here, so their bit patterns order like
                // the values)
                uint32_t key[4];
                int n = 0;
#pragma unroll
                for (int i = 0; i < 4; i++)
                    if (mask & (1 << i)) key[n++] = (__float_as_uint(fmaxf(tn[i], 0.0f)) & ~3u) | (uint32_t)i;
#define CSWAP(a, b) if (key[a] > key[b]) { uint32_t t_ = key[a]; key[a] = key[b]; key[b] = t_; }
                if (n == 2) { CSWAP(0, 1) }
                else if (n == 3) { CSWAP(0, 1) CSWAP(1, 2) CSWAP(0, 1) }
                else if (n == 4) { CSWAP(0, 1) CSWAP(2, 3) CSWAP(0, 2) CSWAP(1, 3) CSWAP(1, 2) }
#undef CSWAP
                for (int k = n - 1; k >= 1; k--) {
                    if (sp < kQStack) {
                        stack_e[sp] = cid[key[k] & 3u];
                        stack_t[sp] = tn[key[k] & 3u];
                        sp++;
                    }
                }
                entry = cid[key[0] & 3u];
                continue;
            }
        } else {
            const int first = (int)((entry & 0x7fffffffu) >> 3);
            const int count = (int)(entry & 7u) + 1;
            for (int k = 0; k < count; k++) {
                const int slot = first + k;
                const float4 a = __ldg(&m.tris[3 * slot]);
                const float4 b = __ldg(&m.tris[3 * slot + 1]);
                const float4 cc = __ldg(&m.tris[3 * slot + 2]);
                if (COUNT) c.prims++;
                float t, u, v;
                if (qtri_test<TRI>(r, a, b, cc, r.tmin, tmax, t, u, v, m.watertight) && t < t_best) {
                    t_best = t; bu = u; bv = v;
                    best = __float_as_int(a.w);
                    if (ANY) return best;
                }
            }
        }
    pop:
        if constexpr (ANY) {
            if (sp == 0) return best;
            entry = stack_e[--sp];
        } else {
            while (true) {
                if (sp == 0) return best;
                --sp;
                if (stack_t[sp] <= t_best) { entry = stack_e[sp]; break; }
            }
        }
    }
}

// Scenes with instanced meshes add them to the mesh category in functions
// of their own (dev/instances.cuh).
template <bool COUNT, int TRI>
__device__ __noinline__ bool mesh_q_inst(const DevScene& S, const Ray& r, Hit& h, Counters& c);
template <bool COUNT, int TRI>
__device__ __noinline__ int mesh_shadow_q_inst(const DevScene& S, const Ray& r, bool mask_aware, ShadowHit& sh,
                                               Counters& c);
template <bool COUNT, int TRI>
__device__ __noinline__ bool mesh_any_q_inst(const DevScene& S, const Ray& r, Counters& c);

// Closest mesh hit over q_all as a hit record (mesh_ref's result).
template <bool COUNT, int TRI>
__device__ __forceinline__ bool mesh_q(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_instances > 0) return mesh_q_inst<COUNT, TRI>(S, r, h, c);
    if (!S.q_all.nodes) return false;
    const QRay q = make_qray(r);
    float t = r.tmax, u = 0.0f, v = 0.0f;
    const int tri = qmesh_trace<false, COUNT, TRI>(S.q_all, q, r.tmax, t, u, v, c);
    if (tri < 0) return false;
    tri_finish(r, S.tris[tri], t, u, v, h);
    h.obj = -(tri + 1);
    return true;
}

// Mesh category of a shadow query (render_kernel.cu:248-267 over
// raycast.h:87): the category's closest hit decides.  With passable
// triangles present, the closest passable hit t_p is found first; any
// blocking hit before it (or anywhere when there is none) makes the closest
// hit blocking; otherwise the passable hit is classified by its material
// (mask-aware when asked).  Returns kClear when the mesh has no hit at all.
template <bool COUNT, int TRI>
__device__ __forceinline__ int mesh_shadow_q(const DevScene& S, const Ray& r, bool mask_aware, ShadowHit& sh,
                                             Counters& c) {
    if (S.num_instances > 0) return mesh_shadow_q_inst<COUNT, TRI>(S, r, mask_aware, sh, c);
    if (!S.q_all.nodes) return kClear;
    const QRay q = make_qray(r);
    if (!S.q_pass.nodes) {
        // No triangle can pass (every material's transmission <= 0.5, and a
        // property map only scales it down): any hit blocks.
        float t = r.tmax, u, v;
        return qmesh_trace<true, COUNT, TRI>(S.q_all, q, r.tmax, t, u, v, c) >= 0 ? kBlocked : kClear;
    }
    float tp = r.tmax, up = 0.0f, vp = 0.0f;
    const int pass_tri = qmesh_trace<false, COUNT, TRI>(S.q_pass, q, r.tmax, tp, up, vp, c);
    if (S.q_block.nodes) {
        float tb = tp, ub, vb;   // strictly closer than the passable hit (or than t_max)
        if (qmesh_trace<true, COUNT, TRI>(S.q_block, q, r.tmax, tb, ub, vb, c) >= 0) return kBlocked;
    }
    if (pass_tri < 0) return kClear;
    Hit h;
    tri_finish(r, S.tris[pass_tri], tp, up, vp, h);
    return classify_shadow_hit(S, h, mask_aware, sh);
}

// Any hit in the opaque categories (render_kernel.cu:413-422, media rays).
template <bool COUNT, int TRI>
__device__ __forceinline__ bool mesh_any_q(const DevScene& S, const Ray& r, Counters& c) {
    if (S.num_instances > 0) return mesh_any_q_inst<COUNT, TRI>(S, r, c);
    if (!S.q_all.nodes) return false;
    const QRay q = make_qray(r);
    float t = r.tmax, u, v;
    return qmesh_trace<true, COUNT, TRI>(S.q_all, q, r.tmax, t, u, v, c) >= 0;
}

// ---- non-triangle categories: culled, near-first walks ------------------
//
// The plain form walks the median BVHs of the other categories in the
// reference's order and tests every primitive whose leaf box the ray
// touches (bvh.h:605-922).  The wavefront form walks the same trees but
// visits the nearer child first and skips every box whose entry distance
// lies beyond the closest hit found so far.  A box is only ever visited when
// the reference's own slab test accepts it, so the primitives tested are a
// subset of the reference's, and the closest hit is the same unless two
// primitives hit at exactly the same distance.  Entry distances are widened
// by 2^-20 relative before the comparison, more than the rounding of the
// slab arithmetic.

// The reference slab test (box_hit_ref) that also returns the entry
// distance (largest of the three entry planes).
__device__ __forceinline__ bool box_enter_ref(const Ray& r, float4 a, float4 b, float& tnear) {
    float ix = 1.0f / r.d.x;
    float tminX = (a.x - r.o.x) * ix, tmaxX = (b.x - r.o.x) * ix;
    if (tminX > tmaxX) { float t = tminX; tminX = tmaxX; tmaxX = t; }
    float iy = 1.0f / r.d.y;
    float tminY = (a.y - r.o.y) * iy, tmaxY = (b.y - r.o.y) * iy;
    if (tminY > tmaxY) { float t = tminY; tminY = tmaxY; tmaxY = t; }
    if (tminX > tmaxY || tminY > tmaxX) return false;
    if (tminY > tminX) tminX = tminY;
    if (tmaxY < tmaxX) tmaxX = tmaxY;
    float iz = 1.0f / r.d.z;
    float tminZ = (a.z - r.o.z) * iz, tmaxZ = (b.z - r.o.z) * iz;
    if (tminZ > tmaxZ) { float t = tminZ; tminZ = tmaxZ; tmaxZ = t; }
    if (tminX > tmaxZ || tminZ > tmaxX) return false;
    if (tminZ > tminX) tminX = tminZ;
    tnear = tminX - fabsf(tminX) * 9.5367431640625e-7f;
    return (tmaxX >= r.tmin) && (tminX <= r.tmax);
}

// `leaf(prim)` tests one primitive and lowers `best` on a closer hit.
template <bool COUNT, class Leaf>
__device__ __forceinline__ void dfs_cull(const BvhNode* __restrict__ nodes, const Ray& r, const float& best,
                                         Counters& c, Leaf leaf) {
    int stack[kRefStack];
    float stack_t[kRefStack];
    int sp = 0;
    {
        const float4 a = __ldg(&nodes[0].a), b = __ldg(&nodes[0].b);
        float tn;
        if (COUNT) c.nodes++;
        if (!box_enter_ref(r, a, b, tn)) return;
        stack[0] = 0;
        stack_t[0] = tn;
        sp = 1;
    }
    while (sp > 0) {
        --sp;
        if (stack_t[sp] > best) continue;       // NaN entry distances are kept
        const int id = stack[sp];
        const float4 a = __ldg(&nodes[id].a), b = __ldg(&nodes[id].b);
        const int left = __float_as_int(a.w), right = __float_as_int(b.w);
        if (left < 0) {
            if (COUNT) c.prims++;
            leaf(~left);
            continue;
        }
        const float4 la = __ldg(&nodes[left].a), lb = __ldg(&nodes[left].b);
        const float4 ra = __ldg(&nodes[right].a), rb = __ldg(&nodes[right].b);
        float tl = 0.0f, tr = 0.0f;
        if (COUNT) c.nodes += 2;
        const bool hl = box_enter_ref(r, la, lb, tl) && !(tl > best);
        const bool hr = box_enter_ref(r, ra, rb, tr) && !(tr > best);
        if (sp > kRefStack - 2) continue;       // cannot happen for the trees built here
        if (hl && hr) {
            const bool l_first = !(tr < tl);
            stack[sp] = l_first ? right : left; stack_t[sp] = l_first ? tr : tl; sp++;
            stack[sp] = l_first ? left : right; stack_t[sp] = l_first ? tl : tr; sp++;
        } else if (hl) {
            stack[sp] = left; stack_t[sp] = tl; sp++;
        } else if (hr) {
            stack[sp] = right; stack_t[sp] = tr; sp++;
        }
    }
}

template <bool COUNT>
__device__ __forceinline__ bool spheres_cull(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_objects == 0 || !S.sphere_bvh) return false;
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.sphere_bvh, r, best, c, [&](int i) {
        const Object o = S.objects[i];
        Hit tmp;
        if (o.type == 0 && sphere_test(r, f3(o.param1), o.param2, tmp) && tmp.t < best) {
            h = tmp; h.mat = o.material_id; h.obj = i; best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool strands_cull(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_strands == 0) return false;
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.strand_bvh, r, best, c, [&](int i) {
        Hit tmp;
        if (strand_test<true>(r, S.strands[i], S.sweep_points, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

// Extension scenes (SheenSceneExt) walk their categories in functions of
// their own, not inlined, so that the kernels' code for the reference's
// shapes is what it is without extensions.
template <bool COUNT>
static __device__ __noinline__ bool hfs_cull_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.hf_bvh, r, best, c, [&](int i) {
        Hit tmp;
        const HfGrid g = hf_grid_of(S, i);
        if ((g.h ? hf_test_grid(r, S.hfs[i], tmp, g) : hf_test(r, S.hfs[i], tmp)) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool hfs_cull(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_hfs == 0) return false;
    if (S.hf_grid) return hfs_cull_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.hf_bvh, r, best, c, [&](int i) {
        Hit tmp;
        if (hf_test(r, S.hfs[i], tmp) && tmp.t < best) { h = tmp; h.obj = -(i + 1); best = tmp.t; any = true; }
    });
    return any;
}

template <bool COUNT>
static __device__ __noinline__ bool ses_cull_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.se_bvh, r, best, c, [&](int i) {
        Hit tmp;
        const float n2 = se_n2_of(S, i);
        if ((n2 > 0.0f ? se_test2(r, S.ses[i], n2, tmp) : se_test<true>(r, S.ses[i], tmp, S.se_polish)) &&
            tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool ses_cull(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_ses == 0) return false;
    if (S.se_n2) return ses_cull_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.se_bvh, r, best, c, [&](int i) {
        Hit tmp;
        if (se_test<true>(r, S.ses[i], tmp, S.se_polish) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
static __device__ __noinline__ bool lathes_cull_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    const LatheRay lr(r);
    dfs_cull<COUNT>(S.lathe_bvh, r, best, c, [&](int i) {
        Hit tmp;
        const int2 run = lathe_run_of(S, i);
        const bool ok = run.y > 0 ? lathe_exact_test(r, S.bz_spans, run, __ldg(&S.lathe_bz_bound[i]),
                                                     S.lathes[i].material_id, tmp)
                                  : lathe_test_pre(r, lr, S.lathes[i], S.lathe_seg, __ldg(&S.lathe_bound[i]), tmp);
        if (ok && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

// Tessellated lathes through the height buckets (DevScene.lathe_grid): the
// ray's t-range inside the cylinder about the Y axis that holds every
// lathe, cut to the buckets' height range, gives the buckets it can meet;
// each segment listed there is tested once (in the first of those buckets
// that lists it), with lathe_test_pre's per-segment test.  The closest hit
// over all lathes is the per-lathe walk's (exact ties between two lathes
// may resolve the other way).
template <bool COUNT>
__device__ __forceinline__ bool lathes_grid(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    const float4 g = __ldg(&S.lathe_grid[0]);
    const int nb = __float_as_int(g.w);
    const LatheRay lr(r);
    // inside the cylinder x^2 + z^2 <= R^2 (q(t) = axz t^2 + 2 bxz t + cxz)
    float ta = r.tmin, tb = r.tmax;
    const float R2 = g.z * g.z;
    if (lr.axz > 0.0f) {
        const float disc = lr.bxz * lr.bxz - lr.axz * (lr.cxz - R2);
        if (!(disc >= 0.0f)) return false;
        const float sq = sqrtf(disc);
        const float c0 = (-lr.bxz - sq) / lr.axz, c1 = (-lr.bxz + sq) / lr.axz;
        const float slack = 1e-5f * (fabsf(c0) + fabsf(c1)) + 1e-6f;
        ta = fmaxf(ta, c0 - slack);
        tb = fminf(tb, c1 + slack);
    } else if (lr.cxz > R2) {
        return false;
    }
    // and inside the buckets' height range
    const float y_lo = g.x, y_hi = g.x + (float)nb / g.y;
    if (r.d.y != 0.0f) {
        const float u0 = (y_lo - r.o.y) * lr.inv[1], u1 = (y_hi - r.o.y) * lr.inv[1];
        ta = fmaxf(ta, fminf(u0, u1));
        tb = fminf(tb, fmaxf(u0, u1));
    } else if (r.o.y < y_lo || r.o.y > y_hi) {
        return false;
    }
    if (ta > tb + 1e-5f * (fabsf(ta) + fabsf(tb)) + 1e-6f) return false;
    const float ya = r.o.y + ta * r.d.y, yb = r.o.y + tb * r.d.y;
    const float ylo = fminf(ya, yb), yhi = fmaxf(ya, yb);
    const float m = 1e-4f * (fabsf(ylo) + fabsf(yhi)) + 1e-5f;
    const int b0 = max(0, min(nb - 1, (int)floorf((ylo - m - g.x) * g.y)));
    const int b1 = max(0, min(nb - 1, (int)floorf((yhi + m - g.x) * g.y)));
    bool any = false;
    float best = r.tmax;
    int lathe = -1;
    for (int b = b0; b <= b1; b++) {
        const int k0 = __ldg(&S.lathe_grid_start[b]), k1 = __ldg(&S.lathe_grid_start[b + 1]);
        for (int k = k0; k < k1; k++) {
            const int it = __ldg(&S.lathe_grid_items[k]);
            const int first = (int)((unsigned)it >> 24);
            if (max(first, b0) != b) continue;
            const int p = it & 0xffffff;
            if (COUNT) c.prims++;
            if (lathe_seg_hit(r, lr, S.lathe_seg, p, best, h)) { any = true; lathe = p; }
        }
    }
    if (!any) return false;
    const int li = __ldg(&S.lathe_of_point[lathe]);
    h.mat = S.lathes[li].material_id;
    h.uv = make_float2(0.0f, 0.0f);
    h.obj = -(li + 1);
    return true;
}

template <bool COUNT>
__device__ __forceinline__ bool lathes_cull(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_lathes == 0) return false;
    if (S.lathe_bz) return lathes_cull_ext<COUNT>(S, r, h, c);
    if (S.lathe_grid) return lathes_grid<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    const LatheRay lr(r);
    dfs_cull<COUNT>(S.lathe_bvh, r, best, c, [&](int i) {
        Hit tmp;
        if (lathe_test_pre(r, lr, S.lathes[i], S.lathe_seg, __ldg(&S.lathe_bound[i]), tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
static __device__ __noinline__ bool prisms_cull_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.prism_bvh, r, best, c, [&](int i) {
        Hit tmp;
        if (prism_any_test(S, r, i, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool prisms_cull(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_prisms == 0) return false;
    if (S.prism_bz) return prisms_cull_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_cull<COUNT>(S.prism_bvh, r, best, c, [&](int i) {
        Hit tmp;
        if (prism_test(r, S.prisms[i], S.prism_points, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

// Scene categories a kernel variant compiles in (a scene outside a
// variant's set runs the full variant).
enum : int {
    kCatSpheres = 1, kCatStrands = 2, kCatMesh = 4, kCatHF = 8, kCatSE = 16, kCatLathe = 32, kCatPrism = 64,
    kCatCSG = 128, kCatPlanes = 256,
    kCatAll = 511,
    kCatSimple = kCatSpheres | kCatMesh | kCatPlanes,
    kCatBasic = kCatSpheres | kCatPlanes,
    // triangle test compiled in (neither bit: chosen per mesh at run time)
    kTriMT = 512, kTriWT = 1024
};

// Query policy of the wavefront form: triangles through the BVH4s, every
// other category through the plain form's code (same category order).
template <int F>
constexpr int tri_of() { return (F & kTriWT) ? 2 : ((F & kTriMT) ? 1 : 0); }

template <bool COUNT, int F = kCatAll>
struct FastTracer {
    __device__ __forceinline__ static bool closest(const DevScene& S, const Ray& r, Hit& rec, Counters& c) {
        float best = r.tmax;
        bool hit = false;
        Hit t;
        if ((F & kCatSpheres) && spheres_cull<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatStrands) && strands_cull<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatMesh) && mesh_q<COUNT, tri_of<F>()>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatHF) && hfs_cull<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatSE) && ses_cull<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatLathe) && lathes_cull<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatPrism) && prisms_cull<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatCSG) && csg_closest(S, r, t, true) && t.t < best) { best = t.t; rec = t; hit = true; }
        if ((F & kCatPlanes) && planes_scan(S, r, t) && t.t < best) { best = t.t; rec = t; hit = true; }
        return hit;
    }
    __device__ __forceinline__ static int shadow(const DevScene& S, const Ray& r, bool mask_aware, ShadowHit& sh,
                                                 Counters& c) {
        Hit h;
        if ((F & kCatSpheres) && spheres_cull<COUNT>(S, r, h, c)) return classify_shadow_hit(S, h, mask_aware, sh);
        if (F & kCatMesh) {
            const int m = mesh_shadow_q<COUNT, tri_of<F>()>(S, r, mask_aware, sh, c);
            if (m != kClear) return m;
        }
        if (((F & kCatHF) && hfs_cull<COUNT>(S, r, h, c)) || ((F & kCatSE) && ses_cull<COUNT>(S, r, h, c)) ||
            ((F & kCatLathe) && lathes_cull<COUNT>(S, r, h, c)) || ((F & kCatPrism) && prisms_cull<COUNT>(S, r, h, c)) ||
            ((F & kCatCSG) && csg_closest(S, r, h, true)) || ((F & kCatPlanes) && planes_scan(S, r, h)))
            return classify_shadow_hit(S, h, mask_aware, sh);
        return kClear;
    }
    // The shadow query split around its mesh category, for callers that walk
    // the mesh themselves: the sphere category (-1 when it has no hit, else
    // its classification) and the categories after the mesh (kClear when
    // none has a hit).  shadow() == pre, else mesh, else post.
    __device__ __forceinline__ static int shadow_pre_mesh(const DevScene& S, const Ray& r, bool mask_aware,
                                                          ShadowHit& sh, Counters& c) {
        Hit h;
        if ((F & kCatSpheres) && spheres_cull<COUNT>(S, r, h, c)) return classify_shadow_hit(S, h, mask_aware, sh);
        return -1;
    }
    __device__ __forceinline__ static int shadow_post_mesh(const DevScene& S, const Ray& r, bool mask_aware,
                                                           ShadowHit& sh, Counters& c) {
        Hit h;
        if (((F & kCatHF) && hfs_cull<COUNT>(S, r, h, c)) || ((F & kCatSE) && ses_cull<COUNT>(S, r, h, c)) ||
            ((F & kCatLathe) && lathes_cull<COUNT>(S, r, h, c)) || ((F & kCatPrism) && prisms_cull<COUNT>(S, r, h, c)) ||
            ((F & kCatCSG) && csg_closest(S, r, h, true)) || ((F & kCatPlanes) && planes_scan(S, r, h)))
            return classify_shadow_hit(S, h, mask_aware, sh);
        return kClear;
    }
    __device__ __forceinline__ static bool occluded(const DevScene& S, const Ray& r, Counters& c) {
        Hit h;
        if ((F & kCatSpheres) && spheres_cull<COUNT>(S, r, h, c)) return true;
        if ((F & kCatMesh) && mesh_any_q<COUNT, tri_of<F>()>(S, r, c)) return true;
        return ((F & kCatHF) && hfs_cull<COUNT>(S, r, h, c)) || ((F & kCatSE) && ses_cull<COUNT>(S, r, h, c)) ||
               ((F & kCatLathe) && lathes_cull<COUNT>(S, r, h, c)) ||
               ((F & kCatPrism) && prisms_cull<COUNT>(S, r, h, c)) ||
               ((F & kCatCSG) && csg_closest(S, r, h, true)) || ((F & kCatPlanes) && planes_scan(S, r, h));
    }
    __device__ __forceinline__ static float strand_depth(const DevScene& S, const Ray& r, Counters& c) {
        return (F & kCatStrands) ? strands_tau_ref<COUNT, true>(S, r, c) : 0.0f;
    }
};

}  // namespace dev
}  // namespace sheen

#include "instances.cuh"
