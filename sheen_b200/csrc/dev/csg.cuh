// csg.cuh -- interval CSG (integrator/csg.h:22-186) without recursion.
//
// The reference evaluates the tree recursively with two 8-interval arrays
// per level on the thread stack (hence its 16 KB stack limit).  Here the
// tree is evaluated post-order with an explicit node stack and a value stack
// of interval lists, bounded by kCsgMaxDepth levels; a deeper tree reports no
// CSG hit (the loader never builds one: .sheen trees are a few levels deep).
// The set algebra and its 8-interval cap are the reference's.
#pragma once
#include "prims.cuh"

namespace sheen {
namespace dev {

constexpr int kCsgMaxDepth = 12;

struct Span {
    float te, tx;
    int mat, leaf, kind;
};

struct SpanList {
    Span s[8];
    int n;
};

// integrator/csg.h:43-112
__device__ __forceinline__ void csg_combine(const SpanList& A, const SpanList& B, int op, SpanList& out) {
    out.n = 0;
    if (op == 0) {
        Span tmp[16];
        int n = 0;
        for (int i = 0; i < A.n && n < 16; i++) tmp[n++] = A.s[i];
        for (int i = 0; i < B.n && n < 16; i++) tmp[n++] = B.s[i];
        for (int i = 1; i < n; i++) {
            Span key = tmp[i];
            int j = i - 1;
            while (j >= 0 && tmp[j].te > key.te) { tmp[j + 1] = tmp[j]; j--; }
            tmp[j + 1] = key;
        }
        for (int i = 0; i < n && out.n < 8; i++) {
            if (out.n == 0 || tmp[i].te > out.s[out.n - 1].tx) out.s[out.n++] = tmp[i];
            else if (tmp[i].tx > out.s[out.n - 1].tx) out.s[out.n - 1].tx = tmp[i].tx;
        }
    } else if (op == 1) {
        for (int i = 0; i < A.n; i++)
            for (int j = 0; j < B.n; j++) {
                float t0 = fmaxf(A.s[i].te, B.s[j].te), t1 = fminf(A.s[i].tx, B.s[j].tx);
                if (t0 < t1 && out.n < 8) { out.s[out.n] = A.s[i]; out.s[out.n].te = t0; out.s[out.n].tx = t1; out.n++; }
            }
    } else if (op == 2) {
        for (int i = 0; i < A.n; i++) {
            float cur = A.s[i].te;
            for (int j = 0; j < B.n; j++) {
                float b0 = B.s[j].te, b1 = B.s[j].tx;
                if (b1 <= cur) continue;
                if (b0 >= A.s[i].tx) break;
                if (b0 > cur && out.n < 8) { out.s[out.n] = A.s[i]; out.s[out.n].te = cur; out.s[out.n].tx = b0; out.n++; }
                cur = fmaxf(cur, b1);
                if (cur >= A.s[i].tx) break;
            }
            if (cur < A.s[i].tx && out.n < 8) { out.s[out.n] = A.s[i]; out.s[out.n].te = cur; out.s[out.n].tx = A.s[i].tx; out.n++; }
        }
    }
}

// Extension leaves (no counterpart in the reference, whose leaves are
// spheres and superellipsoids).  Both solids are convex, so a ray meets
// each in one interval, clipped to [t0, t1] like sphere_span.
__device__ __forceinline__ bool box_span(const Ray& r, float3 lo, float3 hi, float t0, float t1, float& te,
                                         float& tx) {
    const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
    const float l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
    float tn = -3.0e38f, tf = 3.0e38f;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float inv = 1.0f / d[a];
        const float ta = (l[a] - o[a]) * inv, tb = (h[a] - o[a]) * inv;
        tn = fmaxf(tn, fminf(ta, tb));
        tf = fminf(tf, fmaxf(ta, tb));
    }
    if (!(tn <= tf) || tf < t0 || tn > t1) return false;
    te = fmaxf(tn, t0);
    tx = fminf(tf, t1);
    return te <= tx;
}

// Capped cone (frustum) from p0 (radius r0) to p1 (radius r1): the axial
// slab [0, L] intersected with |w|^2 <= (r0 + k h)^2, w the offset from the
// axis, h the axial coordinate, k = (r1 - r0) / L.
__device__ __forceinline__ bool cone_span(const Ray& r, float3 p0, float r0, float3 p1, float r1, float t0, float t1,
                                          float& te, float& tx) {
    const float3 ax = p1 - p0;
    const float L = sqrtf(dot(ax, ax));
    if (!(L > 0.0f)) return false;
    const float3 a = ax / L;
    const float3 oc = r.o - p0;
    const float ho = dot(oc, a), hd = dot(r.d, a);
    float sa, sb;
    if (fabsf(hd) > 1e-30f) {
        sa = (0.0f - ho) / hd;
        sb = (L - ho) / hd;
        if (sa > sb) { const float t = sa; sa = sb; sb = t; }
    } else {
        if (ho < 0.0f || ho > L) return false;
        sa = -3.0e38f;
        sb = 3.0e38f;
    }
    const float k = (r1 - r0) / L, rb = r0 + k * ho, rk = k * hd;
    const float A = dot(r.d, r.d) - hd * hd - rk * rk;
    const float B = 2.0f * (dot(oc, r.d) - ho * hd - rb * rk);
    const float C = dot(oc, oc) - ho * ho - rb * rb;
    float lo = sa, hi = sb;
    if (fabsf(A) <= 1e-12f * (fabsf(B) + fabsf(C) + 1e-30f)) {
        if (B == 0.0f) { if (C > 0.0f) return false; }
        else if (B > 0.0f) hi = fminf(hi, -C / B);
        else lo = fmaxf(lo, -C / B);
    } else {
        const float disc = B * B - 4.0f * A * C;
        if (A > 0.0f) {
            if (disc < 0.0f) return false;
            const float sq = sqrtf(disc);
            lo = fmaxf(lo, (-B - sq) / (2.0f * A));
            hi = fminf(hi, (-B + sq) / (2.0f * A));
        } else if (disc >= 0.0f) {
            // q <= 0 outside the roots: the piece on the frustum's side of
            // the apex (radius r0 + k h >= 0 at its middle)
            const float sq = sqrtf(disc);
            const float ra = (-B + sq) / (2.0f * A), rbb = (-B - sq) / (2.0f * A);   // ra <= rbb
            const float l1 = lo, h1 = fminf(hi, ra), l2 = fmaxf(lo, rbb), h2 = hi;
            const bool ok1 = l1 <= h1, ok2 = l2 <= h2;
            if (ok1 && ok2) {
                const float m1 = 0.5f * (fmaxf(l1, -1e30f) + fminf(h1, 1e30f));
                if (r0 + k * (ho + m1 * hd) >= 0.0f) hi = h1; else lo = l2;
            } else if (ok1) {
                hi = h1;
            } else if (ok2) {
                lo = l2;
            } else {
                return false;
            }
        }
    }
    if (!(lo <= hi) || hi < t0 || lo > t1) return false;
    te = fmaxf(lo, t0);
    tx = fminf(hi, t1);
    return te <= tx;
}

__device__ __forceinline__ float se_n2_of(const DevScene& S, int i) {
    return S.se_n2 ? __ldg(&S.se_n2[i]) : 0.0f;
}

__device__ __forceinline__ void csg_leaf(const DevScene& S, const CSGNode& nd, const Ray& r, float t0, float t1,
                                         SpanList& out) {
    out.n = 0;
    Span sp;
    bool ok = false;
    if (nd.leaf_kind == 0) {
        const Object o = S.objects[nd.leaf_index];
        ok = sphere_span(r, f3(o.param1), o.param2, t0, t1, sp.te, sp.tx);
        sp.mat = o.material_id;
    } else if (nd.leaf_kind == 1) {
        const Superellipsoid se = S.ses[nd.leaf_index];
        const float n2 = se_n2_of(S, nd.leaf_index);
        ok = n2 > 0.0f ? se_span2(r, se, n2, t0, t1, sp.te, sp.tx, nullptr) : se_span(r, se, t0, t1, sp.te, sp.tx);
        sp.mat = se.material_id;
    } else if (nd.leaf_kind == 2 && S.csg_boxes) {
        const float4 lo = __ldg(&S.csg_boxes[2 * nd.leaf_index]), hi = __ldg(&S.csg_boxes[2 * nd.leaf_index + 1]);
        ok = box_span(r, f3(lo.x, lo.y, lo.z), f3(hi.x, hi.y, hi.z), t0, t1, sp.te, sp.tx);
        sp.mat = __float_as_int(lo.w);
    } else if (nd.leaf_kind == 3 && S.csg_cones) {
        const float4 a = __ldg(&S.csg_cones[3 * nd.leaf_index]), b = __ldg(&S.csg_cones[3 * nd.leaf_index + 1]);
        ok = cone_span(r, f3(a.x, a.y, a.z), a.w, f3(b.x, b.y, b.z), b.w, t0, t1, sp.te, sp.tx);
        sp.mat = __float_as_int(__ldg(&S.csg_cones[3 * nd.leaf_index + 2]).x);
    }
    if (ok) {
        sp.leaf = nd.leaf_index;
        sp.kind = nd.leaf_kind;
        out.s[out.n++] = sp;
    }
}

// Outward normal direction of an extension leaf at p.
__device__ __forceinline__ float3 csg_ext_normal(const DevScene& S, int kind, int leaf, float3 p) {
    if (kind == 2) {
        const float4 lo = __ldg(&S.csg_boxes[2 * leaf]), hi = __ldg(&S.csg_boxes[2 * leaf + 1]);
        const float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
        const float e[3] = {0.5f * (hi.x - lo.x), 0.5f * (hi.y - lo.y), 0.5f * (hi.z - lo.z)};
        const float q[3] = {p.x - c[0], p.y - c[1], p.z - c[2]};
        int best = 0;
        float bd = 3.0e38f;
        for (int a = 0; a < 3; a++) {
            const float dd = fabsf(e[a] - fabsf(q[a])) / fmaxf(e[a], 1e-30f);
            if (dd < bd) { bd = dd; best = a; }
        }
        float3 n = f3(0.0f, 0.0f, 0.0f);
        const float sg = q[best] >= 0.0f ? 1.0f : -1.0f;
        if (best == 0) n.x = sg; else if (best == 1) n.y = sg; else n.z = sg;
        return n;
    }
    const float4 a4 = __ldg(&S.csg_cones[3 * leaf]), b4 = __ldg(&S.csg_cones[3 * leaf + 1]);
    const float3 p0 = f3(a4.x, a4.y, a4.z), ax = f3(b4.x, b4.y, b4.z) - p0;
    const float L = sqrtf(dot(ax, ax));
    const float3 a = ax / L;
    const float hh = dot(p - p0, a);
    const float3 w = (p - p0) - hh * a;
    const float k = (b4.w - a4.w) / L, rad = a4.w + k * hh, wl = sqrtf(dot(w, w));
    const float side = fabsf(wl - rad) / fmaxf(fmaxf(a4.w, b4.w), 1e-30f);
    const float cap0 = fabsf(hh) / L, cap1 = fabsf(hh - L) / L;
    if (cap0 < side && cap0 <= cap1) return -a;
    if (cap1 < side) return a;
    // the side: gradient of |w|^2 - (r0 + k h)^2
    return wl > 0.0f ? w - (rad * k) * a : a;
}

// integrator/csg.h:142-186: nearest interval of the tree at `root` -> hit
// record.
static __device__ __noinline__ bool csg_tree_test(const DevScene& S, const Ray& r, Hit& h, int root) {
    const float t0 = r.tmin, t1 = r.tmax;
    int node_stack[kCsgMaxDepth + 1];
    unsigned char phase[kCsgMaxDepth + 1];
    SpanList vals[kCsgMaxDepth + 2];
    int nn = 0, nv = 0;
    node_stack[nn] = root; phase[nn] = 0; nn++;
    while (nn > 0) {
        const int id = node_stack[nn - 1];
        const CSGNode nd = S.csg_nodes[id];
        if (nd.leaf_kind >= 0) {
            if (nv >= kCsgMaxDepth + 2) return false;
            csg_leaf(S, nd, r, t0, t1, vals[nv++]);
            nn--;
            continue;
        }
        const int ph = phase[nn - 1];
        if (ph < 2) {
            phase[nn - 1] = (unsigned char)(ph + 1);
            const int child = ph == 0 ? nd.left : nd.right;
            if (child >= 0) {
                if (nn > kCsgMaxDepth) return false;
                node_stack[nn] = child; phase[nn] = 0; nn++;
            } else {
                if (nv >= kCsgMaxDepth + 2) return false;
                vals[nv++].n = 0;
            }
            continue;
        }
        // both children evaluated: A = vals[nv-2], B = vals[nv-1]
        SpanList out;
        csg_combine(vals[nv - 2], vals[nv - 1], nd.op, out);
        nv -= 2;
        vals[nv++] = out;
        nn--;
    }
    if (nv != 1) return false;
    const SpanList& L = vals[0];
    float best = 1e30f;
    int bi = -1;
    for (int i = 0; i < L.n; i++)
        if (L.s[i].te < best && L.s[i].tx > t0) { best = L.s[i].te; bi = i; }
    if (bi < 0) return false;
    const Span sp = L.s[bi];
    const float t = fmaxf(sp.te, t0);
    if (t < t0 || t > t1) return false;
    h.t = t;
    h.mat = sp.mat;
    h.obj = 0;
    h.p = r.o + t * r.d;
    if (sp.kind == 0) {
        h.n = normalize(h.p - f3(S.objects[sp.leaf].param1));
        h.tan = f3(0.0f, 0.0f, 0.0f);
    } else if (sp.kind == 1) {
        h.n = normalize(se_normal_dir(S.ses[sp.leaf], se_n2_of(S, sp.leaf), h.p));
        h.tan = f3(1.0f, 0.0f, 0.0f);
    } else if (sp.kind == 2 || sp.kind == 3) {
        h.n = normalize(csg_ext_normal(S, sp.kind, sp.leaf, h.p));
        h.tan = f3(1.0f, 0.0f, 0.0f);
    } else {
        h.n = f3(0.0f, 1.0f, 0.0f);
        h.tan = f3(1.0f, 0.0f, 0.0f);
    }
    h.uv = make_float2(h.p.x, h.p.y);
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    return true;
}

// The scene's own tree (integrator/csg.h: a single root).
__device__ __forceinline__ bool csg_test(const DevScene& S, const Ray& r, Hit& h) {
    return csg_tree_test(S, r, h, S.csg_root);
}

// Extension: the closest hit over the further trees of the scene's CSG
// forest, walked through the median BVH over their leaf boxes (boxes beyond
// the closest hit so far are skipped).  Each tree is evaluated over the
// ray's whole [tmin, tmax], as when it is alone.
static __device__ __noinline__ bool csg_forest_test(const DevScene& S, const Ray& r, Hit& h) {
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    bool any = false;
    float best = r.tmax;
    while (sp > 0) {
        const int id = stack[--sp];
        const float4 a = __ldg(&S.csg_root_bvh[id].a), b = __ldg(&S.csg_root_bvh[id].b);
        Ray rb = r;
        rb.tmax = best;
        if (!box_hit_ref(rb, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z))) continue;
        const int left = __float_as_int(a.w), right = __float_as_int(b.w);
        if (left < 0) {
            Hit t;
            if (csg_tree_test(S, r, t, S.csg_roots[~left]) && t.t < best) { h = t; best = t.t; any = true; }
            continue;
        }
        if (sp > 62) continue;   // cannot happen for the trees built here
        stack[sp++] = right;
        stack[sp++] = left;
    }
    return any;
}

// The CSG category with the extension forest: the scene's tree (with
// cull_box, skipped when the ray misses the box of its leaves), then the
// further trees; strict '<' keeps the earlier tree on a tie.  Not inlined:
// scenes without a forest take csg_closest's single-tree path.
static __device__ __noinline__ bool csg_closest_forest(const DevScene& S, const Ray& r, Hit& h, bool cull_box) {
    bool any = false;
    if (S.csg_root >= 0 && (!cull_box || ray_meets_box(r, S.csg_lo, S.csg_hi)) && csg_test(S, r, h)) any = true;
    Hit t;
    if (csg_forest_test(S, r, t) && (!any || t.t < h.t)) { h = t; any = true; }
    return any;
}

// The CSG category (integrator/csg.h: the scene's single tree, culled by the
// box of its leaves when cull_box), or with an extension forest every tree.
__device__ __forceinline__ bool csg_closest(const DevScene& S, const Ray& r, Hit& h, bool cull_box) {
    if (S.num_csg_roots > 0) return csg_closest_forest(S, r, h, cull_box);
    return S.csg_root >= 0 && (!cull_box || ray_meets_box(r, S.csg_lo, S.csg_hi)) && csg_test(S, r, h);
}

__device__ __forceinline__ bool has_csg(const DevScene& S) { return S.csg_root >= 0 || S.num_csg_roots > 0; }

}  // namespace dev
}  // namespace sheen
