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
        ok = se_span(r, se, t0, t1, sp.te, sp.tx);
        sp.mat = se.material_id;
    }
    if (ok) {
        sp.leaf = nd.leaf_index;
        sp.kind = nd.leaf_kind;
        out.s[out.n++] = sp;
    }
}

// integrator/csg.h:142-186: nearest interval of the root -> hit record.
static __device__ __noinline__ bool csg_test(const DevScene& S, const Ray& r, Hit& h) {
    const float t0 = r.tmin, t1 = r.tmax;
    int node_stack[kCsgMaxDepth + 1];
    unsigned char phase[kCsgMaxDepth + 1];
    SpanList vals[kCsgMaxDepth + 2];
    int nn = 0, nv = 0;
    node_stack[nn] = S.csg_root; phase[nn] = 0; nn++;
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
        h.n = normalize(se_gradient(S.ses[sp.leaf], h.p));
        h.tan = f3(1.0f, 0.0f, 0.0f);
    } else {
        h.n = f3(0.0f, 1.0f, 0.0f);
        h.tan = f3(1.0f, 0.0f, 0.0f);
    }
    h.uv = make_float2(h.p.x, h.p.y);
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    return true;
}

}  // namespace dev
}  // namespace sheen
