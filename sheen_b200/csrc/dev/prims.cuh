// prims.cuh -- ray/primitive tests with the reference's semantics.
//
// Each function states the reference lines whose results it reproduces.
// They are shared by every renderer form: the forms differ in how they find
// candidate primitives, never in how a primitive answers.
#pragma once
#include <cfloat>

#include "scene.cuh"
#include "vec.cuh"

namespace sheen {
namespace dev {

// Slab test of bvh.h:578-600.  Note the reference's final check uses the
// interval merged over x and y only (z only rejects disjoint slabs).
__device__ __forceinline__ bool box_hit_ref(const Ray& r, float3 lo, float3 hi) {
    float ix = 1.0f / r.d.x;
    float tminX = (lo.x - r.o.x) * ix, tmaxX = (hi.x - r.o.x) * ix;
    if (tminX > tmaxX) { float t = tminX; tminX = tmaxX; tmaxX = t; }
    float iy = 1.0f / r.d.y;
    float tminY = (lo.y - r.o.y) * iy, tmaxY = (hi.y - r.o.y) * iy;
    if (tminY > tmaxY) { float t = tminY; tminY = tmaxY; tmaxY = t; }
    if (tminX > tmaxY || tminY > tmaxX) return false;
    if (tminY > tminX) tminX = tminY;
    if (tmaxY < tmaxX) tmaxX = tmaxY;
    float iz = 1.0f / r.d.z;
    float tminZ = (lo.z - r.o.z) * iz, tmaxZ = (hi.z - r.o.z) * iz;
    if (tminZ > tmaxZ) { float t = tminZ; tminZ = tmaxZ; tmaxZ = t; }
    if (tminX > tmaxZ || tminZ > tmaxX) return false;
    return (tmaxX >= r.tmin) && (tminX <= r.tmax);
}

// primitives/sphere.h:33-53: near root, else far root, inside [tmin, tmax].
__device__ __forceinline__ bool sphere_test(const Ray& r, float3 c, float rad, Hit& h) {
    float3 oc = r.o - c;
    float a = dot(r.d, r.d);
    float b = 2.0f * dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float t = (-b - sq) / (2.0f * a);
    if (t < r.tmin || t > r.tmax) {
        t = (-b + sq) / (2.0f * a);
        if (t < r.tmin || t > r.tmax) return false;
    }
    h.t = t;
    h.p = r.o + t * r.d;
    h.n = normalize(h.p - c);
    h.tan = f3(0.0f, 0.0f, 0.0f);
    h.uv = make_float2(0.0f, 0.0f);
    return true;
}

// primitives/sphere.h:11-28: [t_enter, t_exit] clipped to [t0, t1].
__device__ __forceinline__ bool sphere_span(const Ray& r, float3 c, float rad, float t0, float t1,
                                            float& te, float& tx) {
    float3 oc = r.o - c;
    float a = dot(r.d, r.d);
    float b = 2.0f * dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float ta = (-b - sq) / (2.0f * a);
    float tb = (-b + sq) / (2.0f * a);
    if (tb < t0 || ta > t1) return false;
    te = fmaxf(ta, t0);
    tx = fminf(tb, t1);
    return te <= tx;
}

// primitives/plane.h:7-24
__device__ __forceinline__ bool plane_test(const Ray& r, float3 n, float d, Hit& h) {
    float den = dot(n, r.d);
    if (fabsf(den) > 1e-6f) {
        float t = -(dot(r.o, n) + d) / den;
        if (t >= r.tmin && t <= r.tmax) {
            h.t = t;
            h.p = r.o + t * r.d;
            h.n = dot(n, r.d) > 0.0f ? -n : n;
            h.tan = f3(0.0f, 0.0f, 0.0f);
            h.uv = make_float2(0.0f, 0.0f);
            return true;
        }
    }
    return false;
}

// primitives/triangle.h:8-47, positions only (Moller-Trumbore, det eps 1e-8,
// u, v in [0, 1]).  Returns t and barycentrics; the hit record is completed
// by tri_finish() once the closest triangle is known.
__device__ __forceinline__ bool tri_test(const Ray& r, float3 v0, float3 v1, float3 v2,
                                         float& t, float& u, float& v) {
    float3 e1 = v1 - v0, e2 = v2 - v0;
    float3 pv = cross(r.d, e2);
    float det = dot(e1, pv);
    if (fabsf(det) < 1e-8f) return false;
    float inv = 1.0f / det;
    float3 tv = r.o - v0;
    u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    float3 qv = cross(tv, e1);
    v = dot(r.d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot(e2, qv) * inv;
    return !(t < r.tmin || t > r.tmax);
}

__device__ __forceinline__ void tri_finish(const Ray& r, const Triangle& tr, float t, float u, float v, Hit& h) {
    float3 v0 = f3(tr.v0), e1 = f3(tr.v1) - v0, e2 = f3(tr.v2) - v0;
    h.t = t;
    h.p = r.o + t * r.d;
    float w = 1.0f - u - v;
    float3 nv = f3(tr.n0) * w + f3(tr.n1) * u + f3(tr.n2) * v;
    h.n = dot(nv, nv) > 1e-12f ? normalize(nv) : normalize(cross(e1, e2));
    h.tan = normalize(e1);
    h.uv = make_float2(tr.uv0.x * w + tr.uv1.x * u + tr.uv2.x * v, tr.uv0.y * w + tr.uv1.y * u + tr.uv2.y * v);
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    h.mat = tr.material_id;
}

// primitives/cone.h:11-73: truncated cone between two sweep points, radial
// normal (no axial term), first root inside the ray range and the segment.
__device__ __forceinline__ bool cone_test(const Ray& r, float3 p0, float r0, float3 p1, float r1, Hit& h) {
    float3 axis = p1 - p0;
    float L2 = dot(axis, axis);
    if (L2 < 1e-12f) return false;
    float L = sqrtf(L2);
    float3 da = axis / L;
    float k = (r1 - r0) / L;
    float3 Q = r.o - p0;
    float u = dot(r.d, da), v = dot(Q, da);
    float3 Dp = r.d - u * da, Qp = Q - v * da;
    float A = dot(Dp, Dp) - k * k * u * u;
    float B = 2.0f * (dot(Dp, Qp) - k * r0 * u - k * k * v * u);
    float C = dot(Qp, Qp) - k * k * v * v - 2.0f * k * r0 * v - r0 * r0;
    float disc = B * B - 4.0f * A * C;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float i2a = 1.0f / (2.0f * A);
    float s1 = (-B - sq) * i2a, s2 = (-B + sq) * i2a;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        float s = i == 0 ? s1 : s2;
        if (s < r.tmin || s > r.tmax) continue;
        float tp = v + s * u;
        if (tp < 0.0f || tp > L) continue;
        h.t = s;
        h.p = r.o + s * r.d;
        h.n = normalize(Qp + s * Dp);
        h.tan = da;
        if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
        return true;
    }
    return false;
}

// primitives/cone.h:78-121: sphere cap kept on the side of `axis`.  The
// reference leaves the tangent unset here; it is zero in this renderer.
__device__ __forceinline__ bool cap_test(const Ray& r, float3 c, float rad, float3 axis, Hit& h) {
    float3 oc = r.o - c;
    float a = dot(r.d, r.d);
    float b = 2.0f * dot(oc, r.d);
    float cc = dot(oc, oc) - rad * rad;
    float disc = b * b - 4.0f * a * cc;
    if (disc < 0.0f) return false;
    float sq = sqrtf(disc);
    float i2a = 1.0f / (2.0f * a);
    float t1 = (-b - sq) * i2a, t2 = (-b + sq) * i2a;
#pragma unroll
    for (int i = 0; i < 2; i++) {
        float t = i == 0 ? t1 : t2;
        if (t < r.tmin || t > r.tmax) continue;
        float3 p = r.o + t * r.d;
        float3 n = normalize(p - c);
        if (dot(n, axis) < 0.0f) continue;
        h.t = t; h.p = p; h.n = dot(n, r.d) > 0.0f ? -n : n;
        h.tan = f3(0.0f, 0.0f, 0.0f);
        return true;
    }
    return false;
}

// primitives/sweep.h:13-90: a strand = caps at both ends + cone pieces with
// caps at the joints; closest of all against the unchanged ray range.
// Whether the ray's line comes within R = half + rmax of the point m.  A
// miss is declared only beyond R by 1e-3 relative plus the cancellation
// error of the squared distance (1e-5 of |w|^2 + R^2), so the pieces it
// skips are ones whose tests report no hit (or no depth):
//   - a piece from a to b with radii up to rmax (its cone and end caps) lies
//     within |b - a| / 2 + rmax of its midpoint;
//   - piece_tau measures the distance between the points o - v t (t >= 0)
//     and a - u s (s in [0, 1]) -- its w = o - a with the reference's signs
//     -- so the depth it can report comes from the segment a .. 2a - b:
//     centre a - u / 2, the same half length.
__device__ __forceinline__ bool piece_in_reach(const Ray& r, float3 m, float half, float rmax) {
    const float R = half + fabsf(rmax);
    const float3 w = m - r.o;
    const float dd = dot(r.d, r.d);
    if (!(dd > 0.0f)) return true;
    const float p = dot(w, r.d);
    const float ww = dot(w, w);
    const float d2 = ww - p * p / dd;
    const float R2 = R * R;
    return !(d2 > R2 * 1.002001f + 1e-5f * (ww + R2));
}

// CULL (the wavefront form): pieces out of reach (piece_in_reach) skip
// their tests; the hits are the same.
template <bool CULL = false>
__device__ __forceinline__ bool strand_test(const Ray& r, const SweepStrand& st, const SweepPoint* pts, Hit& h) {
    const int n = st.point_count;
    if (n < 2) return false;
    const SweepPoint* P = pts + st.point_offset;
    bool any = false;
    float best = r.tmax;
    Hit tmp;
    auto reach = [&](float3 a, float3 b, float ra, float rb) {
        const float3 u = b - a;
        return piece_in_reach(r, 0.5f * (a + b), 0.5f * sqrtf(dot(u, u)), fmaxf(fabsf(ra), fabsf(rb)));
    };
    const bool reach0 = !CULL || reach(f3(P[0].position), f3(P[1].position), P[0].radius, P[1].radius);
    if (reach0 && cap_test(r, f3(P[0].position), P[0].radius, normalize(f3(P[0].position) - f3(P[1].position)), tmp) &&
        tmp.t < best) { h = tmp; best = tmp.t; any = true; }
    for (int i = 0; i < n - 1; i++) {
        float3 a = f3(P[i].position), b = f3(P[i + 1].position);
        if (CULL && !reach(a, b, P[i].radius, P[i + 1].radius)) continue;
        if (cone_test(r, a, P[i].radius, b, P[i + 1].radius, tmp) && tmp.t < best) { h = tmp; best = tmp.t; any = true; }
        if (i < n - 2) {
            float3 ax = normalize(f3(P[i + 2].position) - b);
            if (cap_test(r, b, P[i + 1].radius, ax, tmp) && tmp.t < best) { h = tmp; best = tmp.t; any = true; }
        }
    }
    float3 pl = f3(P[n - 1].position), pp = f3(P[n - 2].position);
    const bool reach1 = !CULL || reach(pp, pl, P[n - 2].radius, P[n - 1].radius);
    if (reach1 && cap_test(r, pl, P[n - 1].radius, normalize(pl - pp), tmp) && tmp.t < best) {
        h = tmp; best = tmp.t; any = true;
    }
    if (any) { h.mat = st.material_id; h.uv = make_float2(0.0f, 0.0f); }
    return any;
}

// primitives/sweep.h:96-137: optical depth of one strand piece for a ray.
__device__ __forceinline__ float piece_tau(const Ray& r, const SweepPoint& a, const SweepPoint& b, float sigma) {
    float3 u = f3(b.position) - f3(a.position);
    float A = dot(u, u);
    if (A < 1e-12f) return 0.0f;
    float3 v = r.d, w = r.o - f3(a.position);
    float B = dot(u, v), C = dot(v, v), D = dot(u, w), E = dot(v, w);
    float den = A * C - B * B;
    float s = (den > 1e-9f) ? (B * E - C * D) / den : 0.0f;
    s = fminf(fmaxf(s, 0.0f), 1.0f);
    float t = (B * s + E) / C;
    if (t < 0.0f) { t = 0.0f; s = fminf(fmaxf(-D / A, 0.0f), 1.0f); }
    if (t > r.tmax) return 0.0f;
    float3 cl = w + u * s - v * t;
    float d2 = dot(cl, cl);
    float rr = a.radius + (b.radius - a.radius) * s;
    float r2 = rr * rr;
    if (d2 >= r2) return 0.0f;
    return sigma * (2.0f * sqrtf(fmaxf(r2 - d2, 0.0f)));
}

template <bool CULL = false>
__device__ __forceinline__ float strand_tau(const Ray& r, const SweepStrand& st, const SweepPoint* pts, float sigma) {
    float tau = 0.0f;
    for (int i = 0; i < st.point_count - 1; i++) {
        const SweepPoint& a = pts[st.point_offset + i];
        const SweepPoint& b = pts[st.point_offset + i + 1];
        // a piece out of reach adds exactly 0 (piece_tau's segment is a .. 2a - b)
        if (CULL) {
            const float3 u = f3(b.position) - f3(a.position);
            if (!piece_in_reach(r, f3(a.position) - 0.5f * u, 0.5f * sqrtf(dot(u, u)),
                                fmaxf(fabsf(a.radius), fabsf(b.radius))))
                continue;
        }
        tau += piece_tau(r, a, b, sigma);
        if (tau > 6.0f) break;
    }
    return tau;
}

// primitives/lathe.h:14-63.  The profile turns about the world Y axis
// (x = z = 0): Lathe.center does not move the surface, as in the reference.
__device__ __forceinline__ bool lathe_test(const Ray& r, const Lathe& l, const LathePoint* pts, Hit& h) {
    if (l.point_count < 2) return false;
    bool any = false;
    float best = r.tmax;
    Hit tmp;
    for (int i = 0; i < l.point_count - 1; i++) {
        const LathePoint a = pts[l.point_offset + i], b = pts[l.point_offset + i + 1];
        if (a.radius <= 0.0f && b.radius <= 0.0f) continue;
        if (cone_test(r, f3(0.0f, a.y, 0.0f), a.radius, f3(0.0f, b.y, 0.0f), b.radius, tmp) && tmp.t < best) {
            tmp.p = r.o + tmp.t * r.d;
            h = tmp; best = tmp.t; any = true;
        }
    }
    if (any) { h.mat = l.material_id; h.uv = make_float2(0.0f, 0.0f); }
    return any;
}

// cone_test's constants of every lathe segment (p0 = (0, y_i, 0), p1 =
// (0, y_{i+1}, 0)), with cone_test's expressions: seg[2p] = {y0, r0, k, L},
// seg[2p + 1] = {da.y, y1, r1, valid}; valid 0 for a segment lathe_test
// skips (both radii <= 0, or L^2 < 1e-12).  The axis has no x / z part, so
// da = (0, da.y, 0) exactly.
static __global__ void lathe_segments_kernel(const Lathe* __restrict__ lathes, int nl, const LathePoint* __restrict__ pts,
                                      float4* __restrict__ seg, float4* __restrict__ bound) {
    const int l = blockIdx.x;
    if (l >= nl) return;
    const Lathe L0 = lathes[l];
    if (threadIdx.x == 0) {
        // the surface's box about the Y axis (cone_test's hits lie on cones
        // between consecutive profile points), widened by 1e-4 relative:
        // far more than the rounding of a hit cone_test accepts
        float R = 0.0f, ylo = FLT_MAX, yhi = -FLT_MAX;
        for (int i = 0; i < L0.point_count; i++) {
            const LathePoint q = pts[L0.point_offset + i];
            R = fmaxf(R, fabsf(q.radius));
            ylo = fminf(ylo, q.y);
            yhi = fmaxf(yhi, q.y);
        }
        const float m = 1e-4f * (R + fabsf(ylo) + fabsf(yhi)) + 1e-6f;
        bound[l] = L0.point_count >= 2 ? make_float4(R + m, ylo - m, yhi + m, 1.0f)
                                        : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    for (int i = threadIdx.x; i < L0.point_count - 1; i += blockDim.x) {
        const int p = L0.point_offset + i;
        const LathePoint a = pts[p], b = pts[p + 1];
        float4 s0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), s1 = s0;
        if (!(a.radius <= 0.0f && b.radius <= 0.0f)) {
            const float3 p0 = f3(0.0f, a.y, 0.0f), p1 = f3(0.0f, b.y, 0.0f);
            const float3 axis = p1 - p0;
            const float L2 = dot(axis, axis);
            if (!(L2 < 1e-12f)) {
                const float L = sqrtf(L2);
                const float3 da = axis / L;
                const float k = (b.radius - a.radius) / L;
                s0 = make_float4(a.y, a.radius, k, L);
                s1 = make_float4(da.y, b.y, b.radius, 1.0f);
            }
        }
        seg[2 * (size_t)p] = s0;
        seg[2 * (size_t)p + 1] = s1;
    }
}

// The ray's terms shared by every lathe test (computed once per ray: the
// reference's lathe bounds are infinite in x and z, so a ray meets every
// lathe whose y range it crosses).
struct LatheRay {
    float inv[3];            // 1 / d
    float axz, bxz, cxz;     // squared distance to the Y axis: axz t^2 + 2 bxz t + cxz
    float tstar;             // its minimum
    __device__ __forceinline__ explicit LatheRay(const Ray& r) {
        inv[0] = 1.0f / r.d.x;
        inv[1] = 1.0f / r.d.y;
        inv[2] = 1.0f / r.d.z;
        axz = r.d.x * r.d.x + r.d.z * r.d.z;
        bxz = r.o.x * r.d.x + r.o.z * r.d.z;
        cxz = r.o.x * r.o.x + r.o.z * r.o.z;
        tstar = axz > 0.0f ? -bxz / axz : 0.0f;
    }
};

// One profile segment p of a tessellated lathe (cone_test on the
// precomputed constants) against the ray: lowers `best` and fills h on a
// closer hit.  The ray's squared distance to the Y axis, q(t) = axz t^2 +
// 2 bxz t + cxz, is convex: the segment is skipped when q stays above its
// largest radius squared over the ray's t-range inside the segment's y-slab
// (1e-4 relative margins in space, 1e-5 relative slack in t and q, far
// above the rounding of a hit cone_test accepts, cancellation included).
__device__ __forceinline__ bool lathe_seg_hit(const Ray& r, const LatheRay& lr, const float4* __restrict__ seg, int p,
                                              float& best, Hit& h) {
    const float idy = lr.inv[1];
    const float axz = lr.axz, bxz = lr.bxz, cxz = lr.cxz, tstar = lr.tstar;
    const float4 s1 = __ldg(&seg[2 * (size_t)p + 1]);
    if (s1.w == 0.0f) return false;
    const float4 s0 = __ldg(&seg[2 * (size_t)p]);
    {
        const float rs = fmaxf(fabsf(s0.y), fabsf(s1.z));
        const float m = 1e-4f * (fabsf(s0.x) + fabsf(s1.y) + rs) + 1e-6f;
        const float ylo = fminf(s0.x, s1.y) - m, yhi = fmaxf(s0.x, s1.y) + m;
        float ta = r.tmin, tb = r.tmax;
        if (r.d.y != 0.0f) {
            const float u0 = (ylo - r.o.y) * idy, u1 = (yhi - r.o.y) * idy;
            ta = fmaxf(ta, fminf(u0, u1));
            tb = fminf(tb, fmaxf(u0, u1));
        } else if (r.o.y < ylo || r.o.y > yhi) {
            return false;
        }
        if (ta > tb + 1e-5f * (fabsf(ta) + fabsf(tb)) + 1e-6f) return false;
        if (ta <= tb) {
            const float tc = fminf(fmaxf(tstar, ta), tb);
            const float q = axz * tc * tc + 2.0f * bxz * tc + cxz;
            const float rr = rs + m;
            const float tol = 1e-5f * (axz * tc * tc + 2.0f * fabsf(bxz * tc) + cxz) + 1e-4f * rr * rr;
            if (q > rr * rr + tol) return false;
        }
    }
    const float3 p0 = f3(0.0f, s0.x, 0.0f);
    const float r0 = s0.y, k = s0.z, L = s0.w;
    const float3 da = f3(0.0f, s1.x, 0.0f);
    const float3 Q = r.o - p0;
    const float u = dot(r.d, da), v = dot(Q, da);
    const float3 Dp = r.d - u * da, Qp = Q - v * da;
    const float A = dot(Dp, Dp) - k * k * u * u;
    const float B = 2.0f * (dot(Dp, Qp) - k * r0 * u - k * k * v * u);
    const float C = dot(Qp, Qp) - k * k * v * v - 2.0f * k * r0 * v - r0 * r0;
    const float disc = B * B - 4.0f * A * C;
    if (disc < 0.0f) return false;
    const float sq = sqrtf(disc);
    const float i2a = 1.0f / (2.0f * A);
    const float s1r = (-B - sq) * i2a, s2r = (-B + sq) * i2a;
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const float sr = j == 0 ? s1r : s2r;
        if (sr < r.tmin || sr > r.tmax) continue;
        const float tp = v + sr * u;
        if (tp < 0.0f || tp > L) continue;
        if (sr < best) {
            h.t = sr;
            h.n = normalize(Qp + sr * Dp);
            h.tan = da;
            if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
            h.p = r.o + sr * r.d;
            best = sr;
            return true;
        }
        return false;   // cone_test reports its first root in range
    }
    return false;
}

// lathe_test with the segment constants precomputed (lathe_segments_kernel):
// cone_test's steps after its axis, L, da and k, so the same hits and
// records, without a square root and four divisions per segment.
__device__ __forceinline__ bool lathe_test_pre(const Ray& r, const LatheRay& lr, const Lathe& l,
                                               const float4* __restrict__ seg, float4 bound, Hit& h) {
    if (l.point_count < 2 || bound.w == 0.0f) return false;
    {
        // slab test against the surface's box (a NaN from 0 * inf leaves
        // that slab unconstrained)
        const float lo[3] = {-bound.x, bound.y, -bound.x}, hi[3] = {bound.x, bound.z, bound.x};
        const float o[3] = {r.o.x, r.o.y, r.o.z};
        float tn = r.tmin, tf = r.tmax;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float inv = lr.inv[a];
            const float t0 = (lo[a] - o[a]) * inv, t1 = (hi[a] - o[a]) * inv;
            tn = fmaxf(tn, fminf(t0, t1));
            tf = fminf(tf, fmaxf(t0, t1));
        }
        if (tn > tf + 1e-5f * (fabsf(tn) + fabsf(tf)) + 1e-6f) return false;
    }
    bool any = false;
    float best = r.tmax;
    for (int i = 0; i < l.point_count - 1; i++) any |= lathe_seg_hit(r, lr, seg, l.point_offset + i, best, h);
    if (any) { h.mat = l.material_id; h.uv = make_float2(0.0f, 0.0f); }
    return any;
}

// Whether the ray's [tmin, tmax] range can meet the box [lo, hi]: a slab
// test that accepts up to 1e-5 relative in t beyond the box, far more than
// the rounding of any hit computed inside it (a NaN from 0 * inf leaves
// that slab unconstrained).
__device__ __forceinline__ bool ray_meets_box(const Ray& r, const float lo[3], const float hi[3]) {
    const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
    float tn = r.tmin, tf = r.tmax;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float inv = 1.0f / d[a];
        const float t0 = (lo[a] - o[a]) * inv, t1 = (hi[a] - o[a]) * inv;
        tn = fmaxf(tn, fminf(t0, t1));
        tf = fminf(tf, fmaxf(t0, t1));
    }
    return !(tn > tf + 1e-5f * (fabsf(tn) + fabsf(tf)) + 1e-6f);
}

// primitives/prism.h:18-63: even-odd containment of (x, z) over the closed
// sub-contours (a contour ends where its first point repeats).
__device__ __forceinline__ bool prism_contains(float x, float z, const Prism& p, const PrismPoint* all) {
    const int base = p.point_offset, cnt = p.point_count;
    bool inside = false;
    int i = 0;
    while (i < cnt) {
        const int start = i;
        const float sx = all[base + start].x, sz = all[base + start].z;
        int j = i + 1;
        while (j < cnt && !(all[base + j].x == sx && all[base + j].z == sz)) j++;
        const int len = j - start;
        if (len >= 3) {
            bool in = false;
            int q = len - 1;
            for (int k = 0; k < len; k++) {
                const PrismPoint pk = all[base + start + k], pq = all[base + start + q];
                if ((pk.z > z) != (pq.z > z)) {
                    float xint = (pq.x - pk.x) * (z - pk.z) / (pq.z - pk.z) + pk.x;
                    if (x < xint) in = !in;
                }
                q = k;
            }
            if (in) inside = !inside;
        }
        i = j < cnt ? j + 1 : j;
    }
    return inside;
}

// primitives/prism.h:68-133: caps (y_min, y_max) and vertical walls.
__device__ __forceinline__ bool prism_test(const Ray& r, const Prism& p, const PrismPoint* pts, Hit& h) {
    const float y0 = p.center.y + p.y_min, y1 = p.center.y + p.y_max;
    float ty0 = (y0 - r.o.y) / r.d.y, ty1 = (y1 - r.o.y) / r.d.y;
    if (ty0 > ty1) { float t = ty0; ty0 = ty1; ty1 = t; }
    if (fmaxf(ty0, r.tmin) > fminf(ty1, r.tmax)) return false;
    bool any = false;
    float best = r.tmax;
    for (int face = 0; face < 2; face++) {
        float yf = face == 0 ? y0 : y1;
        float t = (yf - r.o.y) / r.d.y;
        if (t < r.tmin || t > r.tmax) continue;
        float3 P = r.o + t * r.d;
        if (!prism_contains(P.x - p.center.x, P.z - p.center.z, p, pts)) continue;
        if (t < best) {
            float3 n = f3(0.0f, face == 0 ? -1.0f : 1.0f, 0.0f);
            h.t = t; h.p = P; h.n = dot(n, r.d) > 0.0f ? -n : n;
            h.tan = f3(1.0f, 0.0f, 0.0f);
            best = t; any = true;
        }
    }
    const float dx = r.d.x, dy = r.d.y, dz = r.d.z, ox = r.o.x, oz = r.o.z;
    const int base = p.point_offset, cnt = p.point_count;
    for (int i = 0; i < cnt; i++) {
        const PrismPoint a = pts[base + i], b = pts[base + (i + 1) % cnt];
        if (a.x == b.x && a.z == b.z) continue;
        float ax = a.x + p.center.x, az = a.z + p.center.z;
        float bx = b.x + p.center.x, bz = b.z + p.center.z;
        float ex = bx - ax, ez = bz - az;
        float den = ex * dz - ez * dx;
        if (fabsf(den) < 1e-9f) continue;
        float s = (dx * (az - oz) - dz * (ax - ox)) / den;
        if (s < -0.001f || s > 1.001f) continue;
        float t;
        if (fabsf(dx) > 1e-9f) t = (ax + s * ex - ox) / dx;
        else if (fabsf(dz) > 1e-9f) t = (az + s * ez - oz) / dz;
        else continue;
        if (t < r.tmin || t > r.tmax) continue;
        float yy = r.o.y + dy * t;
        if (yy < y0 - 0.001f || yy > y1 + 0.001f) continue;
        if (t < best) {
            float3 n = normalize(f3(ez, 0.0f, -ex));
            h.t = t; h.p = r.o + t * r.d; h.n = dot(n, r.d) > 0.0f ? -n : n;
            h.tan = f3(0.0f, 1.0f, 0.0f);
            best = t; any = true;
        }
    }
    if (any) { h.mat = p.material_id; h.uv = make_float2(0.0f, 0.0f); }
    return any;
}

// primitives/superellipsoid.h:12-28
__device__ __forceinline__ float se_value(const Superellipsoid& s, float3 p) {
    float qx = (p.x - s.center.x) / s.a, qy = (p.y - s.center.y) / s.b, qz = (p.z - s.center.z) / s.c;
    return powf(fabsf(qx), s.n) + powf(fabsf(qy), s.n) + powf(fabsf(qz), s.n);
}
__device__ __forceinline__ float3 se_gradient(const Superellipsoid& s, float3 p) {
    float qx = (p.x - s.center.x) / s.a, qy = (p.y - s.center.y) / s.b, qz = (p.z - s.center.z) / s.c;
    return f3(s.n * powf(fabsf(qx), s.n - 1.0f) * (qx >= 0.0f ? 1.0f : -1.0f) / s.a,
              s.n * powf(fabsf(qy), s.n - 1.0f) * (qy >= 0.0f ? 1.0f : -1.0f) / s.b,
              s.n * powf(fabsf(qz), s.n - 1.0f) * (qz >= 0.0f ? 1.0f : -1.0f) / s.c);
}

// Extension (no counterpart in the reference): the two-exponent body
// (|qx|^n + |qz|^n)^(n2/n) + |qy|^n2 = 1 -- n the east-west exponent,
// n2 > 0 the north-south one on the y axis; n2 == n is the single-exponent
// body above.
__device__ __forceinline__ float se_value2(const Superellipsoid& s, float n2, float3 p) {
    float qx = (p.x - s.center.x) / s.a, qy = (p.y - s.center.y) / s.b, qz = (p.z - s.center.z) / s.c;
    const float xz = powf(fabsf(qx), s.n) + powf(fabsf(qz), s.n);
    return powf(xz, n2 / s.n) + powf(fabsf(qy), n2);
}
__device__ __forceinline__ float3 se_gradient2(const Superellipsoid& s, float n2, float3 p) {
    float qx = (p.x - s.center.x) / s.a, qy = (p.y - s.center.y) / s.b, qz = (p.z - s.center.z) / s.c;
    const float ax = fabsf(qx), az = fabsf(qz);
    const float xz = powf(ax, s.n) + powf(az, s.n);
    const float k = xz > 0.0f ? n2 * powf(xz, n2 / s.n - 1.0f) : 0.0f;
    return f3(k * powf(ax, s.n - 1.0f) * (qx >= 0.0f ? 1.0f : -1.0f) / s.a,
              n2 * powf(fabsf(qy), n2 - 1.0f) * (qy >= 0.0f ? 1.0f : -1.0f) / s.b,
              k * powf(az, s.n - 1.0f) * (qz >= 0.0f ? 1.0f : -1.0f) / s.c);
}
__device__ __forceinline__ float3 se_normal_dir(const Superellipsoid& s, float n2, float3 p) {
    return n2 > 0.0f ? se_gradient2(s, n2, p) : se_gradient(s, p);
}

// Whether F(p) = |qx|^n + |qy|^n + |qz|^n exceeds 1 -- the only use se_span
// makes of F -- deciding from two bounds before any powf where they can:
//   F <= 3 max|q_i|^n, so max|q_i| < (1/3)^(1/n) means inside;
//   F >= 3 (sum|q_i| / 3)^n for n >= 1 (power means) and F >= sum|q_i| for
//   n < 1 (|x|^n >= |x| on [0, 1]; a |q_i| > 1 is outside anyway), so
//   sum|q_i| above 3^(1 - 1/n), or 1, means outside.
// The thresholds carry a 1e-4 relative margin, far above the few-ulp error
// of powf and the sum, so every decision equals se_value(s, p) > 1; any
// other point (or a NaN) is evaluated exactly with se_value's arithmetic.
// The bounds are evaluated on q from multiplications by 1 / a, 1 / b, 1 / c
// (a few ulp from the quotients, far inside the 1e-4 margins); only a point
// they leave undecided computes the quotients and F with se_value's
// arithmetic.
struct SeSign {
    float thr_in, thr_out;   // on max|q_i| and on sum|q_i|; -1 / +inf: no shortcut
    float ia, ib, ic;
    __device__ __forceinline__ SeSign(float n, const Superellipsoid& s) {
        if (n >= 0.25f && n <= 1e4f) {
            thr_in = powf(1.0f / 3.0f, 1.0f / n) * (1.0f - 1e-4f);
            thr_out = (n >= 1.0f ? powf(3.0f, 1.0f - 1.0f / n) : 1.0f) * (1.0f + 1e-4f);
        } else {
            thr_in = -1.0f;
            thr_out = __int_as_float(0x7f800000);
        }
        ia = 1.0f / s.a;
        ib = 1.0f / s.b;
        ic = 1.0f / s.c;
    }
    __device__ __forceinline__ bool outside(const Superellipsoid& s, float3 p) const {
        const float dx = p.x - s.center.x, dy = p.y - s.center.y, dz = p.z - s.center.z;
        {
            const float ax = fabsf(dx * ia), ay = fabsf(dy * ib), az = fabsf(dz * ic);
            const float sum = ax + ay + az;
            if (sum == sum) {
                if (fmaxf(fmaxf(ax, ay), az) < thr_in) return false;
                if (sum > thr_out) return true;
            }
        }
        const float ax = fabsf(dx / s.a), ay = fabsf(dy / s.b), az = fabsf(dz / s.c);
        return powf(ax, s.n) + powf(ay, s.n) + powf(az, s.n) > 1.0f;
    }
};

__device__ __forceinline__ void se_chord(const Ray& r, const Superellipsoid& s, float& tA, float& tB) {
    const float3 lo = f3(s.center.x - s.a, s.center.y - s.b, s.center.z - s.c);
    const float3 hi = f3(s.center.x + s.a, s.center.y + s.b, s.center.z + s.c);
    float ix = 1.0f / r.d.x;
    float tx0 = (lo.x - r.o.x) * ix, tx1 = (hi.x - r.o.x) * ix;
    if (tx0 > tx1) { float t = tx0; tx0 = tx1; tx1 = t; }
    float iy = 1.0f / r.d.y;
    float ty0 = (lo.y - r.o.y) * iy, ty1 = (hi.y - r.o.y) * iy;
    if (ty0 > ty1) { float t = ty0; ty0 = ty1; ty1 = t; }
    float iz = 1.0f / r.d.z;
    float tz0 = (lo.z - r.o.z) * iz, tz1 = (hi.z - r.o.z) * iz;
    if (tz0 > tz1) { float t = tz0; tz0 = tz1; tz1 = t; }
    tA = fmaxf(fmaxf(tx0, ty0), tz0);
    tB = fminf(fminf(tx1, ty1), tz1);
}

// primitives/superellipsoid.h:41-117: 32 samples of F along the clipped
// chord, 20 bisection steps for the exit.  As in the reference an entry
// found by sampling is not refined (its bisection interval is empty), so
// the entry lies on a sample.
// SIGN: decide the samples through SeSign (the same decisions, fewer powf).
// The march and bisection of se_span over an "outside" predicate.
// make() builds the predicate once the chord is known to be hit.
// ENTRY_ONLY (the closest-hit test, whose result is the entry alone): stop
// at the entry sample.  The exit the march would go on to find lies at or
// after the entry (it is bisected after an inside sample at or after the
// entry, and clamped to t1 >= entry), so the reference's final check
// entry <= exit always holds and the exit never changes the hit; tx is
// then t1.
// [wa, wb]: a window outside which every point of the ray is known to be
// outside the body (se_may_enter's widened bounding-ellipsoid chord); a
// sample or bisection point outside it is decided without evaluating F,
// and once no entry was found and the samples pass wb none can follow.
template <bool ENTRY_ONLY = false, class MakeOut>
__device__ __forceinline__ bool se_span_core(const Ray& r, const Superellipsoid& s, float t0, float t1, float& te,
                                             float& tx, float* te_prev, MakeOut make,
                                             float wa = -INFINITY, float wb = INFINITY) {
    float tA, tB;
    se_chord(r, s, tA, tB);
    if (tB < t0 || tA > t1 || tB < tA) return false;
    t0 = fmaxf(t0, tA);
    t1 = fminf(t1, tB);
    const auto out0 = make();
    const auto out = [&](float t) { return (t < wa || t > wb) ? true : out0(r.o + t * r.d); };
    const float step = (t1 - t0) / 32.0f;
    float tp = t0;
    bool inside = !out(tp);
    bool found_in = inside, found_out = false;
    te = inside ? t0 : -1e30f;
    if (te_prev) *te_prev = te;   // the last sample outside before the entry (te itself: no bracket)
    tx = -1e30f;
    if (ENTRY_ONLY && inside) { tx = t1; return true; }
    for (int i = 1; i <= 32 && !found_out; i++) {
        float t = fminf(t0 + step * (float)i, t1);
        if (!inside && t > wb) break;   // every later sample is outside too
        const bool o = out(t);
        if (inside && o) {
            float lo = tp, hi = t;
            for (int b = 0; b < 20; b++) {
                float mid = 0.5f * (lo + hi);
                if (out(mid)) hi = mid; else lo = mid;
            }
            tx = fminf(0.5f * (lo + hi), t1);
            found_out = true;
            break;
        }
        if (!inside && !o) {
            te = fmaxf(t, t0);   // bisection over [t, t] in the reference
            if (te_prev) *te_prev = tp;
            if (ENTRY_ONLY) { tx = t1; return true; }
            found_in = true;
            inside = true;
        }
        tp = t;
    }
    if (!found_in) return false;
    if (!found_out) tx = t1;
    return te <= tx;
}

// Whether the march over [t0, t1] can find an inside sample at all.  The
// body |qx|^n + |qy|^n + |qz|^n <= 1 lies in the ellipsoid
// qx^2 + qy^2 + qz^2 <= k^2 with k = 1 for n <= 2 (there sum q^2 <=
// (sum |q|^n)^(2/n), the power means) and k^2 = 3^(1 - 2/n) for n > 2
// (sum q^2 / 3 <= (sum |q|^n / 3)^(2/n)).  On a ray that misses that
// ellipsoid widened by 1e-3, every point has F >= (1 + 1e-3)^min(n, 2) - 1
// above 1 -- for n >= 0.25 about 2.5e-4, far beyond the rounding of F in
// FP32 -- so every sample tests outside and the march finds no entry: the
// result is the march's, without its 33 evaluations.
// The widened chord [wa, wb] is returned as se_span_core's window (left
// unbounded where no chord is computed).
__device__ __forceinline__ bool se_may_enter(const Ray& r, const Superellipsoid& s, float t0, float t1, float& wa,
                                             float& wb) {
    wa = -INFINITY;
    wb = INFINITY;
    if (!(s.n >= 0.25f && s.n <= 1e4f)) return true;
    const float k2 = s.n <= 2.0f ? 1.0f : powf(3.0f, 1.0f - 2.0f / s.n);
    const float K = k2 * 1.002001f;   // (k (1 + 1e-3))^2
    const float3 inv = f3(1.0f / s.a, 1.0f / s.b, 1.0f / s.c);
    const float3 oc = f3((r.o.x - s.center.x) * inv.x, (r.o.y - s.center.y) * inv.y, (r.o.z - s.center.z) * inv.z);
    const float3 dd = f3(r.d.x * inv.x, r.d.y * inv.y, r.d.z * inv.z);
    const float A = dot(dd, dd), B = dot(oc, dd), C = dot(oc, oc) - K;
    const float disc = B * B - A * C;
    // a generous slack on the FP32 discriminant before declaring a miss
    if (!(disc < -1e-4f * (B * B + fabsf(A * C)))) {
        if (!(A > 0.0f) || disc <= 0.0f) return true;
        const float sq = sqrtf(disc);
        const float ta = (-B - sq) / A, tb = (-B + sq) / A;
        const float slack = 1e-3f * (fabsf(ta) + fabsf(tb)) + 1e-6f;
        wa = ta - slack;
        wb = tb + slack;
        return !(tb < t0 - slack || ta > t1 + slack);
    }
    return false;
}

// primitives/superellipsoid.h:41-117: 32 samples of F along the clipped
// chord, 20 bisection steps for the exit.  As in the reference an entry
// found by sampling is not refined (its bisection interval is empty), so
// the entry lies on a sample.
// SIGN: decide the samples through SeSign (the same decisions, fewer powf),
// and skip the march of rays that miss the body's bounding ellipsoid
// (se_may_enter: the same result).
template <bool SIGN = false, bool ENTRY_ONLY = false>
__device__ __forceinline__ bool se_span(const Ray& r, const Superellipsoid& s, float t0, float t1,
                                        float& te, float& tx, float* te_prev = nullptr) {
    float wa = -INFINITY, wb = INFINITY;
    if (SIGN && !se_may_enter(r, s, t0, t1, wa, wb)) return false;
    return se_span_core<ENTRY_ONLY>(r, s, t0, t1, te, tx, te_prev, [&]() {
        const SeSign sg(SIGN ? s.n : 0.0f, s);
        return [sg, &s](float3 p) { return SIGN ? sg.outside(s, p) : se_value(s, p) > 1.0f; };
    }, wa, wb);
}

// Extension: the two-exponent body's span (the same march), not inlined so
// that the kernels' code for the reference's body is unchanged.
static __device__ __noinline__ bool se_span2(const Ray& r, const Superellipsoid& s, float n2, float t0, float t1,
                                             float& te, float& tx, float* te_prev, bool entry_only = false) {
    auto make = [&]() { return [&s, n2](float3 p) { return se_value2(s, n2, p) > 1.0f; }; };
    return entry_only ? se_span_core<true>(r, s, t0, t1, te, tx, te_prev, make)
                      : se_span_core<false>(r, s, t0, t1, te, tx, te_prev, make);
}

// Extension (a scene created with "trace.se_polish"; the reference has
// none): the entry that the sampling above leaves on a sample is refined in
// FP64 -- safeguarded Newton on G(t) = F(o + t d) - 1 inside the bracket
// [last outside sample, first inside sample], bisection whenever a Newton
// step leaves the bracket -- so the hit lies on the surface instead of up
// to one sample step (1/32 of the chord) inside it.
static __device__ __noinline__ float se_polish_entry(const Ray& r, const Superellipsoid& s, float t_out, float t_in) {
    const double ox = (double)r.o.x - s.center.x, oy = (double)r.o.y - s.center.y, oz = (double)r.o.z - s.center.z;
    const double dx = r.d.x, dy = r.d.y, dz = r.d.z;
    const double ia = 1.0 / s.a, ib = 1.0 / s.b, ic = 1.0 / s.c, n = s.n;
    auto G = [&](double t, double& dG) {
        const double qx = (ox + t * dx) * ia, qy = (oy + t * dy) * ib, qz = (oz + t * dz) * ic;
        const double ax = fabs(qx), ay = fabs(qy), az = fabs(qz);
        const double px = pow(ax, n - 1.0), py = pow(ay, n - 1.0), pz = pow(az, n - 1.0);
        dG = n * (px * copysign(1.0, qx) * dx * ia + py * copysign(1.0, qy) * dy * ib + pz * copysign(1.0, qz) * dz * ic);
        return px * ax + py * ay + pz * az - 1.0;
    };
    double lo = t_out, hi = t_in, x = t_in, dG = 0.0;
    double g = G(x, dG);
    for (int k = 0; k < 60 && hi - lo > 1e-13 * fmax(fabs(hi), 1.0); k++) {
        double xn = (dG != 0.0) ? x - g / dG : 0.5 * (lo + hi);
        if (!(xn > lo && xn < hi)) xn = 0.5 * (lo + hi);
        x = xn;
        g = G(x, dG);
        if (g > 0.0) lo = x;
        else hi = x;
        if (g == 0.0) break;
    }
    return (float)hi;
}

// primitives/superellipsoid.h:123-161
// primitives/superellipsoid.h:123-161
template <bool SIGN = false>
__device__ __forceinline__ bool se_test(const Ray& r, const Superellipsoid& s, Hit& h, int polish = 0) {
    float t0, t1;
    se_chord(r, s, t0, t1);
    if (t1 < r.tmin || t0 > r.tmax || t1 < t0) return false;
    t0 = fmaxf(t0, r.tmin);
    t1 = fminf(t1, r.tmax);
    float te, tx, te_prev;
    if (!se_span<SIGN, true>(r, s, t0, t1, te, tx, &te_prev)) return false;
    if (polish && te_prev < te) te = se_polish_entry(r, s, te_prev, te);
    h.t = te;
    h.p = r.o + te * r.d;
    h.n = normalize(se_gradient(s, h.p));
    h.tan = f3(1.0f, 0.0f, 0.0f);
    h.uv = make_float2(h.p.x, h.p.y);
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    h.mat = s.material_id;
    return true;
}

// Extension: the two-exponent body (n2 > 0; no polish), not inlined.
static __device__ __noinline__ bool se_test2(const Ray& r, const Superellipsoid& s, float n2, Hit& h) {
    float t0, t1;
    se_chord(r, s, t0, t1);
    if (t1 < r.tmin || t0 > r.tmax || t1 < t0) return false;
    t0 = fmaxf(t0, r.tmin);
    t1 = fminf(t1, r.tmax);
    float te, tx;
    if (!se_span2(r, s, n2, t0, t1, te, tx, nullptr, true)) return false;
    h.t = te;
    h.p = r.o + te * r.d;
    h.n = normalize(se_gradient2(s, n2, h.p));
    h.tan = f3(1.0f, 0.0f, 0.0f);
    h.uv = make_float2(h.p.x, h.p.y);
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    h.mat = s.material_id;
    return true;
}

// primitives/heightfield.h:13-56: lattice hash, smoothed value noise, fBm.
__device__ __forceinline__ float hf_hash(int xi, int zi, int seed) {
    unsigned h = (unsigned)(xi * 374761393 + zi * 668265263 + seed * 974634097);
    h = (h ^ (h >> 13)) * 1274126177u;
    h = h ^ (h >> 16);
    return float(h & 0xffffffu) / 16777216.0f;
}
__device__ __forceinline__ float hf_noise(float fx, float fz, int seed) {
    int x0 = (int)floorf(fx), z0 = (int)floorf(fz);
    float tx = fx - (float)x0, tz = fz - (float)z0;
    tx = tx * tx * (3.0f - 2.0f * tx);
    tz = tz * tz * (3.0f - 2.0f * tz);
    float v00 = hf_hash(x0, z0, seed), v10 = hf_hash(x0 + 1, z0, seed);
    float v01 = hf_hash(x0, z0 + 1, seed), v11 = hf_hash(x0 + 1, z0 + 1, seed);
    float a = v00 + (v10 - v00) * tx, b = v01 + (v11 - v01) * tx;
    return a + (b - a) * tz;
}

// primitives/heightfield.h:58-116: height above the tile base.
// Extension (no counterpart in the reference): an FP32 height grid of
// gw x gh values in [0, 1] replaces the procedural / 8-bit height, sampled
// bilinearly over the same footprint as the 8-bit image.
struct HfGrid {
    const float* h;
    int w, hgt;
};

__device__ __forceinline__ float hf_height(const HeightField& hf, float x, float z, HfGrid g = HfGrid{nullptr, 0, 0}) {
    float lx = (x - hf.center.x) / hf.size_x + 0.5f;
    float lz = (z - hf.center.z) / hf.size_z + 0.5f;
    if (lx < 0.0f || lx > 1.0f || lz < 0.0f || lz > 1.0f) return 0.0f;
    if (g.h) {
        float fu = lx * (float)(g.w - 1), fv = lz * (float)(g.hgt - 1);
        int u0 = (int)fu, v0 = (int)fv;
        int u1 = u0 < g.w - 1 ? u0 + 1 : u0, v1 = v0 < g.hgt - 1 ? v0 + 1 : v0;
        float tx = fu - (float)u0, ty = fv - (float)v0;
        const float h00 = __ldg(&g.h[(size_t)v0 * g.w + u0]), h10 = __ldg(&g.h[(size_t)v0 * g.w + u1]);
        const float h01 = __ldg(&g.h[(size_t)v1 * g.w + u0]), h11 = __ldg(&g.h[(size_t)v1 * g.w + u1]);
        float hh = h00 * (1.0f - tx) * (1.0f - ty) + h10 * tx * (1.0f - ty) + h01 * (1.0f - tx) * ty + h11 * tx * ty;
        return hh * hf.height;
    }
    if (hf.image) {
        if (hf.img_w < 1 || hf.img_h < 1) return 0.0f;
        float fu = lx * (float)(hf.img_w - 1), fv = lz * (float)(hf.img_h - 1);
        int u0 = (int)fu, v0 = (int)fv;
        int u1 = u0 < hf.img_w - 1 ? u0 + 1 : u0, v1 = v0 < hf.img_h - 1 ? v0 + 1 : v0;
        float tx = fu - (float)u0, ty = fv - (float)v0;
        float h00 = (float)hf.image[v0 * hf.img_w + u0] / 255.0f, h10 = (float)hf.image[v0 * hf.img_w + u1] / 255.0f;
        float h01 = (float)hf.image[v1 * hf.img_w + u0] / 255.0f, h11 = (float)hf.image[v1 * hf.img_w + u1] / 255.0f;
        float hh = h00 * (1.0f - tx) * (1.0f - ty) + h10 * tx * (1.0f - ty) + h01 * (1.0f - tx) * ty + h11 * tx * ty;
        return hh * hf.height;
    }
    float fx = lx * hf.freq, fz = lz * hf.freq, amp = 0.5f, sum = 0.0f, nz = 0.0f;
    for (int o = 0; o < hf.octaves; o++) {
        sum += amp * hf_noise(fx, fz, hf.seed + o * 131);
        nz += amp;
        amp *= 0.5f;
        fx *= 2.0f; fz *= 2.0f;
    }
    float t = sum / nz;
    float detail = hf_noise(lx * 7.0f, lz * 7.0f, hf.seed + 7777) * 0.06f;
    t = fminf(t + detail - 0.03f, 1.0f);
    return t * hf.height;
}

// primitives/heightfield.h:121-183: march (diagonal/64 steps, <= 256) then
// 10 bisection steps; finite-difference normal.
__device__ __forceinline__ bool hf_test(const Ray& r, const HeightField& hf, Hit& h, HfGrid g = HfGrid{nullptr, 0, 0}) {
    const float3 lo = f3(hf.center.x - 0.5f * hf.size_x, hf.center.y, hf.center.z - 0.5f * hf.size_z);
    const float3 hi = f3(hf.center.x + 0.5f * hf.size_x, hf.center.y + hf.height, hf.center.z + 0.5f * hf.size_z);
    float ix = 1.0f / r.d.x, iy = 1.0f / r.d.y, iz = 1.0f / r.d.z;
    float tx0 = (lo.x - r.o.x) * ix, tx1 = (hi.x - r.o.x) * ix;
    float ty0 = (lo.y - r.o.y) * iy, ty1 = (hi.y - r.o.y) * iy;
    float tz0 = (lo.z - r.o.z) * iz, tz1 = (hi.z - r.o.z) * iz;
    if (tx0 > tx1) { float t = tx0; tx0 = tx1; tx1 = t; }
    if (ty0 > ty1) { float t = ty0; ty0 = ty1; ty1 = t; }
    if (tz0 > tz1) { float t = tz0; tz0 = tz1; tz1 = t; }
    float t0 = fmaxf(fmaxf(tx0, ty0), tz0), t1 = fminf(fminf(tx1, ty1), tz1);
    if (t1 < r.tmin || t0 > r.tmax || t1 < t0) return false;
    t0 = fmaxf(t0, r.tmin);
    t1 = fminf(t1, r.tmax);
    const float diag = sqrtf(hf.size_x * hf.size_x + hf.size_z * hf.size_z);
    const float step = fmaxf(diag / 64.0f, 1e-4f);
    float t = t0;
    bool inside = false;
    for (int i = 0; i < 256; i++) {
        float3 p = r.o + t * r.d;
        bool below = p.y <= hf_height(hf, p.x, p.z, g) + hf.center.y;
        if (below != inside) {
            float a = t - step, b = t;
            if (a < t0) a = t0;
            for (int k = 0; k < 10; k++) {
                float mid = 0.5f * (a + b);
                float3 pm = r.o + mid * r.d;
                if ((pm.y <= hf_height(hf, pm.x, pm.z, g) + hf.center.y) == below) b = mid; else a = mid;
            }
            float tt = 0.5f * (a + b);
            float3 P = r.o + tt * r.d;
            if (tt >= r.tmin && tt <= r.tmax) {
                const float e = fmaxf(hf.size_x, hf.size_z) / 256.0f;
                float hxp = hf_height(hf, P.x + e, P.z, g), hxm = hf_height(hf, P.x - e, P.z, g);
                float hzp = hf_height(hf, P.x, P.z + e, g), hzm = hf_height(hf, P.x, P.z - e, g);
                h.t = tt;
                h.p = P;
                h.n = normalize(f3(-(hxp - hxm) / (2.0f * e), 1.0f, -(hzp - hzm) / (2.0f * e)));
                h.tan = f3(1.0f, 0.0f, 0.0f);
                h.uv = make_float2(P.x, P.z);
                if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
                h.mat = hf.material_id;
                return true;
            }
            return false;
        }
        inside = below;
        t += step;
        if (t > t1) break;
    }
    return false;
}

// Extension: hf_test over an FP32 height grid, not inlined so that the
// kernels' code for the reference's heights is unchanged.
static __device__ __noinline__ bool hf_test_grid(const Ray& r, const HeightField& hf, Hit& h, HfGrid g) {
    return hf_test(r, hf, h, g);
}

}  // namespace dev
}  // namespace sheen
