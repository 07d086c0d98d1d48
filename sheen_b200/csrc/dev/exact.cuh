// exact.cuh -- scene extensions with no counterpart in the reference: exact
// cubic-Bezier surfaces of revolution and extrusion.
//
// The reference turns Bezier profiles into polylines on the host
// (api/scene_io.cpp:86-102, 791-819) and intersects cone segments
// (primitives/lathe.h:14-95) and straight prism walls
// (primitives/prism.h:18-134).  Here the curves themselves are intersected:
//
//   lathe   profile (y(u), r(u)), turned about the world Y axis (the axis of
//           the reference's tessellated lathe, whose test ignores the
//           lathe's centre).  With the ray o + s d and s = (y(u) - oy) / dy,
//           (ox + s dx)^2 + (oz + s dz)^2 = r(u)^2 becomes, times dy^2,
//             A Y^2 + B dy Y + C dy^2 - dy^2 R^2 = 0,   Y = y(u) - oy,
//           A = dx^2 + dz^2, B = 2 (ox dx + oz dz), C = ox^2 + oz^2:
//           a sextic in u per cubic span.  A ray with dy = 0 solves
//           Y(u) = 0 (a cubic) and then the circle of radius r(u).
//   prism   contour (x(u), z(u)) about the prism's centre, extruded over
//           [y_min, y_max]: a wall hit solves the cubic
//           (x(u) - ox) dz - (z(u) - oz) dx = 0; a cap hit keeps the cap
//           point when the contour crosses the line z = pz an odd number of
//           times at x > px (even-odd rule, the reference's
//           prism_in_contour), the crossings being the cubic
//           z(u) - pz = 0.
//
// The polynomials are formed and their roots in [0, 1] isolated in FP64 in
// the Bernstein basis: de Casteljau halving, an interval whose coefficients
// do not change sign holds no root (variation diminishing), one whose end
// values differ in sign and whose coefficients change sign once holds one
// root, which bisection narrows to 1e-13.  Hit points, normals and
// shading stay FP32.
//
// A profile is a list of spans of four control points (a, b); the host
// joins consecutive spans whose ends differ with straight spans (the limit
// of the reference's polyline, which runs from one span's end straight to
// the next span's first sample) and closes prism contours the same way.
#pragma once
#include "prims.cuh"

namespace sheen {
namespace dev {

constexpr int kBezMaxDepth = 34;   // interval width 2^-34 ~ 6e-11

__device__ __forceinline__ double cubic_at(const double* c, double u) {
    const double v = 1.0 - u;
    return v * v * v * c[0] + 3.0 * v * v * u * c[1] + 3.0 * v * u * u * c[2] + u * u * u * c[3];
}
__device__ __forceinline__ double cubic_d(const double* c, double u) {
    const double v = 1.0 - u;
    return 3.0 * (v * v * (c[1] - c[0]) + 2.0 * v * u * (c[2] - c[1]) + u * u * (c[3] - c[2]));
}

// Bernstein coefficients of the product of two cubics (degree 6):
// (PQ)_k = sum_{i+j=k} C(3,i) C(3,j) / C(6,k) P_i Q_j.
__device__ __forceinline__ void bern_mul33(const double* p, const double* q, double* out) {
    const double b3[4] = {1.0, 3.0, 3.0, 1.0};
    const double b6[7] = {1.0, 6.0, 15.0, 20.0, 15.0, 6.0, 1.0};
#pragma unroll
    for (int k = 0; k < 7; k++) out[k] = 0.0;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) out[i + j] += b3[i] * b3[j] * p[i] * q[j];
#pragma unroll
    for (int k = 0; k < 7; k++) out[k] /= b6[k];
}

// Value of a degree-N Bernstein polynomial at u (de Casteljau).
template <int N>
__device__ __forceinline__ double bern_at(const double* c, double u) {
    double w[N + 1];
#pragma unroll
    for (int i = 0; i <= N; i++) w[i] = c[i];
    for (int r = 1; r <= N; r++)
        for (int i = 0; i <= N - r; i++) w[i] = (1.0 - u) * w[i] + u * w[i + 1];
    return w[0];
}

// Roots in [0, 1] of the degree-N Bernstein polynomial c, in increasing
// order (at most N; a double root without a sign change is not reported).
template <int N>
__device__ __noinline__ int bern_roots(const double* c, double* roots) {
    struct Item {
        double c[N + 1];
        double lo, hi;
        int depth;
    };
    Item stack[kBezMaxDepth + 2];
    int sp = 0;
    int nr = 0;
    Item cur;
#pragma unroll
    for (int i = 0; i <= N; i++) cur.c[i] = c[i];
    cur.lo = 0.0; cur.hi = 1.0; cur.depth = 0;
    while (true) {
        // sign changes of the coefficients
        int changes = 0;
        double prev = cur.c[0];
        bool zero_all = true;
#pragma unroll
        for (int i = 0; i <= N; i++) zero_all &= cur.c[i] == 0.0;
        for (int i = 1; i <= N; i++) {
            if (cur.c[i] == 0.0) continue;
            if (prev != 0.0 && ((prev < 0.0) != (cur.c[i] < 0.0))) changes++;
            prev = cur.c[i];
        }
        bool descend = false;
        if (!zero_all && changes > 0) {
            const bool ends_differ = (cur.c[0] < 0.0) != (cur.c[N] < 0.0) || cur.c[0] == 0.0 || cur.c[N] == 0.0;
            if (changes == 1 && ends_differ) {
                // one root: bisection on the end values
                double lo = cur.lo, hi = cur.hi;
                double flo = cur.c[0];
                if (cur.c[0] == 0.0) {
                    if (nr < N) roots[nr++] = lo;
                } else if (cur.c[N] == 0.0) {
                    if (nr < N) roots[nr++] = hi;
                } else {
                    for (int k = 0; k < 60 && hi - lo > 1e-13; k++) {
                        const double mid = 0.5 * (lo + hi);
                        const double fm = bern_at<N>(c, mid);
                        if (fm == 0.0) { lo = hi = mid; break; }
                        if ((fm < 0.0) == (flo < 0.0)) { lo = mid; flo = fm; }
                        else hi = mid;
                    }
                    if (nr < N) roots[nr++] = 0.5 * (lo + hi);
                }
            } else if (cur.depth >= kBezMaxDepth) {
                // a cluster narrower than 2^-34: one root where the ends differ
                if (((cur.c[0] < 0.0) != (cur.c[N] < 0.0)) && nr < N) roots[nr++] = 0.5 * (cur.lo + cur.hi);
            } else {
                descend = true;
            }
        }
        if (descend && sp < kBezMaxDepth + 2) {
            // de Casteljau halves: left kept in cur, right pushed
            double w[N + 1];
#pragma unroll
            for (int i = 0; i <= N; i++) w[i] = cur.c[i];
            Item right;
            right.c[N] = w[N];
            double left0 = w[0];
            double lc[N + 1];
            lc[0] = left0;
            for (int r = 1; r <= N; r++) {
                for (int i = 0; i <= N - r; i++) w[i] = 0.5 * (w[i] + w[i + 1]);
                lc[r] = w[0];
                right.c[N - r] = w[N - r];
            }
            const double mid = 0.5 * (cur.lo + cur.hi);
            right.lo = mid; right.hi = cur.hi; right.depth = cur.depth + 1;
            stack[sp++] = right;
#pragma unroll
            for (int i = 0; i <= N; i++) cur.c[i] = lc[i];
            cur.hi = mid;
            cur.depth++;
            continue;
        }
        if (sp == 0) break;
        cur = stack[--sp];
    }
    return nr;
}

// Span table of a Bezier profile: spans [first, first + count) of
// bz_span, two float4 each: {a0, b0, a1, b1}, {a2, b2, a3, b3}.
__device__ __forceinline__ void load_span(const float4* spans, int k, double* a, double* b) {
    const float4 p = __ldg(&spans[2 * k]), q = __ldg(&spans[2 * k + 1]);
    a[0] = p.x; b[0] = p.y; a[1] = p.z; b[1] = p.w;
    a[2] = q.x; b[2] = q.y; a[3] = q.z; b[3] = q.w;
}

// Exact Bezier lathe (extension).  run = {first span, span count}; bound =
// {R, y_lo, y_hi, -}: the surface lies in |x|, |z| <= R, y in [y_lo, y_hi].
static __device__ __noinline__ bool lathe_exact_test(const Ray& r, const float4* spans, int2 run, float4 bound,
                                              int material_id, Hit& h) {
    // cylinder bound about the Y axis
    {
        float tn = r.tmin, tf = r.tmax;
        const float lo[3] = {-bound.x, bound.y, -bound.x}, hi[3] = {bound.x, bound.z, bound.x};
        const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float inv = 1.0f / d[a];
            const float t0 = (lo[a] - o[a]) * inv, t1 = (hi[a] - o[a]) * inv;
            tn = fmaxf(tn, fminf(t0, t1));
            tf = fminf(tf, fmaxf(t0, t1));
        }
        if (tn > tf + 1e-5f * (fabsf(tn) + fabsf(tf)) + 1e-6f) return false;
    }
    const double ox = r.o.x, oy = r.o.y, oz = r.o.z, dx = r.d.x, dy = r.d.y, dz = r.d.z;
    const double A = dx * dx + dz * dz, B = 2.0 * (ox * dx + oz * dz), C = ox * ox + oz * oz;
    const double dlen2 = A + dy * dy;
    const bool flat = dy * dy <= 1e-24 * dlen2;
    double best = r.tmax;
    double bu = -1.0;
    int bk = -1;
    for (int k = run.x; k < run.x + run.y; k++) {
        double Y[4], Rr[4];
        load_span(spans, k, Y, Rr);
        // the span lies in the hull of its control points: skip it when the
        // ray's y range up to the closest hit so far misses that hull
        double ylo = Y[0], yhi = Y[0];
        for (int i = 1; i < 4; i++) { ylo = fmin(ylo, Y[i]); yhi = fmax(yhi, Y[i]); }
        {
            const double ya = oy + (double)r.tmin * dy, yb = oy + best * dy;
            const double m = 1e-9 * (fabs(ya) + fabs(yb) + 1.0);
            if (fmax(ya, yb) < ylo - m || fmin(ya, yb) > yhi + m) continue;
        }
        for (int i = 0; i < 4; i++) Y[i] -= oy;
        double roots[6];
        int n;
        if (!flat) {
            double YY[7], RR[7], Y1[7];
            bern_mul33(Y, Y, YY);
            bern_mul33(Rr, Rr, RR);
            const double one[4] = {1.0, 1.0, 1.0, 1.0};
            bern_mul33(Y, one, Y1);
            double p[7];
            for (int i = 0; i < 7; i++) p[i] = A * YY[i] + B * dy * Y1[i] + C * dy * dy - dy * dy * RR[i];
            n = bern_roots<6>(p, roots);
            for (int i = 0; i < n; i++) {
                const double s = cubic_at(Y, roots[i]) / dy;
                if (s >= r.tmin && s < best) { best = s; bu = roots[i]; bk = k; }
            }
        } else {
            n = bern_roots<3>(Y, roots);
            for (int i = 0; i < n; i++) {
                const double rad = cubic_at(Rr, roots[i]);
                const double disc = B * B - 4.0 * A * (C - rad * rad);
                if (disc < 0.0 || A <= 0.0) continue;
                const double sq = sqrt(disc);
                const double s0 = (-B - sq) / (2.0 * A), s1 = (-B + sq) / (2.0 * A);
                if (s0 >= r.tmin && s0 < best) { best = s0; bu = roots[i]; bk = k; }
                else if (s1 >= r.tmin && s1 < best) { best = s1; bu = roots[i]; bk = k; }
            }
        }
    }
    if (bk < 0 || best > r.tmax) return false;
    double Y[4], Rr[4];
    load_span(spans, bk, Y, Rr);
    const float t = (float)best;
    h.t = t;
    h.p = r.o + t * r.d;
    // normal: (y'(u) cos phi, -r'(u) sgn r(u), y'(u) sin phi), (cos phi, sin phi) = (x, z) / rho
    const double yd = cubic_d(Y, bu), rd = cubic_d(Rr, bu), rv = cubic_at(Rr, bu);
    const float rho = sqrtf(h.p.x * h.p.x + h.p.z * h.p.z);
    const float cx = rho > 0.0f ? h.p.x / rho : 1.0f, cz = rho > 0.0f ? h.p.z / rho : 0.0f;
    const float sg = rv < 0.0 ? -1.0f : 1.0f;
    float3 n = f3((float)yd * cx, -(float)rd * sg, (float)yd * cz);
    if (!(dot(n, n) > 0.0f)) n = f3(cx, 0.0f, cz);
    h.n = normalize(n);
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    h.tan = f3(0.0f, 1.0f, 0.0f);
    h.uv = make_float2(0.0f, 0.0f);
    h.mat = material_id;
    return true;
}

// Whether (px, pz) (relative to the prism's centre) is inside the closed
// Bezier contour: crossings of the line z = pz at x > px, counted where the
// contour changes side (even-odd rule).
__device__ __forceinline__ bool bez_contour_inside(const float4* spans, int2 run, double px, double pz) {
    bool inside = false;
    for (int k = run.x; k < run.x + run.y; k++) {
        double X[4], Z[4];
        load_span(spans, k, X, Z);
        double zlo = Z[0], zhi = Z[0], xhi = X[0];
        for (int i = 1; i < 4; i++) { zlo = fmin(zlo, Z[i]); zhi = fmax(zhi, Z[i]); xhi = fmax(xhi, X[i]); }
        if (pz < zlo || pz > zhi || xhi <= px) continue;
        for (int i = 0; i < 4; i++) Z[i] -= pz;
        double roots[3];
        const int n = bern_roots<3>(Z, roots);
        for (int i = 0; i < n; i++) {
            // half-open in u: a crossing at a span's end belongs to the next span
            if (roots[i] >= 1.0) continue;
            if (cubic_at(X, roots[i]) > px) inside = !inside;
        }
    }
    return inside;
}

// Exact Bezier prism (extension): walls and caps of the contour run
// extruded over [y0, y1] (absolute), contour about (cx, cz).
static __device__ __noinline__ bool prism_exact_test(const Ray& r, const Prism& p, const float4* spans, int2 run, Hit& h) {
    const float y0 = p.center.y + p.y_min, y1 = p.center.y + p.y_max;
    {
        float ty0 = (y0 - r.o.y) / r.d.y, ty1 = (y1 - r.o.y) / r.d.y;
        if (ty0 > ty1) { const float t = ty0; ty0 = ty1; ty1 = t; }
        if (fmaxf(ty0, r.tmin) > fminf(ty1, r.tmax)) return false;
    }
    const double cx = p.center.x, cz = p.center.z;
    double best = r.tmax;
    int kind = -1;          // 0 cap, 1 wall
    double bu = 0.0;
    int bk = -1;
    float cap_ny = 0.0f;
    // caps
    for (int face = 0; face < 2; face++) {
        const float yf = face == 0 ? y0 : y1;
        const float t = (yf - r.o.y) / r.d.y;
        if (!(t >= r.tmin && t <= r.tmax) || t >= best) continue;
        const float3 P = r.o + t * r.d;
        if (!bez_contour_inside(spans, run, (double)P.x - cx, (double)P.z - cz)) continue;
        best = t; kind = 0; cap_ny = face == 0 ? -1.0f : 1.0f;
    }
    // walls
    const double ox = (double)r.o.x - cx, oz = (double)r.o.z - cz, dx = r.d.x, dz = r.d.z;
    const double a2 = dx * dx + dz * dz;
    if (a2 > 1e-24 * (a2 + (double)r.d.y * r.d.y)) {
        for (int k = run.x; k < run.x + run.y; k++) {
            double X[4], Z[4];
            load_span(spans, k, X, Z);
            double f[4];
            for (int i = 0; i < 4; i++) f[i] = (X[i] - ox) * dz - (Z[i] - oz) * dx;
            double roots[3];
            const int n = bern_roots<3>(f, roots);
            for (int i = 0; i < n; i++) {
                const double s = ((cubic_at(X, roots[i]) - ox) * dx + (cubic_at(Z, roots[i]) - oz) * dz) / a2;
                if (!(s >= r.tmin && s < best)) continue;
                const double yy = (double)r.o.y + s * r.d.y;
                if (yy < (double)y0 - 1e-6 * fabs(y0) - 1e-7 || yy > (double)y1 + 1e-6 * fabs(y1) + 1e-7) continue;
                best = s; kind = 1; bu = roots[i]; bk = k;
            }
        }
    }
    if (kind < 0) return false;
    const float t = (float)best;
    h.t = t;
    h.p = r.o + t * r.d;
    if (kind == 0) {
        h.n = f3(0.0f, cap_ny, 0.0f);
        h.tan = f3(1.0f, 0.0f, 0.0f);
    } else {
        double X[4], Z[4];
        load_span(spans, bk, X, Z);
        const float ex = (float)cubic_d(X, bu), ez = (float)cubic_d(Z, bu);
        float3 n = f3(ez, 0.0f, -ex);
        h.n = dot(n, n) > 0.0f ? normalize(n) : f3(1.0f, 0.0f, 0.0f);
        h.tan = f3(0.0f, 1.0f, 0.0f);
    }
    if (dot(h.n, r.d) > 0.0f) h.n = -h.n;
    h.uv = make_float2(0.0f, 0.0f);
    h.mat = p.material_id;
    return true;
}

// ---- per-primitive dispatch of the extensions --------------------------

__device__ __forceinline__ HfGrid hf_grid_of(const DevScene& S, int i) {
    if (!S.hf_grid) return HfGrid{nullptr, 0, 0};
    const int4 g = __ldg(&S.hf_grid[i]);
    if (g.x < 0) return HfGrid{nullptr, 0, 0};
    return HfGrid{S.hf_heights + g.x, g.y, g.z};
}

__device__ __forceinline__ int2 lathe_run_of(const DevScene& S, int i) {
    if (!S.lathe_bz) return make_int2(0, 0);
    const int4 r = __ldg(&S.lathe_bz[i]);
    return make_int2(r.x, r.y);
}

__device__ __forceinline__ int2 prism_run_of(const DevScene& S, int i) {
    if (!S.prism_bz) return make_int2(0, 0);
    const int4 r = __ldg(&S.prism_bz[i]);
    return make_int2(r.x, r.y);
}

// Lathe i: its exact Bezier surface when it has one, else the reference's
// tessellated test (primitives/lathe.h:30-59).
__device__ __forceinline__ bool lathe_any_test(const DevScene& S, const Ray& r, int i, Hit& h) {
    const int2 run = lathe_run_of(S, i);
    if (run.y > 0) return lathe_exact_test(r, S.bz_spans, run, __ldg(&S.lathe_bz_bound[i]), S.lathes[i].material_id, h);
    return lathe_test(r, S.lathes[i], S.lathe_points, h);
}

// Prism i: its exact Bezier contour when it has one, else the reference's
// polygon test (primitives/prism.h:70-134).
__device__ __forceinline__ bool prism_any_test(const DevScene& S, const Ray& r, int i, Hit& h) {
    const int2 run = prism_run_of(S, i);
    if (run.y > 0) return prism_exact_test(r, S.prisms[i], S.bz_spans, run, h);
    return prism_test(r, S.prisms[i], S.prism_points, h);
}

}  // namespace dev
}  // namespace sheen
