/*
 * sheen_oracle.c -- C restatement of Sheen's per-pixel ray-casting path.
 *
 * TEST INFRASTRUCTURE ONLY (see sheen_oracle.h).  Built twice: with
 * ORACLE_REAL=float (the reference's precision; rsqrtf is taken as the exact
 * 1/sqrt) and ORACLE_REAL=double (the FP64 hit-distance oracle).
 *
 * Every function names the reference lines it restates.  Quirks of the
 * reference that affect results are restated on purpose and marked QUIRK.
 */
#include "sheen_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;

#define R(x) ((real)(x))

/* ------------------------------------------------------------------ */
/* vectors                                                             */
/* ------------------------------------------------------------------ */
typedef struct { real x, y, z; } V;
static inline V v3(real x, real y, real z) { V r = {x, y, z}; return r; }
static inline V fv(sheen_float3 a) { return v3(a.x, a.y, a.z); }
static inline V add(V a, V b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V sub(V a, V b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V mul(V a, real s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V vmul(V a, V b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V neg(V a) { return v3(-a.x, -a.y, -a.z); }
static inline real dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V cross(V a, V b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
/* types.h:314-317 (rsqrtf -> exact reciprocal square root) */
static inline V nrm(V a) { real il = R(1) / sqrt(dot(a, a)); return mul(a, il); }
static inline real rmin(real a, real b) { return a < b ? a : b; }   /* fminf for non-NaN */
static inline real rmax(real a, real b) { return a > b ? a : b; }
static inline real rfmin(real a, real b) { return (real)fmin((double)a, (double)b); }
static inline real rfmax(real a, real b) { return (real)fmax((double)a, (double)b); }
static inline real rpow(real a, real b) { return (real)pow((double)a, (double)b); }

typedef struct { V o, d; real tmin, tmax; } Ray;

typedef struct {
    real t;
    int mat, obj;          /* material_id, object_id as the reference sets them */
    int cat, prim;         /* category and index within it (oracle bookkeeping) */
    V p, n, tan;
    real u, v;
} Hit;

enum { CAT_SPHERE, CAT_STRAND, CAT_MESH, CAT_HF, CAT_SE, CAT_LATHE, CAT_PRISM, CAT_CSG, CAT_PLANE };

/* ------------------------------------------------------------------ */
/* sampling/aa.h:15-71 -- pixel sample layout and counter-based RNG    */
/* ------------------------------------------------------------------ */
static inline uint32_t aa_hash(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static inline real aa_rand(uint32_t seed) { return R((float)(aa_hash(seed) & 0xffffffu) / 16777216.0f); }

static void aa_offset(int s, int n, int x, int y, real* ox, real* oy) {
    uint32_t seed = (uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)s * 83492791u;
    if (n <= 4) {
        static const float cell[4][2] = {{0.25f, 0.25f}, {0.75f, 0.25f}, {0.25f, 0.75f}, {0.75f, 0.75f}};
        int k = s < 3 ? s : 3;
        real jx = aa_rand(seed) - R(0.5), jy = aa_rand(seed ^ 0x9e3779b9u) - R(0.5);
        *ox = R(cell[k][0]) + jx * R(0.5);
        *oy = R(cell[k][1]) + jy * R(0.5);
        return;
    }
    int side = 2;
    while (side * side < n) side++;
    real inv = R(1) / (real)side;
    *ox = ((real)(s % side) + aa_rand(seed)) * inv;
    *oy = ((real)(s / side) + aa_rand(seed ^ 0x9e3779b9u)) * inv;
}

/* Extension (no reference counterpart): sample positions without jitter --
 * the pixel centre at 1 spp, the centres of the same cells otherwise. */
static void aa_offset_centered(int s, int n, real* ox, real* oy) {
    if (n <= 1) { *ox = R(0.5); *oy = R(0.5); return; }
    if (n <= 4) {
        *ox = (s == 0 || s == 2) ? R(0.25) : R(0.75);
        *oy = s < 2 ? R(0.25) : R(0.75);
        return;
    }
    int side = 2;
    while (side * side < n) side++;
    real inv = R(1) / (real)side;
    *ox = ((real)(s % side) + R(0.5)) * inv;
    *oy = ((real)(s / side) + R(0.5)) * inv;
}

/* ------------------------------------------------------------------ */
/* scene                                                               */
/* ------------------------------------------------------------------ */
typedef struct { unsigned char* px; int w, h, mips; } Tex;

struct OracleScene {
    SheenScene s;                       /* pointers into the copies below */
    Object* objects; SweepPoint* sweep_points; SweepStrand* strands; Triangle* tris;
    HeightField* hfs; Superellipsoid* ses; LathePoint* lpts; Lathe* lathes;
    PrismPoint* ppts; Prism* prisms; CSGNode* csg; Plane* planes; Material* mats;
    Light* lights; Medium* media;
    Tex* tex; int ntex;
    unsigned char** hf_img;
    /* photon map (render_kernel.h:47-53) */
    sheen_float3* ph_pos; sheen_float3* ph_dir; sheen_float3* ph_nrm; sheen_float3* ph_flux;
    int nph; int* cell_start; int* cell_count; int num_cells; real cell;
    int centered;                       /* samples without jitter (extension) */
    int knn;                            /* k-nearest-photon gather (extension; 0: the reference's) */
    /* scene extensions (SheenSceneExt); NULL / 0 when absent */
    float* se_n2;                       /* per superellipsoid: north-south exponent (> 0: two-exponent) */
    int* hfg;                           /* per heightfield: offset (< 0 none), w, h */
    float* hf_heights;
    int* lathe_run;                     /* per lathe: first span, spans */
    int* prism_run;                     /* per prism */
    double* spans;                      /* 8 per cubic span: a0 b0 a1 b1 a2 b2 a3 b3 */
    int nspans;
    int* csg_roots; int ncsg_roots;
    SheenCsgBox* csg_boxes; int ncsg_boxes;
    SheenCsgCone* csg_cones; int ncsg_cones;
    int bounces;                        /* reflect + refract recursion depth (> 1: render_deep) */
};

static void sample_pos(const OracleScene* S, int s, int n, int x, int y, real* ox, real* oy) {
    if (S->centered) aa_offset_centered(s, n, ox, oy);
    else aa_offset(s, n, x, y, ox, oy);
}

/* ------------------------------------------------------------------ */
/* bvh.h:578-600 -- slab test exactly as the reference writes it        */
/* (QUIRK: the final range check uses the x/y-merged interval only)     */
/* ------------------------------------------------------------------ */
static int slab(const Ray* r, V lo, V hi) {
    real ix = R(1) / r->d.x;
    real tminX = (lo.x - r->o.x) * ix, tmaxX = (hi.x - r->o.x) * ix;
    if (tminX > tmaxX) { real t = tminX; tminX = tmaxX; tmaxX = t; }
    real iy = R(1) / r->d.y;
    real tminY = (lo.y - r->o.y) * iy, tmaxY = (hi.y - r->o.y) * iy;
    if (tminY > tmaxY) { real t = tminY; tminY = tmaxY; tmaxY = t; }
    if (tminX > tmaxY || tminY > tmaxX) return 0;
    if (tminY > tminX) tminX = tminY;
    if (tmaxY < tmaxX) tmaxX = tmaxY;
    real iz = R(1) / r->d.z;
    real tminZ = (lo.z - r->o.z) * iz, tmaxZ = (hi.z - r->o.z) * iz;
    if (tminZ > tmaxZ) { real t = tminZ; tminZ = tmaxZ; tmaxZ = t; }
    if (tminX > tmaxZ || tminZ > tmaxX) return 0;
    return (tmaxX >= r->tmin) && (tminX <= r->tmax);
}

/* Leaf boxes of the reference BVHs (bvh.h:24-35, 40-62, 235-242, 304-309,
 * 314-316, 321-332, 394-407).  They are float boxes in the reference; the
 * FP64 build widens them by a relative 1e-6 so that rounding can never cull
 * a hit the FP32 box admits. */
static void widen(V* lo, V* hi) {
    if (sizeof(real) == sizeof(float)) return;
    real ex = R(1e-6) * (fabs(lo->x) + fabs(hi->x)) + R(1e-12);
    real ey = R(1e-6) * (fabs(lo->y) + fabs(hi->y)) + R(1e-12);
    real ez = R(1e-6) * (fabs(lo->z) + fabs(hi->z)) + R(1e-12);
    lo->x -= ex; lo->y -= ey; lo->z -= ez; hi->x += ex; hi->y += ey; hi->z += ez;
}

/* ------------------------------------------------------------------ */
/* primitives/sphere.h:8-53                                            */
/* ------------------------------------------------------------------ */
static int sphere_hit(const Ray* r, V c, real rad, Hit* h) {
    V oc = sub(r->o, c);
    real a = dot(r->d, r->d), b = R(2) * dot(oc, r->d), cc = dot(oc, oc) - rad * rad;
    real disc = b * b - R(4) * a * cc;
    if (disc < 0) return 0;
    real sq = sqrt(disc);
    real t = (-b - sq) / (R(2) * a);
    if (t < r->tmin || t > r->tmax) {
        t = (-b + sq) / (R(2) * a);
        if (t < r->tmin || t > r->tmax) return 0;
    }
    h->t = t;
    h->p = add(r->o, mul(r->d, t));
    h->n = nrm(sub(h->p, c));
    h->tan = v3(0, 0, 0);
    h->u = h->v = 0;   /* the reference leaves uv unset for spheres */
    return 1;
}

static int sphere_iv(const Ray* r, V c, real rad, real t0, real t1, real* te, real* tx) {
    V oc = sub(r->o, c);
    real a = dot(r->d, r->d), b = R(2) * dot(oc, r->d), cc = dot(oc, oc) - rad * rad;
    real disc = b * b - R(4) * a * cc;
    if (disc < 0) return 0;
    real sq = sqrt(disc);
    real ta = (-b - sq) / (R(2) * a), tb = (-b + sq) / (R(2) * a);
    if (tb < t0 || ta > t1) return 0;
    *te = rfmax(ta, t0);
    *tx = rfmin(tb, t1);
    return *te <= *tx;
}

/* primitives/plane.h:7-24 */
static int plane_hit(const Ray* r, V n, real d, Hit* h) {
    real den = dot(n, r->d);
    if (fabs(den) > R(1e-6)) {
        real t = -(dot(r->o, n) + d) / den;
        if (t >= r->tmin && t <= r->tmax) {
            h->t = t;
            h->p = add(r->o, mul(r->d, t));
            h->n = n;
            h->tan = v3(0, 0, 0);
            h->u = h->v = 0;
            if (dot(h->n, r->d) > 0) h->n = neg(h->n);
            return 1;
        }
    }
    return 0;
}

/* primitives/triangle.h:8-47 (Moller-Trumbore) */
static int tri_hit(const Ray* r, const Triangle* tr, Hit* h) {
    V v0 = fv(tr->v0), e1 = sub(fv(tr->v1), v0), e2 = sub(fv(tr->v2), v0);
    V pv = cross(r->d, e2);
    real det = dot(e1, pv);
    if (fabs(det) < R(1e-8)) return 0;
    real inv = R(1) / det;
    V tv = sub(r->o, v0);
    real u = dot(tv, pv) * inv;
    if (u < 0 || u > 1) return 0;
    V qv = cross(tv, e1);
    real v = dot(r->d, qv) * inv;
    if (v < 0 || u + v > 1) return 0;
    real t = dot(e2, qv) * inv;
    if (t < r->tmin || t > r->tmax) return 0;
    h->t = t;
    h->p = add(r->o, mul(r->d, t));
    real w = R(1) - u - v;
    V nv = add(add(mul(fv(tr->n0), w), mul(fv(tr->n1), u)), mul(fv(tr->n2), v));
    if (dot(nv, nv) > R(1e-12)) h->n = nrm(nv);
    else h->n = nrm(cross(e1, e2));
    h->tan = nrm(e1);
    h->u = tr->uv0.x * w + tr->uv1.x * u + tr->uv2.x * v;
    h->v = tr->uv0.y * w + tr->uv1.y * u + tr->uv2.y * v;
    if (dot(h->n, r->d) > 0) h->n = neg(h->n);
    return 1;
}

/* primitives/cone.h:11-73 -- cone segment between two sweep points */
static int cone_hit(const Ray* r, V p0, real r0, V p1, real r1, Hit* h) {
    V axis = sub(p1, p0);
    real L2 = dot(axis, axis);
    if (L2 < R(1e-12)) return 0;
    real L = sqrt(L2);
    V da = mul(axis, R(1) / L);   /* axis / L */
    da = v3(axis.x / L, axis.y / L, axis.z / L);
    real k = (r1 - r0) / L;
    V Q = sub(r->o, p0);
    real u = dot(r->d, da), v = dot(Q, da);
    V Dp = sub(r->d, mul(da, u)), Qp = sub(Q, mul(da, v));
    real A = dot(Dp, Dp) - k * k * u * u;
    real B = R(2) * (dot(Dp, Qp) - k * r0 * u - k * k * v * u);
    real C = dot(Qp, Qp) - k * k * v * v - R(2) * k * r0 * v - r0 * r0;
    real disc = B * B - R(4) * A * C;
    if (disc < 0) return 0;
    real sq = sqrt(disc), i2a = R(1) / (R(2) * A);
    real s1 = (-B - sq) * i2a, s2 = (-B + sq) * i2a;
    for (int i = 0; i < 2; i++) {
        real s = i == 0 ? s1 : s2;
        if (s < r->tmin || s > r->tmax) continue;
        real tp = v + s * u;
        if (tp < 0 || tp > L) continue;
        h->t = s;
        h->p = add(r->o, mul(r->d, s));
        h->n = nrm(add(Qp, mul(Dp, s)));
        h->tan = da;
        if (dot(h->n, r->d) > 0) h->n = neg(h->n);
        return 1;
    }
    return 0;
}

/* primitives/cone.h:78-121 -- hemisphere cap (the reference leaves the
 * tangent unset here; the oracle uses 0) */
static int hemi_hit(const Ray* r, V c, real rad, V axis, Hit* h) {
    V oc = sub(r->o, c);
    real a = dot(r->d, r->d), b = R(2) * dot(oc, r->d), cc = dot(oc, oc) - rad * rad;
    real disc = b * b - R(4) * a * cc;
    if (disc < 0) return 0;
    real sq = sqrt(disc), i2a = R(1) / (R(2) * a);
    real t1 = (-b - sq) * i2a, t2 = (-b + sq) * i2a;
    for (int i = 0; i < 2; i++) {
        real t = i == 0 ? t1 : t2;
        if (t < r->tmin || t > r->tmax) continue;
        V p = add(r->o, mul(r->d, t));
        V n = nrm(sub(p, c));
        if (dot(n, axis) < 0) continue;
        h->t = t; h->p = p; h->n = n; h->tan = v3(0, 0, 0);
        if (dot(h->n, r->d) > 0) h->n = neg(h->n);
        return 1;
    }
    return 0;
}

/* primitives/sweep.h:13-90 -- whole strand: caps + segments + joints */
static int sweep_hit(const Ray* r, const SweepStrand* st, const SweepPoint* pts, Hit* h) {
    if (st->point_count < 2) return 0;
    int any = 0;
    real best = r->tmax;
    Hit tmp;
    const SweepPoint* P = pts + st->point_offset;
    int n = st->point_count;
#define TAKE() do { if (tmp.t < best) { *h = tmp; h->mat = st->material_id; best = tmp.t; any = 1; } } while (0)
    if (hemi_hit(r, fv(P[0].position), P[0].radius, nrm(sub(fv(P[0].position), fv(P[1].position))), &tmp)) TAKE();
    for (int i = 0; i < n - 1; i++) {
        if (cone_hit(r, fv(P[i].position), P[i].radius, fv(P[i + 1].position), P[i + 1].radius, &tmp)) TAKE();
        if (i < n - 2) {
            V ax = nrm(sub(fv(P[i + 2].position), fv(P[i + 1].position)));
            if (hemi_hit(r, fv(P[i + 1].position), P[i + 1].radius, ax, &tmp)) TAKE();
        }
    }
    if (hemi_hit(r, fv(P[n - 1].position), P[n - 1].radius,
                 nrm(sub(fv(P[n - 1].position), fv(P[n - 2].position))), &tmp)) TAKE();
#undef TAKE
    h->u = h->v = 0;
    return any;
}

/* primitives/sweep.h:96-148 -- optical depth of strands along a shadow ray */
static real seg_tau(const Ray* r, const SweepPoint* a, const SweepPoint* b, real sigma) {
    V u = sub(fv(b->position), fv(a->position));
    real A = dot(u, u);
    if (A < R(1e-12)) return 0;
    V v = r->d, w = sub(r->o, fv(a->position));
    real B = dot(u, v), C = dot(v, v), D = dot(u, w), E = dot(v, w);
    real den = A * C - B * B;
    real s = den > R(1e-9) ? (B * E - C * D) / den : R(0);
    s = rfmin(rfmax(s, 0), 1);
    real t = (B * s + E) / C;
    if (t < 0) { t = 0; s = rfmin(rfmax(-D / A, 0), 1); }
    if (t > r->tmax) return 0;
    V cl = sub(add(w, mul(u, s)), mul(v, t));
    real d2 = dot(cl, cl);
    real rr = a->radius + (b->radius - a->radius) * s;
    real r2 = rr * rr;
    if (d2 >= r2) return 0;
    return sigma * (R(2) * sqrt(rfmax(r2 - d2, 0)));
}

static void strand_box(const OracleScene* S, int i, V* lo, V* hi) {
    const SweepStrand* st = &S->strands[i];
    *lo = v3(1e10f, 1e10f, 1e10f);
    *hi = v3(-1e10f, -1e10f, -1e10f);
    for (int k = 0; k < st->point_count; k++) {
        const SweepPoint* p = &S->sweep_points[st->point_offset + k];
        real rr = p->radius;
        *lo = v3(rfmin(lo->x, p->position.x - rr), rfmin(lo->y, p->position.y - rr), rfmin(lo->z, p->position.z - rr));
        *hi = v3(rfmax(hi->x, p->position.x + rr), rfmax(hi->y, p->position.y + rr), rfmax(hi->z, p->position.z + rr));
    }
    widen(lo, hi);
}

/* bvh.h:928-960 (scan order instead of DFS order; the early exit at tau > 6
 * makes the exact sum order dependent only beyond exp(-6)) */
static real strands_tau(const OracleScene* S, const Ray* r, real sigma) {
    real tau = 0;
    for (int i = 0; i < S->s.num_sweep_strands; i++) {
        V lo, hi;
        strand_box(S, i, &lo, &hi);
        if (!slab(r, lo, hi)) continue;
        const SweepStrand* st = &S->strands[i];
        real ts = 0;
        for (int k = 0; k < st->point_count - 1; k++) {
            ts += seg_tau(r, &S->sweep_points[st->point_offset + k], &S->sweep_points[st->point_offset + k + 1], sigma);
            if (ts > R(6)) break;
        }
        tau += ts;
        if (tau > R(6)) return tau;
    }
    return tau;
}

/* primitives/lathe.h:14-63.  QUIRK: the profile is revolved about the world
 * Y axis at x = z = 0; Lathe.center is ignored by the test. */
static int lathe_hit(const Ray* r, const Lathe* l, const LathePoint* pts, Hit* h) {
    if (l->point_count < 2) return 0;
    int any = 0;
    real best = r->tmax;
    Hit tmp;
    for (int i = 0; i < l->point_count - 1; i++) {
        const LathePoint* a = &pts[l->point_offset + i];
        const LathePoint* b = &pts[l->point_offset + i + 1];
        if (a->radius <= 0 && b->radius <= 0) continue;
        if (cone_hit(r, v3(0, a->y, 0), a->radius, v3(0, b->y, 0), b->radius, &tmp)) {
            if (tmp.t < best) {
                tmp.p = add(r->o, mul(r->d, tmp.t));
                *h = tmp;
                h->mat = l->material_id;
                best = tmp.t;
                any = 1;
            }
        }
    }
    h->u = h->v = 0;
    return any;
}

/* bvh.h:394-407.  QUIRK: the x/z extent starts at center -/+ 1e30, so only the
 * y range (which does use center.y) ever culls. */
static void lathe_box(const Lathe* l, const LathePoint* pts, V* lo, V* hi) {
    *lo = v3(l->center.x - 1e30f, 1e30f, l->center.z - 1e30f);
    *hi = v3(l->center.x + 1e30f, -1e30f, l->center.z + 1e30f);
    for (int i = 0; i < l->point_count; i++) {
        const LathePoint* p = &pts[l->point_offset + i];
        real rr = p->radius;
        if (rr < 0) continue;
        *lo = v3(rfmin(lo->x, l->center.x - rr), rfmin(lo->y, l->center.y + p->y - rr), rfmin(lo->z, l->center.z - rr));
        *hi = v3(rfmax(hi->x, l->center.x + rr), rfmax(hi->y, l->center.y + p->y + rr), rfmax(hi->z, l->center.z + rr));
    }
    if (lo->x > hi->x) { *lo = *hi = v3(0, 0, 0); }
    widen(lo, hi);
}

/* primitives/prism.h:18-63 -- even-odd containment over closed sub-contours */
static int prism_in_contour(real x, real z, const PrismPoint* pts, int base, int count) {
    int inside = 0;
    int j = count - 1;
    for (int i = 0; i < count; i++) {
        const PrismPoint* pi = &pts[base + i];
        const PrismPoint* pj = &pts[base + j];
        if ((pi->z > z) != (pj->z > z)) {
            real xint = (R(pj->x) - pi->x) * (z - pi->z) / (R(pj->z) - pi->z) + pi->x;
            if (x < xint) inside = !inside;
        }
        j = i;
    }
    return inside;
}

static int prism_inside(real x, real z, const Prism* p, const PrismPoint* all) {
    int base = p->point_offset, cnt = p->point_count, i = 0, inside = 0;
    while (i < cnt) {
        int start = i, j = i + 1;
        while (j < cnt) {
            if (all[base + j].x == all[base + start].x && all[base + j].z == all[base + start].z) break;
            j++;
        }
        if (j - start >= 3 && prism_in_contour(x, z, all, base + start, j - start)) inside = !inside;
        i = j < cnt ? j + 1 : j;
    }
    return inside;
}

/* primitives/prism.h:68-133 -- caps and vertical walls */
static int prism_hit(const Ray* r, const Prism* p, const PrismPoint* pts, Hit* h) {
    real y0 = R(p->center.y) + p->y_min, y1 = R(p->center.y) + p->y_max;
    real ty0 = (y0 - r->o.y) / r->d.y, ty1 = (y1 - r->o.y) / r->d.y;
    if (ty0 > ty1) { real t = ty0; ty0 = ty1; ty1 = t; }
    if (rfmax(ty0, r->tmin) > rfmin(ty1, r->tmax)) return 0;
    int any = 0;
    real best = r->tmax;
    for (int face = 0; face < 2; face++) {
        real yf = face == 0 ? y0 : y1;
        real t = (yf - r->o.y) / r->d.y;
        if (t < r->tmin || t > r->tmax) continue;
        V P = add(r->o, mul(r->d, t));
        if (!prism_inside(P.x - p->center.x, P.z - p->center.z, p, pts)) continue;
        if (t < best) {
            h->t = t; h->p = P;
            h->n = v3(0, face == 0 ? -1 : 1, 0);
            if (dot(h->n, r->d) > 0) h->n = neg(h->n);
            h->tan = v3(1, 0, 0);
            h->mat = p->material_id;
            best = t; any = 1;
        }
    }
    real dx = r->d.x, dy = r->d.y, dz = r->d.z, ox = r->o.x, oz = r->o.z;
    int base = p->point_offset, cnt = p->point_count;
    for (int i = 0; i < cnt; i++) {
        int j = (i + 1) % cnt;
        const PrismPoint* a = &pts[base + i];
        const PrismPoint* b = &pts[base + j];
        if (a->x == b->x && a->z == b->z) continue;
        real ax = R(a->x) + p->center.x, az = R(a->z) + p->center.z;
        real bx = R(b->x) + p->center.x, bz = R(b->z) + p->center.z;
        real ex = bx - ax, ez = bz - az;
        real den = ex * dz - ez * dx;
        if (fabs(den) < R(1e-9)) continue;
        real s = (dx * (az - oz) - dz * (ax - ox)) / den;
        if (s < R(-0.001) || s > R(1.001)) continue;
        real t;
        if (fabs(dx) > R(1e-9)) t = (ax + s * ex - ox) / dx;
        else if (fabs(dz) > R(1e-9)) t = (az + s * ez - oz) / dz;
        else continue;
        if (t < r->tmin || t > r->tmax) continue;
        real yy = r->o.y + dy * t;
        if (yy < y0 - R(0.001) || yy > y1 + R(0.001)) continue;
        if (t < best) {
            h->t = t; h->p = add(r->o, mul(r->d, t));
            h->n = nrm(v3(ez, 0, -ex));
            h->tan = v3(0, 1, 0);
            if (dot(h->n, r->d) > 0) h->n = neg(h->n);
            h->mat = p->material_id;
            best = t; any = 1;
        }
    }
    h->u = h->v = 0;
    return any;
}

static void prism_box(const Prism* p, const PrismPoint* pts, V* lo, V* hi) {
    *lo = v3(1e30f, p->center.y + p->y_min, 1e30f);
    *hi = v3(-1e30f, p->center.y + p->y_max, -1e30f);
    for (int i = 0; i < p->point_count; i++) {
        const PrismPoint* q = &pts[p->point_offset + i];
        lo->x = rfmin(lo->x, p->center.x + q->x); hi->x = rfmax(hi->x, p->center.x + q->x);
        lo->z = rfmin(lo->z, p->center.z + q->z); hi->z = rfmax(hi->z, p->center.z + q->z);
    }
    if (lo->x > hi->x) { *lo = *hi = v3(0, p->center.y, 0); }
    widen(lo, hi);
}

/* ------------------------------------------------------------------ */
/* primitives/superellipsoid.h:12-161                                  */
/* ------------------------------------------------------------------ */
/* n2 > 0 (extension, no counterpart in the reference): the two-exponent
 * body (|qx|^n + |qz|^n)^(n2/n) + |qy|^n2. */
static real se_f(const Superellipsoid* s, V p, real n2) {
    real qx = (p.x - s->center.x) / s->a, qy = (p.y - s->center.y) / s->b, qz = (p.z - s->center.z) / s->c;
    if (n2 > 0) return rpow(rpow(fabs(qx), s->n) + rpow(fabs(qz), s->n), n2 / s->n) + rpow(fabs(qy), n2);
    return rpow(fabs(qx), s->n) + rpow(fabs(qy), s->n) + rpow(fabs(qz), s->n);
}

static V se_grad(const Superellipsoid* s, V p, real n2) {
    real qx = (p.x - s->center.x) / s->a, qy = (p.y - s->center.y) / s->b, qz = (p.z - s->center.z) / s->c;
    real n = s->n;
    if (n2 > 0) {
        real xz = rpow(fabs(qx), n) + rpow(fabs(qz), n);
        real k = xz > 0 ? n2 * rpow(xz, n2 / n - 1) : 0;
        return v3(k * rpow(fabs(qx), n - 1) * (qx >= 0 ? 1 : -1) / s->a,
                  n2 * rpow(fabs(qy), n2 - 1) * (qy >= 0 ? 1 : -1) / s->b,
                  k * rpow(fabs(qz), n - 1) * (qz >= 0 ? 1 : -1) / s->c);
    }
    return v3(n * rpow(fabs(qx), n - 1) * (qx >= 0 ? 1 : -1) / s->a,
              n * rpow(fabs(qy), n - 1) * (qy >= 0 ? 1 : -1) / s->b,
              n * rpow(fabs(qz), n - 1) * (qz >= 0 ? 1 : -1) / s->c);
}

static int se_clip(const Ray* r, const Superellipsoid* s, real* tA, real* tB) {
    V lo = v3(R(s->center.x) - s->a, R(s->center.y) - s->b, R(s->center.z) - s->c);
    V hi = v3(R(s->center.x) + s->a, R(s->center.y) + s->b, R(s->center.z) + s->c);
    real ix = R(1) / r->d.x, iy = R(1) / r->d.y, iz = R(1) / r->d.z;
    real tx0 = (lo.x - r->o.x) * ix, tx1 = (hi.x - r->o.x) * ix;
    if (tx0 > tx1) { real t = tx0; tx0 = tx1; tx1 = t; }
    real ty0 = (lo.y - r->o.y) * iy, ty1 = (hi.y - r->o.y) * iy;
    if (ty0 > ty1) { real t = ty0; ty0 = ty1; ty1 = t; }
    real tz0 = (lo.z - r->o.z) * iz, tz1 = (hi.z - r->o.z) * iz;
    if (tz0 > tz1) { real t = tz0; tz0 = tz1; tz1 = t; }
    *tA = rfmax(rfmax(tx0, ty0), tz0);
    *tB = rfmin(rfmin(tx1, ty1), tz1);
    return 1;
}

/* superellipsoid.h:41-117.  QUIRK: on an outside->inside crossing the
 * bisection runs on [t, t] (t_prev was already advanced), so the entry point
 * is the sample itself. */
static int se_intervals(const Ray* r, const Superellipsoid* s, real t0, real t1, real* te, real* tx, real n2) {
    real tA, tB;
    se_clip(r, s, &tA, &tB);
    if (tB < t0 || tA > t1 || tB < tA) return 0;
    t0 = rfmax(t0, tA);
    t1 = rfmin(t1, tB);
    const real EPS = 1;
    const int NS = 32;
    real step = (t1 - t0) / (real)NS;
    real tp = t0;
    real Fp = se_f(s, add(r->o, mul(r->d, tp)), n2);
    int inside = Fp <= EPS, fe = 0, fx = 0;
    *te = R(-1e30); *tx = R(-1e30);
    if (inside) { *te = t0; fe = 1; }
    for (int i = 1; i <= NS && !fx; i++) {
        real t = rfmin(t0 + step * (real)i, t1);
        real F = se_f(s, add(r->o, mul(r->d, t)), n2);
        if (inside && F > EPS) {
            real lo = tp, hi = t;
            for (int b = 0; b < 20; b++) {
                real mid = R(0.5) * (lo + hi);
                if (se_f(s, add(r->o, mul(r->d, mid)), n2) > EPS) hi = mid; else lo = mid;
            }
            *tx = R(0.5) * (lo + hi);
            if (*tx > t1) *tx = t1;
            fx = 1;
            break;
        }
        tp = t;
        Fp = F;
        if (!inside && F <= EPS) {
            real lo = tp, hi = t;
            for (int b = 0; b < 20; b++) {
                real mid = R(0.5) * (lo + hi);
                if (se_f(s, add(r->o, mul(r->d, mid)), n2) <= EPS) hi = mid; else lo = mid;
            }
            *te = R(0.5) * (lo + hi);
            if (*te < t0) *te = t0;
            fe = 1;
            inside = 1;
        }
    }
    (void)Fp;
    if (!fe) return 0;
    if (!fx) *tx = t1;
    return *te <= *tx;
}

static int se_hit(const Ray* r, const Superellipsoid* s, Hit* h, real n2) {
    real t0, t1;
    se_clip(r, s, &t0, &t1);
    if (t1 < r->tmin || t0 > r->tmax || t1 < t0) return 0;
    t0 = rfmax(t0, r->tmin);
    t1 = rfmin(t1, r->tmax);
    real te, tx;
    if (!se_intervals(r, s, t0, t1, &te, &tx, n2)) return 0;
    h->t = te;
    h->p = add(r->o, mul(r->d, te));
    h->n = nrm(se_grad(s, h->p, n2));
    h->tan = v3(1, 0, 0);
    h->u = h->p.x; h->v = h->p.y;
    if (dot(h->n, r->d) > 0) h->n = neg(h->n);
    return 1;
}

/* ------------------------------------------------------------------ */
/* primitives/heightfield.h:13-183                                     */
/* ------------------------------------------------------------------ */
static real hf_cell_hash(int xi, int zi, int seed) {
    uint32_t h = (uint32_t)xi * 374761393u + (uint32_t)zi * 668265263u + (uint32_t)seed * 974634097u;
    h = (h ^ (h >> 13)) * 1274126177u;
    h = h ^ (h >> 16);
    return R((float)(h & 0xffffffu) / 16777216.0f);
}

static real hf_noise(real fx, real fz, int seed) {
    int x0 = (int)floor(fx), z0 = (int)floor(fz);
    real tx = fx - (real)x0, tz = fz - (real)z0;
    tx = tx * tx * (R(3) - R(2) * tx);
    tz = tz * tz * (R(3) - R(2) * tz);
    real v00 = hf_cell_hash(x0, z0, seed), v10 = hf_cell_hash(x0 + 1, z0, seed);
    real v01 = hf_cell_hash(x0, z0 + 1, seed), v11 = hf_cell_hash(x0 + 1, z0 + 1, seed);
    real a = v00 + (v10 - v00) * tx, b = v01 + (v11 - v01) * tx;
    return a + (b - a) * tz;
}

static real hf_fbm(real x, real z, real freq, int octaves, int seed) {
    real fx = x * freq, fz = z * freq, amp = R(0.5), sum = 0, nrmz = 0;
    for (int o = 0; o < octaves; o++) {
        sum += amp * hf_noise(fx, fz, seed + o * 131);
        nrmz += amp;
        amp *= R(0.5);
        fx *= 2; fz *= 2;
    }
    return sum / nrmz;
}

/* grid (extension): gw x gh FP32 heights in [0, 1], bilinear over the
 * footprint, scaled by height; replaces the procedural / 8-bit height. */
typedef struct { const float* h; int w, hgt; } Grid;

static real hf_eval(const HeightField* hf, const unsigned char* img, real x, real z, Grid g) {
    real lx = (x - hf->center.x) / hf->size_x + R(0.5);
    real lz = (z - hf->center.z) / hf->size_z + R(0.5);
    if (lx < 0 || lx > 1 || lz < 0 || lz > 1) return 0;
    if (g.h) {
        real fu = lx * (real)(g.w - 1), fvv = lz * (real)(g.hgt - 1);
        int u0 = (int)fu, v0 = (int)fvv;
        int u1 = u0 < g.w - 1 ? u0 + 1 : u0, v1 = v0 < g.hgt - 1 ? v0 + 1 : v0;
        real tx = fu - (real)u0, ty = fvv - (real)v0;
#define GV(u, v) ((real)g.h[(size_t)(v) * g.w + (u)])
        real hh = GV(u0, v0) * (1 - tx) * (1 - ty) + GV(u1, v0) * tx * (1 - ty) + GV(u0, v1) * (1 - tx) * ty +
                  GV(u1, v1) * tx * ty;
#undef GV
        return hh * hf->height;
    }
    if (img) {
        if (hf->img_w < 1 || hf->img_h < 1) return 0;
        real fu = lx * (real)(hf->img_w - 1), fvv = lz * (real)(hf->img_h - 1);
        int u0 = (int)fu, v0 = (int)fvv;
        int u1 = u0 < hf->img_w - 1 ? u0 + 1 : u0, v1 = v0 < hf->img_h - 1 ? v0 + 1 : v0;
        real tx = fu - (real)u0, ty = fvv - (real)v0;
#define PX(u, v) ((real)img[(v) * hf->img_w + (u)] / R(255))
        real hh = PX(u0, v0) * (1 - tx) * (1 - ty) + PX(u1, v0) * tx * (1 - ty) +
                  PX(u0, v1) * (1 - tx) * ty + PX(u1, v1) * tx * ty;
#undef PX
        return hh * hf->height;
    }
    real t = hf_fbm(lx, lz, hf->freq, hf->octaves, hf->seed);
    real detail = hf_noise(lx * R(7), lz * R(7), hf->seed + 7777) * R(0.06);
    t = rfmin(t + detail - R(0.03), 1);
    return t * hf->height;
}

static int hf_hit(const Ray* r, const HeightField* hf, const unsigned char* img, Hit* h, Grid g) {
    V lo = v3(R(hf->center.x) - R(0.5) * hf->size_x, hf->center.y, R(hf->center.z) - R(0.5) * hf->size_z);
    V hi = v3(R(hf->center.x) + R(0.5) * hf->size_x, R(hf->center.y) + hf->height, R(hf->center.z) + R(0.5) * hf->size_z);
    real ix = R(1) / r->d.x, iy = R(1) / r->d.y, iz = R(1) / r->d.z;
    real tx0 = (lo.x - r->o.x) * ix, tx1 = (hi.x - r->o.x) * ix;
    real ty0 = (lo.y - r->o.y) * iy, ty1 = (hi.y - r->o.y) * iy;
    real tz0 = (lo.z - r->o.z) * iz, tz1 = (hi.z - r->o.z) * iz;
    if (tx0 > tx1) { real t = tx0; tx0 = tx1; tx1 = t; }
    if (ty0 > ty1) { real t = ty0; ty0 = ty1; ty1 = t; }
    if (tz0 > tz1) { real t = tz0; tz0 = tz1; tz1 = t; }
    real t0 = rfmax(rfmax(tx0, ty0), tz0), t1 = rfmin(rfmin(tx1, ty1), tz1);
    if (t1 < r->tmin || t0 > r->tmax || t1 < t0) return 0;
    t0 = rfmax(t0, r->tmin);
    t1 = rfmin(t1, r->tmax);
    real diag = sqrt(R(hf->size_x) * hf->size_x + R(hf->size_z) * hf->size_z);
    real step = rfmax(diag / R(64), R(1e-4));
    real t = t0;
    int inside = 0;
    for (int i = 0; i < 256; i++) {
        V p = add(r->o, mul(r->d, t));
        real hg = hf_eval(hf, img, p.x, p.z, g) + hf->center.y;
        int iyy = p.y <= hg;
        if (iyy != inside) {
            real a = t - step, b = t;
            if (a < t0) a = t0;
            for (int k = 0; k < 10; k++) {
                real mid = R(0.5) * (a + b);
                V pm = add(r->o, mul(r->d, mid));
                real hm = hf_eval(hf, img, pm.x, pm.z, g) + hf->center.y;
                if ((pm.y <= hm) == iyy) b = mid; else a = mid;
            }
            real tt = R(0.5) * (a + b);
            V P = add(r->o, mul(r->d, tt));
            if (tt >= r->tmin && tt <= r->tmax) {
                h->t = tt;
                h->p = P;
                real e = rfmax(hf->size_x, hf->size_z) / R(256);
                real hxp = hf_eval(hf, img, P.x + e, P.z, g), hxm = hf_eval(hf, img, P.x - e, P.z, g);
                real hzp = hf_eval(hf, img, P.x, P.z + e, g), hzm = hf_eval(hf, img, P.x, P.z - e, g);
                h->n = nrm(v3(-(hxp - hxm) / (R(2) * e), 1, -(hzp - hzm) / (R(2) * e)));
                h->tan = v3(1, 0, 0);
                h->u = P.x; h->v = P.z;
                if (dot(h->n, r->d) > 0) h->n = neg(h->n);
                return 1;
            }
            break;
        }
        inside = iyy;
        t += step;
        if (t > t1) break;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* integrator/csg.h:22-186 -- interval CSG, 8 intervals per node        */
/* ------------------------------------------------------------------ */
/* ------------------------------------------------------------------ */
/* Extension: exact cubic-Bezier lathes and prisms (no counterpart in the */
/* reference, which tessellates Bezier profiles on the host,             */
/* api/scene_io.cpp:86-102, 791-819).  Independent of the library's      */
/* Bernstein root isolation: each span's polynomial is evaluated directly */
/* at 4096 points and every sign change bisected to the last bit, in      */
/* double whatever the build's precision.                                 */
/* ------------------------------------------------------------------ */
static double bz(const double* c, double u) {
    double v = 1.0 - u;
    return v * v * v * c[0] + 3.0 * v * v * u * c[1] + 3.0 * v * u * u * c[2] + u * u * u * c[3];
}
static double bzd(const double* c, double u) {
    double v = 1.0 - u;
    return 3.0 * (v * v * (c[1] - c[0]) + 2.0 * v * u * (c[2] - c[1]) + u * u * (c[3] - c[2]));
}
static void span_ab(const OracleScene* S, int k, double a[4], double b[4]) {
    const double* q = S->spans + 8 * (size_t)k;
    for (int i = 0; i < 4; i++) { a[i] = q[2 * i]; b[i] = q[2 * i + 1]; }
}

/* Sign-change roots in [0, 1) of f (sampled at n points, bisected). */
typedef double (*ufun)(const void* ctx, double u);
static int sampled_roots(ufun f, const void* ctx, int n, double* roots, int max_roots) {
    int nr = 0;
    double u0 = 0.0, f0 = f(ctx, 0.0);
    for (int i = 1; i <= n && nr < max_roots; i++) {
        double u1 = (double)i / n, f1 = f(ctx, u1);
        if (f0 == 0.0) { roots[nr++] = u0; }
        else if ((f0 < 0.0) != (f1 < 0.0) && f1 != 0.0) {
            double lo = u0, hi = u1, flo = f0;
            for (int k = 0; k < 80 && hi - lo > 0.0; k++) {
                double mid = 0.5 * (lo + hi);
                if (mid <= lo || mid >= hi) break;
                double fm = f(ctx, mid);
                if ((fm < 0.0) == (flo < 0.0)) { lo = mid; flo = fm; } else hi = mid;
            }
            roots[nr++] = 0.5 * (lo + hi);
        }
        u0 = u1; f0 = f1;
    }
    return nr;
}

typedef struct { double Y[4], Rr[4], A, B, C, dy; } LatheCtx;
static double lathe_f(const void* c, double u) {
    const LatheCtx* L = (const LatheCtx*)c;
    double y = bz(L->Y, u), rr = bz(L->Rr, u);
    return L->A * y * y + L->B * L->dy * y + L->C * L->dy * L->dy - L->dy * L->dy * rr * rr;
}
static double cubic_f(const void* c, double u) { return bz((const double*)c, u); }

static int lathe_exact_hit(const OracleScene* S, const Ray* r, int i, Hit* h) {
    const int first = S->lathe_run[2 * i], cnt = S->lathe_run[2 * i + 1];
    double ox = r->o.x, oy = r->o.y, oz = r->o.z, dx = r->d.x, dy = r->d.y, dz = r->d.z;
    double A = dx * dx + dz * dz, B = 2 * (ox * dx + oz * dz), C = ox * ox + oz * oz;
    int flat = dy * dy <= 1e-24 * (A + dy * dy);
    double best = r->tmax, bu = 0;
    int bk = -1;
    for (int k = first; k < first + cnt; k++) {
        LatheCtx L;
        span_ab(S, k, L.Y, L.Rr);
        for (int j = 0; j < 4; j++) L.Y[j] -= oy;
        double roots[64];
        if (!flat) {
            L.A = A; L.B = B; L.C = C; L.dy = dy;
            int n = sampled_roots(lathe_f, &L, 4096, roots, 64);
            for (int j = 0; j < n; j++) {
                double sv = bz(L.Y, roots[j]) / dy;
                if (sv >= r->tmin && sv < best) { best = sv; bu = roots[j]; bk = k; }
            }
        } else {
            int n = sampled_roots(cubic_f, L.Y, 4096, roots, 64);
            for (int j = 0; j < n; j++) {
                double rad = bz(L.Rr, roots[j]), disc = B * B - 4 * A * (C - rad * rad);
                if (disc < 0 || A <= 0) continue;
                double sq = sqrt(disc), s0 = (-B - sq) / (2 * A), s1 = (-B + sq) / (2 * A);
                if (s0 >= r->tmin && s0 < best) { best = s0; bu = roots[j]; bk = k; }
                else if (s1 >= r->tmin && s1 < best) { best = s1; bu = roots[j]; bk = k; }
            }
        }
    }
    if (bk < 0 || best > r->tmax) return 0;
    double Y[4], Rr[4];
    span_ab(S, bk, Y, Rr);
    h->t = (real)best;
    h->p = add(r->o, mul(r->d, h->t));
    double yd = bzd(Y, bu), rd = bzd(Rr, bu), rv = bz(Rr, bu);
    double rho = sqrt((double)h->p.x * h->p.x + (double)h->p.z * h->p.z);
    double cx = rho > 0 ? h->p.x / rho : 1, cz = rho > 0 ? h->p.z / rho : 0;
    h->n = nrm(v3((real)(yd * cx), (real)(-rd * (rv < 0 ? -1 : 1)), (real)(yd * cz)));
    if (dot(h->n, r->d) > 0) h->n = neg(h->n);
    h->tan = v3(0, 1, 0);
    h->u = 0; h->v = 0;
    h->mat = S->lathes[i].material_id;
    return 1;
}

static void lathe_exact_box(const OracleScene* S, int i, V* lo, V* hi) {
    const int first = S->lathe_run[2 * i], cnt = S->lathe_run[2 * i + 1];
    double R = 0, y0 = 1e300, y1 = -1e300;
    for (int k = first; k < first + cnt; k++)
        for (int j = 0; j < 4; j++) {
            const double* q = S->spans + 8 * (size_t)k + 2 * j;
            y0 = fmin(y0, q[0]); y1 = fmax(y1, q[0]); R = fmax(R, fabs(q[1]));
        }
    *lo = v3((real)-R, (real)y0, (real)-R);
    *hi = v3((real)R, (real)y1, (real)R);
    widen(lo, hi);
}

/* even-odd: crossings of z = pz at x > px, u in [0, 1) per span */
static int bez_inside(const OracleScene* S, int first, int cnt, double px, double pz) {
    int inside = 0;
    for (int k = first; k < first + cnt; k++) {
        double X[4], Z[4], roots[64];
        span_ab(S, k, X, Z);
        for (int j = 0; j < 4; j++) Z[j] -= pz;
        int n = sampled_roots(cubic_f, Z, 4096, roots, 64);
        for (int j = 0; j < n; j++)
            if (roots[j] < 1.0 && bz(X, roots[j]) > px) inside = !inside;
    }
    return inside;
}

typedef struct { double X[4], Z[4], ox, oz, dx, dz; } WallCtx;
static double wall_f(const void* c, double u) {
    const WallCtx* w = (const WallCtx*)c;
    return (bz(w->X, u) - w->ox) * w->dz - (bz(w->Z, u) - w->oz) * w->dx;
}

static int prism_exact_hit(const OracleScene* S, const Ray* r, int i, Hit* h) {
    const Prism* p = &S->prisms[i];
    const int first = S->prism_run[2 * i], cnt = S->prism_run[2 * i + 1];
    double y0 = (double)p->center.y + p->y_min, y1 = (double)p->center.y + p->y_max;
    double best = r->tmax, bu = 0, capn = 0;
    int kind = -1, bk = -1;
    for (int face = 0; face < 2; face++) {
        double yf = face == 0 ? y0 : y1;
        double t = (yf - r->o.y) / r->d.y;
        if (!(t >= r->tmin && t <= r->tmax) || t >= best) continue;
        double Px = r->o.x + t * r->d.x, Pz = r->o.z + t * r->d.z;
        if (!bez_inside(S, first, cnt, Px - p->center.x, Pz - p->center.z)) continue;
        best = t; kind = 0; capn = face == 0 ? -1 : 1;
    }
    WallCtx w;
    w.ox = (double)r->o.x - p->center.x; w.oz = (double)r->o.z - p->center.z; w.dx = r->d.x; w.dz = r->d.z;
    double a2 = w.dx * w.dx + w.dz * w.dz;
    if (a2 > 1e-24 * (a2 + (double)r->d.y * r->d.y)) {
        for (int k = first; k < first + cnt; k++) {
            double roots[64];
            span_ab(S, k, w.X, w.Z);
            int n = sampled_roots(wall_f, &w, 4096, roots, 64);
            for (int j = 0; j < n; j++) {
                double sv = ((bz(w.X, roots[j]) - w.ox) * w.dx + (bz(w.Z, roots[j]) - w.oz) * w.dz) / a2;
                if (!(sv >= r->tmin && sv < best)) continue;
                double yy = r->o.y + sv * r->d.y;
                if (yy < y0 - 1e-6 * fabs(y0) - 1e-7 || yy > y1 + 1e-6 * fabs(y1) + 1e-7) continue;
                best = sv; kind = 1; bu = roots[j]; bk = k;
            }
        }
    }
    if (kind < 0) return 0;
    h->t = (real)best;
    h->p = add(r->o, mul(r->d, h->t));
    if (kind == 0) { h->n = v3(0, (real)capn, 0); h->tan = v3(1, 0, 0); }
    else {
        double X[4], Z[4];
        span_ab(S, bk, X, Z);
        h->n = nrm(v3((real)bzd(Z, bu), 0, (real)-bzd(X, bu)));
        h->tan = v3(0, 1, 0);
    }
    if (dot(h->n, r->d) > 0) h->n = neg(h->n);
    h->u = 0; h->v = 0;
    h->mat = p->material_id;
    return 1;
}

static void prism_exact_box(const OracleScene* S, int i, V* lo, V* hi) {
    const Prism* p = &S->prisms[i];
    const int first = S->prism_run[2 * i], cnt = S->prism_run[2 * i + 1];
    double x0 = 1e300, x1 = -1e300, z0 = 1e300, z1 = -1e300;
    for (int k = first; k < first + cnt; k++)
        for (int j = 0; j < 4; j++) {
            const double* q = S->spans + 8 * (size_t)k + 2 * j;
            x0 = fmin(x0, q[0]); x1 = fmax(x1, q[0]); z0 = fmin(z0, q[1]); z1 = fmax(z1, q[1]);
        }
    *lo = v3((real)(p->center.x + x0), (real)(p->center.y + p->y_min), (real)(p->center.z + z0));
    *hi = v3((real)(p->center.x + x1), (real)(p->center.y + p->y_max), (real)(p->center.z + z1));
    widen(lo, hi);
}

/* Extension CSG leaves: axis-aligned box and capped cone, one interval each
 * (both convex), clipped to [t0, t1]. */
static int box_iv(const Ray* r, const SheenCsgBox* b, real t0, real t1, real* te, real* tx) {
    real lo[3] = {b->lo.x, b->lo.y, b->lo.z}, hi[3] = {b->hi.x, b->hi.y, b->hi.z};
    real o[3] = {r->o.x, r->o.y, r->o.z}, d[3] = {r->d.x, r->d.y, r->d.z};
    real tn = R(-1e300), tf = R(1e300);
    for (int a = 0; a < 3; a++) {
        if (d[a] == 0) { if (o[a] < lo[a] || o[a] > hi[a]) return 0; continue; }
        real ta = (lo[a] - o[a]) / d[a], tb = (hi[a] - o[a]) / d[a];
        if (ta > tb) { real t = ta; ta = tb; tb = t; }
        tn = rfmax(tn, ta); tf = rfmin(tf, tb);
    }
    if (!(tn <= tf) || tf < t0 || tn > t1) return 0;
    *te = rfmax(tn, t0); *tx = rfmin(tf, t1);
    return *te <= *tx;
}

static int cone_iv(const Ray* r, const SheenCsgCone* c, real t0, real t1, real* te, real* tx) {
    V p0 = v3(c->p0.x, c->p0.y, c->p0.z), ax = sub(v3(c->p1.x, c->p1.y, c->p1.z), p0);
    real L = sqrt(dot(ax, ax));
    if (!(L > 0)) return 0;
    V a = mul(ax, 1 / L), oc = sub(r->o, p0);
    real ho = dot(oc, a), hd = dot(r->d, a);
    real sa, sb;
    if (hd != 0) { sa = -ho / hd; sb = (L - ho) / hd; if (sa > sb) { real t = sa; sa = sb; sb = t; } }
    else { if (ho < 0 || ho > L) return 0; sa = R(-1e300); sb = R(1e300); }
    real k = (c->r1 - c->r0) / L, rb = c->r0 + k * ho, rk = k * hd;
    real A = dot(r->d, r->d) - hd * hd - rk * rk;
    real B = 2 * (dot(oc, r->d) - ho * hd - rb * rk);
    real Cc = dot(oc, oc) - ho * ho - rb * rb;
    real lo = sa, hi = sb;
    if (fabs(A) <= 1e-12 * (fabs(B) + fabs(Cc) + 1e-300)) {
        if (B == 0) { if (Cc > 0) return 0; }
        else if (B > 0) hi = rfmin(hi, -Cc / B);
        else lo = rfmax(lo, -Cc / B);
    } else {
        real disc = B * B - 4 * A * Cc;
        if (A > 0) {
            if (disc < 0) return 0;
            real sq = sqrt(disc);
            lo = rfmax(lo, (-B - sq) / (2 * A)); hi = rfmin(hi, (-B + sq) / (2 * A));
        } else if (disc >= 0) {
            real sq = sqrt(disc), ra = (-B + sq) / (2 * A), rbb = (-B - sq) / (2 * A);
            real l1 = lo, h1 = rfmin(hi, ra), l2 = rfmax(lo, rbb), h2 = hi;
            int ok1 = l1 <= h1, ok2 = l2 <= h2;
            if (ok1 && ok2) {
                real m1 = R(0.5) * (rfmax(l1, R(-1e30)) + rfmin(h1, R(1e30)));
                if (c->r0 + k * (ho + m1 * hd) >= 0) hi = h1; else lo = l2;
            } else if (ok1) hi = h1;
            else if (ok2) lo = l2;
            else return 0;
        }
    }
    if (!(lo <= hi) || hi < t0 || lo > t1) return 0;
    *te = rfmax(lo, t0); *tx = rfmin(hi, t1);
    return *te <= *tx;
}

static V csg_ext_normal(const OracleScene* S, int kind, int leaf, V p) {
    if (kind == 2) {
        const SheenCsgBox* b = &S->csg_boxes[leaf];
        real c[3] = {R(0.5) * (b->lo.x + b->hi.x), R(0.5) * (b->lo.y + b->hi.y), R(0.5) * (b->lo.z + b->hi.z)};
        real e[3] = {R(0.5) * (b->hi.x - b->lo.x), R(0.5) * (b->hi.y - b->lo.y), R(0.5) * (b->hi.z - b->lo.z)};
        real q[3] = {p.x - c[0], p.y - c[1], p.z - c[2]};
        int best = 0; real bd = R(1e300);
        for (int a = 0; a < 3; a++) {
            real dd = fabs(e[a] - fabs(q[a])) / rfmax(e[a], R(1e-30));
            if (dd < bd) { bd = dd; best = a; }
        }
        real n[3] = {0, 0, 0};
        n[best] = q[best] >= 0 ? 1 : -1;
        return v3(n[0], n[1], n[2]);
    }
    const SheenCsgCone* c = &S->csg_cones[leaf];
    V p0 = v3(c->p0.x, c->p0.y, c->p0.z), ax = sub(v3(c->p1.x, c->p1.y, c->p1.z), p0);
    real L = sqrt(dot(ax, ax));
    V a = mul(ax, 1 / L);
    real hh = dot(sub(p, p0), a);
    V w = sub(sub(p, p0), mul(a, hh));
    real k = (c->r1 - c->r0) / L, rad = c->r0 + k * hh, wl = sqrt(dot(w, w));
    real side = fabs(wl - rad) / rfmax(rfmax(c->r0, c->r1), R(1e-30));
    real cap0 = fabs(hh) / L, cap1 = fabs(hh - L) / L;
    if (cap0 < side && cap0 <= cap1) return neg(a);
    if (cap1 < side) return a;
    return wl > 0 ? sub(w, mul(a, rad * k)) : a;
}

typedef struct { real te, tx; int mat, leaf, kind; } Iv;

static void csg_merge(const Iv* A, int nA, const Iv* B, int nB, int op, Iv* out, int* nOut) {
    int n = 0;
    *nOut = 0;
    if (op == 0) {
        Iv tmp[16];
        for (int i = 0; i < nA && n < 16; i++) tmp[n++] = A[i];
        for (int i = 0; i < nB && n < 16; i++) tmp[n++] = B[i];
        for (int i = 1; i < n; i++) {
            Iv key = tmp[i];
            int j = i - 1;
            while (j >= 0 && tmp[j].te > key.te) { tmp[j + 1] = tmp[j]; j--; }
            tmp[j + 1] = key;
        }
        for (int i = 0; i < n && *nOut < 8; i++) {
            if (*nOut == 0 || tmp[i].te > out[*nOut - 1].tx) out[(*nOut)++] = tmp[i];
            else if (tmp[i].tx > out[*nOut - 1].tx) out[*nOut - 1].tx = tmp[i].tx;
        }
    } else if (op == 1) {
        for (int i = 0; i < nA; i++)
            for (int j = 0; j < nB; j++) {
                real t0 = rfmax(A[i].te, B[j].te), t1 = rfmin(A[i].tx, B[j].tx);
                if (t0 < t1 && *nOut < 8) { out[*nOut] = A[i]; out[*nOut].te = t0; out[*nOut].tx = t1; (*nOut)++; }
            }
    } else if (op == 2) {
        for (int i = 0; i < nA; i++) {
            real cur = A[i].te;
            for (int j = 0; j < nB; j++) {
                real b0 = B[j].te, b1 = B[j].tx;
                if (b1 <= cur) continue;
                if (b0 >= A[i].tx) break;
                if (b0 > cur && *nOut < 8) { out[*nOut] = A[i]; out[*nOut].te = cur; out[*nOut].tx = b0; (*nOut)++; }
                cur = rfmax(cur, b1);
                if (cur >= A[i].tx) break;
            }
            if (cur < A[i].tx && *nOut < 8) { out[*nOut] = A[i]; out[*nOut].te = cur; out[*nOut].tx = A[i].tx; (*nOut)++; }
        }
    }
}

static void csg_collect(const OracleScene* S, int node, const Ray* r, real t0, real t1, Iv* out, int* nOut) {
    const CSGNode* n = &S->csg[node];
    *nOut = 0;
    if (n->leaf_kind >= 0) {
        Iv iv;
        int ok = 0;
        if (n->leaf_kind == 0) {
            const Object* o = &S->objects[n->leaf_index];
            ok = sphere_iv(r, fv(o->param1), o->param2, t0, t1, &iv.te, &iv.tx);
            iv.mat = o->material_id;
        } else if (n->leaf_kind == 1) {
            const Superellipsoid* se = &S->ses[n->leaf_index];
            ok = se_intervals(r, se, t0, t1, &iv.te, &iv.tx, S->se_n2 ? S->se_n2[n->leaf_index] : 0);
            iv.mat = se->material_id;
        } else if (n->leaf_kind == 2 && S->csg_boxes) {
            ok = box_iv(r, &S->csg_boxes[n->leaf_index], t0, t1, &iv.te, &iv.tx);
            iv.mat = S->csg_boxes[n->leaf_index].material_id;
        } else if (n->leaf_kind == 3 && S->csg_cones) {
            ok = cone_iv(r, &S->csg_cones[n->leaf_index], t0, t1, &iv.te, &iv.tx);
            iv.mat = S->csg_cones[n->leaf_index].material_id;
        }
        if (ok) { iv.leaf = n->leaf_index; iv.kind = n->leaf_kind; out[(*nOut)++] = iv; }
        return;
    }
    Iv A[8], B[8];
    int nA = 0, nB = 0;
    if (n->left >= 0) csg_collect(S, n->left, r, t0, t1, A, &nA);
    if (n->right >= 0) csg_collect(S, n->right, r, t0, t1, B, &nB);
    csg_merge(A, nA, B, nB, n->op, out, nOut);
}

static int csg_tree_hit(const OracleScene* S, int root, const Ray* r, Hit* h) {
    Iv iv[8];
    int cnt = 0;
    real t0 = r->tmin, t1 = r->tmax;
    csg_collect(S, root, r, t0, t1, iv, &cnt);
    real best = R(1e30);
    int bi = -1;
    for (int i = 0; i < cnt; i++)
        if (iv[i].te < best && iv[i].tx > t0) { best = iv[i].te; bi = i; }
    if (bi < 0) return 0;
    real t = rfmax(iv[bi].te, t0);
    if (t < t0 || t > t1) return 0;
    h->t = t;
    h->mat = iv[bi].mat;
    h->p = add(r->o, mul(r->d, t));
    if (iv[bi].kind == 0) {
        h->n = nrm(sub(h->p, fv(S->objects[iv[bi].leaf].param1)));
        h->tan = v3(0, 0, 0);
    } else if (iv[bi].kind == 1) {
        h->n = nrm(se_grad(&S->ses[iv[bi].leaf], h->p, S->se_n2 ? S->se_n2[iv[bi].leaf] : 0));
        h->tan = v3(1, 0, 0);
    } else if (iv[bi].kind == 2 || iv[bi].kind == 3) {
        h->n = nrm(csg_ext_normal(S, iv[bi].kind, iv[bi].leaf, h->p));
        h->tan = v3(1, 0, 0);
    } else {
        h->n = v3(0, 1, 0);
        h->tan = v3(1, 0, 0);
    }
    h->u = h->p.x; h->v = h->p.y;
    if (dot(h->n, r->d) > 0) h->n = neg(h->n);
    h->obj = 0;
    h->prim = bi;
    return 1;
}

/* The CSG category: the scene's tree, then the extension trees in index
 * order; a later tree replaces the hit only when strictly closer. */
static int csg_hit(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0;
    if (S->s.csg_root >= 0 && csg_tree_hit(S, S->s.csg_root, r, h)) any = 1;
    for (int k = 0; k < S->ncsg_roots; k++) {
        Hit t;
        if (csg_tree_hit(S, S->csg_roots[k], r, &t) && (!any || t.t < h->t)) { *h = t; any = 1; }
    }
    return any;
}

/* ------------------------------------------------------------------ */
/* per-category closest hit (bvh.h:605-922 semantics, linear scan)       */
/* ------------------------------------------------------------------ */
static int cat_spheres(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_objects; i++) {
        const Object* o = &S->objects[i];
        if (o->type != 0) continue;
        V c = fv(o->param1);
        V lo = v3(c.x - o->param2, c.y - o->param2, c.z - o->param2);
        V hi = v3(c.x + o->param2, c.y + o->param2, c.z + o->param2);
        lo = v3(o->param1.x - o->param2, o->param1.y - o->param2, o->param1.z - o->param2);
        hi = v3(o->param1.x + o->param2, o->param1.y + o->param2, o->param1.z + o->param2);
        widen(&lo, &hi);
        if (!slab(r, lo, hi)) continue;
        if (sphere_hit(r, c, o->param2, &tmp) && tmp.t < best) {
            *h = tmp; h->mat = o->material_id; h->obj = i; h->cat = CAT_SPHERE; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static int cat_strands(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_sweep_strands; i++) {
        V lo, hi;
        strand_box(S, i, &lo, &hi);
        if (!slab(r, lo, hi)) continue;
        if (sweep_hit(r, &S->strands[i], S->sweep_points, &tmp) && tmp.t < best) {
            *h = tmp; h->obj = -(i + 1); h->cat = CAT_STRAND; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static void tri_box(const Triangle* t, V* lo, V* hi) {
    *lo = v3(fminf(t->v0.x, fminf(t->v1.x, t->v2.x)), fminf(t->v0.y, fminf(t->v1.y, t->v2.y)),
             fminf(t->v0.z, fminf(t->v1.z, t->v2.z)));
    *hi = v3(fmaxf(t->v0.x, fmaxf(t->v1.x, t->v2.x)), fmaxf(t->v0.y, fmaxf(t->v1.y, t->v2.y)),
             fmaxf(t->v0.z, fmaxf(t->v1.z, t->v2.z)));
    widen(lo, hi);
}

static int cat_mesh(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_triangles; i++) {
        V lo, hi;
        tri_box(&S->tris[i], &lo, &hi);
        if (!slab(r, lo, hi)) continue;
        if (tri_hit(r, &S->tris[i], &tmp) && tmp.t < best) {
            *h = tmp; h->mat = S->tris[i].material_id; h->obj = -(i + 1); h->cat = CAT_MESH; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static int cat_hf(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_heightfields; i++) {
        const HeightField* hf = &S->hfs[i];
        V lo = v3(hf->center.x - 0.5f * hf->size_x, hf->center.y, hf->center.z - 0.5f * hf->size_z);
        V hi = v3(hf->center.x + 0.5f * hf->size_x, hf->center.y + hf->height, hf->center.z + 0.5f * hf->size_z);
        widen(&lo, &hi);
        if (!slab(r, lo, hi)) continue;
        Grid g = {NULL, 0, 0};
        if (S->hfg && S->hfg[3 * i] >= 0) { g.h = S->hf_heights + S->hfg[3 * i]; g.w = S->hfg[3 * i + 1]; g.hgt = S->hfg[3 * i + 2]; }
        if (hf_hit(r, hf, S->hf_img[i], &tmp, g) && tmp.t < best) {
            *h = tmp; h->mat = hf->material_id; h->obj = -(i + 1); h->cat = CAT_HF; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static int cat_se(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_superellipsoids; i++) {
        const Superellipsoid* se = &S->ses[i];
        V lo = v3(se->center.x - se->a, se->center.y - se->b, se->center.z - se->c);
        V hi = v3(se->center.x + se->a, se->center.y + se->b, se->center.z + se->c);
        widen(&lo, &hi);
        if (!slab(r, lo, hi)) continue;
        if (se_hit(r, se, &tmp, S->se_n2 ? S->se_n2[i] : 0) && tmp.t < best) {
            *h = tmp; h->mat = se->material_id; h->obj = -(i + 1); h->cat = CAT_SE; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static int cat_lathe(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_lathes; i++) {
        V lo, hi;
        const int exact = S->lathe_run && S->lathe_run[2 * i + 1] > 0;
        if (exact) lathe_exact_box(S, i, &lo, &hi);
        else lathe_box(&S->lathes[i], S->lpts, &lo, &hi);
        if (!slab(r, lo, hi)) continue;
        if ((exact ? lathe_exact_hit(S, r, i, &tmp) : lathe_hit(r, &S->lathes[i], S->lpts, &tmp)) && tmp.t < best) {
            *h = tmp; h->obj = -(i + 1); h->cat = CAT_LATHE; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static int cat_prism(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_prisms; i++) {
        V lo, hi;
        const int exact = S->prism_run && S->prism_run[2 * i + 1] > 0;
        if (exact) prism_exact_box(S, i, &lo, &hi);
        else prism_box(&S->prisms[i], S->ppts, &lo, &hi);
        if (!slab(r, lo, hi)) continue;
        if ((exact ? prism_exact_hit(S, r, i, &tmp) : prism_hit(r, &S->prisms[i], S->ppts, &tmp)) && tmp.t < best) {
            *h = tmp; h->obj = -(i + 1); h->cat = CAT_PRISM; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

static int cat_planes(const OracleScene* S, const Ray* r, Hit* h) {
    int any = 0; real best = r->tmax; Hit tmp;
    for (int i = 0; i < S->s.num_planes; i++) {
        const Plane* p = &S->planes[i];
        if (plane_hit(r, fv(p->normal), p->d, &tmp) && tmp.t < best) {
            *h = tmp; h->mat = p->material_id; h->obj = -1 - i; h->cat = CAT_PLANE; h->prim = i;
            best = tmp.t; any = 1;
        }
    }
    return any;
}

/* Scene queries issued by this thread (every scene_hit / scene_hit_opaque
 * call): the ray count of the throughput metric -- primary, each glass pass
 * of a shadow ray, every mirror / refraction segment, beam and medium shadow
 * rays. */
static _Thread_local unsigned long long tl_queries;

/* integrator/raycast.h:14-70 -- closest hit over the categories in order */
static int scene_hit(const OracleScene* S, const Ray* r, Hit* rec) {
    tl_queries++;
    real best = r->tmax;
    int hit = 0;
    Hit t;
#define CAT(call) if ((call) && t.t < best) { best = t.t; *rec = t; hit = 1; }
    CAT(cat_spheres(S, r, &t))
    CAT(cat_strands(S, r, &t))
    CAT(cat_mesh(S, r, &t))
    CAT(cat_hf(S, r, &t))
    CAT(cat_se(S, r, &t))
    CAT(cat_lathe(S, r, &t))
    CAT(cat_prism(S, r, &t))
    if (S->s.csg_root >= 0 || S->ncsg_roots > 0) { CAT(csg_hit(S, r, &t) && ((t.cat = CAT_CSG), 1)) }
    CAT(cat_planes(S, r, &t))
#undef CAT
    return hit;
}

/* integrator/raycast.h:74-97 -- QUIRK: the first category with any hit wins
 * (its closest hit), strands excluded */
static int scene_hit_opaque(const OracleScene* S, const Ray* r, Hit* rec) {
    tl_queries++;
    if (cat_spheres(S, r, rec)) return 1;
    if (cat_mesh(S, r, rec)) return 1;
    if (cat_hf(S, r, rec)) return 1;
    if (cat_se(S, r, rec)) return 1;
    if (cat_lathe(S, r, rec)) return 1;
    if (cat_prism(S, r, rec)) return 1;
    if ((S->s.csg_root >= 0 || S->ncsg_roots > 0) && csg_hit(S, r, rec)) { rec->cat = CAT_CSG; return 1; }
    return cat_planes(S, r, rec);
}

/* ------------------------------------------------------------------ */
/* integrator/shading.h:10-175 -- textures and BRDFs                   */
/* ------------------------------------------------------------------ */
static real tex_lod(const Tex* t, real uv_fp) { return (real)log2(rfmax(uv_fp * (real)t->w, 1)); }

static V tex_sample_lod(const Tex* t, real uu, real vv, real lod) {
    int level = (int)floor(lod + R(0.5));
    if (level < 0) level = 0;
    if (level >= t->mips) level = t->mips - 1;
    int w = t->w, h = t->h;
    size_t off = 0;
    for (int i = 0; i < level; i++) {
        off += (size_t)w * h * 3;
        w = w > 1 ? w / 2 : 1;
        h = h > 1 ? h / 2 : 1;
    }
    const unsigned char* base = t->px + off;
    real u = uu - floor(uu);
    real v = R(1) - (vv - floor(vv));
    real fx = u * (real)(w - 1), fy = v * (real)(h - 1);
    int x0 = (int)fx, y0 = (int)fy, x1 = (x0 + 1) % w, y1 = (y0 + 1) % h;
    real tx = fx - (real)x0, ty = fy - (real)y0;
#define AT(x, y) v3(base[((size_t)(y) * w + (x)) * 3] / R(255), base[((size_t)(y) * w + (x)) * 3 + 1] / R(255), \
                    base[((size_t)(y) * w + (x)) * 3 + 2] / R(255))
    V c00 = AT(x0, y0), c10 = AT(x1, y0), c01 = AT(x0, y1), c11 = AT(x1, y1);
#undef AT
    V a = add(mul(c00, 1 - tx), mul(c10, tx));
    V b = add(mul(c01, 1 - tx), mul(c11, tx));
    return add(mul(a, 1 - ty), mul(b, ty));
}

typedef struct { V p, n, tan, view; real u, v, uv_fp; } Shade;

static V albedo(const OracleScene* S, const Material* m, const Shade* in) {
    if (m->texture_id >= 0 && m->texture_id < S->ntex) {
        const Tex* t = &S->tex[m->texture_id];
        return tex_sample_lod(t, in->u, in->v, tex_lod(t, in->uv_fp));
    }
    return fv(m->diffuse_color);
}

static int has_mask(const OracleScene* S, const Material* m) { return m->mask_id >= 0 && m->mask_id < S->ntex; }

static real rough_to_shin(real r) {
    real rr = rfmax(r, R(0.02)), r2 = rr * rr;
    return rfmin(rfmax(R(2) / (r2 * r2) - R(2), 1), R(4096));
}

static real hit_transmission(const OracleScene* S, const Hit* h, const Material* m) {
    if (m->transmission <= 0) return 0;
    if (has_mask(S, m)) return m->transmission * tex_sample_lod(&S->tex[m->mask_id], h->u, h->v, 0).x;
    return m->transmission;
}

static real hit_ior(const OracleScene* S, const Hit* h, const Material* m) {
    if (has_mask(S, m)) return R(1) + tex_sample_lod(&S->tex[m->mask_id], h->u, h->v, 0).y;
    return m->ior;
}

static V shade_hair(const Material* m, const Shade* in, V L, V rad) {
    V T = in->tan, N = in->n, Vv = in->view;
    real tl = dot(T, L);
    real sin_tl = sqrt(rfmax(1 - tl * tl, 0));
    real back = rfmax(-tl, 0);
    real diffuse = sin_tl + m->hair_backlight * back * back;
    V res = mul(vmul(fv(m->diffuse_color), rad), diffuse * R(0.75));
    real wr = m->hair_spec_r, wt = m->hair_spec_t, er = m->hair_exp_r, et = m->hair_exp_t;
    if (wr <= 0 && wt <= 0) { wr = m->specular; er = m->shininess; }
    V H = nrm(add(L, Vv));
    if (wr > 0) {
        V Tr = nrm(add(T, mul(N, m->hair_shift)));
        real sr = dot(Tr, H);
        res = add(res, mul(rad, wr * rpow(sqrt(rfmax(1 - sr * sr, 0)), rfmax(er, 1))));
    }
    if (wt > 0) {
        V Tt = nrm(sub(T, mul(N, m->hair_shift)));
        real st = dot(Tt, H);
        res = add(res, mul(rad, wt * rpow(sqrt(rfmax(1 - st * st, 0)), rfmax(et, 1))));
    }
    return res;
}

static V shade_direct(const OracleScene* S, const Material* m, const Shade* in, V L, V rad, real shin) {
    if (m->anisotropy > 0) return shade_hair(m, in, L, rad);
    V base = albedo(S, m, in);
    real diff = rfmax(dot(in->n, L), 0);
    V res = mul(vmul(base, rad), diff);
    if (m->specular > 0 && diff > 0) {
        V hv = nrm(add(L, in->view));
        real sp = rpow(rfmax(dot(in->n, hv), 0), shin);
        res = add(res, mul(rad, m->specular * sp));
    }
    return res;
}

/* render_kernel.h:55-111 */
static int cell_hash(int ix, int iy, int iz, int num_cells) {
    uint32_t h = (uint32_t)ix * 73856093u ^ (uint32_t)iy * 19349663u ^ (uint32_t)iz * 83492791u;
    h ^= h >> 16; h *= 0x7feb352du;
    h ^= h >> 15; h *= 0x846ca68bu;
    h ^= h >> 16;
    return (int)(h & (uint32_t)(num_cells - 1));
}

static V photon_gather(const OracleScene* S, V p, V n, real radius, int max_samples) {
    V acc = v3(0, 0, 0);
    if (!S->nph || S->num_cells <= 0 || S->cell <= 0) return acc;
    real c = S->cell;
    int x0 = (int)floor((p.x - radius) / c), x1 = (int)floor((p.x + radius) / c);
    int y0 = (int)floor((p.y - radius) / c), y1 = (int)floor((p.y + radius) / c);
    int z0 = (int)floor((p.z - radius) / c), z1 = (int)floor((p.z + radius) / c);
    real r2 = radius * radius;
    int cells[8], nc = 0, taken = 0;
    for (int iz = z0; iz <= z1; iz++)
        for (int iy = y0; iy <= y1; iy++)
            for (int ix = x0; ix <= x1; ix++) {
                int hc = cell_hash(ix, iy, iz, S->num_cells), seen = 0;
                for (int q = 0; q < nc; q++) if (cells[q] == hc) { seen = 1; break; }
                if (!seen && nc < 8) cells[nc++] = hc;
            }
    for (int q = 0; q < nc && taken < max_samples; q++) {
        int st = S->cell_start[cells[q]], cnt = S->cell_count[cells[q]];
        for (int k = 0; k < cnt && taken < max_samples; k++) {
            V d = sub(fv(S->ph_pos[st + k]), p);
            if (dot(d, d) > r2) continue;
            if (dot(fv(S->ph_nrm[st + k]), n) < R(0.1)) continue;
            acc = add(acc, fv(S->ph_flux[st + k]));
            taken++;
        }
    }
    return acc;
}

/* Extension (no reference counterpart): the k nearest photons within rmax
 * facing n, found by a full sort of the candidates' squared distances (the
 * library uses a heap); the estimate's radius is the k-th distance, or rmax
 * when fewer are found.  Returns their flux sum, *r2 the radius squared. */
static int cmp_real(const void* a, const void* b) {
    const real x = *(const real*)a, y = *(const real*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

static V photon_knn(const OracleScene* S, V p, V n, real rmax, int k, real* r2_out) {
    V acc = v3(0, 0, 0);
    *r2_out = rmax * rmax;
    if (!S->nph || S->num_cells <= 0 || S->cell <= 0 || k <= 0) return acc;
    real c = S->cell;
    int x0 = (int)floor((p.x - rmax) / c), x1 = (int)floor((p.x + rmax) / c);
    int y0 = (int)floor((p.y - rmax) / c), y1 = (int)floor((p.y + rmax) / c);
    int z0 = (int)floor((p.z - rmax) / c), z1 = (int)floor((p.z + rmax) / c);
    int cells[27], nc = 0;
    for (int iz = z0; iz <= z1; iz++)
        for (int iy = y0; iy <= y1; iy++)
            for (int ix = x0; ix <= x1; ix++) {
                int hc = cell_hash(ix, iy, iz, S->num_cells), seen = 0;
                for (int q = 0; q < nc; q++) if (cells[q] == hc) { seen = 1; break; }
                if (!seen && nc < 27) cells[nc++] = hc;
            }
    real rmax2 = rmax * rmax;
    int total = 0;
    for (int q = 0; q < nc; q++) total += S->cell_count[cells[q]];
    real* d2s = (real*)malloc(sizeof(real) * (size_t)(total > 0 ? total : 1));
    int m = 0;
    for (int q = 0; q < nc; q++) {
        int st = S->cell_start[cells[q]], cnt = S->cell_count[cells[q]];
        for (int j = 0; j < cnt; j++) {
            V d = sub(fv(S->ph_pos[st + j]), p);
            real d2 = dot(d, d);
            if (d2 > rmax2) continue;
            if (dot(fv(S->ph_nrm[st + j]), n) < R(0.1)) continue;
            d2s[m++] = d2;
        }
    }
    real r2 = rmax2;
    if (m >= k) {
        qsort(d2s, (size_t)m, sizeof(real), cmp_real);
        r2 = d2s[k - 1];
    }
    free(d2s);
    *r2_out = r2;
    for (int q = 0; q < nc; q++) {
        int st = S->cell_start[cells[q]], cnt = S->cell_count[cells[q]];
        for (int j = 0; j < cnt; j++) {
            V d = sub(fv(S->ph_pos[st + j]), p);
            if (dot(d, d) > r2) continue;
            if (dot(fv(S->ph_nrm[st + j]), n) < R(0.1)) continue;
            acc = add(acc, fv(S->ph_flux[st + j]));
        }
    }
    return acc;
}

static V up_for(V a) { return fabs(a.y) < R(0.9) ? v3(0, 1, 0) : v3(1, 0, 0); }

/* render_kernel.cu:13-24 */
static V sun_dir(const Light* l, uint32_t seed) {
    V base = neg(fv(l->direction));
    if (l->angle <= 0) return base;
    V up = up_for(base);
    V t1 = nrm(cross(base, up)), t2 = cross(base, t1);
    real r = sqrt(aa_rand(seed ^ 0x68e31da4u)) * (real)tan(l->angle);
    real phi = R(6.2831853) * aa_rand(seed ^ 0xb5297a4du);
    return nrm(add(add(base, mul(t1, cos(phi) * r)), mul(t2, sin(phi) * r)));
}

/* render_kernel.cu:26-298 */
static V lighting(const OracleScene* S, const Hit* rec, V view, real footprint, uint32_t seed) {
    const Material* m = &S->mats[rec->mat];
    Shade in;
    in.p = rec->p; in.n = rec->n; in.tan = rec->tan; in.u = rec->u; in.v = rec->v; in.view = view;
    real uv_fp = footprint;
    V tan_u = v3(0, 0, 0), tan_v = v3(0, 0, 0);
    /* QUIRK: any negative object id is read as a triangle index when the
     * scene has triangles (render_kernel.cu:82-84). */
    if (rec->obj < 0 && S->s.num_triangles > 0) {
        int ti = -rec->obj - 1;
        if (ti >= 0 && ti < S->s.num_triangles) {
            const Triangle* tr = &S->tris[ti];
            V e1 = sub(fv(tr->v1), fv(tr->v0)), e2 = sub(fv(tr->v2), fv(tr->v0));
            real d1x = R(tr->uv1.x) - tr->uv0.x, d1y = R(tr->uv1.y) - tr->uv0.y;
            real d2x = R(tr->uv2.x) - tr->uv0.x, d2y = R(tr->uv2.y) - tr->uv0.y;
            real w1 = sqrt(dot(e1, e1)), w2 = sqrt(dot(e2, e2));
            real u1 = sqrt(d1x * d1x + d1y * d1y), u2 = sqrt(d2x * d2x + d2y * d2y);
            real a1 = w1 > R(1e-6) ? u1 / w1 : 0, a2 = w2 > R(1e-6) ? u2 / w2 : 0;
            real dens = a1 > a2 ? a1 : a2;
            if (dens > R(1e-6)) uv_fp = footprint * dens;
            real det = d1x * d2y - d2x * d1y;
            if (fabs(det) > R(1e-8)) {
                V du = mul(sub(mul(e1, d2y), mul(e2, d1y)), R(1) / det);
                V dv = mul(sub(mul(e2, d1x), mul(e1, d2x)), R(1) / det);
                du = v3((e1.x * d2y - e2.x * d1y) / det, (e1.y * d2y - e2.y * d1y) / det, (e1.z * d2y - e2.z * d1y) / det);
                dv = v3((e2.x * d1x - e1.x * d2x) / det, (e2.y * d1x - e1.y * d2x) / det, (e2.z * d1x - e1.z * d2x) / det);
                V n0 = rec->n;
                du = sub(du, mul(n0, dot(du, n0)));
                dv = sub(dv, mul(n0, dot(dv, n0)));
                real lu = dot(du, du);
                if (lu > R(1e-12)) {
                    tan_u = mul(du, R(1) / sqrt(lu));
                    dv = sub(dv, mul(tan_u, dot(dv, tan_u)));
                    real lv = dot(dv, dv);
                    if (lv > R(1e-12)) tan_v = mul(dv, R(1) / sqrt(lv));
                }
            }
        }
    }
    in.uv_fp = uv_fp;
    if (m->normal_id >= 0 && m->normal_id < S->ntex) {
        const Tex* nt = &S->tex[m->normal_id];
        V nx3 = tex_sample_lod(nt, in.u, in.v, tex_lod(nt, in.uv_fp));
        real nx = (nx3.x * 2 - 1) * m->normal_strength, ny = (nx3.y * 2 - 1) * m->normal_strength;
        V n0 = in.n, t1, t2;
        if (dot(tan_u, tan_u) > R(0.5) && dot(tan_v, tan_v) > R(0.5)) { t1 = tan_u; t2 = tan_v; }
        else { V up = up_for(n0); t1 = nrm(cross(up, n0)); t2 = cross(n0, t1); }
        in.n = nrm(add(add(n0, mul(t1, nx)), mul(t2, ny)));
    }
    V base = albedo(S, m, &in);
    V result = add(mul(base, m->ambient), mul(fv(m->emission_color), m->emission));
    real shin = m->shininess;
    if (has_mask(S, m)) {
        const Tex* mt = &S->tex[m->mask_id];
        shin = rough_to_shin(tex_sample_lod(mt, in.u, in.v, tex_lod(mt, in.uv_fp)).z);
    }
    for (int i = 0; i < S->s.num_lights; i++) {
        const Light* L = &S->lights[i];
        uint32_t ls = seed ^ ((uint32_t)i * 2654435761u);
        V Ld, radiance, target;
        real tmax = R(1e10);
        if (L->type == 0) {
            Ld = sun_dir(L, ls);
            radiance = mul(fv(L->color), L->intensity);
            target = add(rec->p, mul(Ld, R(1e6)));
        } else {
            V sp = fv(L->position);
            if (L->type == 2) {
                real ru = aa_rand(ls) * 2 - 1, rv = aa_rand(ls ^ 0x9e3779b9u) * 2 - 1;
                sp = add(add(fv(L->position), mul(fv(L->u_axis), ru)), mul(fv(L->v_axis), rv));
            }
            V tl = sub(sp, rec->p);
            real d2 = rfmax(dot(tl, tl), R(1e-4)), dist = sqrt(d2);
            Ld = mul(tl, R(1) / dist);
            Ld = v3(tl.x / dist, tl.y / dist, tl.z / dist);
            if ((L->type == 1 || L->type == 3) && L->radius > 0) {
                V up = up_for(Ld);
                V t1 = nrm(cross(Ld, up)), t2 = cross(Ld, t1);
                real rr = sqrt(aa_rand(ls ^ 0x85ebca6bu)) * L->radius;
                real phi = R(6.2831853) * aa_rand(ls ^ 0xc2b2ae35u);
                sp = add(add(sp, mul(t1, cos(phi) * rr)), mul(t2, sin(phi) * rr));
                tl = sub(sp, rec->p);
                d2 = rfmax(dot(tl, tl), R(1e-4));
                dist = sqrt(d2);
                Ld = v3(tl.x / dist, tl.y / dist, tl.z / dist);
            }
            real att = L->intensity / (R(12.5663706) * d2);
            V gobo = v3(1, 1, 1);
            if (L->type == 2) {
                V n = nrm(cross(fv(L->u_axis), fv(L->v_axis)));
                real cl = dot(n, Ld);
                if (cl <= 0) continue;
                att *= cl;
            } else if (L->type == 3) {
                V ts = nrm(sub(rec->p, sp));
                real c = dot(ts, fv(L->direction));
                real ch = (real)cos(L->angle);
                if (c <= ch) continue;
                real bl = rfmin(rfmax(L->blend, 0), 1);
                real cs = (real)cos(L->angle * (1 - bl));
                if (cs > ch + R(1e-4)) att *= rfmin((c - ch) / (cs - ch), 1);
                if (L->texture_id >= 0 && L->texture_id < S->ntex) {
                    V ax = fv(L->direction), up = up_for(ax);
                    V t1 = nrm(cross(ax, up)), t2 = cross(ax, t1);
                    real th = (real)tan(rfmax(L->angle, R(1e-3)));
                    real gu = R(0.5) + R(0.5) * dot(ts, t1) / th, gv = R(0.5) + R(0.5) * dot(ts, t2) / th;
                    gobo = tex_sample_lod(&S->tex[L->texture_id], gu, gv, 0);
                }
            }
            radiance = vmul(mul(fv(L->color), att), gobo);
            target = sp;
            tmax = dist * R(0.999);
        }
        Ray sr;
        sr.o = add(rec->p, mul(rec->n, R(0.002)));
        sr.d = nrm(sub(target, sr.o));
        sr.tmin = R(0.001);
        sr.tmax = tmax;
        Ray r2 = sr;
        int blocked = 0;
        for (int pass = 0; pass < 3; pass++) {
            Hit sh;
            if (!scene_hit_opaque(S, &r2, &sh)) { blocked = 0; break; }
            if (hit_transmission(S, &sh, &S->mats[sh.mat]) > R(0.5)) {
                /* QUIRK: t_max is not reduced after a glass pass */
                r2.o = add(sh.p, mul(r2.d, R(0.002)));
                continue;
            }
            blocked = 1;
            break;
        }
        if (m->shininess < 0) return blocked ? v3(1, 0, 0) : v3(0, 1, 0);
        if (blocked) continue;
        real trans = 1;
        if (m->anisotropy <= 0) trans = (real)exp(-strands_tau(S, &sr, R(6)));
        result = add(result, mul(shade_direct(S, m, &in, Ld, radiance, shin), trans));
    }
    if (S->nph && S->s.caustics > 0) {
        real r = S->cell * R(0.5);
        if (S->knn > 0) {
            real r2;
            V flux = photon_knn(S, rec->p, rec->n, r, S->knn, &r2);
            result = add(result, mul(vmul(base, flux), S->s.caustics / (R(9.8696044) * r2)));
        } else {
            V flux = photon_gather(S, rec->p, rec->n, r, 128);
            result = add(result, mul(vmul(base, flux), S->s.caustics / (R(9.8696044) * r * r)));
        }
    }
    return result;
}

/* render_kernel.cu:302-334 */
static int ray_box(const Ray* r, V c, V hh, real* t0, real* t1) {
    *t0 = R(-1e30); *t1 = R(1e30);
    real o[3] = {r->o.x, r->o.y, r->o.z}, d[3] = {r->d.x, r->d.y, r->d.z};
    real cc[3] = {c.x, c.y, c.z}, h[3] = {hh.x, hh.y, hh.z};
    for (int a = 0; a < 3; a++) {
        if (fabs(d[a]) < R(1e-8)) {
            if (o[a] < cc[a] - h[a] || o[a] > cc[a] + h[a]) return 0;
            continue;
        }
        real inv = R(1) / d[a];
        real tn = (cc[a] - h[a] - o[a]) * inv, tf = (cc[a] + h[a] - o[a]) * inv;
        if (tn > tf) { real t = tn; tn = tf; tf = t; }
        *t0 = rfmax(*t0, tn);
        *t1 = rfmin(*t1, tf);
        if (*t0 > *t1) return 0;
    }
    return 1;
}

static V sky(V d) {
    real t = R(0.5) * (d.y + 1);
    return v3((1 - t) * 1 + t * R(0.5), (1 - t) * 1 + t * R(0.7), (1 - t) * 1 + t * 1);
}

/* render_kernel.cu:339-436 */
static V media_march(const OracleScene* S, const Ray* ray, real t_surf, uint32_t seed, real* tau_out) {
    V ins = v3(0, 0, 0);
    real tau_total = 0;
    for (int mi = 0; mi < S->s.num_media; mi++) {
        const Medium* md = &S->media[mi];
        if (md->samples <= 0) continue;
        real m0, m1;
        if (!ray_box(ray, fv(md->center), fv(md->half), &m0, &m1)) continue;
        m0 = rfmax(m0, ray->tmin);
        m1 = rfmin(m1, t_surf);
        if (m1 <= m0) continue;
        int n = md->samples > 64 ? 64 : md->samples;
        real dt = (m1 - m0) / (real)n, tau = 0;
        for (int k = 0; k < n; k++) {
            real jit = aa_rand(seed ^ ((uint32_t)mi * 9781u) ^ ((uint32_t)k * 6271u));
            real t = m0 + ((real)k + jit) * dt;
            V p = add(ray->o, mul(ray->d, t));
            V rad = v3(0, 0, 0);
            for (int i = 0; i < S->s.num_lights; i++) {
                const Light* L = &S->lights[i];
                if (!(L->flags & 1)) continue;
                V ld, lr;
                real ldist;
                if (L->type == 0) {
                    ld = sun_dir(L, seed ^ ((uint32_t)i * 2654435761u) ^ ((uint32_t)k * 2246822519u));
                    ldist = R(1e9);
                    lr = mul(fv(L->color), L->intensity);
                } else {
                    V tl = sub(fv(L->position), p);
                    real d2 = rfmax(dot(tl, tl), R(1e-4));
                    ldist = sqrt(d2);
                    ld = v3(tl.x / ldist, tl.y / ldist, tl.z / ldist);
                    lr = mul(fv(L->color), L->intensity / (R(12.5663706) * d2));
                    if (L->type == 3) {
                        real c = dot(neg(ld), fv(L->direction)), ch = (real)cos(L->angle);
                        if (c <= ch) continue;
                        real bl = rfmin(rfmax(L->blend, 0), 1), cs = (real)cos(L->angle * (1 - bl));
                        if (cs > ch + R(1e-4)) lr = mul(lr, rfmin((c - ch) / (cs - ch), 1));
                    }
                }
                Ray sr;
                sr.o = p; sr.d = ld; sr.tmin = R(0.002); sr.tmax = ldist;
                Hit sh;
                if (scene_hit_opaque(S, &sr, &sh)) continue;
                rad = add(rad, lr);
            }
            V sc = mul(vmul(fv(md->sigma_s), rad), R(0.07957747));
            ins = add(ins, mul(sc, (real)exp(-tau) * dt));
            tau += md->sigma_t * dt;
        }
        tau_total += tau;
    }
    *tau_out = tau_total;
    return ins;
}

/* render_kernel.cu:560-652 -- visible spot-light cones along one ray */
static V beams(const OracleScene* S, const Ray* ray, int hit, real t_hit, uint32_t seed) {
    V total = v3(0, 0, 0);
    for (int i = 0; i < S->s.num_lights; i++) {
        const Light* L = &S->lights[i];
        if (L->type != 3 || L->beam <= 0) continue;
        real t_end = hit ? rfmin(t_hit, 30) : R(30);
        if (t_end <= 0) continue;
        const int STEPS = 6;
        real dt = t_end / (real)STEPS, ch = (real)cos(L->angle);
        real bl = rfmin(rfmax(L->blend, 0), 1), cs = (real)cos(L->angle * (1 - bl));
        V bacc = v3(0, 0, 0);
        for (int k = 0; k < STEPS; k++) {
            real t = ((real)k + R(0.5)) * dt;
            V p = add(ray->o, mul(ray->d, t));
            V vv = sub(p, fv(L->position));
            real d2 = rfmax(dot(vv, vv), R(1e-4));
            real c = dot(vv, fv(L->direction)) * (R(1) / sqrt(d2));
            if (c <= ch) continue;
            real w = 1;
            if (cs > ch + R(1e-4)) w = rfmin((c - ch) / (cs - ch), 1);
            real dens = L->beam * L->intensity * R(1e-3) / (1 + R(0.25) * d2);
            V target = fv(L->position);
            if (L->radius > 0) {
                V axis = nrm(neg(vv)), up = up_for(axis);
                V t1 = nrm(cross(axis, up)), t2 = cross(axis, t1);
                real rr = sqrt(aa_rand(seed ^ ((uint32_t)k * 2654435761u) ^ 0x85ebca6bu)) * L->radius;
                real ph = R(6.2831853) * aa_rand(seed ^ ((uint32_t)k * 2246822519u) ^ 0xc2b2ae35u);
                target = add(add(fv(L->position), mul(t1, cos(ph) * rr)), mul(t2, sin(ph) * rr));
            }
            V tl = sub(target, p);
            real ld = sqrt(rfmax(dot(tl, tl), R(1e-8)));
            V ldir = v3(tl.x / ld, tl.y / ld, tl.z / ld);
            real remain = ld * R(0.999);
            Ray sr;
            sr.o = p; sr.d = ldir; sr.tmin = R(0.002); sr.tmax = remain;
            int blocked = 0;
            for (int pass = 0; pass < 3; pass++) {
                Hit sh;
                if (!scene_hit_opaque(S, &sr, &sh)) { blocked = 0; break; }
                if (S->mats[sh.mat].transmission > R(0.5)) {
                    remain -= sh.t + R(0.002);
                    if (remain <= 0) { blocked = 0; break; }
                    sr.o = add(sh.p, mul(ldir, R(0.002)));
                    sr.tmax = remain;
                    continue;
                }
                blocked = 1;
                break;
            }
            if (blocked) continue;
            bacc = add(bacc, mul(fv(L->color), dens * w * dt));
        }
        total = add(total, bacc);
    }
    return total;
}

/* Extension, no counterpart in the reference: reflect + refract recursion to
 * S->bounces bounces.  Below the limit every hit blends as the reference's
 * primary hit does (render_kernel.cu:730-731, 805): its lighting times
 * (1 - wr)(1 - wt), a mirror ray times wr (1 - wt), a refracted ray times the
 * face's transmission (wr = min(reflect, 1), wt = min(transmission, 1)); at
 * the limit a hit gives its lighting alone.  A refracted ray crosses the face
 * (exit eta = ior after an entry); a mirror ray and a totally reflected ray
 * stay on their side.  Media act on every segment, beams on the primary ray
 * only.  Paths are summed depth first in the order a stack gives (the mirror
 * child is pushed last, so it is walked first), the device's order. */
typedef struct { V o, d, w; int depth, inside; } DeepNode;

static V render_deep(const OracleScene* S, Ray ray0, real pix, uint32_t seed) {
    DeepNode st[10];
    int sp = 0;
    const int D = S->bounces < 8 ? S->bounces : 8;
    st[sp].o = ray0.o; st[sp].d = ray0.d; st[sp].w = v3(1, 1, 1); st[sp].depth = 0; st[sp].inside = 0; sp++;
    V color = v3(0, 0, 0);
    while (sp > 0) {
        const DeepNode nd = st[--sp];
        Ray r;
        r.o = nd.o; r.d = nd.d; r.tmin = R(0.001); r.tmax = R(1e10);
        Hit h;
        int hit = scene_hit(S, &r, &h);
        V local = hit ? lighting(S, &h, neg(r.d), h.t * pix, seed) : sky(r.d);
        if (nd.depth == 0) local = add(local, beams(S, &r, hit, hit ? h.t : 0, seed));
        if (S->s.num_media > 0) {
            real tau = 0;
            V ins = media_march(S, &r, hit ? h.t : R(1e9), seed, &tau);
            local = add(mul(local, (real)exp(-tau)), ins);
        }
        if (!hit || nd.depth >= D) { color = add(color, vmul(nd.w, local)); continue; }
        const Material* m = &S->mats[h.mat];
        real wr = m->reflect > 0 ? rfmin(m->reflect, 1) : 0;
        real gtr = hit_transmission(S, &h, m);
        real wt = gtr > 0 ? rfmin(gtr, 1) : 0;
        color = add(color, mul(vmul(nd.w, local), (1 - wr) * (1 - wt)));
        if (gtr > 0 && sp < 10) {
            real ior = rfmax(hit_ior(S, &h, m), 1);
            real eta = nd.inside ? ior : R(1) / ior;
            real cosi = rfmax(-dot(r.d, h.n), R(1e-4));
            real k = 1 - eta * eta * (1 - cosi * cosi);
            V td = k < 0 ? nrm(add(r.d, mul(h.n, R(2) * cosi)))
                         : nrm(add(mul(r.d, eta), mul(h.n, eta * cosi - sqrt(k))));
            DeepNode c;
            c.o = add(h.p, mul(td, R(0.002))); c.d = td; c.w = mul(nd.w, gtr);
            c.depth = nd.depth + 1; c.inside = k < 0 ? nd.inside : !nd.inside;
            st[sp++] = c;
        }
        if (wr > 0 && sp < 10) {
            DeepNode c;
            c.o = add(h.p, mul(h.n, R(0.002)));
            c.d = nrm(sub(r.d, mul(h.n, R(2) * dot(r.d, h.n))));
            c.w = mul(nd.w, wr * (1 - wt));
            c.depth = nd.depth + 1; c.inside = nd.inside;
            st[sp++] = c;
        }
    }
    return color;
}

/* render_kernel.cu:438-814 -- one pixel */
static void render_pixel(const OracleScene* S, int x, int y, int W, int H, int aa, float* out) {
    const CameraData* cam = &S->s.camera;
    const int ns = aa < 1 ? 1 : (aa > 64 ? 64 : aa);
    V acc = v3(0, 0, 0);
    for (int s = 0; s < ns; s++) {
        real ox, oy;
        sample_pos(S, s, ns, x, y, &ox, &oy);
        real u = ((real)x + ox) / (real)W * 2 - 1;
        real v = 1 - ((real)y + oy) / (real)H * 2;
        uint32_t seed = aa_hash((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)s * 83492791u);
        real tan_h = 1, tan_x = 1, tan_y = 1;
        if (cam->focal_length > 0) {
            tan_h = R(0.5) * cam->sensor_width / cam->focal_length;
            if (W >= H) { tan_x = tan_h; tan_y = tan_h * (real)H / (real)W; }
            else { tan_y = tan_h; tan_x = tan_h * (real)W / (real)H; }
        }
        Ray ray;
        ray.o = fv(cam->position);
        ray.d = nrm(add(add(fv(cam->forward), mul(fv(cam->right), u * tan_x + cam->shift_x * tan_h)),
                        mul(fv(cam->up), v * tan_y + cam->shift_y * tan_h)));
        ray.tmin = R(0.001);
        ray.tmax = R(1e10);
        const real pix = R(2) * tan_x / (real)W;
        if (S->bounces > 1) { acc = add(acc, render_deep(S, ray, pix, seed)); continue; }
        Hit rec;
        int hit = scene_hit(S, &ray, &rec);
        V color = hit ? lighting(S, &rec, neg(ray.d), rec.t * pix, seed) : sky(ray.d);
        color = add(color, beams(S, &ray, hit, hit ? rec.t : 0, seed));
        if (S->s.num_media > 0) {
            real tau = 0;
            V ins = media_march(S, &ray, hit ? rec.t : R(1e9), seed, &tau);
            color = add(mul(color, (real)exp(-tau)), ins);
        }
        if (hit) {
            const Material* pm = &S->mats[rec.mat];
            if (pm->reflect > 0) {
                V rd = sub(ray.d, mul(rec.n, R(2) * dot(ray.d, rec.n)));
                Ray rr;
                rr.o = add(rec.p, mul(rec.n, R(0.002)));
                rr.d = nrm(rd);
                rr.tmin = R(0.001);
                rr.tmax = R(1e10);
                Hit rh;
                int rhit = scene_hit(S, &rr, &rh);
                V rcol = rhit ? lighting(S, &rh, neg(rr.d), rh.t * pix, seed) : sky(rr.d);
                if (S->s.num_media > 0) {
                    real rt = 0;
                    V ri = media_march(S, &rr, rhit ? rh.t : R(1e9), seed, &rt);
                    rcol = add(mul(rcol, (real)exp(-rt)), ri);
                }
                real w = rfmin(pm->reflect, 1);
                color = add(mul(color, 1 - w), mul(rcol, w));
            }
        }
        if (hit) {
            const Material* gm = &S->mats[rec.mat];
            real gtr = hit_transmission(S, &rec, gm);
            if (gtr > 0) {
                V through = v3(0, 0, 0);
                real w = 1;
                Ray gr = ray;
                Hit gh = rec;
                int entering = 1;
                for (int b = 0; b < 3; b++) {
                    const Material* sm = &S->mats[gh.mat];
                    V n = gh.n, d = gr.d;
                    real ior = rfmax(hit_ior(S, &gh, sm), 1);
                    real eta = entering ? R(1) / ior : ior;
                    real cosi = rfmax(-dot(d, n), R(1e-4));
                    real k = 1 - eta * eta * (1 - cosi * cosi);
                    V td = k < 0 ? nrm(add(d, mul(n, R(2) * cosi)))
                                 : nrm(add(mul(d, eta), mul(n, eta * cosi - sqrt(k))));
                    w *= hit_transmission(S, &gh, sm);
                    gr.o = add(gh.p, mul(td, R(0.002)));
                    gr.d = td;
                    gr.tmin = R(0.001);
                    gr.tmax = R(1e10);
                    Hit nh;
                    if (!scene_hit(S, &gr, &nh)) { through = add(through, mul(sky(td), w)); break; }
                    if (hit_transmission(S, &nh, &S->mats[nh.mat]) > 0) { entering = !entering; gh = nh; continue; }
                    through = add(through, mul(lighting(S, &nh, neg(td), nh.t * pix, seed), w));
                    break;
                }
                color = add(mul(color, 1 - rfmin(gtr, 1)), through);
            }
        }
        acc = add(acc, color);
    }
    real inv = R(1) / (real)ns;
    out[0] = (float)(acc.x * inv);
    out[1] = (float)(acc.y * inv);
    out[2] = (float)(acc.z * inv);
    out[3] = 1.0f;
}

/* ------------------------------------------------------------------ */
/* photon pass: render_kernel.cu:820-926 emission, :992-1045 map build   */
/* ------------------------------------------------------------------ */
static int emit_photon(const OracleScene* S, int idx, int per_light, sheen_float3 out[4]) {
    const Light* L = &S->lights[idx / per_light];
    if (L->type == 0) return 0;
    uint32_t sd = aa_hash(0x5eed1234u + (uint32_t)idx * 2654435761u);
    real u1 = aa_rand(sd), u2 = aa_rand(sd ^ 0x9e3779b9u), u3 = aa_rand(sd ^ 0x85ebca6bu);
    V pos = fv(L->position), dir;
    if (L->type == 3) {
        real ch = (real)cos(L->angle);
        real ct = ch + (1 - ch) * u1, st = sqrt(rfmax(1 - ct * ct, 0)), phi = R(6.2831853) * u2;
        V ax = fv(L->direction), up = up_for(ax);
        V t1 = nrm(cross(ax, up)), t2 = cross(ax, t1);
        dir = nrm(add(add(mul(ax, ct), mul(t1, cos(phi) * st)), mul(t2, sin(phi) * st)));
    } else if (L->type == 2) {
        pos = add(add(fv(L->position), mul(fv(L->u_axis), u1 * 2 - 1)), mul(fv(L->v_axis), u2 * 2 - 1));
        V n = nrm(cross(fv(L->u_axis), fv(L->v_axis))), up = up_for(n);
        V t1 = nrm(cross(n, up)), t2 = cross(n, t1);
        real cz = sqrt(rfmax(1 - u3, 0)), r = sqrt(u3), phi = R(6.2831853) * aa_rand(sd ^ 0xc2b2ae35u);
        dir = nrm(add(add(mul(n, cz), mul(t1, cos(phi) * r)), mul(t2, sin(phi) * r)));
    } else {
        real cz = 2 * u1 - 1, st = sqrt(rfmax(1 - cz * cz, 0)), phi = R(6.2831853) * u2;
        dir = v3(st * cos(phi), cz, st * sin(phi));
    }
    V flux = mul(fv(L->color), L->intensity / (real)per_light);
    Ray ray;
    ray.o = pos; ray.d = dir; ray.tmin = R(0.001); ray.tmax = R(1e10);
    for (int b = 0; b < 4; b++) {
        Hit h;
        if (!scene_hit(S, &ray, &h)) return 0;
        const Material* m = &S->mats[h.mat];
        if (m->transmission > R(0.5)) {
            /* QUIRK: eta = 1/ior on every face (render_kernel.cu:896-902) */
            V n = h.n;
            real ior = rfmax(m->ior, 1), eta = R(1) / ior;
            real cosi = rfmax(-dot(ray.d, n), R(1e-4));
            real k = 1 - eta * eta * (1 - cosi * cosi);
            V td = k < 0 ? nrm(add(ray.d, mul(n, 2 * cosi))) : nrm(add(mul(ray.d, eta), mul(n, eta * cosi - sqrt(k))));
            flux = mul(flux, m->transmission);
            ray.o = add(h.p, mul(td, R(0.002)));
            ray.d = td;
            continue;
        }
        if (m->reflect > R(0.5)) {
            V rd = sub(ray.d, mul(h.n, 2 * dot(ray.d, h.n)));
            ray.o = add(h.p, mul(h.n, R(0.002)));
            ray.d = nrm(rd);
            continue;
        }
        out[0] = (sheen_float3){(float)h.p.x, (float)h.p.y, (float)h.p.z};
        out[1] = (sheen_float3){(float)-ray.d.x, (float)-ray.d.y, (float)-ray.d.z};
        out[2] = (sheen_float3){(float)h.n.x, (float)h.n.y, (float)h.n.z};
        out[3] = (sheen_float3){(float)flux.x, (float)flux.y, (float)flux.z};
        return 1;
    }
    return 0;
}

static void build_photons(OracleScene* S) {
    int per = S->s.photons, nl = S->s.num_lights;
    long long total = (long long)per * nl;
    if (total <= 0) return;
    sheen_float3* tmp = (sheen_float3*)malloc((size_t)total * 4 * sizeof(sheen_float3));
    unsigned char* ok = (unsigned char*)calloc((size_t)total, 1);
#pragma omp parallel for schedule(dynamic, 4096)
    for (long long i = 0; i < total; i++) ok[i] = (unsigned char)emit_photon(S, (int)i, per, tmp + 4 * i);
    long long n = 0;
    for (long long i = 0; i < total; i++) if (ok[i]) n++;
    if (n > 4000000) n = 4000000;   /* C-API cap, api/sheen_c_api.cu:276-278 */
    S->nph = (int)n;
    S->num_cells = 1 << 18;
    S->cell = R(S->s.photon_cell > 0 ? S->s.photon_cell : 0.25f);
    S->cell_count = (int*)calloc((size_t)S->num_cells, sizeof(int));
    S->cell_start = (int*)calloc((size_t)S->num_cells + 1, sizeof(int));
    S->ph_pos = (sheen_float3*)malloc((size_t)(n ? n : 1) * sizeof(sheen_float3));
    S->ph_dir = (sheen_float3*)malloc((size_t)(n ? n : 1) * sizeof(sheen_float3));
    S->ph_nrm = (sheen_float3*)malloc((size_t)(n ? n : 1) * sizeof(sheen_float3));
    S->ph_flux = (sheen_float3*)malloc((size_t)(n ? n : 1) * sizeof(sheen_float3));
    int* cell_of = (int*)malloc((size_t)(n ? n : 1) * sizeof(int));
    long long* src = (long long*)malloc((size_t)(n ? n : 1) * sizeof(long long));
    long long k = 0;
    for (long long i = 0; i < total && k < n; i++) {
        if (!ok[i]) continue;
        sheen_float3 p = tmp[4 * i];
        int ix = (int)floorf(p.x / (float)S->cell), iy = (int)floorf(p.y / (float)S->cell), iz = (int)floorf(p.z / (float)S->cell);
        cell_of[k] = cell_hash(ix, iy, iz, S->num_cells);
        src[k] = i;
        S->cell_count[cell_of[k]]++;
        k++;
    }
    int acc = 0;
    for (int c = 0; c < S->num_cells; c++) { S->cell_start[c] = acc; acc += S->cell_count[c]; }
    S->cell_start[S->num_cells] = acc;
    int* cur = (int*)malloc((size_t)S->num_cells * sizeof(int));
    memcpy(cur, S->cell_start, (size_t)S->num_cells * sizeof(int));
    for (long long j = 0; j < n; j++) {
        int slot = cur[cell_of[j]]++;
        S->ph_pos[slot] = tmp[4 * src[j]];
        S->ph_dir[slot] = tmp[4 * src[j] + 1];
        S->ph_nrm[slot] = tmp[4 * src[j] + 2];
        S->ph_flux[slot] = tmp[4 * src[j] + 3];
    }
    free(cur); free(cell_of); free(src); free(tmp); free(ok);
}

/* ------------------------------------------------------------------ */
/* scene setup; mips as scene.h:230-261 (2x2 box, clamped, rounded)     */
/* ------------------------------------------------------------------ */
static void* dup(const void* p, size_t n) {
    if (!p || !n) return NULL;
    void* q = malloc(n);
    memcpy(q, p, n);
    return q;
}

static void build_tex(Tex* t, const unsigned char* px, int w, int h) {
    size_t total = 0;
    int sw = w, sh = h, mips = 1;
    total = (size_t)w * h * 3;
    while (sw > 1 || sh > 1) {
        sw = sw > 1 ? sw / 2 : 1; sh = sh > 1 ? sh / 2 : 1;
        total += (size_t)sw * sh * 3;
        mips++;
    }
    if (w < 2 && h < 2) mips = 1;
    t->px = (unsigned char*)malloc(total);
    memcpy(t->px, px, (size_t)w * h * 3);
    t->w = w; t->h = h; t->mips = mips;
    size_t src = 0, dst = (size_t)w * h * 3;
    sw = w; sh = h;
    for (int l = 1; l < mips; l++) {
        int nw = sw > 1 ? sw / 2 : 1, nh = sh > 1 ? sh / 2 : 1;
        for (int y = 0; y < nh; y++) {
            int y0 = 2 * y < sh ? 2 * y : sh - 1, y1 = 2 * y + 1 < sh ? 2 * y + 1 : sh - 1;
            for (int x = 0; x < nw; x++) {
                int x0 = 2 * x < sw ? 2 * x : sw - 1, x1 = 2 * x + 1 < sw ? 2 * x + 1 : sw - 1;
                for (int c = 0; c < 3; c++) {
                    int s = t->px[src + ((size_t)y0 * sw + x0) * 3 + c] + t->px[src + ((size_t)y0 * sw + x1) * 3 + c] +
                            t->px[src + ((size_t)y1 * sw + x0) * 3 + c] + t->px[src + ((size_t)y1 * sw + x1) * 3 + c];
                    t->px[dst + ((size_t)y * nw + x) * 3 + c] = (unsigned char)((s + 2) / 4);
                }
            }
        }
        src = dst;
        dst += (size_t)nw * nh * 3;
        sw = nw; sh = nh;
    }
}

/* Bezier runs -> cubic spans: consecutive spans joined, and prism contours
 * closed, by straight spans where their ends differ (the limit of the
 * reference's host polyline). */
static void add_runs(OracleScene* S, const SheenSceneExt* x, const SheenBezierRun* runs, int n, int close,
                     int** out_run) {
    if (!runs || n <= 0) return;
    *out_run = (int*)calloc((size_t)n * 2, sizeof(int));
    for (int i = 0; i < n; i++) {
        const SheenBezierRun* r = &runs[i];
        if (r->ctrl_count < 4) continue;
        const float* c = x->bezier_ctrl + 2 * (size_t)r->ctrl_offset;
        int ns = r->ctrl_count / 4, first = S->nspans;
        S->spans = (double*)realloc(S->spans, sizeof(double) * 8 * (size_t)(S->nspans + 2 * ns + 1));
#define PUSH8(a0, b0, a1, b1, a2, b2, a3, b3) do { double v8_[8] = {a0, b0, a1, b1, a2, b2, a3, b3}; \
        memcpy(S->spans + 8 * (size_t)S->nspans++, v8_, sizeof(v8_)); } while (0)
#define LINE(pa, pb, qa, qb) PUSH8(pa, pb, pa + (qa - pa) / 3.0, pb + (qb - pb) / 3.0, \
        pa + 2.0 * (qa - pa) / 3.0, pb + 2.0 * (qb - pb) / 3.0, qa, qb)
        for (int k = 0; k < ns; k++) {
            const float* q = c + 8 * k;
            if (k > 0 && (q[-2] != q[0] || q[-1] != q[1])) LINE((double)q[-2], (double)q[-1], (double)q[0], (double)q[1]);
            PUSH8(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]);
        }
        const float* last = c + 8 * (ns - 1) + 6;
        if (close && (last[0] != c[0] || last[1] != c[1])) LINE((double)last[0], (double)last[1], (double)c[0], (double)c[1]);
#undef LINE
#undef PUSH8
        (*out_run)[2 * i] = first;
        (*out_run)[2 * i + 1] = S->nspans - first;
    }
}

/* Instanced meshes (extension): flattened after the scene's own triangles,
 * instance by instance, so that triangle k of instance j has the index
 * num_triangles + base_j + k the library reports.  Positions go through the
 * object-to-world map and vertex normals through its inverse transpose,
 * both in double and rounded once; the triangles take the instance's
 * material. */
static Triangle* flatten_instances(const SheenScene* in, const SheenSceneExt* x, int* count) {
    long long n = in->num_triangles > 0 ? in->num_triangles : 0;
    for (int j = 0; j < x->num_instances; j++) n += x->meshes[x->instances[j].mesh].tri_count;
    Triangle* out = (Triangle*)calloc((size_t)(n > 0 ? n : 1), sizeof(Triangle));
    if (in->num_triangles > 0) memcpy(out, in->triangles, sizeof(Triangle) * (size_t)in->num_triangles);
    long long k = in->num_triangles > 0 ? in->num_triangles : 0;
    for (int j = 0; j < x->num_instances; j++) {
        const SheenInstance* I = &x->instances[j];
        const float* f = I->xform;
        double M[3][3], T[3], A[3][3];
        for (int r = 0; r < 3; r++) { for (int c = 0; c < 3; c++) M[r][c] = f[4 * r + c]; T[r] = f[4 * r + 3]; }
        double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                     M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        /* inverse transpose = cofactor matrix / det */
        A[0][0] = (M[1][1] * M[2][2] - M[1][2] * M[2][1]) / det;
        A[0][1] = (M[1][2] * M[2][0] - M[1][0] * M[2][2]) / det;
        A[0][2] = (M[1][0] * M[2][1] - M[1][1] * M[2][0]) / det;
        A[1][0] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) / det;
        A[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) / det;
        A[1][2] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) / det;
        A[2][0] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) / det;
        A[2][1] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) / det;
        A[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) / det;
        const SheenMesh* me = &x->meshes[I->mesh];
        for (int t = 0; t < me->tri_count; t++, k++) {
            Triangle tr = x->mesh_triangles[me->tri_offset + t];
            sheen_float3* vs[3] = {&tr.v0, &tr.v1, &tr.v2};
            sheen_float3* ns[3] = {&tr.n0, &tr.n1, &tr.n2};
            for (int v = 0; v < 3; v++) {
                const double p[3] = {vs[v]->x, vs[v]->y, vs[v]->z}, q[3] = {ns[v]->x, ns[v]->y, ns[v]->z};
                double w[3], m[3];
                for (int r = 0; r < 3; r++) {
                    w[r] = M[r][0] * p[0] + M[r][1] * p[1] + M[r][2] * p[2] + T[r];
                    m[r] = A[r][0] * q[0] + A[r][1] * q[1] + A[r][2] * q[2];
                }
                vs[v]->x = (float)w[0]; vs[v]->y = (float)w[1]; vs[v]->z = (float)w[2];
                ns[v]->x = (float)m[0]; ns[v]->y = (float)m[1]; ns[v]->z = (float)m[2];
            }
            tr.material_id = I->material_id;
            out[k] = tr;
        }
    }
    *count = (int)n;
    return out;
}

OracleScene* oracle_scene_create_ext(const SheenScene* in, const SheenSceneExt* x) {
    OracleScene* S;
    if (in && x && x->num_instances > 0) {
        SheenScene flat = *in;
        int n = 0;
        Triangle* tris = flatten_instances(in, x, &n);
        flat.triangles = tris;
        flat.num_triangles = n;
        S = oracle_scene_create(&flat);
        free(tris);
    } else {
        S = oracle_scene_create(in);
    }
    if (!S || !x) return S;
    if (x->se_n2 && in->num_superellipsoids > 0) S->se_n2 = (float*)dup(x->se_n2, sizeof(float) * (size_t)in->num_superellipsoids);
    if (x->hf_grid && in->num_heightfields > 0) {
        S->hfg = (int*)calloc((size_t)in->num_heightfields * 3, sizeof(int));
        for (int i = 0; i < in->num_heightfields; i++) {
            S->hfg[3 * i] = x->hf_grid[i].offset; S->hfg[3 * i + 1] = x->hf_grid[i].w; S->hfg[3 * i + 2] = x->hf_grid[i].h;
        }
        if (x->num_hf_heights > 0) S->hf_heights = (float*)dup(x->hf_heights, sizeof(float) * (size_t)x->num_hf_heights);
    }
    add_runs(S, x, x->lathe_bezier, in->num_lathes, 0, &S->lathe_run);
    add_runs(S, x, x->prism_bezier, in->num_prisms, 1, &S->prism_run);
    if (x->num_csg_roots > 0) { S->csg_roots = (int*)dup(x->csg_roots, sizeof(int) * (size_t)x->num_csg_roots); S->ncsg_roots = x->num_csg_roots; }
    if (x->num_csg_boxes > 0) { S->csg_boxes = (SheenCsgBox*)dup(x->csg_boxes, sizeof(SheenCsgBox) * (size_t)x->num_csg_boxes); S->ncsg_boxes = x->num_csg_boxes; }
    if (x->num_csg_cones > 0) { S->csg_cones = (SheenCsgCone*)dup(x->csg_cones, sizeof(SheenCsgCone) * (size_t)x->num_csg_cones); S->ncsg_cones = x->num_csg_cones; }
    S->bounces = x->max_depth > 1 ? (x->max_depth < 8 ? x->max_depth : 8) : 0;
    return S;
}

OracleScene* oracle_scene_create(const SheenScene* in) {
    if (!in) return NULL;
    OracleScene* S = (OracleScene*)calloc(1, sizeof(OracleScene));
    S->s = *in;
#define CP(dst, field, T, cnt) S->dst = (T*)dup(in->field, sizeof(T) * (size_t)(in->cnt)); S->s.field = S->dst;
    CP(objects, objects, Object, num_objects)
    CP(sweep_points, sweep_points, SweepPoint, num_sweep_points)
    CP(strands, sweep_strands, SweepStrand, num_sweep_strands)
    CP(tris, triangles, Triangle, num_triangles)
    CP(hfs, heightfields, HeightField, num_heightfields)
    CP(ses, superellipsoids, Superellipsoid, num_superellipsoids)
    CP(lpts, lathe_points, LathePoint, num_lathe_points)
    CP(lathes, lathes, Lathe, num_lathes)
    CP(ppts, prism_points, PrismPoint, num_prism_points)
    CP(prisms, prisms, Prism, num_prisms)
    CP(csg, csg_nodes, CSGNode, num_csg_nodes)
    CP(planes, planes, Plane, num_planes)
    CP(mats, materials, Material, num_materials)
    CP(lights, lights, Light, num_lights)
    CP(media, media, Medium, num_media)
#undef CP
    S->hf_img = (unsigned char**)calloc((size_t)(in->num_heightfields > 0 ? in->num_heightfields : 1), sizeof(void*));
    for (int i = 0; i < in->num_heightfields; i++) {
        const HeightField* hf = &in->heightfields[i];
        if (hf->image && hf->img_w > 0 && hf->img_h > 0)
            S->hf_img[i] = (unsigned char*)dup(hf->image, (size_t)hf->img_w * hf->img_h);
    }
    S->ntex = in->num_textures;
    S->tex = (Tex*)calloc((size_t)(S->ntex > 0 ? S->ntex : 1), sizeof(Tex));
    for (int i = 0; i < S->ntex; i++) {
        int w = in->texture_widths ? in->texture_widths[i] : 0, h = in->texture_heights ? in->texture_heights[i] : 0;
        if (in->texture_pixels && in->texture_pixels[i] && w > 0 && h > 0) build_tex(&S->tex[i], in->texture_pixels[i], w, h);
    }
    if (in->photons > 0 && in->num_lights > 0) build_photons(S);
    return S;
}

void oracle_scene_destroy(OracleScene* S) {
    if (!S) return;
    free(S->objects); free(S->sweep_points); free(S->strands); free(S->tris); free(S->hfs);
    free(S->ses); free(S->lpts); free(S->lathes); free(S->ppts); free(S->prisms); free(S->csg);
    free(S->planes); free(S->mats); free(S->lights); free(S->media);
    for (int i = 0; i < S->s.num_heightfields; i++) free(S->hf_img[i]);
    free(S->hf_img);
    for (int i = 0; i < S->ntex; i++) free(S->tex[i].px);
    free(S->tex);
    free(S->ph_pos); free(S->ph_dir); free(S->ph_nrm); free(S->ph_flux);
    free(S->cell_start); free(S->cell_count);
    free(S->se_n2); free(S->hfg); free(S->hf_heights); free(S->lathe_run); free(S->prism_run); free(S->spans);
    free(S->csg_roots); free(S->csg_boxes); free(S->csg_cones);
    free(S);
}

int oracle_scene_photon_count(const OracleScene* S) { return S ? S->nph : 0; }

void oracle_scene_set_centered(OracleScene* S, int centered) {
    if (S) S->centered = centered;
}

void oracle_scene_set_knn(OracleScene* S, int k) {
    if (S) S->knn = k;
}

int oracle_render(const OracleScene* S, int W, int H, int aa, float* out, int y0, int y1, int nthreads) {
    if (!S || W <= 0 || H <= 0 || !out) return -1;
    if (y1 <= 0 || y1 > H) y1 = H;
    if (y0 < 0) y0 = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int y = y0; y < y1; y++)
        for (int x = 0; x < W; x++) render_pixel(S, x, y, W, H, aa, out + 4 * ((size_t)y * W + x));
    return 0;
}

/* Closest hit of the camera ray of sample s of pixel (x, y) (the camera of
 * render_kernel.cu:500-521 in the oracle's precision). */
static int primary_sample(const OracleScene* S, int W, int H, int ns, int x, int y, int s, Hit* h) {
    const CameraData* cam = &S->s.camera;
    real ox, oy;
    sample_pos(S, s, ns, x, y, &ox, &oy);
    real u = ((real)x + ox) / (real)W * 2 - 1, v = 1 - ((real)y + oy) / (real)H * 2;
    real tan_h = 1, tan_x = 1, tan_y = 1;
    if (cam->focal_length > 0) {
        tan_h = R(0.5) * cam->sensor_width / cam->focal_length;
        if (W >= H) { tan_x = tan_h; tan_y = tan_h * (real)H / (real)W; }
        else { tan_y = tan_h; tan_x = tan_h * (real)W / (real)H; }
    }
    Ray ray;
    ray.o = fv(cam->position);
    ray.d = nrm(add(add(fv(cam->forward), mul(fv(cam->right), u * tan_x + cam->shift_x * tan_h)),
                    mul(fv(cam->up), v * tan_y + cam->shift_y * tan_h)));
    ray.tmin = R(0.001);
    ray.tmax = R(1e10);
    return scene_hit(S, &ray, h);
}

int oracle_primary_hits(const OracleScene* S, int W, int H, int aa, int* cat, int* prim, double* tt, int nthreads) {
    if (!S) return -1;
    const int ns = aa < 1 ? 1 : (aa > 64 ? 64 : aa);
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int y = 0; y < H; y++)
        for (int x = 0; x < W; x++)
            for (int s = 0; s < ns; s++) {
                Hit h;
                size_t k = ((size_t)y * W + x) * ns + s;
                if (primary_sample(S, W, H, ns, x, y, s, &h)) { cat[k] = h.cat; prim[k] = h.prim; tt[k] = (double)h.t; }
                else { cat[k] = -1; prim[k] = -1; tt[k] = -1.0; }
            }
    return 0;
}

int oracle_primary_hits_px(const OracleScene* S, int W, int H, int aa, int n, const int* pixels, int* cat,
                           int* prim, double* tt, int nthreads) {
    if (!S || n < 0 || (n > 0 && !pixels)) return -1;
    const int ns = aa < 1 ? 1 : (aa > 64 ? 64 : aa);
    for (int i = 0; i < n; i++)
        if (pixels[i] < 0 || pixels[i] >= W * H) return -1;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int i = 0; i < n; i++)
        for (int s = 0; s < ns; s++) {
            Hit h;
            const int x = pixels[i] % W, y = pixels[i] / W;
            size_t k = (size_t)i * ns + s;
            if (primary_sample(S, W, H, ns, x, y, s, &h)) { cat[k] = h.cat; prim[k] = h.prim; tt[k] = (double)h.t; }
            else { cat[k] = -1; prim[k] = -1; tt[k] = -1.0; }
        }
    return 0;
}

int oracle_render_region(const OracleScene* S, int W, int H, int aa, int x0, int y0, int x1, int y1, float* out,
                         int nthreads, unsigned long long* queries) {
    if (!S || W <= 0 || H <= 0 || !out || x0 < 0 || y0 < 0 || x1 > W || y1 > H || x0 >= x1 || y0 >= y1) return -1;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    (void)nthreads;
    unsigned long long total = 0;
#pragma omp parallel num_threads(nthreads) reduction(+ : total)
    {
        const unsigned long long q0 = tl_queries;
#pragma omp for schedule(dynamic, 1)
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) render_pixel(S, x, y, W, H, aa, out + 4 * ((size_t)y * W + x));
        total += tl_queries - q0;
    }
    if (queries) *queries = total;
    return 0;
}

int oracle_trace(const OracleScene* S, int n, const double* rays, int* cat, int* prim, double* tt, int nthreads) {
    if (!S) return -1;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#endif
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
    for (int i = 0; i < n; i++) {
        Ray r;
        r.o = v3((real)rays[6 * i], (real)rays[6 * i + 1], (real)rays[6 * i + 2]);
        r.d = v3((real)rays[6 * i + 3], (real)rays[6 * i + 4], (real)rays[6 * i + 5]);
        r.tmin = R(0.001);
        r.tmax = R(1e10);
        Hit h;
        if (scene_hit(S, &r, &h)) { cat[i] = h.cat; prim[i] = h.prim; tt[i] = (double)h.t; }
        else { cat[i] = -1; prim[i] = -1; tt[i] = -1.0; }
    }
    return 0;
}
