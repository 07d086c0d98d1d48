/*
 * sheen_oracle.h -- C restatement of Sheen's per-pixel ray-casting path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this (as libsheen_oracle.so, FP32, and
 * libsheen_oracle64.so, the same source built with double precision); the
 * product never links it.
 *
 * It restates render_kernel.cu:13-814 and every function it calls, plus the
 * photon pass (render_kernel.cu:820-1045, render_kernel.h:55-111), in plain
 * C.  Acceleration structures are deliberately absent: every category is a
 * linear scan in index order, each primitive first gated by the slab test of
 * its own bounding box (the leaf box of the reference's BVH, bvh.h:24-600).
 * Closest hit with a strict '<' therefore matches the reference except when
 * two primitives give exactly the same t (the reference then keeps the one
 * its DFS visits first, this scan the lower index).
 *
 * Parity status: pinned against the reference's own code built for the
 * host (oracle/_ref/libsheen_ref_host.so) by tests/test_oracle_pin.py and
 * against committed fixtures in tests/golden/.
 */
#ifndef SHEEN_ORACLE_H
#define SHEEN_ORACLE_H

#include "sheen_c_api.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleScene OracleScene;

/* Copies the scene, builds texture mips and (if scene->photons > 0 and there
 * are lights) runs the photon pass with the reference's fixed seed.  Photon
 * slots follow emission order. */
OracleScene* oracle_scene_create(const SheenScene* scene);
/* With scene extensions (SheenSceneExt; no counterpart in the reference):
 * two-exponent superellipsoids, FP32 height grids, exact Bezier lathes and
 * prisms (found by dense sampling and bisection in double), CSG forests
 * with box and cone leaves.  ext may be NULL. */
OracleScene* oracle_scene_create_ext(const SheenScene* scene, const SheenSceneExt* ext);
void oracle_scene_destroy(OracleScene* s);
int oracle_scene_photon_count(const OracleScene* s);
/* Extension: camera samples without jitter (the library's "camera.centered"). */
void oracle_scene_set_centered(OracleScene* s, int centered);
/* Extension: k-nearest-photon caustic gather (the library's "caustic.knn"). */
void oracle_scene_set_knn(OracleScene* s, int k);

/* RGBA (width*height*4 floats) for pixel rows [y0, y1) (y1 <= 0: all rows). */
int oracle_render(const OracleScene* s, int width, int height, int aa,
                  float* out_rgba, int y0, int y1, int nthreads);

/* Primary closest hits: width*height*ns entries, index (y*width+x)*ns+s.
 * category: -1 miss, 0 sphere, 1 strand, 2 mesh, 3 heightfield,
 * 4 superellipsoid, 5 lathe, 6 prism, 7 csg, 8 plane.  prim = index within
 * the category.  t in the oracle's precision, cast to double. */
int oracle_primary_hits(const OracleScene* s, int width, int height, int aa,
                        int* category, int* prim, double* t, int nthreads);

/* Primary closest hits of the n pixels pixels[i] = y*width + x: n*ns
 * entries, index i*ns + s, as oracle_primary_hits. */
int oracle_primary_hits_px(const OracleScene* s, int width, int height, int aa, int n, const int* pixels,
                           int* category, int* prim, double* t, int nthreads);

/* RGBA of the pixel rectangle [x0, x1) x [y0, y1) into out_rgba (the whole
 * width*height*4 image; other pixels untouched) and the number of scene
 * queries the rectangle issued (*queries, may be NULL): primary rays, each
 * glass pass of a shadow ray, every mirror / refraction segment, beam and
 * medium shadow rays -- the ray count of the throughput metric. */
int oracle_render_region(const OracleScene* s, int width, int height, int aa, int x0, int y0, int x1, int y1,
                         float* out_rgba, int nthreads, unsigned long long* queries);

/* Closest hit of arbitrary rays (origin, direction as 6 doubles per ray,
 * t_min 1e-3, t_max 1e10): category, prim, t. */
int oracle_trace(const OracleScene* s, int n, const double* rays,
                 int* category, int* prim, double* t, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
