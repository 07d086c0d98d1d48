// bvh4_rules.h -- the arithmetic of the wavefront form's BVH4 build, shared
// by the host builder (bvh4.cpp) and the device builder (bvh4_gpu.cu) so the
// two make the same decisions bit for bit.
//
// Every float operation is written as an explicitly rounded add / multiply
// / divide: nvcc would otherwise contract a*b + c into one FMA on the
// device, which rounds once where the host rounds twice.  Triangle box
// coordinates are canonicalised (-0 becomes +0) because min/max of -0 and
// +0 depends on the order of the operands and the device reduces in no
// fixed order.
#pragma once
#include <cfloat>
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define BVH_HD __host__ __device__ __forceinline__
#else
#define BVH_HD inline
#endif

namespace sheen {
namespace bvhr {

constexpr int kBins = 16;      // SAH bins per axis over the centroid box
constexpr int kMaxLeaf = 8;    // triangles per leaf at most

BVH_HD float add(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
BVH_HD float sub(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
BVH_HD float mul(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
BVH_HD float div(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}

// -0 -> +0 (x + 0 rounds -0 to +0 and leaves everything else unchanged).
BVH_HD float canon(float x) { return add(x, 0.0f); }

// Surface area of a box (0 for an empty box, judged by its x extent).
BVH_HD float area(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float dx = sub(hx, lx), dy = sub(hy, ly), dz = sub(hz, lz);
    if (dx < 0.0f) return 0.0f;
    return mul(2.0f, add(add(mul(dx, dy), mul(dy, dz)), mul(dz, dx)));
}

// SAH cost of a split: area_l * n_l + area_r * n_r.
BVH_HD float split_cost(float area_l, int n_l, float area_r, int n_r) {
    return add(mul(area_l, (float)n_l), mul(area_r, (float)n_r));
}

// Centroid coordinate of a box.
BVH_HD float centroid(float lo, float hi) { return mul(0.5f, add(lo, hi)); }

// Bin of a centroid coordinate: trunc((c - lo) * k) clamped to the bins,
// where k = kBins / extent.  A NaN product lands in bin 0 on both sides.
BVH_HD int bin_of(float c, float lo, float k) {
    const float f = mul(sub(c, lo), k);
    if (!(f == f)) return 0;
    int b;
    if (f >= 2147483520.0f) b = kBins - 1;
    else if (f <= -2147483520.0f) b = 0;
    else b = (int)f;
    return b < 0 ? 0 : (b > kBins - 1 ? kBins - 1 : b);
}

BVH_HD float bin_scale(float ext) { return div((float)kBins, ext); }

// Leaf or split for a node of n <= kMaxLeaf triangles with box area pa and
// best split cost best_cost (both sides' area x count): the leaf wins when
// its n tests cost no more than one node visit (node_cost, in triangle
// tests, scaled by the area) plus the split's tests.  node_cost 1 is exact
// (1 * pa == pa).
BVH_HD bool leaf_wins(float pa, int n, float best_cost, float node_cost) {
    return mul(pa, (float)n) <= add(mul(node_cost, pa), best_cost);
}

// node_cost from the "build.node_cost" setting (quarters of a triangle test).
BVH_HD float node_cost_of(int quarters) { return (float)quarters * 0.25f; }

// Smallest e with 2^e >= v for v > 0 (frexp is exact; log2 is not).
BVH_HD int ceil_log2(double v) {
    int x = 0;
    const double m = frexp(v, &x);   // v = m * 2^x, m in [0.5, 1)
    return m == 0.5 ? x - 1 : x;
}

// Exponent of the per-axis scale 2^e of a node frame over [lo, hi]: the
// extent fits in 254 steps, and q = 255 decoded with the device's fmaf
// reaches hi.
BVH_HD int frame_exponent(float lo, float hi) {
    const double ext = (double)hi - (double)lo;
    int e = ext > 0.0 ? ceil_log2(ext / 254.0) : -20;
    e = e < -100 ? -100 : (e > 100 ? 100 : e);
    while (fmaf(255.0f, ldexpf(1.0f, e), lo) < hi && e < 100) e++;
    return e;
}

// Outward quantisation of a child interval [a, b] in a frame starting at
// `origin` with step `scale`: floor/ceil in double, then moved outward
// until fmaf(q, scale, origin) -- the device decode -- contains [a, b].
BVH_HD void quantize_axis(float origin, float scale, float a, float b, uint8_t& qlo, uint8_t& qhi) {
    const double fl = floor(((double)a - (double)origin) / (double)scale);
    const double fh = ceil(((double)b - (double)origin) / (double)scale);
    double tl = (fl < 255.0) ? fl : 255.0;
    tl = (0.0 < tl) ? tl : 0.0;
    double th = (fh < 255.0) ? fh : 255.0;
    th = (0.0 < th) ? th : 0.0;
    int lo = (int)tl, hi = (int)th;
    while (lo > 0 && fmaf((float)lo, scale, origin) > a) lo--;
    while (hi < 255 && fmaf((float)hi, scale, origin) < b) hi++;
    qlo = (uint8_t)lo;
    qhi = (uint8_t)hi;
}

}  // namespace bvhr
}  // namespace sheen
