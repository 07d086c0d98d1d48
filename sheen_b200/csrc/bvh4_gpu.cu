// bvh4_gpu.cu -- the wavefront form's triangle BVH4, built on the device.
//
// Same algorithm and the same arithmetic (bvh4_rules.h) as the host builder
// (bvh4.cpp), so both produce byte-identical node and triangle arrays:
//   1. triangle boxes of the subset, root box and root centroid box;
//   2. large nodes (more than kSmall triangles), one tree level per pass:
//      binned SAH (16 bins per axis over the centroid box) counted in
//      shared memory per 4096-triangle chunk and merged with atomics,
//      split chosen by one warp per node, stable partition by a scan over
//      the chunks in order;
//   3. small nodes: one block builds the whole subtree in shared memory,
//      continuing with the smaller child and stacking the larger;
//   4. collapse to 4-wide nodes breadth first, one level per pass (the
//      host's greedy rule: open the inner child of largest area until there
//      are four), child boxes quantised outward in the node's frame, and the
//      triangles written in leaf order.
// Node numbering of the intermediate binary tree differs from the host's;
// the collapse walks the tree structure only, so the output does not.
// Min/max reductions run as integer atomics on an order-preserving encoding
// of the floats; they are exact, so reduction order does not matter.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "bvh4_rules.h"
#include "engine.h"

namespace sheen {
namespace bvhg {

using namespace bvhr;

constexpr int kSmall = 1024;                      // subtree size built by one block
constexpr int kSmallThreads = 128;
constexpr int kSmallPer = kSmall / kSmallThreads;
constexpr int kChunk = 4096;                      // triangles per block in the large passes
constexpr int kChunkThreads = 256;
constexpr int kChunkPer = kChunk / kChunkThreads;
constexpr int kBinWords = 13;                     // count, box lo/hi, centroid lo/hi
constexpr int kNodeBins = 3 * kBins * kBinWords;
constexpr int kMaxLargeLevels = 4096;

__device__ __forceinline__ int ford(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float funord(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// Initial value of word w of a bin (count 0, empty boxes).
__device__ __forceinline__ int bin_init(int w) {
    const int k = w % kBinWords;
    if (k == 0) return 0;
    const bool is_lo = (k >= 1 && k <= 3) || (k >= 7 && k <= 9);
    return ford(is_lo ? FLT_MAX : -FLT_MAX);
}

// Binary node of the build.
struct __align__(16) BNode {
    float lo[3], hi[3];     // box of the triangle boxes
    float clo[3], chi[3];   // box of the triangle centroids
    int first, count;       // triangle range in idx
    int left, right;        // children, -1 for a leaf
};
static_assert(sizeof(BNode) == 64, "BNode is 64 bytes");

__device__ __forceinline__ void add_to_bin(int* B, const float l[3], const float h[3], const float c[3]) {
    atomicAdd(B, 1);
#pragma unroll
    for (int q = 0; q < 3; q++) {
        atomicMin(B + 1 + q, ford(l[q]));
        atomicMax(B + 4 + q, ford(h[q]));
        atomicMin(B + 7 + q, ford(c[q]));
        atomicMax(B + 10 + q, ford(c[q]));
    }
}

// Adds each active lane's triangle (box l, h, centroid c) to bin b[a] of
// every axis a with axis_on[a] (bins of axis a start at A + a * kBins *
// kBinWords).  On an axis where all active lanes of the warp share one bin
// the warp reduces first and one lane adds the result: mesh order puts runs
// of neighbouring triangles into the same bin, where one atomic per lane on
// the same words serialises.  Integer min / max of the ordered keys give the
// same words as the per-lane atomics.  Called by all 32 lanes with the same
// axis_on.
__device__ __forceinline__ void add_to_bins_warp(int* A, const int b[3], bool act, const bool axis_on[3],
                                                 const float l[3], const float h[3], const float c[3]) {
    const unsigned full = 0xffffffffu;
    const unsigned active = __ballot_sync(full, act);
    if (!active) return;
    const int src = __ffs(active) - 1;
    bool uni[3];
    bool any_uni = false;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const int b0 = __shfl_sync(full, b[a], src);
        uni[a] = axis_on[a] && __all_sync(full, !act || b[a] == b0);
        any_uni |= uni[a];
        if (axis_on[a] && !uni[a] && act) add_to_bin(A + (a * kBins + b[a]) * kBinWords, l, h, c);
    }
    if (!any_uni) return;
    int k[12];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        k[q] = act ? ford(l[q]) : INT_MAX;
        k[3 + q] = act ? ford(h[q]) : INT_MIN;
        k[6 + q] = act ? ford(c[q]) : INT_MAX;
        k[9 + q] = act ? ford(c[q]) : INT_MIN;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 12; q++) {
            const int v = __shfl_xor_sync(full, k[q], o);
            k[q] = (q < 3 || (q >= 6 && q < 9)) ? min(k[q], v) : max(k[q], v);
        }
    }
    if ((threadIdx.x & 31) == src) {
        const int cnt = __popc(active);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (!uni[a]) continue;
            int* B = A + (a * kBins + b[a]) * kBinWords;
            atomicAdd(B, cnt);
#pragma unroll
            for (int q = 0; q < 3; q++) {
                atomicMin(B + 1 + q, k[q]);
                atomicMax(B + 4 + q, k[3 + q]);
                atomicMin(B + 7 + q, k[6 + q]);
                atomicMax(B + 10 + q, k[9 + q]);
            }
        }
    }
}

// add_to_bin without the centroid words (1 + 6 atomics): for bins whose
// centroid bounds nobody reads (the warp-built subtrees, which take each
// node's bounds from warp reductions; axis_best_bins reads count and box).
__device__ __forceinline__ void add_to_bin_box(int* B, const float l[3], const float h[3]) {
    atomicAdd(B, 1);
#pragma unroll
    for (int q = 0; q < 3; q++) {
        atomicMin(B + 1 + q, ford(l[q]));
        atomicMax(B + 4 + q, ford(h[q]));
    }
}

// Union of bins [b0, b1] of one axis into box/centroid box; returns the count.
__device__ __forceinline__ int bin_union(const int* A, int b0, int b1, float lo[3], float hi[3], float clo[3],
                                         float chi[3]) {
    int n = 0;
    for (int q = 0; q < 3; q++) { lo[q] = FLT_MAX; hi[q] = -FLT_MAX; clo[q] = FLT_MAX; chi[q] = -FLT_MAX; }
    for (int i = b0; i <= b1; i++) {
        const int* b = A + i * kBinWords;
        n += b[0];
        for (int q = 0; q < 3; q++) {
            lo[q] = fminf(lo[q], funord(b[1 + q]));
            hi[q] = fmaxf(hi[q], funord(b[4 + q]));
            clo[q] = fminf(clo[q], funord(b[7 + q]));
            chi[q] = fmaxf(chi[q], funord(b[10 + q]));
        }
    }
    return n;
}

// Best split over the bins of a node, computed by one warp: for each axis,
// lanes 0..15 hold one bin each, shuffle scans give every lane the union of
// the bins up to it (left side) and from it on (right side), lane s prices
// the split after bin s.  The result is candidate axis * 15 + split with the
// lowest cost, ties to the lowest index (the host's strict "<" in candidate
// order), or INT_MAX when no split qualifies (flat axes or an empty side).
// Every lane gets the result.  Min/max unions are exact and the counts are
// integers, so the scan order does not change any value.
// One axis of warp_best, from that axis's 16 bins A: the lowest-cost split
// (ties to the lower split) as candidate a * 15 + split, or FLT_MAX /
// INT_MAX.  ext is the axis's centroid extent.
__device__ __forceinline__ void axis_best_bins(const int* A, float ext, int a, float& best_cost, int& best) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    best_cost = FLT_MAX;
    best = INT_MAX;
    {
        if (!(ext > 0.0f)) return;
        int lc = 0;
        float l0[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, l1[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        if (lane < kBins) {
            const int* b = A + lane * kBinWords;
            lc = b[0];
            for (int q = 0; q < 3; q++) { l0[q] = funord(b[1 + q]); l1[q] = funord(b[4 + q]); }
        }
        int rc = lc;
        float r0[3] = {l0[0], l0[1], l0[2]}, r1[3] = {l1[0], l1[1], l1[2]};
        for (int o = 1; o < kBins; o <<= 1) {
            const int cu = __shfl_up_sync(full, lc, o), cd = __shfl_down_sync(full, rc, o);
            float u0[3], u1[3], d0[3], d1[3];
            for (int q = 0; q < 3; q++) {
                u0[q] = __shfl_up_sync(full, l0[q], o);
                u1[q] = __shfl_up_sync(full, l1[q], o);
                d0[q] = __shfl_down_sync(full, r0[q], o);
                d1[q] = __shfl_down_sync(full, r1[q], o);
            }
            if (lane >= o) {
                lc += cu;
                for (int q = 0; q < 3; q++) { l0[q] = fminf(l0[q], u0[q]); l1[q] = fmaxf(l1[q], u1[q]); }
            }
            if (lane + o < kBins) {
                rc += cd;
                for (int q = 0; q < 3; q++) { r0[q] = fminf(r0[q], d0[q]); r1[q] = fmaxf(r1[q], d1[q]); }
            }
        }
        // right side of the split after bin s = suffix starting at s + 1
        const int nrc = __shfl_down_sync(full, rc, 1);
        float n0[3], n1[3];
        for (int q = 0; q < 3; q++) {
            n0[q] = __shfl_down_sync(full, r0[q], 1);
            n1[q] = __shfl_down_sync(full, r1[q], 1);
        }
        float cost = FLT_MAX;
        int cand = INT_MAX;
        if (lane < kBins - 1 && lc > 0 && nrc > 0) {
            const float c = split_cost(area(l0[0], l0[1], l0[2], l1[0], l1[1], l1[2]), lc,
                                       area(n0[0], n0[1], n0[2], n1[0], n1[1], n1[2]), nrc);
            if (c < FLT_MAX) { cost = c; cand = a * (kBins - 1) + lane; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float oc = __shfl_xor_sync(full, cost, o);
            const int ob = __shfl_xor_sync(full, cand, o);
            if (oc < cost || (oc == cost && ob < cand)) { cost = oc; cand = ob; }
        }
        best_cost = cost;
        best = cand;
    }
}

__device__ __forceinline__ void axis_best(const int* bins, const float clo[3], const float chi[3], int a,
                                          float& best_cost, int& best) {
    axis_best_bins(bins + a * kBins * kBinWords, sub(chi[a], clo[a]), a, best_cost, best);
}

__device__ __forceinline__ void warp_best(const int* bins, const float clo[3], const float chi[3], float& best_cost,
                                          int& best) {
    best_cost = FLT_MAX;
    best = INT_MAX;
    for (int a = 0; a < 3; a++) {
        float c;
        int b;
        axis_best(bins, clo, chi, a, c, b);
        if (c < best_cost) { best_cost = c; best = b; }   // earlier axes win ties
    }
}

// ---- 1. triangle boxes ----------------------------------------------------

__global__ void k_init_ord(int* ord, int n12) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n12) {
        const int k = i % 12;
        ord[i] = ford((k < 3 || (k >= 6 && k < 9)) ? FLT_MAX : -FLT_MAX);
    }
}

// ord layout per record: lo[3], hi[3], clo[3], chi[3]
__global__ void __launch_bounds__(256) k_prep(const Triangle* __restrict__ tris, const int* __restrict__ subset, int n,
                                              float4* __restrict__ plo, float4* __restrict__ phi,
                                              int* __restrict__ idx, int* __restrict__ root_ord) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Triangle& t = tris[subset ? subset[i] : i];
        const float v0[3] = {t.v0.x, t.v0.y, t.v0.z}, v1[3] = {t.v1.x, t.v1.y, t.v1.z},
                    v2[3] = {t.v2.x, t.v2.y, t.v2.z};
        float bl[3], bh[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            bl[k] = canon(fminf(fminf(fminf(FLT_MAX, v0[k]), v1[k]), v2[k]));
            bh[k] = canon(fmaxf(fmaxf(fmaxf(-FLT_MAX, v0[k]), v1[k]), v2[k]));
            const float c = centroid(bl[k], bh[k]);
            lo[k] = fminf(lo[k], bl[k]); hi[k] = fmaxf(hi[k], bh[k]);
            clo[k] = fminf(clo[k], c); chi[k] = fmaxf(chi[k], c);
        }
        plo[i] = make_float4(bl[0], bl[1], bl[2], 0.0f);
        phi[i] = make_float4(bh[0], bh[1], bh[2], 0.0f);
        idx[i] = i;
    }
#pragma unroll
    for (int k = 0; k < 3; k++)
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            clo[k] = fminf(clo[k], __shfl_xor_sync(0xffffffffu, clo[k], o));
            chi[k] = fmaxf(chi[k], __shfl_xor_sync(0xffffffffu, chi[k], o));
        }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; k++) {
            atomicMin(&root_ord[k], ford(lo[k]));
            atomicMax(&root_ord[3 + k], ford(hi[k]));
            atomicMin(&root_ord[6 + k], ford(clo[k]));
            atomicMax(&root_ord[9 + k], ford(chi[k]));
        }
    }
}

__global__ void k_root(const int* __restrict__ root_ord, int n, BNode* __restrict__ nodes) {
    if (threadIdx.x != 0) return;
    BNode r;
    for (int k = 0; k < 3; k++) {
        r.lo[k] = funord(root_ord[k]);
        r.hi[k] = funord(root_ord[3 + k]);
        r.clo[k] = funord(root_ord[6 + k]);
        r.chi[k] = funord(root_ord[9 + k]);
    }
    r.first = 0;
    r.count = n;
    r.left = r.right = -1;
    nodes[0] = r;
}

// ---- 2. large nodes --------------------------------------------------------

// Node slot of chunk c: the last j with chunk_base[j] <= c.
__device__ __forceinline__ int chunk_node(const int* __restrict__ chunk_base, int m, int c) {
    int lo = 0, hi = m - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (chunk_base[mid] <= c) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_init_bins(int* __restrict__ bins, int words) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < words) bins[i] = bin_init(i % kNodeBins);
}

__global__ void __launch_bounds__(kChunkThreads) k_bin_large(const int* __restrict__ work, const int* __restrict__ chunk_base,
                                                             int m, const BNode* __restrict__ nodes,
                                                             const float4* __restrict__ plo, const float4* __restrict__ phi,
                                                             const int* __restrict__ idx, int* __restrict__ gbins) {
    __shared__ int sb[kNodeBins];
    const int c = blockIdx.x;
    const int j = chunk_node(chunk_base, m, c);
    const BNode nd = nodes[work[j]];
    const int start = nd.first + (c - chunk_base[j]) * kChunk;
    const int end = min(start + kChunk, nd.first + nd.count);
    for (int w = threadIdx.x; w < kNodeBins; w += kChunkThreads) sb[w] = bin_init(w);
    __syncthreads();
    float kk[3];
    bool on[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float ext = sub(nd.chi[a], nd.clo[a]);
        on[a] = ext > 0.0f;
        kk[a] = on[a] ? bin_scale(ext) : 0.0f;
    }
    for (int base = start; base < end; base += kChunkThreads) {   // uniform trip count per warp
        const int pos = base + threadIdx.x;
        const bool act = pos < end;
        float l[3] = {0.0f, 0.0f, 0.0f}, h[3] = {0.0f, 0.0f, 0.0f};
        if (act) {
            const int p = idx[pos];
            const float4 L = plo[p], H = phi[p];
            l[0] = L.x; l[1] = L.y; l[2] = L.z;
            h[0] = H.x; h[1] = H.y; h[2] = H.z;
        }
        const float cc[3] = {centroid(l[0], h[0]), centroid(l[1], h[1]), centroid(l[2], h[2])};
        int b[3];
#pragma unroll
        for (int a = 0; a < 3; a++) b[a] = on[a] ? bin_of(cc[a], nd.clo[a], kk[a]) : 0;
        add_to_bins_warp(sb, b, act, on, l, h, cc);
    }
    __syncthreads();
    int* G = gbins + (size_t)j * kNodeBins;
    for (int w = threadIdx.x; w < kNodeBins; w += kChunkThreads) {
        const int v = sb[w];
        const int k = w % kBinWords;
        if (k == 0) {
            if (v) atomicAdd(&G[w], v);
        } else if (v != bin_init(w)) {
            const bool is_lo = (k >= 1 && k <= 3) || (k >= 7 && k <= 9);
            if (is_lo) atomicMin(&G[w], v);
            else atomicMax(&G[w], v);
        }
    }
}

// split[j] = {axis or -1 (list split in half), bin, left count, 0}
__global__ void __launch_bounds__(32) k_split_large(const int* __restrict__ work, int m, int next_id,
                                                    BNode* __restrict__ nodes, const int* __restrict__ gbins,
                                                    int4* __restrict__ split, int2* __restrict__ child_fc) {
    const int j = blockIdx.x;
    const int id = work[j];
    const BNode nd = nodes[id];
    const int* B = gbins + (size_t)j * kNodeBins;
    float best_cost;
    int best;
    warp_best(B, nd.clo, nd.chi, best_cost, best);
    if (threadIdx.x != 0) return;
    const int n = nd.count;                  // > kSmall > kMaxLeaf: never a leaf
    const int left_id = next_id + 2 * j, right_id = left_id + 1;
    BNode L, R;
    int nleft;
    if (best != INT_MAX) {
        const int a = best / (kBins - 1), s = best % (kBins - 1);
        const int* A = B + a * kBins * kBinWords;
        nleft = bin_union(A, 0, s, L.lo, L.hi, L.clo, L.chi);
        bin_union(A, s + 1, kBins - 1, R.lo, R.hi, R.clo, R.chi);
        split[j] = make_int4(a, s, nleft, 0);
    } else {
        nleft = n / 2;                          // bounds filled in by k_list_split_bounds
        for (int q = 0; q < 3; q++) {
            L.lo[q] = R.lo[q] = FLT_MAX; L.hi[q] = R.hi[q] = -FLT_MAX;
            L.clo[q] = R.clo[q] = FLT_MAX; L.chi[q] = R.chi[q] = -FLT_MAX;
        }
        split[j] = make_int4(-1, 0, nleft, 0);
    }
    L.first = nd.first; L.count = nleft; L.left = L.right = -1;
    R.first = nd.first + nleft; R.count = n - nleft; R.left = R.right = -1;
    nodes[left_id] = L;
    nodes[right_id] = R;
    nodes[id].left = left_id;
    nodes[id].right = right_id;
    child_fc[2 * j] = make_int2(L.first, L.count);
    child_fc[2 * j + 1] = make_int2(R.first, R.count);
}

__device__ __forceinline__ bool goes_left_large(const BNode& nd, int4 sp, float k_axis, int pos, int p,
                                                const float4* __restrict__ plo, const float4* __restrict__ phi) {
    if (sp.x < 0) return pos - nd.first < sp.z;
    const float4 L = plo[p], H = phi[p];
    const float lo = sp.x == 0 ? L.x : (sp.x == 1 ? L.y : L.z);
    const float hi = sp.x == 0 ? H.x : (sp.x == 1 ? H.y : H.z);
    return bin_of(centroid(lo, hi), nd.clo[sp.x], k_axis) <= sp.y;
}

__device__ __forceinline__ float split_scale(const BNode& nd, int4 sp) {
    return sp.x >= 0 ? bin_scale(sub(nd.chi[sp.x], nd.clo[sp.x])) : 0.0f;
}

// Bounds of the two halves of a list split (every centroid equal): rare.
__global__ void __launch_bounds__(kChunkThreads) k_list_split_bounds(const int* __restrict__ work, const int* __restrict__ chunk_base,
                                                                     int m, const BNode* __restrict__ nodes,
                                                                     const int4* __restrict__ split,
                                                                     const float4* __restrict__ plo,
                                                                     const float4* __restrict__ phi,
                                                                     const int* __restrict__ idx, int* __restrict__ child_ord) {
    const int c = blockIdx.x;
    const int j = chunk_node(chunk_base, m, c);
    const int4 sp = split[j];
    if (sp.x >= 0) return;
    const BNode nd = nodes[work[j]];
    const int start = nd.first + (c - chunk_base[j]) * kChunk;
    const int end = min(start + kChunk, nd.first + nd.count);
    for (int pos = start + threadIdx.x; pos < end; pos += kChunkThreads) {
        const int p = idx[pos];
        const float4 L = plo[p], H = phi[p];
        const float l[3] = {L.x, L.y, L.z}, h[3] = {H.x, H.y, H.z};
        int* o = child_ord + (size_t)(2 * j + (pos - nd.first < sp.z ? 0 : 1)) * 12;
        for (int q = 0; q < 3; q++) {
            const float cc = centroid(l[q], h[q]);
            atomicMin(&o[q], ford(l[q]));
            atomicMax(&o[3 + q], ford(h[q]));
            atomicMin(&o[6 + q], ford(cc));
            atomicMax(&o[9 + q], ford(cc));
        }
    }
}

__global__ void k_list_split_write(int m, int next_id, const int4* __restrict__ split, const int* __restrict__ child_ord,
                                   BNode* __restrict__ nodes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;   // child slot 0 .. 2m-1
    if (i >= 2 * m || split[i / 2].x >= 0) return;
    BNode& c = nodes[next_id + i];
    const int* o = child_ord + (size_t)i * 12;
    for (int q = 0; q < 3; q++) {
        c.lo[q] = funord(o[q]);
        c.hi[q] = funord(o[3 + q]);
        c.clo[q] = funord(o[6 + q]);
        c.chi[q] = funord(o[9 + q]);
    }
}

__global__ void __launch_bounds__(kChunkThreads) k_part_count(const int* __restrict__ work, const int* __restrict__ chunk_base,
                                                              int m, const BNode* __restrict__ nodes,
                                                              const int4* __restrict__ split,
                                                              const float4* __restrict__ plo,
                                                              const float4* __restrict__ phi,
                                                              const int* __restrict__ idx, int* __restrict__ chunk_left) {
    typedef cub::BlockReduce<int, kChunkThreads> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const int c = blockIdx.x;
    const int j = chunk_node(chunk_base, m, c);
    const BNode nd = nodes[work[j]];
    const int4 sp = split[j];
    const float k_axis = split_scale(nd, sp);
    const int start = nd.first + (c - chunk_base[j]) * kChunk;
    const int end = min(start + kChunk, nd.first + nd.count);
    int cnt = 0;
    for (int pos = start + threadIdx.x; pos < end; pos += kChunkThreads)
        cnt += goes_left_large(nd, sp, k_axis, pos, idx[pos], plo, phi) ? 1 : 0;
    const int total = Reduce(tmp).Sum(cnt);
    if (threadIdx.x == 0) chunk_left[c] = total;
}

// Stable scatter of each chunk into its node's left / right ranges of tmp.
__global__ void __launch_bounds__(kChunkThreads) k_part_scatter(const int* __restrict__ work, const int* __restrict__ chunk_base,
                                                                int m, const BNode* __restrict__ nodes,
                                                                const int4* __restrict__ split,
                                                                const float4* __restrict__ plo,
                                                                const float4* __restrict__ phi,
                                                                const int* __restrict__ idx,
                                                                const int* __restrict__ chunk_off, int* __restrict__ tmp,
                                                                int* __restrict__ err) {
    typedef cub::BlockScan<int, kChunkThreads> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;
    const int c = blockIdx.x;
    const int j = chunk_node(chunk_base, m, c);
    const BNode nd = nodes[work[j]];
    const int4 sp = split[j];
    const float k_axis = split_scale(nd, sp);
    const int start = nd.first + (c - chunk_base[j]) * kChunk;
    const int end = min(start + kChunk, nd.first + nd.count);
    const int left_before = chunk_off[c] - chunk_off[chunk_base[j]];
    const int right_before = (start - nd.first) - left_before;
    int p[kChunkPer];
    bool f[kChunkPer];
    int cnt = 0;
    const int t0 = start + threadIdx.x * kChunkPer;
#pragma unroll
    for (int e = 0; e < kChunkPer; e++) {
        const int pos = t0 + e;
        f[e] = false;
        p[e] = 0;
        if (pos < end) {
            p[e] = idx[pos];
            f[e] = goes_left_large(nd, sp, k_axis, pos, p[e], plo, phi);
            cnt += f[e] ? 1 : 0;
        }
    }
    int lpos;
    Scan(scan_tmp).ExclusiveSum(cnt, lpos);
    int rpos = min(threadIdx.x * kChunkPer, end - start) - lpos;
    lpos += nd.first + left_before;
    rpos += nd.first + sp.z + right_before;
    // Both sides stay inside the node (the bins and this pass classify with
    // the same function); a position outside it is recorded, not written.
    const int lend = nd.first + sp.z, rend = nd.first + nd.count;
#pragma unroll
    for (int e = 0; e < kChunkPer; e++) {
        if (t0 + e >= end) break;
        if (f[e]) {
            if (lpos < lend) tmp[lpos++] = p[e];
            else *err = 2;
        } else {
            if (rpos >= lend && rpos < rend) tmp[rpos++] = p[e];
            else *err = 2;
        }
    }
}

__global__ void k_copy_back(const int* __restrict__ work, const int* __restrict__ chunk_base, int m,
                            const BNode* __restrict__ nodes, const int* __restrict__ tmp, int* __restrict__ idx) {
    const int c = blockIdx.x;
    const int j = chunk_node(chunk_base, m, c);
    const BNode nd = nodes[work[j]];
    const int start = nd.first + (c - chunk_base[j]) * kChunk;
    const int end = min(start + kChunk, nd.first + nd.count);
    for (int pos = start + threadIdx.x; pos < end; pos += blockDim.x) idx[pos] = tmp[pos];
}

// ---- 3. small subtrees -----------------------------------------------------

// ---- subtrees of at most 32 triangles: one warp each ----------------------
//
// One triangle per lane; every sub-node's box and centroid box are warp
// min / max reductions over its triangles (exactly the unions of its bins),
// bins live in a per-warp array of one axis, partitions are ballots.  The
// decisions are the block path's, on the same values.

constexpr int kTiny = 32;
constexpr int kTinyCap = 128;     // tiny subtree roots listed per block (packed words)
constexpr int kTinyStack = 8;     // smaller child first: depth <= log2(32) + 1
constexpr int kAxisWords = kBins * kBinWords;

struct TinyFrame {
    unsigned short first, count;  // range in the block's permutation
    int id;                       // binary node id
};

__device__ __forceinline__ float warp_min(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Builds the subtree of `root` (count <= 32) with the calling warp.  perm:
// the block's permutation of local triangle slots; box: their boxes
// (6 x kSmall); bins: this warp's kAxisWords ints; stack: this warp's
// kTinyStack frames; next_id: the block's id counter.
__device__ void build_tiny(TinyFrame root, float node_cost, unsigned short* __restrict__ perm,
                           const float (*box)[kSmall], int gfirst,
                           int* __restrict__ bins, TinyFrame* __restrict__ stack, int* next_id,
                           BNode* __restrict__ nodes, int* __restrict__ err) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int sp = 0;
    TinyFrame cur = root;
    while (true) {
        const int m = cur.count, first = cur.first;
        const bool act = lane < m;
        const int s = act ? perm[first + lane] : 0;
        float l[3], h[3], c[3];
        for (int q = 0; q < 3; q++) {
            l[q] = act ? box[q][s] : FLT_MAX;
            h[q] = act ? box[3 + q][s] : -FLT_MAX;
            c[q] = act ? centroid(l[q], h[q]) : FLT_MAX;
        }
        float lo[3], hi[3], clo[3], chi[3];
        for (int q = 0; q < 3; q++) {
            lo[q] = warp_min(l[q]);
            hi[q] = warp_max(h[q]);
            clo[q] = warp_min(c[q]);
            chi[q] = warp_max(act ? c[q] : -FLT_MAX);
        }
        bool leaf = m <= 2;
        int best = -1;
        if (!leaf) {
            float bc = FLT_MAX;
            int bi = INT_MAX;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const float ext = sub(chi[a], clo[a]);
                if (!(ext > 0.0f)) continue;
                for (int w = lane; w < kAxisWords; w += 32) bins[w] = bin_init(w);
                __syncwarp();
                if (act) add_to_bin_box(bins + bin_of(c[a], clo[a], bin_scale(ext)) * kBinWords, l, h);
                __syncwarp();
                float cost;
                int cand;
                axis_best_bins(bins, ext, a, cost, cand);
                if (cost < bc) { bc = cost; bi = cand; }   // earlier axes win ties
                __syncwarp();
            }
            best = bi == INT_MAX ? -1 : bi;
            const float pa = area(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
            if (best < 0 || (m <= kMaxLeaf && leaf_wins(pa, m, bc, node_cost))) leaf = m <= kMaxLeaf;
        }
        BNode o;
        for (int q = 0; q < 3; q++) { o.lo[q] = lo[q]; o.hi[q] = hi[q]; o.clo[q] = clo[q]; o.chi[q] = chi[q]; }
        o.first = gfirst + first;
        o.count = m;
        if (leaf) {
            o.left = o.right = -1;
            if (lane == 0) nodes[cur.id] = o;
            if (sp == 0) break;
            cur = stack[--sp];
            continue;
        }
        // stable partition by ballot
        const int axis = best >= 0 ? best / (kBins - 1) : -1;
        const int sbin = best >= 0 ? best % (kBins - 1) : 0;
        const float ca = axis == 0 ? c[0] : (axis == 1 ? c[1] : c[2]);
        const float la = axis == 0 ? clo[0] : (axis == 1 ? clo[1] : clo[2]);
        const float ha = axis == 0 ? chi[0] : (axis == 1 ? chi[1] : chi[2]);
        bool f = false;
        if (act) f = axis >= 0 ? bin_of(ca, la, bin_scale(sub(ha, la))) <= sbin : lane < m / 2;
        const unsigned left_mask = __ballot_sync(full, act && f);
        const int nleft = __popc(left_mask);
        const int before = __popc(left_mask & ((1u << lane) - 1u));
        __syncwarp();
        if (act) perm[first + (f ? before : nleft + (lane - before))] = (unsigned short)s;
        __syncwarp();
        int mid = first + (axis >= 0 ? nleft : m / 2);
        if (mid == first || mid == first + m) mid = first + m / 2;
        int base = 0;
        if (lane == 0) base = atomicAdd(next_id, 2);
        base = __shfl_sync(full, base, 0);
        o.left = base;
        o.right = base + 1;
        if (lane == 0) nodes[cur.id] = o;
        TinyFrame L, R;
        L.first = (unsigned short)first; L.count = (unsigned short)(mid - first); L.id = base;
        R.first = (unsigned short)mid; R.count = (unsigned short)(first + m - mid); R.id = base + 1;
        if (sp >= kTinyStack) {
            if (lane == 0) *err = 3;
            break;
        }
        if (R.count >= L.count) { stack[sp++] = R; cur = L; }
        else { stack[sp++] = L; cur = R; }
    }
    __syncwarp();
}

struct SmallFrame {
    int first, count, id, pad;
    float lo[3], hi[3], clo[3], chi[3];
};

// Smaller child first: a frame is pushed only when descending into a child
// of at most half its parent's count, so the stack holds at most
// log2(kSmall) = 10 frames.
constexpr int kSmallStack = 16;

// List word of a tiny subtree root: first (10 bits) | count - 1 (5 bits) |
// node id - the block's first id (11 bits; 2047 for the block's root).
static_assert(kSmall <= 1024 && kTiny <= 32 && 2 * kSmall - 2 < 2047, "tiny list word");

__global__ void __launch_bounds__(kSmallThreads, 6) k_small(const int* __restrict__ list, const int* __restrict__ id_base,
                                                         const float4* __restrict__ plo, const float4* __restrict__ phi,
                                                         int* __restrict__ idx, BNode* __restrict__ nodes,
                                                         int* __restrict__ err, float node_cost) {
    __shared__ float s_box[6][kSmall];
    __shared__ int s_pid[kSmall];
    __shared__ unsigned short s_perm[kSmall];
    __shared__ __align__(16) unsigned short s_tmp[kSmall];
    __shared__ int s_bins[kNodeBins];
    __shared__ int s_cb[24];
    __shared__ __align__(16) SmallFrame s_stack[kSmallStack];
    __shared__ SmallFrame s_cur;
    __shared__ unsigned s_tiny[kTinyCap];
    __shared__ int s_sp, s_next, s_done, s_best, s_leaf, s_ntiny;
    __shared__ float s_axis_cost[3];
    __shared__ int s_axis_cand[3];
    typedef cub::BlockScan<int, kSmallThreads> Scan;
    __shared__ typename Scan::TempStorage s_scan;

    const int tid = threadIdx.x;
    const int root = list[blockIdx.x];
    const int gfirst = nodes[root].first, n0 = nodes[root].count;
    for (int k = tid; k < n0; k += kSmallThreads) {
        const int p = idx[gfirst + k];
        const float4 l = plo[p], h = phi[p];
        s_box[0][k] = l.x; s_box[1][k] = l.y; s_box[2][k] = l.z;
        s_box[3][k] = h.x; s_box[4][k] = h.y; s_box[5][k] = h.z;
        s_pid[k] = p;
        s_perm[k] = (unsigned short)k;
    }
    if (tid == 0) {
        const BNode r = nodes[root];
        s_cur.first = 0; s_cur.count = n0; s_cur.id = root; s_cur.pad = 0;
        for (int q = 0; q < 3; q++) {
            s_cur.lo[q] = r.lo[q]; s_cur.hi[q] = r.hi[q]; s_cur.clo[q] = r.clo[q]; s_cur.chi[q] = r.chi[q];
        }
        s_sp = 0;
        s_next = id_base[blockIdx.x];
        s_done = 0;
        s_ntiny = 0;
    }
    __syncthreads();
    while (true) {
        const SmallFrame cur = s_cur;
        const int ntiny = s_ntiny;
        __syncthreads();   // every thread has its copies before thread 0 may replace them
        const int n = cur.count;
        if (n <= kTiny && ntiny < kTinyCap) {
            // left to one warp after the block phase (a full list falls back
            // to the block path below)
            if (tid == 0) {
                const unsigned rel = cur.id == root ? 2047u : (unsigned)(cur.id - id_base[blockIdx.x]);
                s_tiny[ntiny] = (unsigned)cur.first | (unsigned)(n - 1) << 10 | rel << 15;
                s_ntiny = ntiny + 1;
                if (s_sp == 0) s_done = 1;
                else s_cur = s_stack[--s_sp];
            }
            __syncthreads();
            if (s_done) break;
            continue;
        }
        bool leaf = n <= 2;
        if (!leaf) {
            for (int w = tid; w < kNodeBins; w += kSmallThreads) s_bins[w] = bin_init(w);
            __syncthreads();
            float kk[3];
            bool on[3];
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const float ext = sub(cur.chi[a], cur.clo[a]);
                on[a] = ext > 0.0f;
                kk[a] = on[a] ? bin_scale(ext) : 0.0f;
            }
            for (int k0 = 0; k0 < n; k0 += kSmallThreads) {   // uniform trip count per warp
                const int k = k0 + tid;
                const bool act = k < n;
                const int s = act ? s_perm[cur.first + k] : 0;
                const float l[3] = {s_box[0][s], s_box[1][s], s_box[2][s]};
                const float h[3] = {s_box[3][s], s_box[4][s], s_box[5][s]};
                const float cc[3] = {centroid(l[0], h[0]), centroid(l[1], h[1]), centroid(l[2], h[2])};
                int b[3];
#pragma unroll
                for (int a = 0; a < 3; a++) b[a] = on[a] ? bin_of(cc[a], cur.clo[a], kk[a]) : 0;
                add_to_bins_warp(s_bins, b, act, on, l, h, cc);
            }
            __syncthreads();
            // one warp per axis, then thread 0 takes the lowest cost (ties
            // to the lower axis, as warp_best)
            const int warp = tid >> 5;
            if (warp < 3) {
                float c;
                int b;
                axis_best(s_bins, cur.clo, cur.chi, warp, c, b);
                if ((tid & 31) == 0) { s_axis_cost[warp] = c; s_axis_cand[warp] = b; }
            }
            __syncthreads();
            {
                if (tid == 0) {
                    float bc = FLT_MAX;
                    int bi = INT_MAX;
                    for (int a = 0; a < 3; a++)
                        if (s_axis_cost[a] < bc) { bc = s_axis_cost[a]; bi = s_axis_cand[a]; }
                    const int best = bi == INT_MAX ? -1 : bi;
                    const float pa = area(cur.lo[0], cur.lo[1], cur.lo[2], cur.hi[0], cur.hi[1], cur.hi[2]);
                    int lf = 0;
                    if (best < 0 || (n <= kMaxLeaf && leaf_wins(pa, n, bc, node_cost))) {
                        if (n <= kMaxLeaf) lf = 1;
                    }
                    s_best = best;
                    s_leaf = lf;
                }
            }
            __syncthreads();
            leaf = s_leaf != 0;
        }
        if (leaf) {
            if (tid == 0) {
                BNode o;
                for (int q = 0; q < 3; q++) {
                    o.lo[q] = cur.lo[q]; o.hi[q] = cur.hi[q]; o.clo[q] = cur.clo[q]; o.chi[q] = cur.chi[q];
                }
                o.first = gfirst + cur.first;
                o.count = n;
                o.left = o.right = -1;
                nodes[cur.id] = o;
                if (s_sp == 0) s_done = 1;
                else s_cur = s_stack[--s_sp];
            }
            __syncthreads();
            if (s_done) break;
            continue;
        }
        // Stable partition of s_perm[cur.first, cur.first + n).
        const int best = s_best;
        const int axis = best >= 0 ? best / (kBins - 1) : -1;
        const int sbin = best >= 0 ? best % (kBins - 1) : 0;
        const float k_axis = axis >= 0 ? bin_scale(sub(cur.chi[axis], cur.clo[axis])) : 0.0f;
        bool f[kSmallPer];
        int cnt = 0;
#pragma unroll
        for (int e = 0; e < kSmallPer; e++) {
            const int k = tid * kSmallPer + e;
            f[e] = false;
            if (k < n) {
                if (axis >= 0) {
                    const int s = s_perm[cur.first + k];
                    f[e] = bin_of(centroid(s_box[axis][s], s_box[3 + axis][s]), cur.clo[axis], k_axis) <= sbin;
                } else {
                    f[e] = k < n / 2;
                }
                cnt += f[e] ? 1 : 0;
            }
        }
        int lpos, nleft;
        Scan(s_scan).ExclusiveSum(cnt, lpos, nleft);
        int rpos = min(tid * kSmallPer, n) - lpos;
#pragma unroll
        for (int e = 0; e < kSmallPer; e++) {
            const int k = tid * kSmallPer + e;
            if (k >= n) break;
            const unsigned short v = s_perm[cur.first + k];
            if (f[e]) s_tmp[cur.first + lpos++] = v;
            else s_tmp[cur.first + nleft + rpos++] = v;
        }
        __syncthreads();
        for (int k = tid; k < n; k += kSmallThreads) s_perm[cur.first + k] = s_tmp[cur.first + k];
        int mid = cur.first + (axis >= 0 ? nleft : n / 2);
        bool forced = false;
        if (mid == cur.first || mid == cur.first + n) { mid = cur.first + n / 2; forced = true; }
        const bool from_bins = axis >= 0 && !forced;
        if (!from_bins) {
            if (tid < 24) s_cb[tid] = ford(((tid % 12) < 3 || ((tid % 12) >= 6 && (tid % 12) < 9)) ? FLT_MAX : -FLT_MAX);
            __syncthreads();
            for (int k = tid; k < n; k += kSmallThreads) {
                const int s = s_perm[cur.first + k];
                int* o = s_cb + (cur.first + k < mid ? 0 : 12);
                for (int q = 0; q < 3; q++) {
                    const float lq = s_box[q][s], hq = s_box[3 + q][s], cq = centroid(lq, hq);
                    atomicMin(&o[q], ford(lq));
                    atomicMax(&o[3 + q], ford(hq));
                    atomicMin(&o[6 + q], ford(cq));
                    atomicMax(&o[9 + q], ford(cq));
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            SmallFrame L, R;
            L.first = cur.first; L.count = mid - cur.first; L.pad = 0;
            R.first = mid; R.count = cur.first + n - mid; R.pad = 0;
            if (from_bins) {
                const int* A = s_bins + axis * kBins * kBinWords;
                bin_union(A, 0, sbin, L.lo, L.hi, L.clo, L.chi);
                bin_union(A, sbin + 1, kBins - 1, R.lo, R.hi, R.clo, R.chi);
            } else {
                for (int q = 0; q < 3; q++) {
                    L.lo[q] = funord(s_cb[q]); L.hi[q] = funord(s_cb[3 + q]);
                    L.clo[q] = funord(s_cb[6 + q]); L.chi[q] = funord(s_cb[9 + q]);
                    R.lo[q] = funord(s_cb[12 + q]); R.hi[q] = funord(s_cb[15 + q]);
                    R.clo[q] = funord(s_cb[18 + q]); R.chi[q] = funord(s_cb[21 + q]);
                }
            }
            L.id = s_next;
            R.id = s_next + 1;
            s_next += 2;
            BNode o;
            for (int q = 0; q < 3; q++) {
                o.lo[q] = cur.lo[q]; o.hi[q] = cur.hi[q]; o.clo[q] = cur.clo[q]; o.chi[q] = cur.chi[q];
            }
            o.first = gfirst + cur.first;
            o.count = n;
            o.left = L.id;
            o.right = R.id;
            nodes[cur.id] = o;
            if (s_sp >= kSmallStack) {
                *err = 1;
                s_done = 1;
            } else if (R.count >= L.count) {
                s_stack[s_sp++] = R;
                s_cur = L;
            } else {
                s_stack[s_sp++] = L;
                s_cur = R;
            }
        }
        __syncthreads();
        if (s_done) break;
    }
    __syncthreads();
    {
        // Subtrees of at most kTiny triangles, one warp each.  The block
        // phase's bins (three warps) and partition buffer (the fourth) hold
        // the warps' bins, its frame stack their stacks.
        static_assert(3 * kAxisWords <= kNodeBins && kAxisWords * 4 <= (int)sizeof(s_tmp), "tiny bins fit");
        static_assert(4 * kTinyStack * sizeof(TinyFrame) <= sizeof(s_stack), "tiny stacks fit");
        static_assert(kSmallThreads == 128, "four warps");
        const int warp = tid >> 5;
        int* wbins = warp < 3 ? s_bins + warp * kAxisWords : reinterpret_cast<int*>(s_tmp);
        TinyFrame* wstack = reinterpret_cast<TinyFrame*>(s_stack) + warp * kTinyStack;
        const int nt = s_ntiny, id0 = id_base[blockIdx.x];
        for (int t = warp; t < nt; t += kSmallThreads / 32) {
            const unsigned w = s_tiny[t];
            TinyFrame f;
            f.first = (unsigned short)(w & 1023u);
            f.count = (unsigned short)(((w >> 10) & 31u) + 1u);
            const unsigned rel = w >> 15;
            f.id = rel == 2047u ? root : id0 + (int)rel;
            build_tiny(f, node_cost, s_perm, s_box, gfirst, wbins, wstack, &s_next, nodes, err);
        }
    }
    __syncthreads();
    for (int k = tid; k < n0; k += kSmallThreads) idx[gfirst + k] = s_pid[s_perm[k]];
    // Ids reserved for this subtree but not used (a tree with leaves of
    // several triangles has fewer than 2 n0 - 1 nodes) are marked empty
    // (count 0), so that passes over every id see only real nodes.
    const int id_end = id_base[blockIdx.x] + max(0, 2 * n0 - 2);
    for (int k = s_next + tid; k < id_end; k += kSmallThreads) {
        nodes[k].count = 0;
        nodes[k].first = 0;
        nodes[k].left = nodes[k].right = -1;
    }
}

// ---- 4. collapse to BVH4 ---------------------------------------------------

__device__ __forceinline__ float node_area(const BNode& c) {
    return area(c.lo[0], c.lo[1], c.lo[2], c.hi[0], c.hi[1], c.hi[2]);
}

__global__ void k_collapse_count(const int* __restrict__ level, int m, const BNode* __restrict__ nodes,
                                 int4* __restrict__ kids, int* __restrict__ nkids, int* __restrict__ ninner) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const int b = level[j];
    int k[4] = {-1, -1, -1, -1};
    int nk;
    const BNode nb = nodes[b];
    if (nb.left < 0) {
        k[0] = b;   // a leaf root: one node with one leaf child
        nk = 1;
    } else {
        k[0] = nb.left;
        k[1] = nb.right;
        nk = 2;
        while (nk < 4) {
            int pick = -1;
            float best = -1.0f;
            for (int q = 0; q < nk; q++) {
                const BNode& c = nodes[k[q]];
                if (c.left >= 0) {
                    const float ar = node_area(c);
                    if (ar > best) { best = ar; pick = q; }
                }
            }
            if (pick < 0) break;
            const int opened = k[pick];
            k[pick] = nodes[opened].left;
            k[nk++] = nodes[opened].right;
        }
    }
    int inner = 0;
    for (int q = 0; q < nk; q++) inner += nodes[k[q]].left >= 0 ? 1 : 0;
    kids[j] = make_int4(k[0], k[1], k[2], k[3]);
    nkids[j] = nk;
    ninner[j] = inner;
}

__global__ void k_collapse_emit(const int* __restrict__ level, int m, int base, const int4* __restrict__ kids,
                                const int* __restrict__ nkids, const int* __restrict__ off,
                                const BNode* __restrict__ nodes, dev::QNode4* __restrict__ out,
                                int* __restrict__ next_level) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= m) return;
    const int4 kv = kids[j];
    const int k[4] = {kv.x, kv.y, kv.z, kv.w};
    const int nk = nkids[j];
    float nlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, nhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int q = 0; q < nk; q++) {
        const BNode& c = nodes[k[q]];
        for (int a = 0; a < 3; a++) { nlo[a] = fminf(nlo[a], c.lo[a]); nhi[a] = fmaxf(nhi[a], c.hi[a]); }
    }
    float scale[3];
    uint32_t packed = (uint32_t)nk << 24;
    for (int a = 0; a < 3; a++) {
        const int e = frame_exponent(nlo[a], nhi[a]);
        scale[a] = ldexpf(1.0f, e);
        packed |= (uint32_t)(e + 127) << (8 * a);
    }
    uint8_t q6[6][4];
    for (int r = 0; r < 6; r++)
        for (int c = 0; c < 4; c++) q6[r][c] = 0;
    uint32_t child[4] = {0, 0, 0, 0};
    int r = 0;
    for (int q = 0; q < nk; q++) {
        const BNode& c = nodes[k[q]];
        for (int a = 0; a < 3; a++) quantize_axis(nlo[a], scale[a], c.lo[a], c.hi[a], q6[2 * a][q], q6[2 * a + 1][q]);
        if (c.left < 0) {
            child[q] = 0x80000000u | ((uint32_t)c.first << 3) | (uint32_t)(c.count - 1);
        } else {
            child[q] = (uint32_t)(base + m + off[j] + r);
            next_level[off[j] + r] = k[q];
            r++;
        }
    }
    auto word = [&](int row) {
        return (uint32_t)q6[row][0] | ((uint32_t)q6[row][1] << 8) | ((uint32_t)q6[row][2] << 16) |
               ((uint32_t)q6[row][3] << 24);
    };
    dev::QNode4 o;
    o.origin_exp = make_float4(nlo[0], nlo[1], nlo[2], __uint_as_float(packed));
    o.child = make_uint4(child[0], child[1], child[2], child[3]);
    o.qbox = make_uint4(word(0), word(1), word(2), word(3));
    o.qz = make_uint2(word(4), word(5));
    o.pad = make_uint2(0, 0);
    out[base + j] = o;
}

__global__ void k_emit_tris(const Triangle* __restrict__ tris, const int* __restrict__ subset,
                            const int* __restrict__ idx, int n, float4* __restrict__ out, bool vertices) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = idx[i];
    const int orig = subset ? subset[s] : s;
    const Triangle& t = tris[orig];
    out[3 * (size_t)i] = make_float4(t.v0.x, t.v0.y, t.v0.z, __int_as_float(orig));
    if (vertices) {
        out[3 * (size_t)i + 1] = make_float4(t.v1.x, t.v1.y, t.v1.z, 0.0f);
        out[3 * (size_t)i + 2] = make_float4(t.v2.x, t.v2.y, t.v2.z, 0.0f);
    } else {
        out[3 * (size_t)i + 1] = make_float4(sub(t.v1.x, t.v0.x), sub(t.v1.y, t.v0.y), sub(t.v1.z, t.v0.z), 0.0f);
        out[3 * (size_t)i + 2] = make_float4(sub(t.v2.x, t.v0.x), sub(t.v2.y, t.v0.y), sub(t.v2.z, t.v0.z), 0.0f);
    }
}

// ---- subsets: triangles that can / cannot pass a shadow ray ----------------

__global__ void k_pass_flags(const Triangle* __restrict__ tris, int n, const Material* __restrict__ mats, int nm,
                             int* __restrict__ iota, unsigned char* __restrict__ pass, unsigned char* __restrict__ block) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = tris[i].material_id;
    const bool p = m >= 0 && m < nm && mats[m].transmission > 0.5f;
    iota[i] = i;
    pass[i] = p ? 1 : 0;
    block[i] = p ? 0 : 1;
}

// ---- 6. the tree over a kept subset, derived from the built one -----------
//
// The binary tree over all triangles restricted to those with keep[t]: a
// leaf keeps its kept triangles (none: it goes), an inner node left with one
// child is replaced by that child, boxes are refitted to the kept triangles
// bottom up, and the result is collapsed like a built tree.  Kept leaf slot
// p moves to pre[p] (the exclusive prefix count of kept slots).

// kp[p] = 1 when leaf slot p is kept (p < n); kp[n] = 0 so that the scan
// yields the total in pre[n].
__global__ void k_keep_pos(const int* __restrict__ idx, int n, const unsigned char* __restrict__ keep,
                           int* __restrict__ kp) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) kp[p] = keep[idx[p]] ? 1 : 0;
    else if (p == n) kp[p] = 0;
}

// Kept count kc of every node (0 for ids marked empty), parent links, and
// the refit counters cleared.
__global__ void k_prune_count(const BNode* __restrict__ nodes, int nb, const int* __restrict__ pre,
                              int* __restrict__ kc, int* __restrict__ parent, int* __restrict__ visit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const BNode& b = nodes[i];
    const int cnt = b.count;
    kc[i] = cnt > 0 ? pre[b.first + cnt] - pre[b.first] : 0;
    visit[i] = 0;
    if (cnt > 0 && b.left >= 0) {
        parent[b.left] = i;
        parent[b.right] = i;
    }
    if (i == 0) parent[0] = -1;
}

// Bottom-up refit: every kept leaf writes its box, then climbs; at a parent
// with both children kept the first arrival stops and the second unites the
// two boxes (min / max are exact, so the order of arrival does not matter).
__global__ void k_prune_refit(const BNode* __restrict__ nodes, int nb, const int* __restrict__ kc,
                              const int* __restrict__ pre, const int* __restrict__ parent, const int* __restrict__ idx,
                              const unsigned char* __restrict__ keep, const float4* __restrict__ plo,
                              const float4* __restrict__ phi, BNode* __restrict__ Q, int* __restrict__ visit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const BNode b = nodes[i];
    if (!(b.count > 0 && b.left < 0 && kc[i] > 0)) return;
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int p = b.first; p < b.first + b.count; p++) {
        const int t = idx[p];
        if (!keep[t]) continue;
        const float4 l = plo[t], h = phi[t];
        lo[0] = fminf(lo[0], l.x); lo[1] = fminf(lo[1], l.y); lo[2] = fminf(lo[2], l.z);
        hi[0] = fmaxf(hi[0], h.x); hi[1] = fmaxf(hi[1], h.y); hi[2] = fmaxf(hi[2], h.z);
    }
    BNode& o = Q[i];
    for (int q = 0; q < 3; q++) { o.lo[q] = lo[q]; o.hi[q] = hi[q]; }
    o.first = pre[b.first];
    o.count = kc[i];
    o.left = o.right = -1;
    int j = i;
    while (true) {
        const int p = parent[j];
        if (p < 0) break;
        const int sib = nodes[p].left == j ? nodes[p].right : nodes[p].left;
        if (kc[sib] > 0) {
            __threadfence();
            if (atomicAdd(&visit[p], 1) == 0) return;   // the sibling's climb continues
            __threadfence();
            const float* sl = Q[sib].lo;
            const float* sh = Q[sib].hi;
            for (int q = 0; q < 3; q++) {
                lo[q] = fminf(lo[q], __ldcg(sl + q));
                hi[q] = fmaxf(hi[q], __ldcg(sh + q));
            }
        }
        for (int q = 0; q < 3; q++) { Q[p].lo[q] = lo[q]; Q[p].hi[q] = hi[q]; }
        j = p;
    }
}

// The kept node that stands for node x: x itself, or down the chain of
// nodes with one kept child.
__device__ __forceinline__ int prune_resolve(const BNode* __restrict__ nodes, const int* __restrict__ kc, int x) {
    while (true) {
        const BNode& c = nodes[x];
        if (c.left < 0) return x;
        const bool l = kc[c.left] > 0, r = kc[c.right] > 0;
        if (l && r) return x;
        x = l ? c.left : c.right;
    }
}

// Links of the kept inner nodes (both children kept); thread 0 also puts
// the kept root into level[0].
__global__ void k_prune_link(const BNode* __restrict__ nodes, int nb, const int* __restrict__ kc,
                             const int* __restrict__ pre, BNode* __restrict__ Q, int* __restrict__ level) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    if (i == 0) level[0] = prune_resolve(nodes, kc, 0);
    const BNode& b = nodes[i];
    if (!(b.count > 0 && b.left >= 0 && kc[i] > 0 && kc[b.left] > 0 && kc[b.right] > 0)) return;
    Q[i].first = pre[b.first];
    Q[i].count = kc[i];
    Q[i].left = prune_resolve(nodes, kc, b.left);
    Q[i].right = prune_resolve(nodes, kc, b.right);
}

// kept slot list: out[pre[p]] = idx[p] for every kept slot p.
__global__ void k_prune_compact(const int* __restrict__ idx, int n, const int* __restrict__ kp,
                                const int* __restrict__ pre, int* __restrict__ out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n && kp[p]) out[pre[p]] = idx[p];
}

// Carves 256-byte aligned arrays from one block.
struct Carver {
    char* p;
    size_t used = 0;
    template <class T>
    T* take(size_t count) {
        T* r = reinterpret_cast<T*>(p + used);
        used += (count * sizeof(T) + 255) & ~(size_t)255;
        return r;
    }
};

}  // namespace bvhg

namespace {
std::mutex g_build_stream_mu;
cudaStream_t g_build_streams[64] = {};
}  // namespace

namespace {
bool g_carveout_set[64] = {};
}  // namespace

// The small-subtree kernel asks for the largest shared-memory carveout.
static void set_small_carveout() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(g_build_stream_mu);
    if (g_carveout_set[dev]) return;
    cudaFuncSetAttribute(bvhg::k_small, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    g_carveout_set[dev] = true;
}


// Device-built BVH4 over triangles tris[subset[i]] (subset null: all n).
// Allocates out.nodes (exact size) and out.tris (3 float4 per triangle);
// everything else is temporary.  Synchronises `stream` once per tree level.
// With keep (per triangle, subset null) it also derives the BVH4 over the
// triangles with keep[t] != 0 into *kept_out (build_qbvh4_with_kept's).
cudaError_t build_qbvh4_device(const Triangle* tris, const int* subset, int n, DevQBvh& out, cudaStream_t stream,
                               bool vertices, const unsigned char* keep, DevQBvh* kept_out) {
    using namespace bvhg;
    out = DevQBvh{};
    if (kept_out) *kept_out = DevQBvh{};
    if (keep && (subset || !kept_out)) return cudaErrorInvalidValue;
    if (n <= 0) return cudaSuccess;
    if (n > (1 << 27)) return cudaErrorInvalidValue;   // leaf words hold first < 2^28
    const size_t N = (size_t)n;
    const int max_work = n / kSmall + 2;
    const int max_chunks = n / kChunk + max_work + 2;
    size_t cub_a = 0, cub_b = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, cub_a, (int*)nullptr, (int*)nullptr, max_chunks);
    if (e != cudaSuccess) return e;
    e = cub::DeviceScan::ExclusiveSum(nullptr, cub_b, (int*)nullptr, (int*)nullptr, n + 1);
    if (e != cudaSuccess) return e;
    const size_t cub_bytes = std::max(cub_a, cub_b);

    // Temporary block: sized by a dry carve.
    struct Ptrs {
        float4 *plo, *phi;
        int *idx, *tmp;
        BNode* nodes;
        dev::QNode4* qtmp;
        int4* kids;
        int *nk, *ninner, *off, *lvl_a, *lvl_b;
        int *gbins, *work, *chunk_base, *chunk_left, *chunk_off, *child_ord, *root_ord, *err;
        int4* split;
        int2* child_fc;
        void* cub;
        int *kp, *pre, *kc, *parent, *visit;   // kept-subset derivation
        BNode* Q;
    } P;
    auto carve = [&](Carver& c) {
        P.plo = c.take<float4>(N);
        P.phi = c.take<float4>(N);
        P.idx = c.take<int>(N);
        P.tmp = c.take<int>(N);
        P.nodes = c.take<BNode>(2 * N);
        P.qtmp = c.take<dev::QNode4>(N);
        P.kids = c.take<int4>(N);
        P.nk = c.take<int>(N);
        P.ninner = c.take<int>(N);
        P.off = c.take<int>(N);
        P.lvl_a = c.take<int>(N);
        P.lvl_b = c.take<int>(N);
        P.gbins = c.take<int>((size_t)max_work * kNodeBins);
        P.work = c.take<int>((size_t)max_work);
        P.chunk_base = c.take<int>((size_t)max_work + 1);
        P.chunk_left = c.take<int>((size_t)max_chunks);
        P.chunk_off = c.take<int>((size_t)max_chunks);
        P.child_ord = c.take<int>((size_t)2 * max_work * 12);
        P.root_ord = c.take<int>(12);
        P.err = c.take<int>(1);
        P.split = c.take<int4>((size_t)max_work);
        P.child_fc = c.take<int2>((size_t)2 * max_work);
        P.cub = c.take<char>(cub_bytes);
        if (keep) {
            P.kp = c.take<int>(N + 1);
            P.pre = c.take<int>(N + 1);
            P.kc = c.take<int>(2 * N);
            P.parent = c.take<int>(2 * N);
            P.visit = c.take<int>(2 * N);
            P.Q = c.take<BNode>(2 * N);
        }
    };
    Carver dry{nullptr};
    carve(dry);
    void* block = nullptr;
    if ((e = dmalloc_async(&block, dry.used, stream)) != cudaSuccess) return e;
    Carver real{static_cast<char*>(block)};
    carve(real);
    int* small_buf = nullptr;
    dev::QNode4* nodes_out = nullptr;
    float4* tris_out = nullptr;
    dev::QNode4* kept_nodes = nullptr;
    float4* kept_tris = nullptr;
    int num_q = 0, depth = 0, num_kq = 0, kdepth = 0, nkept = 0;
#define CK(x) do { if ((e = (x)) != cudaSuccess) goto done; } while (0)
    {
        // 1. boxes and root
        CK(cudaMemsetAsync(P.err, 0, sizeof(int), stream));
        k_init_ord<<<1, 32, 0, stream>>>(P.root_ord, 12);
        const int prep_blocks = (int)std::min<size_t>((N + 255) / 256, 148 * 8);
        k_prep<<<prep_blocks, 256, 0, stream>>>(tris, subset, n, P.plo, P.phi, P.idx, P.root_ord);
        k_root<<<1, 32, 0, stream>>>(P.root_ord, n, P.nodes);
        CK(cudaGetLastError());

        // 2. large nodes, one level per pass
        std::vector<int> work, work_count, small_ids, small_count;
        if (n > kSmall) { work.push_back(0); work_count.push_back(n); }
        else { small_ids.push_back(0); small_count.push_back(n); }
        int next_id = 1;
        std::vector<int> chunk_base;
        std::vector<int4> split_h;
        std::vector<int2> fc_h;
        int levels = 0;
        while (!work.empty()) {
            if (++levels > kMaxLargeLevels) { e = cudaErrorInvalidValue; goto done; }
            const int m = (int)work.size();
            chunk_base.assign((size_t)m + 1, 0);
            for (int j = 0; j < m; j++) chunk_base[(size_t)j + 1] = chunk_base[(size_t)j] + (work_count[(size_t)j] + kChunk - 1) / kChunk;
            const int chunks = chunk_base[(size_t)m];
            CK(cudaMemcpyAsync(P.work, work.data(), (size_t)m * sizeof(int), cudaMemcpyHostToDevice, stream));
            CK(cudaMemcpyAsync(P.chunk_base, chunk_base.data(), ((size_t)m + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
            const int words = m * kNodeBins;
            k_init_bins<<<(words + 255) / 256, 256, 0, stream>>>(P.gbins, words);
            k_bin_large<<<chunks, kChunkThreads, 0, stream>>>(P.work, P.chunk_base, m, P.nodes, P.plo, P.phi, P.idx, P.gbins);
            k_split_large<<<m, 32, 0, stream>>>(P.work, m, next_id, P.nodes, P.gbins, P.split, P.child_fc);
            k_init_ord<<<(2 * m * 12 + 255) / 256, 256, 0, stream>>>(P.child_ord, 2 * m * 12);
            k_list_split_bounds<<<chunks, kChunkThreads, 0, stream>>>(P.work, P.chunk_base, m, P.nodes, P.split, P.plo,
                                                                      P.phi, P.idx, P.child_ord);
            k_list_split_write<<<(2 * m + 127) / 128, 128, 0, stream>>>(m, next_id, P.split, P.child_ord, P.nodes);
            k_part_count<<<chunks, kChunkThreads, 0, stream>>>(P.work, P.chunk_base, m, P.nodes, P.split, P.plo, P.phi,
                                                              P.idx, P.chunk_left);
            size_t cb = cub_bytes;
            CK(cub::DeviceScan::ExclusiveSum(P.cub, cb, P.chunk_left, P.chunk_off, chunks, stream));
            k_part_scatter<<<chunks, kChunkThreads, 0, stream>>>(P.work, P.chunk_base, m, P.nodes, P.split, P.plo,
                                                                P.phi, P.idx, P.chunk_off, P.tmp, P.err);
            k_copy_back<<<chunks, kChunkThreads, 0, stream>>>(P.work, P.chunk_base, m, P.nodes, P.tmp, P.idx);
            CK(cudaGetLastError());
            fc_h.resize((size_t)2 * m);
            CK(cudaMemcpyAsync(fc_h.data(), P.child_fc, (size_t)2 * m * sizeof(int2), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            std::vector<int> nwork, ncount;
            for (int i = 0; i < 2 * m; i++) {
                const int id = next_id + i, cnt = fc_h[(size_t)i].y;
                if (cnt > kSmall) { nwork.push_back(id); ncount.push_back(cnt); }
                else { small_ids.push_back(id); small_count.push_back(cnt); }
            }
            next_id += 2 * m;
            work.swap(nwork);
            work_count.swap(ncount);
        }

        // 3. small subtrees
        const int ns = (int)small_ids.size();
        std::vector<int> small_h((size_t)2 * ns);
        int id = next_id;
        for (int b = 0; b < ns; b++) {
            small_h[(size_t)b] = small_ids[(size_t)b];
            small_h[(size_t)ns + b] = id;
            id += std::max(0, 2 * small_count[(size_t)b] - 2);
        }
        if ((size_t)id > 2 * N) { e = cudaErrorInvalidValue; goto done; }
        CK(dmalloc_async(&small_buf, (size_t)2 * ns * sizeof(int), stream));
        CK(cudaMemcpyAsync(small_buf, small_h.data(), (size_t)2 * ns * sizeof(int), cudaMemcpyHostToDevice, stream));
        {
            // 37.6 KB of static shared memory a block: ask for the largest
            // shared-memory carveout so that six blocks fit on an SM
            // (a per-context hint: set once per device, and again after
            // sheen_cleanup's device reset)
            set_small_carveout();
        }
        k_small<<<ns, kSmallThreads, 0, stream>>>(small_buf, small_buf + ns, P.plo, P.phi, P.idx, P.nodes, P.err,
                                                  node_cost_of(tuning().node_cost));
        CK(cudaGetLastError());

        // 4. collapse, breadth first from the binary node in P.lvl_a[0]: the
        // 4-wide nodes go to P.qtmp; returns their count and the depth
        auto collapse = [&](const BNode* tree, int ntris, int& count, int& levels) -> cudaError_t {
            cudaError_t ce = cudaSuccess;
            int m = 1, base = 0;
            int* cur = P.lvl_a;
            int* nxt = P.lvl_b;
            levels = 0;
            while (m > 0) {
                levels++;
                k_collapse_count<<<(m + 127) / 128, 128, 0, stream>>>(cur, m, tree, P.kids, P.nk, P.ninner);
                size_t cb = cub_bytes;
                if ((ce = cub::DeviceScan::ExclusiveSum(P.cub, cb, P.ninner, P.off, m, stream)) != cudaSuccess) return ce;
                k_collapse_emit<<<(m + 127) / 128, 128, 0, stream>>>(cur, m, base, P.kids, P.nk, P.off, tree, P.qtmp,
                                                                     nxt);
                if ((ce = cudaGetLastError()) != cudaSuccess) return ce;
                int last[2] = {0, 0};
                if ((ce = cudaMemcpyAsync(&last[0], P.off + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, stream)) !=
                    cudaSuccess)
                    return ce;
                if ((ce = cudaMemcpyAsync(&last[1], P.ninner + (m - 1), sizeof(int), cudaMemcpyDeviceToHost, stream)) !=
                    cudaSuccess)
                    return ce;
                if ((ce = cudaStreamSynchronize(stream)) != cudaSuccess) return ce;
                base += m;
                m = last[0] + last[1];
                std::swap(cur, nxt);
                if (base + m > ntris) return cudaErrorInvalidValue;
            }
            count = base;
            return cudaSuccess;
        };
        CK(cudaMemsetAsync(P.lvl_a, 0, sizeof(int), stream));   // the root, binary node 0
        CK(collapse(P.nodes, n, num_q, depth));
        int err_h = 0;
        CK(cudaMemcpyAsync(&err_h, P.err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (err_h) { e = cudaErrorInvalidValue; goto done; }

        // outputs
        CK(dmalloc_async(&nodes_out, (size_t)num_q * sizeof(dev::QNode4), stream));
        CK(dmalloc_async(&tris_out, 3 * N * sizeof(float4), stream));
        CK(cudaMemcpyAsync(nodes_out, P.qtmp, (size_t)num_q * sizeof(dev::QNode4), cudaMemcpyDeviceToDevice, stream));
        k_emit_tris<<<(n + 255) / 256, 256, 0, stream>>>(tris, subset, P.idx, n, tris_out, vertices);
        CK(cudaGetLastError());

        // 6. the kept subset's tree, derived from this one
        if (keep) {
            const int nb = id;   // every id below is a node (or marked empty)
            k_keep_pos<<<(n + 1 + 255) / 256, 256, 0, stream>>>(P.idx, n, keep, P.kp);
            size_t cb = cub_bytes;
            CK(cub::DeviceScan::ExclusiveSum(P.cub, cb, P.kp, P.pre, n + 1, stream));
            CK(cudaMemcpyAsync(&nkept, P.pre + n, sizeof(int), cudaMemcpyDeviceToHost, stream));
            CK(cudaStreamSynchronize(stream));
            if (nkept > 0) {
                const int g = (nb + 255) / 256;
                k_prune_count<<<g, 256, 0, stream>>>(P.nodes, nb, P.pre, P.kc, P.parent, P.visit);
                k_prune_refit<<<g, 256, 0, stream>>>(P.nodes, nb, P.kc, P.pre, P.parent, P.idx, keep, P.plo, P.phi, P.Q,
                                                     P.visit);
                k_prune_link<<<g, 256, 0, stream>>>(P.nodes, nb, P.kc, P.pre, P.Q, P.lvl_a);
                CK(cudaGetLastError());
                CK(collapse(P.Q, nkept, num_kq, kdepth));
                CK(dmalloc_async(&kept_nodes, (size_t)num_kq * sizeof(dev::QNode4), stream));
                CK(dmalloc_async(&kept_tris, 3 * (size_t)nkept * sizeof(float4), stream));
                CK(cudaMemcpyAsync(kept_nodes, P.qtmp, (size_t)num_kq * sizeof(dev::QNode4), cudaMemcpyDeviceToDevice,
                                   stream));
                k_prune_compact<<<(n + 255) / 256, 256, 0, stream>>>(P.idx, n, P.kp, P.pre, P.tmp);
                k_emit_tris<<<(nkept + 255) / 256, 256, 0, stream>>>(tris, nullptr, P.tmp, nkept, kept_tris, vertices);
                CK(cudaGetLastError());
            }
        }
        CK(cudaStreamSynchronize(stream));
    }
done:
#undef CK
    dfree_async(small_buf, stream);
    dfree_async(block, stream);
    if (e != cudaSuccess) {
        dfree_async(nodes_out, stream);
        dfree_async(tris_out, stream);
        dfree_async(kept_nodes, stream);
        dfree_async(kept_tris, stream);
        return e;
    }
    if (kept_out && nkept > 0) {
        kept_out->nodes = kept_nodes;
        kept_out->tris = kept_tris;
        kept_out->num_nodes = num_kq;
        kept_out->num_tris = nkept;
        kept_out->max_depth = kdepth;
    }
    out.nodes = nodes_out;
    out.tris = tris_out;
    out.num_nodes = num_q;
    out.num_tris = n;
    out.max_depth = depth;
    return cudaSuccess;
}

// The wavefront form's three triangle BVH4s of a resident scene (triangles
// and materials already in the arena), built on the device.  The subsets
// are the host's: passable = material transmission > 0.5 (in range), in
// index order.  The blocking triangles' tree is derived from the tree over
// all triangles (build_qbvh4_with_kept); the passable triangles' tree is
// built at the same time from a second host thread on a second stream.
// Allocations go to s.extra.
// The second build stream of a device, created once and kept: memory the
// pool hands out and takes back on the same stream is reused in stream
// order, where a fresh stream per call can make the pool map new memory.
void release_build_streams() {
    std::lock_guard<std::mutex> lk(g_build_stream_mu);
    for (auto& c : g_carveout_set) c = false;
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < 64; d++) {
        if (!g_build_streams[d]) continue;
        cudaSetDevice(d);
        cudaStreamDestroy(g_build_streams[d]);
        g_build_streams[d] = nullptr;
    }
    cudaSetDevice(cur);
}

static cudaError_t build_stream2(cudaStream_t* out) {
    auto& mu = g_build_stream_mu;
    auto& streams = g_build_streams;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(mu);
    if (!streams[dev] && (e = cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking)) != cudaSuccess) {
        streams[dev] = nullptr;
        return e;
    }
    *out = streams[dev];
    return cudaSuccess;
}

cudaError_t build_wave_meshes_device(DeviceScene& s, cudaStream_t stream) {
    dev::DevScene& v = s.view;
    const int n = v.num_tris;
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    DevQBvh all, blk, pas;
    int* iota = nullptr;
    int* sel = nullptr;
    unsigned char* flags = nullptr;
    void* cub_tmp = nullptr;
    int* num_sel = nullptr;
    int npass = 0;
    size_t cb = 0;
    cudaStream_t st2 = nullptr;
    cudaError_t e_all = cudaSuccess, e_sub = cudaSuccess;
    const bool wt = tuning().watertight != 0;
#define CK(x) do { if ((e = (x)) != cudaSuccess) goto done; } while (0)
    CK(build_stream2(&st2));
    CK(dmalloc_async(&iota, (size_t)n * sizeof(int), stream));
    CK(dmalloc_async(&sel, (size_t)2 * n * sizeof(int), stream));
    CK(dmalloc_async(&flags, (size_t)2 * n, stream));
    CK(dmalloc_async(&num_sel, 2 * sizeof(int), stream));
    bvhg::k_pass_flags<<<(n + 255) / 256, 256, 0, stream>>>(v.tris, n, v.materials, v.num_materials, iota, flags,
                                                             flags + n);
    CK(cudaGetLastError());
    CK(cub::DeviceSelect::Flagged(nullptr, cb, iota, flags, sel, num_sel, n, stream));
    CK(dmalloc_async(&cub_tmp, cb, stream));
    CK(cub::DeviceSelect::Flagged(cub_tmp, cb, iota, flags, sel + n, num_sel, n, stream));          // passable
    CK(cudaMemcpyAsync(&npass, num_sel, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    {
        int dev_id = 0;
        CK(cudaGetDevice(&dev_id));
        auto subset_trees = [&] {
            cudaSetDevice(dev_id);
            if (npass > 0) e_sub = build_qbvh4_device(v.tris, sel + n, npass, pas, st2, wt);
        };
        // with passable triangles present: the blocking ones' tree from the
        // tree over all (flags + n: the blocking flags)
        const unsigned char* keep = npass > 0 ? flags + n : nullptr;
        if (tuning().build_concurrent) {
            std::thread subsets(subset_trees);
            e_all = build_qbvh4_device(v.tris, nullptr, n, all, stream, wt, keep, keep ? &blk : nullptr);
            subsets.join();
        } else {
            e_all = build_qbvh4_device(v.tris, nullptr, n, all, stream, wt, keep, keep ? &blk : nullptr);
            subset_trees();
        }
        e = e_all != cudaSuccess ? e_all : e_sub;
    }
done:
#undef CK
    dfree_async(iota, stream);
    dfree_async(sel, stream);
    dfree_async(flags, stream);
    dfree_async(cub_tmp, stream);
    dfree_async(num_sel, stream);
    if (st2) cudaStreamSynchronize(st2);
    auto keep = [&](const DevQBvh& q) {
        if (q.nodes) s.extra.push_back(q.nodes);
        if (q.tris) s.extra.push_back(q.tris);
        s.extra_bytes += (size_t)q.num_nodes * sizeof(dev::QNode4) + (size_t)q.num_tris * 3 * sizeof(float4);
    };
    keep(all);
    keep(blk);
    keep(pas);
    if (e != cudaSuccess) return e;
    auto qmesh = [wt](const DevQBvh& q) {
        dev::QMesh m;
        m.nodes = q.nodes;
        m.tris = q.tris;
        m.num_nodes = q.num_nodes;
        m.num_tris = q.num_tris;
        m.watertight = wt ? 1 : 0;
        return m;
    };
    v.q_all = qmesh(all);
    v.q_block = qmesh(blk);
    v.q_pass = qmesh(pas);
    s.wave_depth = std::max(all.max_depth, std::max(blk.max_depth, pas.max_depth));
    return cudaSuccess;
}

}  // namespace sheen

// Both builders on one scene, compared byte for byte (a parity check of the
// device builder; no rendering).  Returns 0 when the three BVH4s (all /
// blocking / passable triangles) are identical, 1 + 10*set for a differing
// node count, 2 + 10*set for differing node bytes, 3 + 10*set for differing
// triangle records, 4 + 10*set for a differing depth (set 0 all, 1
// blocking, 2 passable), -1 on error.  times_ms (may be NULL) receives the
// host and the device build times.
extern "C" int sheen_bvh4_compare_builders(const SheenScene* scene, double* times_ms) {
    using namespace sheen;
    if (!scene || scene->num_triangles <= 0 || !scene->triangles) { set_error("scene has no triangles"); return -1; }
    const int n = scene->num_triangles;
    std::vector<int> all, pass;
    std::vector<unsigned char> blocking((size_t)n);
    for (int i = 0; i < n; i++) {
        all.push_back(i);
        const int m = scene->triangles[i].material_id;
        const bool passable = m >= 0 && m < scene->num_materials && scene->materials[m].transmission > 0.5f;
        if (passable) pass.push_back(i);
        blocking[(size_t)i] = passable ? 0 : 1;
    }
    const double h0 = now_ms();
    QBvh hq[3];
    const bool wt = tuning().watertight != 0;   // both builders use the record layout in force
    if (!pass.empty()) {
        build_qbvh4_with_kept(scene->triangles, n, blocking, hq[0], hq[1], wt);
        build_qbvh4(scene->triangles, pass, hq[2], wt);
    } else {
        build_qbvh4(scene->triangles, all, hq[0], wt);
    }
    const double host_ms = now_ms() - h0;

    DeviceScene ds;
    Triangle* dt = nullptr;
    Material* dm = nullptr;
    int rc = 0;
    cudaError_t e = dmalloc(&dt, (size_t)n * sizeof(Triangle));
    if (e == cudaSuccess) e = dmalloc(&dm, (size_t)std::max(scene->num_materials, 1) * sizeof(Material));
    if (e == cudaSuccess) e = cudaMemcpy(dt, scene->triangles, (size_t)n * sizeof(Triangle), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && scene->num_materials > 0)
        e = cudaMemcpy(dm, scene->materials, (size_t)scene->num_materials * sizeof(Material), cudaMemcpyHostToDevice);
    double dev_ms = 0.0;
    if (e == cudaSuccess) {
        ds.form = SHEEN_FORM_WAVEFRONT;
        ds.view.tris = dt;
        ds.view.num_tris = n;
        ds.view.materials = dm;
        ds.view.num_materials = scene->num_materials;
        e = cudaDeviceSynchronize();
        const double d0 = now_ms();
        if (e == cudaSuccess) e = build_wave_meshes_device(ds, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        dev_ms = now_ms() - d0;
    }
    const dev::QMesh dq[3] = {ds.view.q_all, ds.view.q_block, ds.view.q_pass};
    for (int k = 0; k < 3 && e == cudaSuccess && rc == 0; k++) {
        const QBvh& h = hq[k];
        if ((size_t)dq[k].num_nodes != h.nodes.size() || (size_t)dq[k].num_tris * 3 != h.tris.size()) {
            rc = 1 + 10 * k;
            break;
        }
        if (h.nodes.empty()) continue;
        std::vector<dev::QNode4> nodes(h.nodes.size());
        std::vector<float4> tris(h.tris.size());
        e = cudaMemcpy(nodes.data(), dq[k].nodes, nodes.size() * sizeof(dev::QNode4), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(tris.data(), dq[k].tris, tris.size() * sizeof(float4), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) break;
        if (std::memcmp(nodes.data(), h.nodes.data(), nodes.size() * sizeof(dev::QNode4)) != 0) rc = 2 + 10 * k;
        else if (std::memcmp(tris.data(), h.tris.data(), tris.size() * sizeof(float4)) != 0) rc = 3 + 10 * k;
    }
    if (e == cudaSuccess && rc == 0) {
        const int hd = std::max(hq[0].max_depth, std::max(hq[1].max_depth, hq[2].max_depth));
        if (hd != ds.wave_depth) rc = 4;
    }
    for (void* p : ds.extra) dfree(p);
    dfree(dt);
    dfree(dm);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return -1; }
    if (times_ms) { times_ms[0] = host_ms; times_ms[1] = dev_ms; }
    return rc;
}
