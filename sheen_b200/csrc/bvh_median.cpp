// bvh_median.cpp -- median-split BVH of the plain form.
//
// Same splitting rule as the reference builders (bvh.h:71-576) so the plain
// form's trees have the same shape and DFS order as the reference's: node box
// = union of primitive boxes; a single primitive makes a leaf; otherwise pick
// the axis with the largest extent (first of x, y, z on ties), partition the
// index range at count/2 with std::nth_element on box centroids, recurse on
// [start, mid) then [mid, end).  Centroids are the float midpoint of each
// primitive box, as the reference computes them.
//
// Subtrees below the top levels are built on worker threads into their own
// node vectors and spliced in afterwards; nth_element runs on the same
// sub-ranges in the same order either way, so the tree is identical to the
// serial build (only node numbering differs, which traversal never sees).
#include <algorithm>
#include <cmath>
#include <thread>

#include "engine.h"

namespace sheen {

namespace {

struct Builder {
    const float* lo;
    const float* hi;
    std::vector<float> cen;   // 3 per primitive id
    bool axis_from_centroids;

    void build(std::vector<int>& idx, int start, int end, int depth, std::vector<HostNode>& nodes) {
        const int node = (int)nodes.size();
        nodes.push_back(HostNode{});
        float bl[3] = {1e30f, 1e30f, 1e30f}, bh[3] = {-1e30f, -1e30f, -1e30f};
        float cl[3] = {1e30f, 1e30f, 1e30f}, ch[3] = {-1e30f, -1e30f, -1e30f};
        if (axis_from_centroids) {
            for (int k = 0; k < 3; k++) { bl[k] = 1e10f; bh[k] = -1e10f; cl[k] = 1e10f; ch[k] = -1e10f; }
        }
        for (int i = start; i < end; i++) {
            const int p = idx[(size_t)i];
            for (int k = 0; k < 3; k++) {
                bl[k] = fminf(bl[k], lo[3 * (size_t)p + k]);
                bh[k] = fmaxf(bh[k], hi[3 * (size_t)p + k]);
                cl[k] = fminf(cl[k], cen[3 * (size_t)p + k]);
                ch[k] = fmaxf(ch[k], cen[3 * (size_t)p + k]);
            }
        }
        HostNode& n = nodes[(size_t)node];
        for (int k = 0; k < 3; k++) { n.lo[k] = bl[k]; n.hi[k] = bh[k]; }
        const int count = end - start;
        if (count <= 1) {
            n.left = n.right = ~idx[(size_t)start];
            return;
        }
        float ext[3];
        for (int k = 0; k < 3; k++) ext[k] = axis_from_centroids ? ch[k] - cl[k] : bh[k] - bl[k];
        int axis = 0;
        if (ext[1] > ext[0] && ext[1] > ext[2]) axis = 1;
        if (ext[2] > ext[0] && ext[2] > ext[1]) axis = 2;
        const int mid = start + count / 2;
        const float* c = cen.data();
        std::nth_element(idx.begin() + start, idx.begin() + mid, idx.begin() + end,
                         [c, axis](int a, int b) { return c[3 * (size_t)a + axis] < c[3 * (size_t)b + axis]; });
        if (depth < 4 && count > 65536) {
            std::vector<HostNode> right_nodes;
            std::thread worker([&] { build(idx, mid, end, depth + 1, right_nodes); });
            const int left = (int)nodes.size();
            build(idx, start, mid, depth + 1, nodes);
            worker.join();
            const int right = (int)nodes.size();
            for (HostNode rn : right_nodes) {
                if (rn.left >= 0) { rn.left += right; rn.right += right; }
                nodes.push_back(rn);
            }
            nodes[(size_t)node].left = left;
            nodes[(size_t)node].right = right;
        } else {
            const int left = (int)nodes.size();
            build(idx, start, mid, depth + 1, nodes);
            const int right = (int)nodes.size();
            build(idx, mid, end, depth + 1, nodes);
            nodes[(size_t)node].left = left;
            nodes[(size_t)node].right = right;
        }
    }
};

}  // namespace

void build_median_bvh(const std::vector<float>& lo, const std::vector<float>& hi, const std::vector<int>& prims,
                      bool axis_from_centroids, std::vector<HostNode>& out) {
    out.clear();
    if (prims.empty()) return;
    Builder b;
    b.lo = lo.data();
    b.hi = hi.data();
    b.axis_from_centroids = axis_from_centroids;
    b.cen.resize(lo.size());
    for (size_t i = 0; i < lo.size(); i++) b.cen[i] = (lo[i] + hi[i]) * 0.5f;
    std::vector<int> idx = prims;
    out.reserve(2 * prims.size());
    b.build(idx, 0, (int)idx.size(), 0, out);
}

}  // namespace sheen
