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

// One primitive as the builder moves it: its centroid, box and id side by
// side, so partitions and box unions read contiguous memory instead of
// gathering through an id array (the gathers dominated the build).
struct Item {
    float c[3];
    float lo[3];
    float hi[3];
    int id;
};

struct Builder {
    bool axis_from_centroids;

    void build(std::vector<Item>& it, int start, int end, int depth, std::vector<HostNode>& nodes) {
        const int node = (int)nodes.size();
        nodes.push_back(HostNode{});
        float bl[3] = {1e30f, 1e30f, 1e30f}, bh[3] = {-1e30f, -1e30f, -1e30f};
        float cl[3] = {1e30f, 1e30f, 1e30f}, ch[3] = {-1e30f, -1e30f, -1e30f};
        if (axis_from_centroids) {
            for (int k = 0; k < 3; k++) { bl[k] = 1e10f; bh[k] = -1e10f; cl[k] = 1e10f; ch[k] = -1e10f; }
        }
        for (int i = start; i < end; i++) {
            const Item& p = it[(size_t)i];
            for (int k = 0; k < 3; k++) {
                bl[k] = fminf(bl[k], p.lo[k]);
                bh[k] = fmaxf(bh[k], p.hi[k]);
                cl[k] = fminf(cl[k], p.c[k]);
                ch[k] = fmaxf(ch[k], p.c[k]);
            }
        }
        HostNode& n = nodes[(size_t)node];
        for (int k = 0; k < 3; k++) { n.lo[k] = bl[k]; n.hi[k] = bh[k]; }
        const int count = end - start;
        if (count <= 1) {
            n.left = n.right = ~it[(size_t)start].id;
            return;
        }
        float ext[3];
        for (int k = 0; k < 3; k++) ext[k] = axis_from_centroids ? ch[k] - cl[k] : bh[k] - bl[k];
        int axis = 0;
        if (ext[1] > ext[0] && ext[1] > ext[2]) axis = 1;
        if (ext[2] > ext[0] && ext[2] > ext[1]) axis = 2;
        const int mid = start + count / 2;
        // the comparisons, and so the permutation nth_element makes, are the
        // ones an id array ordered by the same keys would get
        std::nth_element(it.begin() + start, it.begin() + mid, it.begin() + end,
                         [axis](const Item& a, const Item& b) { return a.c[axis] < b.c[axis]; });
        if (depth < 4 && count > 65536) {
            std::vector<HostNode> right_nodes;
            std::thread worker([&] { build(it, mid, end, depth + 1, right_nodes); });
            const int left = (int)nodes.size();
            build(it, start, mid, depth + 1, nodes);
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
            build(it, start, mid, depth + 1, nodes);
            const int right = (int)nodes.size();
            build(it, mid, end, depth + 1, nodes);
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
    b.axis_from_centroids = axis_from_centroids;
    std::vector<Item> it(prims.size());
    for (size_t i = 0; i < prims.size(); i++) {
        const size_t p = (size_t)prims[i];
        Item& m = it[i];
        for (int k = 0; k < 3; k++) {
            m.lo[k] = lo[3 * p + k];
            m.hi[k] = hi[3 * p + k];
            m.c[k] = (lo[3 * p + k] + hi[3 * p + k]) * 0.5f;
        }
        m.id = prims[i];
    }
    out.reserve(2 * prims.size());
    b.build(it, 0, (int)it.size(), 0, out);
}

}  // namespace sheen
