// bvh4.cpp -- triangle BVH of the wavefront form: binned SAH, collapsed to
// 4-wide nodes whose child boxes are stored as 8-bit integers in a per-node
// frame, rounded outward so that the decoded box always contains the
// original one.
//
// Node (dev::QNode4, 64 bytes, four 128-bit loads):
//   origin_exp.xyz  frame origin (the node's box minimum)
//   origin_exp.w    bits 0-7 / 8-15 / 16-23: biased exponents ex, ey, ez of
//                   the per-axis scale 2^(e-127); bits 24-31: child count
//   child[i]        inner child: node index; leaf: 0x80000000 |
//                   (first triangle << 3) | (count - 1), count <= 8
//   qbox.x..w       byte i of each word: child i's qlo.x, qhi.x, qlo.y, qhi.y
//   qz.x, qz.y      byte i: child i's qlo.z, qhi.z
// A child box decodes as lo = fmaf(qlo, 2^e, origin), hi = fmaf(qhi, 2^e,
// origin).  The builder computes the same fmaf in float and moves each
// integer outward until the decoded box contains the exact child box.
//
// Triangles are stored in leaf order as three float4: {v0, original index},
// then {e1 = v1 - v0, 0}, {e2 = v2 - v0, 0} for the Moller-Trumbore test
// (the same float subtractions the reference performs per test,
// primitives/triangle.h:9-10, so its results are unchanged), or {v1, 0},
// {v2, 0} for the watertight test, which needs the vertices themselves.
//
// The tree over a subset of the triangles (the blocking ones) can be derived
// from the tree over all of them instead of built (build_qbvh4_with_kept):
// leaves lose the other triangles, nodes left with one child are spliced
// out, boxes are refitted.  Where the subset is most of the triangles its
// derived tree is nearly the built one, at a fraction of the build's cost.
//
// The arithmetic of every decision (bins, SAH costs, frame exponents,
// quantisation) is in bvh4_rules.h, shared with the device builder
// (bvh4_gpu.cu); partitions are stable.  The two builders therefore produce
// byte-identical trees, which the tests check.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "bvh4_rules.h"
#include "engine.h"

namespace sheen {

namespace {

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const Box& b) {
        for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
    }
    void grow(const float p[3]) {
        for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
    }
    float area() const { return bvhr::area(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]); }
};

struct BNode {
    Box box;
    int left = -1, right = -1;   // inner
    int first = 0, count = 0;    // leaf when count > 0
};

constexpr int kBins = bvhr::kBins;
constexpr int kMaxLeaf = bvhr::kMaxLeaf;

struct SahBuilder {
    float node_cost = 1.0f;   // a node visit in triangle tests ("build.node_cost")
    std::vector<Box> tri_box;
    std::vector<float> cen;   // 3 per triangle
    std::vector<int> idx;

    // Builds the subtree of idx[first, first+n) into `out`; returns its root.
    int build(int first, int n, int depth, std::vector<BNode>& out) {
        const int me = (int)out.size();
        out.emplace_back();
        Box b, cb;
        for (int i = first; i < first + n; i++) {
            b.grow(tri_box[(size_t)idx[(size_t)i]]);
            cb.grow(&cen[3 * (size_t)idx[(size_t)i]]);
        }
        out[(size_t)me].box = b;
        if (n <= 2) { out[(size_t)me].first = first; out[(size_t)me].count = n; return me; }
        // Binned SAH over the centroid box.
        float best_cost = FLT_MAX;
        int best_axis = -1, best_split = -1;
        for (int axis = 0; axis < 3; axis++) {
            const float ext = cb.hi[axis] - cb.lo[axis];
            if (!(ext > 0.0f)) continue;
            Box bins[kBins];
            int cnt[kBins] = {0};
            const float k = bvhr::bin_scale(ext);
            for (int i = first; i < first + n; i++) {
                const int t = idx[(size_t)i];
                const int bi = bvhr::bin_of(cen[3 * (size_t)t + axis], cb.lo[axis], k);
                cnt[bi]++;
                bins[bi].grow(tri_box[(size_t)t]);
            }
            float right_area[kBins];
            int right_cnt[kBins];
            Box acc;
            int c = 0;
            for (int i = kBins - 1; i > 0; i--) {
                acc.grow(bins[i]);
                c += cnt[i];
                right_area[i] = acc.area();
                right_cnt[i] = c;
            }
            Box lacc;
            int lc = 0;
            for (int i = 0; i < kBins - 1; i++) {
                lacc.grow(bins[i]);
                lc += cnt[i];
                if (lc == 0 || right_cnt[i + 1] == 0) continue;
                const float cost = bvhr::split_cost(lacc.area(), lc, right_area[i + 1], right_cnt[i + 1]);
                if (cost < best_cost) { best_cost = cost; best_axis = axis; best_split = i; }
            }
        }
        // cost model: a node visit node_cost, a triangle test 1 (both scaled by the area)
        if (best_axis < 0 || (n <= kMaxLeaf && bvhr::leaf_wins(b.area(), n, best_cost, node_cost))) {
            if (n <= kMaxLeaf) { out[(size_t)me].first = first; out[(size_t)me].count = n; return me; }
        }
        int mid;
        if (best_axis >= 0) {
            const int axis = best_axis;
            const float k = bvhr::bin_scale(cb.hi[axis] - cb.lo[axis]);
            const float lo = cb.lo[axis];
            auto it = std::stable_partition(idx.begin() + first, idx.begin() + first + n, [&](int t) {
                return bvhr::bin_of(cen[3 * (size_t)t + axis], lo, k) <= best_split;
            });
            mid = (int)(it - idx.begin());
        } else {
            mid = first + n / 2;   // all centroids coincide: split the list
        }
        if (mid == first || mid == first + n) mid = first + n / 2;
        int l, r;
        if (depth < 5 && n > 50000) {
            std::vector<BNode> right_nodes;
            int rroot = 0;
            std::thread worker([&] { rroot = build(mid, first + n - mid, depth + 1, right_nodes); });
            l = build(first, mid - first, depth + 1, out);
            worker.join();
            const int off = (int)out.size();
            for (BNode rn : right_nodes) {
                if (rn.count == 0) { rn.left += off; rn.right += off; }
                out.push_back(rn);
            }
            r = rroot + off;
        } else {
            l = build(first, mid - first, depth + 1, out);
            r = build(mid, first + n - mid, depth + 1, out);
        }
        out[(size_t)me].left = l;
        out[(size_t)me].right = r;
        return me;
    }
};

// Binned SAH tree over tris[subset[i]]: box and centroid of every
// triangle, then the recursive build.  Returns the root of `bn`.
int sah_build(const Triangle* tris, const std::vector<int>& subset, SahBuilder& sb, std::vector<BNode>& bn) {
    const int n = (int)subset.size();
    sb.node_cost = bvhr::node_cost_of(tuning().node_cost);
    sb.tri_box.resize((size_t)n);
    sb.cen.resize(3 * (size_t)n);
    sb.idx.resize((size_t)n);
    for (int i = 0; i < n; i++) {
        const Triangle& t = tris[subset[(size_t)i]];
        const float v[3][3] = {{t.v0.x, t.v0.y, t.v0.z}, {t.v1.x, t.v1.y, t.v1.z}, {t.v2.x, t.v2.y, t.v2.z}};
        Box b;
        for (int k = 0; k < 3; k++) b.grow(v[k]);
        for (int k = 0; k < 3; k++) { b.lo[k] = bvhr::canon(b.lo[k]); b.hi[k] = bvhr::canon(b.hi[k]); }
        sb.tri_box[(size_t)i] = b;
        for (int k = 0; k < 3; k++) sb.cen[3 * (size_t)i + k] = bvhr::centroid(b.lo[k], b.hi[k]);
        sb.idx[(size_t)i] = i;
    }
    bn.reserve((size_t)n);
    return sb.build(0, n, 0, bn);
}

// Triangle records of `out` in leaf order; order[i] is the original index of
// leaf slot i.
void emit_tris(const Triangle* tris, const std::vector<int>& order, QBvh& out, bool vertices) {
    const size_t n = order.size();
    out.tris.resize(3 * n);
    for (size_t i = 0; i < n; i++) {
        const int orig = order[i];
        const Triangle& t = tris[orig];
        float fi;
        std::memcpy(&fi, &orig, 4);
        out.tris[3 * i] = make_float4(t.v0.x, t.v0.y, t.v0.z, fi);
        if (vertices) {
            out.tris[3 * i + 1] = make_float4(t.v1.x, t.v1.y, t.v1.z, 0.0f);
            out.tris[3 * i + 2] = make_float4(t.v2.x, t.v2.y, t.v2.z, 0.0f);
        } else {
            out.tris[3 * i + 1] = make_float4(t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z, 0.0f);
            out.tris[3 * i + 2] = make_float4(t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z, 0.0f);
        }
    }
}

// Collapses the binary tree bn (root `root`; a leaf has count > 0) into
// 4-wide nodes, breadth first from the root, each inner node opening its
// largest-area inner child until it has four children.
void collapse(const std::vector<BNode>& bn, int root, QBvh& out) {
    struct Pending { int bnode; int slot; };
    std::vector<Pending> queue;
    std::vector<int> ndepth;
    int cur_depth = 0;
    auto emit = [&](int b) {
        const int id = (int)out.nodes.size();
        ndepth.push_back(cur_depth + 1);
        out.max_depth = std::max(out.max_depth, cur_depth + 1);
        out.nodes.emplace_back();
        std::memset(&out.nodes.back(), 0, sizeof(dev::QNode4));
        queue.push_back({b, id});
        return id;
    };
    if (bn[(size_t)root].count > 0) {
        // A single leaf: wrap it in one node with one child.
        const int id = emit(root);
        queue.clear();
        queue.push_back({-1 - root, id});
    } else {
        emit(root);
    }
    for (size_t qi = 0; qi < queue.size(); qi++) {
        const int b = queue[qi].bnode;
        const int id = queue[qi].slot;
        cur_depth = ndepth[(size_t)id];
        std::vector<int> kids;
        if (b < 0) {
            kids.push_back(-1 - b);
        } else {
            kids = {bn[(size_t)b].left, bn[(size_t)b].right};
            while (kids.size() < 4) {
                int pick = -1;
                float best = -1.0f;
                for (size_t k = 0; k < kids.size(); k++) {
                    const BNode& c = bn[(size_t)kids[k]];
                    if (c.count == 0 && c.box.area() > best) { best = c.box.area(); pick = (int)k; }
                }
                if (pick < 0) break;
                const BNode c = bn[(size_t)kids[(size_t)pick]];
                kids[(size_t)pick] = c.left;
                kids.push_back(c.right);
            }
        }
        Box nb;
        for (int k : kids) nb.grow(bn[(size_t)k].box);
        float origin[3], scale[3];
        int ebits[3];
        for (int a = 0; a < 3; a++) {
            origin[a] = nb.lo[a];
            const int e = bvhr::frame_exponent(nb.lo[a], nb.hi[a]);
            scale[a] = std::ldexp(1.0f, e);
            ebits[a] = e + 127;
        }
        uint32_t packed = (uint32_t)ebits[0] | ((uint32_t)ebits[1] << 8) | ((uint32_t)ebits[2] << 16) |
                          ((uint32_t)kids.size() << 24);
        float pw;
        std::memcpy(&pw, &packed, 4);
        uint8_t q[6][4] = {{0}};
        uint32_t child[4] = {0, 0, 0, 0};
        for (size_t k = 0; k < kids.size(); k++) {
            const BNode& c = bn[(size_t)kids[k]];
            for (int a = 0; a < 3; a++)
                bvhr::quantize_axis(origin[a], scale[a], c.box.lo[a], c.box.hi[a], q[2 * a][k], q[2 * a + 1][k]);
            if (c.count > 0) {
                child[k] = 0x80000000u | ((uint32_t)c.first << 3) | (uint32_t)(c.count - 1);
            } else {
                child[k] = (uint32_t)emit(kids[k]);
            }
        }
        dev::QNode4& node = out.nodes[(size_t)id];
        node.origin_exp = make_float4(origin[0], origin[1], origin[2], pw);
        node.child = make_uint4(child[0], child[1], child[2], child[3]);
        auto word = [&](int row) {
            return (uint32_t)q[row][0] | ((uint32_t)q[row][1] << 8) | ((uint32_t)q[row][2] << 16) |
                   ((uint32_t)q[row][3] << 24);
        };
        node.qbox = make_uint4(word(0), word(1), word(2), word(3));
        node.qz = make_uint2(word(4), word(5));
        node.pad = make_uint2(0, 0);
    }
    out.leaf_size_max = kMaxLeaf;
}

// The binary tree bn restricted to the leaf slots `kept` marks (pre: its
// prefix counts, so kept slot i moves to pre[i]): a leaf keeps its kept
// triangles (none: the leaf goes), an inner node with one child left is
// replaced by that child, and every box is the union of the kept triangle
// boxes below it.  Returns the new root in `out`, or -1 when nothing is kept.
int prune(const std::vector<BNode>& bn, int i, const std::vector<int>& pre, const std::vector<unsigned char>& kept,
          const SahBuilder& sb, std::vector<BNode>& out) {
    const BNode& b = bn[(size_t)i];
    if (b.count > 0) {
        const int kc = pre[(size_t)(b.first + b.count)] - pre[(size_t)b.first];
        if (kc == 0) return -1;
        BNode o;
        o.first = pre[(size_t)b.first];
        o.count = kc;
        for (int p = b.first; p < b.first + b.count; p++)
            if (kept[(size_t)p]) o.box.grow(sb.tri_box[(size_t)sb.idx[(size_t)p]]);
        out.push_back(o);
        return (int)out.size() - 1;
    }
    const int l = prune(bn, b.left, pre, kept, sb, out);
    const int r = prune(bn, b.right, pre, kept, sb, out);
    if (l < 0) return r;
    if (r < 0) return l;
    BNode o;
    o.left = l;
    o.right = r;
    o.box = out[(size_t)l].box;
    o.box.grow(out[(size_t)r].box);
    out.push_back(o);
    return (int)out.size() - 1;
}

void reset(QBvh& q, bool vertices) {
    q.nodes.clear();
    q.tris.clear();
    q.max_depth = 0;
    q.vertices = vertices;
}

}  // namespace

void build_qbvh4(const Triangle* tris, const std::vector<int>& subset, QBvh& out, bool vertices) {
    reset(out, vertices);
    const int n = (int)subset.size();
    if (n <= 0) return;
    SahBuilder sb;
    std::vector<BNode> bn;
    const int root = sah_build(tris, subset, sb, bn);
    std::vector<int> order((size_t)n);
    for (int i = 0; i < n; i++) order[(size_t)i] = subset[(size_t)sb.idx[(size_t)i]];
    emit_tris(tris, order, out, vertices);
    collapse(bn, root, out);
}

void build_qbvh4_with_kept(const Triangle* tris, int n, const std::vector<unsigned char>& keep, QBvh& all,
                           QBvh& kept_out, bool vertices) {
    reset(all, vertices);
    reset(kept_out, vertices);
    if (n <= 0) return;
    std::vector<int> subset((size_t)n);
    for (int i = 0; i < n; i++) subset[(size_t)i] = i;
    SahBuilder sb;
    std::vector<BNode> bn;
    const int root = sah_build(tris, subset, sb, bn);
    std::vector<int> order((size_t)n), kept_order;
    std::vector<unsigned char> kept((size_t)n);
    std::vector<int> pre((size_t)n + 1, 0);
    for (int i = 0; i < n; i++) {
        order[(size_t)i] = sb.idx[(size_t)i];
        kept[(size_t)i] = keep[(size_t)order[(size_t)i]] ? 1 : 0;
        pre[(size_t)i + 1] = pre[(size_t)i] + kept[(size_t)i];
        if (kept[(size_t)i]) kept_order.push_back(order[(size_t)i]);
    }
    emit_tris(tris, order, all, vertices);
    collapse(bn, root, all);
    if (kept_order.empty()) return;
    std::vector<BNode> pn;
    pn.reserve(bn.size());
    const int proot = prune(bn, root, pre, kept, sb, pn);
    emit_tris(tris, kept_order, kept_out, vertices);
    collapse(pn, proot, kept_out);
}

// Structural check of a BVH4 (host only): every triangle slot is referenced
// by exactly one leaf, every decoded child box contains the boxes of all
// triangles below it, and the depth fits the traversal stack.  Returns 0 or
// a negative code; `depth` gets the tree depth.
int check_qbvh4(const QBvh& q, int& depth) {
    depth = 0;
    const size_t ntri = q.tris.size() / 3;
    if (q.nodes.empty()) return ntri == 0 ? 0 : -1;
    std::vector<int> seen(ntri, 0);
    struct Item { uint32_t e; int d; Box bound; };
    std::vector<Item> st;
    Box root_bound;
    for (int k = 0; k < 3; k++) { root_bound.lo[k] = -FLT_MAX; root_bound.hi[k] = FLT_MAX; }
    st.push_back({0u, 1, root_bound});
    while (!st.empty()) {
        Item it = st.back();
        st.pop_back();
        depth = std::max(depth, it.d);
        if (it.e & 0x80000000u) {
            const uint32_t first = (it.e & 0x7fffffffu) >> 3, count = (it.e & 7u) + 1;
            for (uint32_t k = 0; k < count; k++) {
                const size_t slot = first + k;
                if (slot >= ntri) return -2;
                seen[slot]++;
                const float4 a = q.tris[3 * slot], b = q.tris[3 * slot + 1], c = q.tris[3 * slot + 2];
                float v[3][3] = {{a.x, a.y, a.z}, {b.x, b.y, b.z}, {c.x, c.y, c.z}};
                if (!q.vertices)
                    for (int p = 1; p < 3; p++)
                        for (int ax = 0; ax < 3; ax++) v[p][ax] += v[0][ax];
                for (int p = 0; p < 3; p++)
                    for (int ax = 0; ax < 3; ax++) {
                        // v0 + (v1 - v0) may round by an ulp: allow it for edge records
                        const float tol = q.vertices ? 0.0f : 1e-6f * (std::fabs(v[p][ax]) + 1.0f);
                        if (v[p][ax] < it.bound.lo[ax] - tol || v[p][ax] > it.bound.hi[ax] + tol) return -3;
                    }
            }
            continue;
        }
        if (it.e >= q.nodes.size()) return -4;
        const dev::QNode4& n = q.nodes[it.e];
        uint32_t packed;
        std::memcpy(&packed, &n.origin_exp.w, 4);
        const int count = (int)(packed >> 24);
        if (count < 1 || count > 4) return -5;
        const float org[3] = {n.origin_exp.x, n.origin_exp.y, n.origin_exp.z};
        float s[3];
        for (int a = 0; a < 3; a++) {
            uint32_t bits = ((packed >> (8 * a)) & 0xffu) << 23;
            std::memcpy(&s[a], &bits, 4);
        }
        const uint32_t words[6] = {n.qbox.x, n.qbox.y, n.qbox.z, n.qbox.w, n.qz.x, n.qz.y};
        const uint32_t ch[4] = {n.child.x, n.child.y, n.child.z, n.child.w};
        for (int i = 0; i < count; i++) {
            Box b;
            for (int a = 0; a < 3; a++) {
                b.lo[a] = std::fmaf((float)((words[2 * a] >> (8 * i)) & 0xffu), s[a], org[a]);
                b.hi[a] = std::fmaf((float)((words[2 * a + 1] >> (8 * i)) & 0xffu), s[a], org[a]);
            }
            st.push_back({ch[i], it.d + 1, b});
        }
    }
    for (int v : seen)
        if (v != 1) return -6;
    return 0;
}

// Tightness of a BVH4 against the triangles it was built from: every child
// box is exactly the outward quantisation, in its node's frame, of the union
// of the (canonical) boxes of the original triangles below it, and every
// frame is the one the builder derives from the union of its children.
// Returns 0 or a negative code.
namespace {
int tight_box(const QBvh& q, const Triangle* tris, uint32_t e, Box& out) {
    out = Box();
    if (e & 0x80000000u) {
        const uint32_t first = (e & 0x7fffffffu) >> 3, count = (e & 7u) + 1;
        for (uint32_t k = 0; k < count; k++) {
            int orig;
            std::memcpy(&orig, &q.tris[3 * (size_t)(first + k)].w, 4);
            const Triangle& t = tris[orig];
            const float v[3][3] = {{t.v0.x, t.v0.y, t.v0.z}, {t.v1.x, t.v1.y, t.v1.z}, {t.v2.x, t.v2.y, t.v2.z}};
            Box b;
            for (int p = 0; p < 3; p++) b.grow(v[p]);
            for (int a = 0; a < 3; a++) { b.lo[a] = bvhr::canon(b.lo[a]); b.hi[a] = bvhr::canon(b.hi[a]); }
            out.grow(b);
        }
        return 0;
    }
    const dev::QNode4& n = q.nodes[e];
    uint32_t packed;
    std::memcpy(&packed, &n.origin_exp.w, 4);
    const int count = (int)(packed >> 24);
    const uint32_t ch[4] = {n.child.x, n.child.y, n.child.z, n.child.w};
    const uint32_t words[6] = {n.qbox.x, n.qbox.y, n.qbox.z, n.qbox.w, n.qz.x, n.qz.y};
    Box kb[4];
    for (int i = 0; i < count; i++) {
        const int rc = tight_box(q, tris, ch[i], kb[i]);
        if (rc) return rc;
        out.grow(kb[i]);
    }
    for (int a = 0; a < 3; a++) {
        if (n.origin_exp.x != out.lo[0] || n.origin_exp.y != out.lo[1] || n.origin_exp.z != out.lo[2]) return -11;
        const int ex = bvhr::frame_exponent(out.lo[a], out.hi[a]);
        if ((int)((packed >> (8 * a)) & 0xffu) != ex + 127) return -12;
        const float scale = std::ldexp(1.0f, ex);
        for (int i = 0; i < count; i++) {
            uint8_t ql, qh;
            bvhr::quantize_axis(out.lo[a], scale, kb[i].lo[a], kb[i].hi[a], ql, qh);
            if (((words[2 * a] >> (8 * i)) & 0xffu) != ql || ((words[2 * a + 1] >> (8 * i)) & 0xffu) != qh) return -13;
        }
    }
    return 0;
}
}  // namespace

int check_qbvh4_tight(const QBvh& q, const Triangle* tris) {
    if (q.nodes.empty()) return 0;
    Box b;
    return tight_box(q, tris, 0u, b);
}

}  // namespace sheen

// Host-side self check of the wavefront form's triangle BVH for a scene:
// builds it and runs check_qbvh4.  Returns the tree depth (>= 0) or a
// negative error code.  No device work.
extern "C" int sheen_selfcheck_bvh4(const SheenScene* scene) {
    if (!scene || scene->num_triangles <= 0) return -1;
    std::vector<int> all((size_t)scene->num_triangles);
    for (int i = 0; i < scene->num_triangles; i++) all[(size_t)i] = i;
    sheen::QBvh q;
    sheen::build_qbvh4(scene->triangles, all, q);
    int depth = 0;
    const int rc = sheen::check_qbvh4(q, depth);
    return rc < 0 ? rc : depth;
}

// Host-side self check of the blocking triangles' BVH4 derived from the tree
// over all triangles (build_qbvh4_with_kept, blocking = material
// transmission <= 0.5): the tree over all equals build_qbvh4's byte for byte,
// both trees pass check_qbvh4 and check_qbvh4_tight, and the derived tree
// holds each blocking triangle exactly once.  Returns the derived tree's
// depth (0 when nothing blocks) or a negative code.  No device work.
extern "C" int sheen_selfcheck_bvh4_kept(const SheenScene* scene) {
    using namespace sheen;
    if (!scene || scene->num_triangles <= 0) return -1;
    const int n = scene->num_triangles;
    std::vector<int> all((size_t)n);
    std::vector<unsigned char> blocking((size_t)n);
    int nblock = 0;
    for (int i = 0; i < n; i++) {
        all[(size_t)i] = i;
        const int m = scene->triangles[i].material_id;
        const bool passable = m >= 0 && m < scene->num_materials && scene->materials[m].transmission > 0.5f;
        blocking[(size_t)i] = passable ? 0 : 1;
        nblock += passable ? 0 : 1;
    }
    QBvh built, q_all, q_kept;
    build_qbvh4(scene->triangles, all, built);
    build_qbvh4_with_kept(scene->triangles, n, blocking, q_all, q_kept);
    if (built.nodes.size() != q_all.nodes.size() || built.tris.size() != q_all.tris.size() ||
        std::memcmp(built.nodes.data(), q_all.nodes.data(), built.nodes.size() * sizeof(dev::QNode4)) != 0 ||
        std::memcmp(built.tris.data(), q_all.tris.data(), built.tris.size() * sizeof(float4)) != 0)
        return -20;
    int d_all = 0, d_kept = 0;
    int rc = check_qbvh4(q_all, d_all);
    if (rc < 0) return rc;
    if ((rc = check_qbvh4_tight(q_all, scene->triangles)) < 0) return rc;
    if ((int)(q_kept.tris.size() / 3) != nblock) return -21;
    if (nblock == 0) return q_kept.nodes.empty() ? 0 : -22;
    if ((rc = check_qbvh4(q_kept, d_kept)) < 0) return rc - 30;
    if ((rc = check_qbvh4_tight(q_kept, scene->triangles)) < 0) return rc - 30;
    std::vector<int> seen((size_t)n, 0);
    for (size_t k = 0; k < q_kept.tris.size() / 3; k++) {
        int orig;
        std::memcpy(&orig, &q_kept.tris[3 * k].w, 4);
        if (orig < 0 || orig >= n || !blocking[(size_t)orig] || seen[(size_t)orig]++) return -23;
    }
    if (d_kept > d_all) return -24;
    return d_kept;
}
