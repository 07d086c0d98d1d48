// trace_ref.cuh -- scene queries of the plain form, in the reference's order.
//
// One binary BVH per primitive class with one primitive per leaf (built on
// the host with the reference's median split, bvh_median.cpp), traversed
// depth first exactly as bvh.h:605-922 does: pop, test the box against the
// ray's [t_min, t_max], at a leaf test the primitive and keep it if strictly
// closer, else push left then right.  No culling against the closest hit
// and no child ordering: the plain form visits the same boxes and tests the
// same primitives in the same order as the reference kernel, so even ties
// between equal-distance primitives resolve the same way.
#pragma once
#include "csg.cuh"
#include "exact.cuh"

namespace sheen {
namespace dev {

struct Counters {
    unsigned long long nodes = 0, prims = 0;
    // the part of nodes / prims spent on the glass-aware shadow queries of
    // the lighting loop (the wavefront form's shadow stage)
    unsigned long long shadow_nodes = 0, shadow_prims = 0;
};

constexpr int kRefStack = 64;

// Walks `nodes` and calls leaf(prim) for every leaf whose box the ray
// crosses.  Children are pushed only while the fixed stack has room; the
// median-split trees built here are at most ~log2(n)+1 deep, far below it.
template <bool COUNT, class Leaf>
__device__ __forceinline__ void dfs_ref(const BvhNode* nodes, const Ray& r, Counters& c, Leaf leaf) {
    int stack[kRefStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int id = stack[--sp];
        const float4 a = __ldg(&nodes[id].a), b = __ldg(&nodes[id].b);
        if (COUNT) c.nodes++;
        if (!box_hit_ref(r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z))) continue;
        const int left = __float_as_int(a.w), right = __float_as_int(b.w);
        if (left < 0) {
            if (COUNT) c.prims++;
            leaf(~left);
        } else if (sp <= kRefStack - 2) {
            stack[sp++] = left;
            stack[sp++] = right;
        }
    }
}

template <bool COUNT>
__device__ __forceinline__ bool spheres_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_objects == 0 || !S.sphere_bvh) return false;
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.sphere_bvh, r, c, [&](int i) {
        const Object o = S.objects[i];
        Hit tmp;
        if (o.type == 0 && sphere_test(r, f3(o.param1), o.param2, tmp) && tmp.t < best) {
            h = tmp; h.mat = o.material_id; h.obj = i; best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool strands_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_strands == 0) return false;
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.strand_bvh, r, c, [&](int i) {
        Hit tmp;
        if (strand_test(r, S.strands[i], S.sweep_points, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool mesh_ref_flat(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_tris == 0) return false;
    float best = r.tmax, bu = 0.0f, bv = 0.0f;
    int bi = -1;
    dfs_ref<COUNT>(S.mesh_bvh, r, c, [&](int i) {
        const float4 p0 = __ldg(&S.tri_verts[3 * i]), p1 = __ldg(&S.tri_verts[3 * i + 1]),
                     p2 = __ldg(&S.tri_verts[3 * i + 2]);
        float t, u, v;
        if (tri_test(r, f3(p0.x, p0.y, p0.z), f3(p1.x, p1.y, p1.z), f3(p2.x, p2.y, p2.z), t, u, v) && t < best) {
            best = t; bu = u; bv = v; bi = i;
        }
    });
    if (bi < 0) return false;
    tri_finish(r, S.tris[bi], best, bu, bv, h);
    h.obj = -(bi + 1);
    return true;
}

// Scenes with instanced meshes (dev/instances.cuh) add them to the category.
template <bool COUNT>
__device__ __noinline__ bool mesh_ref_inst(const DevScene& S, const Ray& r, Hit& h, Counters& c);

template <bool COUNT>
__device__ __forceinline__ bool mesh_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_instances > 0) return mesh_ref_inst<COUNT>(S, r, h, c);
    return mesh_ref_flat<COUNT>(S, r, h, c);
}

// Extension scenes (SheenSceneExt) walk their categories in functions of
// their own, not inlined, so that the plain kernel's code for the
// reference's shapes is what it is without extensions.
template <bool COUNT>
static __device__ __noinline__ bool hfs_ref_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.hf_bvh, r, c, [&](int i) {
        Hit tmp;
        const HfGrid g = hf_grid_of(S, i);
        if ((g.h ? hf_test_grid(r, S.hfs[i], tmp, g) : hf_test(r, S.hfs[i], tmp)) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool hfs_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_hfs == 0) return false;
    if (S.hf_grid) return hfs_ref_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.hf_bvh, r, c, [&](int i) {
        Hit tmp;
        if (hf_test(r, S.hfs[i], tmp) && tmp.t < best) { h = tmp; h.obj = -(i + 1); best = tmp.t; any = true; }
    });
    return any;
}

template <bool COUNT>
static __device__ __noinline__ bool ses_ref_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.se_bvh, r, c, [&](int i) {
        Hit tmp;
        const float n2 = se_n2_of(S, i);
        if ((n2 > 0.0f ? se_test2(r, S.ses[i], n2, tmp) : se_test(r, S.ses[i], tmp, S.se_polish)) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool ses_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_ses == 0) return false;
    if (S.se_n2) return ses_ref_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.se_bvh, r, c, [&](int i) {
        Hit tmp;
        if (se_test(r, S.ses[i], tmp, S.se_polish) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
static __device__ __noinline__ bool lathes_ref_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.lathe_bvh, r, c, [&](int i) {
        Hit tmp;
        if (lathe_any_test(S, r, i, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool lathes_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_lathes == 0) return false;
    if (S.lathe_bz) return lathes_ref_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.lathe_bvh, r, c, [&](int i) {
        Hit tmp;
        if (lathe_test(r, S.lathes[i], S.lathe_points, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
static __device__ __noinline__ bool prisms_ref_ext(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.prism_bvh, r, c, [&](int i) {
        Hit tmp;
        if (prism_any_test(S, r, i, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

template <bool COUNT>
__device__ __forceinline__ bool prisms_ref(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
    if (S.num_prisms == 0) return false;
    if (S.prism_bz) return prisms_ref_ext<COUNT>(S, r, h, c);
    bool any = false;
    float best = r.tmax;
    dfs_ref<COUNT>(S.prism_bvh, r, c, [&](int i) {
        Hit tmp;
        if (prism_test(r, S.prisms[i], S.prism_points, tmp) && tmp.t < best) {
            h = tmp; h.obj = -(i + 1); best = tmp.t; any = true;
        }
    });
    return any;
}

__device__ __forceinline__ bool planes_scan(const DevScene& S, const Ray& r, Hit& h) {
    bool any = false;
    float best = r.tmax;
    for (int i = 0; i < S.num_planes; i++) {
        const Plane p = S.planes[i];
        Hit tmp;
        if (plane_test(r, f3(p.normal), p.d, tmp) && tmp.t < best) {
            h = tmp; h.mat = p.material_id; h.obj = -1 - i; best = tmp.t; any = true;
        }
    }
    return any;
}

// integrator/raycast.h:14-70: closest over the categories; a later category
// replaces the current hit only when strictly closer.
template <bool COUNT>
__device__ __noinline__ bool closest_ref(const DevScene& S, const Ray& r, Hit& rec, Counters& c) {
    float best = r.tmax;
    bool hit = false;
    Hit t;
    if (spheres_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (strands_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (mesh_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (hfs_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (ses_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (lathes_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (prisms_ref<COUNT>(S, r, t, c) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (csg_closest(S, r, t, false) && t.t < best) { best = t.t; rec = t; hit = true; }
    if (planes_scan(S, r, t) && t.t < best) { best = t.t; rec = t; hit = true; }
    return hit;
}

// integrator/raycast.h:74-97: the first category (strands excluded) that
// reports a hit answers with its closest hit.
template <bool COUNT>
__device__ __noinline__ bool opaque_ref(const DevScene& S, const Ray& r, Hit& rec, Counters& c) {
    if (spheres_ref<COUNT>(S, r, rec, c)) return true;
    if (mesh_ref<COUNT>(S, r, rec, c)) return true;
    if (hfs_ref<COUNT>(S, r, rec, c)) return true;
    if (ses_ref<COUNT>(S, r, rec, c)) return true;
    if (lathes_ref<COUNT>(S, r, rec, c)) return true;
    if (prisms_ref<COUNT>(S, r, rec, c)) return true;
    if (csg_closest(S, r, rec, false)) return true;
    return planes_scan(S, r, rec);
}

// bvh.h:928-960: strand optical depth along a shadow ray, stopping once
// tau exceeds 6.
template <bool COUNT, bool CULL = false>
__device__ __noinline__ float strands_tau_ref(const DevScene& S, const Ray& r, Counters& c) {
    if (S.num_strands == 0) return 0.0f;
    float tau = 0.0f;
    int stack[kRefStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int id = stack[--sp];
        const float4 a = __ldg(&S.strand_bvh[id].a), b = __ldg(&S.strand_bvh[id].b);
        if (COUNT) c.nodes++;
        if (!box_hit_ref(r, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z))) continue;
        const int left = __float_as_int(a.w), right = __float_as_int(b.w);
        if (left < 0) {
            if (COUNT) c.prims++;
            tau += strand_tau<CULL>(r, S.strands[~left], S.sweep_points, 6.0f);
            if (tau > 6.0f) return tau;
        } else if (sp <= kRefStack - 2) {
            stack[sp++] = left;
            stack[sp++] = right;
        }
    }
    return tau;
}

// Result of the shadow (opaque-set) query.
enum : int { kClear = 0, kBlocked = 1, kPass = 2 };
struct ShadowHit {
    float t;
    float3 p;
};

// Glass test of a shadow hit: transmission above 0.5, read through the
// material's property map when mask_aware (render_kernel.cu:261-262), from
// the material alone otherwise (the beam's test, render_kernel.cu:637).
__device__ __forceinline__ int classify_shadow_hit(const DevScene& S, const Hit& h, bool mask_aware, ShadowHit& sh) {
    const Material& m = S.materials[h.mat];
    float tr;
    if (mask_aware) {
        tr = 0.0f;
        if (m.transmission > 0.0f) {
            tr = m.transmission;
            if (m.mask_id >= 0 && m.mask_id < S.num_textures) {
                // transmission_at without the shade.cuh dependency: R of the map at level 0
                const TextureRef& t = S.textures[m.mask_id];
                float u = h.uv.x - floorf(h.uv.x), v = 1.0f - (h.uv.y - floorf(h.uv.y));
                float fx = u * (float)(t.width - 1), fy = v * (float)(t.height - 1);
                int x0 = (int)fx, y0 = (int)fy, x1 = (x0 + 1) % t.width, y1 = (y0 + 1) % t.height;
                float tx = fx - (float)x0, ty = fy - (float)y0;
                auto R = [&](int x, int y) { return t.pixels[(size_t)(y * t.width + x) * 3] / 255.0f; };
                float a = R(x0, y0) * (1.0f - tx) + R(x1, y0) * tx;
                float b = R(x0, y1) * (1.0f - tx) + R(x1, y1) * tx;
                tr *= a * (1.0f - ty) + b * ty;
            }
        }
    } else {
        tr = m.transmission;
    }
    sh.t = h.t;
    sh.p = h.p;
    return tr > 0.5f ? kPass : kBlocked;
}

// The plain form's query policy for the shared integrator.
template <bool COUNT>
struct RefTracer {
    __device__ __forceinline__ static bool closest(const DevScene& S, const Ray& r, Hit& h, Counters& c) {
        return closest_ref<COUNT>(S, r, h, c);
    }
    __device__ __forceinline__ static int shadow(const DevScene& S, const Ray& r, bool mask_aware, ShadowHit& sh,
                                                 Counters& c) {
        Hit h;
        if (!opaque_ref<COUNT>(S, r, h, c)) return kClear;
        return classify_shadow_hit(S, h, mask_aware, sh);
    }
    __device__ __forceinline__ static bool occluded(const DevScene& S, const Ray& r, Counters& c) {
        Hit h;
        return opaque_ref<COUNT>(S, r, h, c);
    }
    __device__ __forceinline__ static float strand_depth(const DevScene& S, const Ray& r, Counters& c) {
        return strands_tau_ref<COUNT>(S, r, c);
    }
};

}  // namespace dev
}  // namespace sheen
