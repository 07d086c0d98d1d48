// integrator.cuh -- the per-sample integrator of render_kernel.cu:487-809,
// written once over a query policy T so that the plain megakernel
// (reference-order BVHs) and the BVH4 megakernel share every line of
// shading.  T provides:
//   closest(S, r, hit, c)                 scene_intersect (raycast.h:14-70)
//   shadow(S, r, mask_aware, sh, c)       scene_intersect_opaque plus the
//                                         glass test of its hit: kClear,
//                                         kBlocked or kPass (sh = hit t, point)
//   occluded(S, r, c)                     scene_intersect_opaque's boolean
//   strand_depth(S, r, c)                 strand_bvh_tau (bvh.h:928-960)
#pragma once
#include "shade.cuh"
#include "trace_bvh4.cuh"   // both query policies, instanced meshes

namespace sheen {
namespace dev {

// Rays issued, counted the way the throughput metric counts them: every
// scene query is one ray (primary, each glass pass of a shadow ray, every
// reflection/refraction segment, beam and medium shadow rays).
struct RayTally {
    unsigned int primary = 0, shadow = 0, secondary = 0;
};

// Shadow query with glass passes (render_kernel.cu:243-268): up to three
// opaque-set queries; a hit whose transmission exceeds 0.5 is passed by
// moving the origin 0.002 past it (t_max kept, as in the reference).
template <class T, bool COUNT>
__device__ __forceinline__ bool shadow_blocked(const DevScene& S, Ray r, RayTally& rt, Counters& c) {
    for (int pass = 0; pass < 3; pass++) {
        rt.shadow++;
        ShadowHit sh;
        const unsigned long long n0 = c.nodes, p0 = c.prims;
        const int q = T::shadow(S, r, true, sh, c);
        if (COUNT) {
            c.shadow_nodes += c.nodes - n0;
            c.shadow_prims += c.prims - p0;
        }
        if (q == kClear) return false;
        if (q == kBlocked) return true;
        r.o = sh.p + r.d * 0.002f;
    }
    return false;
}

// render_kernel.cu:26-298
template <class T, bool COUNT>
__device__ float3 lighting(const DevScene& S, const Hit& h, float3 view, float footprint, uint32_t seed,
                           RayTally& rt, Counters& c) {
    const ShadePoint sp = shade_prepare(S, h, view, footprint);
    const Material& m = S.materials[h.mat];
    float3 result = shade_emitted(S, sp);
    for (int i = 0; i < S.num_lights; i++) {
        LightSample ls;
        if (!light_sample(S, sp, i, seed, ls)) continue;
        Ray sr;
        sr.o = sp.p + sp.ng * 0.002f;
        sr.d = normalize(ls.target - sr.o);
        sr.tmin = 0.001f;
        sr.tmax = ls.tmax;
        const bool blocked = shadow_blocked<T, COUNT>(S, sr, rt, c);
        if (m.shininess < 0.0f) return blocked ? f3(1.0f, 0.0f, 0.0f) : f3(0.0f, 1.0f, 0.0f);
        if (blocked) continue;
        float trans = 1.0f;
        if (m.anisotropy <= 0.0f && S.num_strands > 0) trans = expf(-T::strand_depth(S, sr, c));
        result += brdf(S, sp, ls.L, ls.radiance) * trans;
    }
    result += caustic_term(S, sp);
    return result;
}

// render_kernel.cu:339-436: single-scatter march through the boxed media.
template <class T, bool COUNT>
__device__ float3 media_march(const DevScene& S, const Ray& ray, float t_surf, uint32_t seed, float& tau_out,
                              RayTally& rt, Counters& c) {
    float3 ins = f3(0.0f, 0.0f, 0.0f);
    float tau_total = 0.0f;
    for (int mi = 0; mi < S.num_media; mi++) {
        const Medium md = S.media[mi];
        if (md.samples <= 0) continue;
        float m0, m1;
        if (!medium_span(ray, f3(md.center), f3(md.half), m0, m1)) continue;
        m0 = fmaxf(m0, ray.tmin);
        m1 = fminf(m1, t_surf);
        if (m1 <= m0) continue;
        const int n = md.samples > 64 ? 64 : md.samples;
        const float dt = (m1 - m0) / (float)n;
        float tau = 0.0f;
        for (int k = 0; k < n; k++) {
            float jit = rand01(seed ^ (uint32_t)(mi * 9781u) ^ (uint32_t)(k * 6271u));
            float t = m0 + ((float)k + jit) * dt;
            float3 p = ray.o + ray.d * t;
            float3 rad = f3(0.0f, 0.0f, 0.0f);
            for (int i = 0; i < S.num_lights; i++) {
                const Light& l = S.lights[i];
                if (!(l.flags & 1)) continue;
                float3 ld, lr;
                float ldist;
                if (l.type == 0) {
                    ld = sun_direction(l, seed ^ (uint32_t)(i * 2654435761u) ^ (uint32_t)(k * 2246822519u));
                    ldist = 1.0e9f;
                    lr = f3(l.color) * l.intensity;
                } else {
                    float3 tl = f3(l.position) - p;
                    float d2 = fmaxf(dot(tl, tl), 1.0e-4f);
                    ldist = sqrtf(d2);
                    ld = tl / ldist;
                    lr = f3(l.color) * (l.intensity / (12.5663706f * d2));
                    if (l.type == 3) {
                        float cc = dot(-ld, f3(l.direction));
                        float ch = cosf(l.angle);
                        if (cc <= ch) continue;
                        float bl = fminf(fmaxf(l.blend, 0.0f), 1.0f);
                        float cs = cosf(l.angle * (1.0f - bl));
                        if (cs > ch + 1.0e-4f) lr = lr * fminf((cc - ch) / (cs - ch), 1.0f);
                    }
                }
                Ray sr;
                sr.o = p; sr.d = ld; sr.tmin = 0.002f; sr.tmax = ldist;
                rt.shadow++;
                if (T::occluded(S, sr, c)) continue;
                rad += lr;
            }
            float3 sc = f3(md.sigma_s) * rad * 0.07957747f;
            ins += sc * (expf(-tau) * dt);
            tau += md.sigma_t * dt;
        }
        tau_total += tau;
    }
    tau_out = tau_total;
    return ins;
}

// render_kernel.cu:560-652: visible spot-light cones, 6 steps, each step
// with its own glass-aware shadow ray (here t_max shrinks per glass pass).
template <class T, bool COUNT>
__device__ float3 beams(const DevScene& S, const Ray& ray, bool hit, float t_hit, uint32_t seed,
                        RayTally& rt, Counters& c) {
    float3 total = f3(0.0f, 0.0f, 0.0f);
    for (int i = 0; i < S.num_lights; i++) {
        const Light& l = S.lights[i];
        if (l.type != 3 || l.beam <= 0.0f) continue;
        const float t_end = hit ? fminf(t_hit, 30.0f) : 30.0f;
        if (t_end <= 0.0f) continue;
        const float dt = t_end / 6.0f;
        const float ch = cosf(l.angle);
        const float bl = fminf(fmaxf(l.blend, 0.0f), 1.0f);
        const float cs = cosf(l.angle * (1.0f - bl));
        float3 acc = f3(0.0f, 0.0f, 0.0f);
        for (int k = 0; k < 6; k++) {
            float t = ((float)k + 0.5f) * dt;
            float3 p = ray.o + ray.d * t;
            float3 v = p - f3(l.position);
            float d2 = fmaxf(dot(v, v), 1.0e-4f);
            float cc = dot(v, f3(l.direction)) * rsqrtf(d2);
            if (cc <= ch) continue;
            float w = 1.0f;
            if (cs > ch + 1.0e-4f) w = fminf((cc - ch) / (cs - ch), 1.0f);
            float dens = l.beam * l.intensity * 1.0e-3f / (1.0f + 0.25f * d2);
            float3 target = f3(l.position);
            if (l.radius > 0.0f) {
                float3 axis = normalize(-v);
                float3 t1 = normalize(cross(axis, up_for(axis)));
                float3 t2 = cross(axis, t1);
                float rr = sqrtf(rand01(seed ^ (uint32_t)(k * 2654435761u) ^ 0x85ebca6bu)) * l.radius;
                float ph = 6.2831853f * rand01(seed ^ (uint32_t)(k * 2246822519u) ^ 0xc2b2ae35u);
                target = f3(l.position) + t1 * (cosf(ph) * rr) + t2 * (sinf(ph) * rr);
            }
            float3 tl = target - p;
            float ld = sqrtf(fmaxf(dot(tl, tl), 1.0e-8f));
            float3 ldir = tl / ld;
            float remain = ld * 0.999f;
            Ray sr;
            sr.o = p; sr.d = ldir; sr.tmin = 0.002f; sr.tmax = remain;
            bool blocked = false;
            for (int pass = 0; pass < 3; pass++) {
                ShadowHit sh;
                rt.shadow++;
                const int q = T::shadow(S, sr, false, sh, c);
                if (q == kClear) { blocked = false; break; }
                if (q == kPass) {
                    remain -= sh.t + 0.002f;
                    if (remain <= 0.0f) { blocked = false; break; }
                    sr.o = sh.p + ldir * 0.002f;
                    sr.tmax = remain;
                    continue;
                }
                blocked = true;
                break;
            }
            if (blocked) continue;
            acc += f3(l.color) * (dens * w * dt);
        }
        total += acc;
    }
    return total;
}

// Camera ray of sample (s of ns) in pixel (x, y): render_kernel.cu:491-521.
// centered: no jitter (sample_offset_centered), an extension.
__device__ __forceinline__ Ray camera_ray(const CameraData& cam, int x, int y, int s, int ns, int W, int H,
                                          float& pix_angle, int centered) {
    float2 off = centered ? sample_offset_centered(s, ns) : sample_offset(s, ns, x, y);
    float u = (float(x) + off.x) / float(W) * 2.0f - 1.0f;
    float v = 1.0f - (float(y) + off.y) / float(H) * 2.0f;
    float tan_h = 1.0f, tan_x = 1.0f, tan_y = 1.0f;
    if (cam.focal_length > 0.0f) {
        tan_h = 0.5f * cam.sensor_width / cam.focal_length;
        if (W >= H) { tan_x = tan_h; tan_y = tan_h * float(H) / float(W); }
        else { tan_y = tan_h; tan_x = tan_h * float(W) / float(H); }
    }
    Ray r;
    r.o = f3(cam.position);
    r.d = normalize(f3(cam.forward) + f3(cam.right) * (u * tan_x + cam.shift_x * tan_h) +
                    f3(cam.up) * (v * tan_y + cam.shift_y * tan_h));
    r.tmin = 0.001f;
    r.tmax = 1e10f;
    pix_angle = 2.0f * tan_x / (float)W;
    return r;
}

__device__ __forceinline__ uint32_t sample_seed(int x, int y, int s) {
    return hash32((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)s * 83492791u);
}

// One sample of one pixel: render_kernel.cu:491-809.
template <class T, bool COUNT>
__device__ float3 render_sample(const DevScene& S, int x, int y, int s, int ns, int W, int H,
                                RayTally& rt, Counters& c) {
    float pix;
    const Ray ray = camera_ray(S.cam, x, y, s, ns, W, H, pix, S.aa_centered);
    const uint32_t seed = sample_seed(x, y, s);
    Hit rec;
    rt.primary++;
    const bool hit = T::closest(S, ray, rec, c);
    float3 color = hit ? lighting<T, COUNT>(S, rec, -ray.d, rec.t * pix, seed, rt, c) : sky(ray.d);
    color += beams<T, COUNT>(S, ray, hit, hit ? rec.t : 0.0f, seed, rt, c);
    if (S.num_media > 0) {
        float tau = 0.0f;
        float3 ins = media_march<T, COUNT>(S, ray, hit ? rec.t : 1.0e9f, seed, tau, rt, c);
        color = color * expf(-tau) + ins;
    }
    if (!hit) return color;
    const Material pm = S.materials[rec.mat];
    if (pm.reflect > 0.0f) {
        Ray rr;
        rr.o = rec.p + rec.n * 0.002f;
        rr.d = normalize(ray.d - rec.n * (2.0f * dot(ray.d, rec.n)));
        rr.tmin = 0.001f;
        rr.tmax = 1.0e10f;
        Hit rh;
        rt.secondary++;
        const bool rhit = T::closest(S, rr, rh, c);
        float3 rcol = rhit ? lighting<T, COUNT>(S, rh, -rr.d, rh.t * pix, seed, rt, c) : sky(rr.d);
        if (S.num_media > 0) {
            float rtau = 0.0f;
            float3 rins = media_march<T, COUNT>(S, rr, rhit ? rh.t : 1.0e9f, seed, rtau, rt, c);
            rcol = rcol * expf(-rtau) + rins;
        }
        const float w = fminf(pm.reflect, 1.0f);
        color = color * (1.0f - w) + rcol * w;
    }
    const float gtr = transmission_at(S, pm, rec.uv);
    if (gtr > 0.0f) {
        float3 through = f3(0.0f, 0.0f, 0.0f);
        float w = 1.0f;
        Ray gr = ray;
        Hit gh = rec;
        bool entering = true;
        for (int b = 0; b < 3; b++) {
            const Material sm = S.materials[gh.mat];
            const float3 n = gh.n, d = gr.d;
            const float ior = fmaxf(ior_at(S, sm, gh.uv), 1.0f);
            const float eta = entering ? 1.0f / ior : ior;
            const float cosi = fmaxf(-dot(d, n), 1.0e-4f);
            const float k = 1.0f - eta * eta * (1.0f - cosi * cosi);
            const float3 td = k < 0.0f ? normalize(d + 2.0f * cosi * n) : normalize(eta * d + (eta * cosi - sqrtf(k)) * n);
            w *= transmission_at(S, sm, gh.uv);
            gr.o = gh.p + td * 0.002f;
            gr.d = td;
            gr.tmin = 0.001f;
            gr.tmax = 1.0e10f;
            Hit nh;
            rt.secondary++;
            if (!T::closest(S, gr, nh, c)) { through += w * sky(td); break; }
            if (transmission_at(S, S.materials[nh.mat], nh.uv) > 0.0f) { entering = !entering; gh = nh; continue; }
            through += w * lighting<T, COUNT>(S, nh, -td, nh.t * pix, seed, rt, c);
            break;
        }
        color = color * (1.0f - fminf(gtr, 1.0f)) + through;
    }
    return color;
}

// Extension (no counterpart in the reference, whose mirror ray stops at
// depth 1 and whose refraction follows at most three faces): reflect +
// refract recursion to S.bounces bounces.  Every hit below the depth
// limit blends as the reference's primary hit does (render_kernel.cu:
// 730-731, 805) -- its lighting weighted by (1 - wr)(1 - wt), a mirror ray by
// wr (1 - wt) and a refracted ray by the face's transmission, wr =
// min(reflect, 1), wt = min(transmission, 1) -- and a hit at the limit
// contributes its lighting alone, as the reference's depth-1 mirror hit
// does.  A refracted ray crosses the face (the next glass face it meets is
// an exit: eta = ior, then an entry again); a mirror ray, and a ray turned
// back by total internal reflection, stays on its side.  Media act on every
// segment (the reference marches them on the primary and the mirror ray),
// beams on the primary ray only.  Paths are walked depth first with an
// explicit stack (at most one pending sibling per bounce); the sum runs in
// that fixed order.
template <class T, bool COUNT>
__device__ __noinline__ float3 render_sample_deep(const DevScene& S, int x, int y, int s, int ns, int W, int H,
                                                  RayTally& rt, Counters& c) {
    struct Node {
        float3 o, d, w;
        int depth, inside;
    };
    float pix;
    const Ray ray0 = camera_ray(S.cam, x, y, s, ns, W, H, pix, S.aa_centered);
    const uint32_t seed = sample_seed(x, y, s);
    const int D = S.bounces < kMaxDeepBounces ? S.bounces : kMaxDeepBounces;
    Node st[kMaxDeepBounces + 2];
    int sp = 0;
    st[sp++] = Node{ray0.o, ray0.d, f3(1.0f, 1.0f, 1.0f), 0, 0};
    float3 color = f3(0.0f, 0.0f, 0.0f);
    while (sp > 0) {
        const Node nd = st[--sp];
        Ray r;
        r.o = nd.o; r.d = nd.d; r.tmin = 0.001f; r.tmax = 1.0e10f;
        Hit h;
        if (nd.depth == 0) rt.primary++;
        else rt.secondary++;
        const bool hit = T::closest(S, r, h, c);
        float3 local = hit ? lighting<T, COUNT>(S, h, -r.d, h.t * pix, seed, rt, c) : sky(r.d);
        if (nd.depth == 0) local += beams<T, COUNT>(S, r, hit, hit ? h.t : 0.0f, seed, rt, c);
        if (S.num_media > 0) {
            float tau = 0.0f;
            const float3 ins = media_march<T, COUNT>(S, r, hit ? h.t : 1.0e9f, seed, tau, rt, c);
            local = local * expf(-tau) + ins;
        }
        if (!hit || nd.depth >= D) { color += nd.w * local; continue; }
        const Material m = S.materials[h.mat];
        const float wr = m.reflect > 0.0f ? fminf(m.reflect, 1.0f) : 0.0f;
        const float gtr = transmission_at(S, m, h.uv);
        const float wt = gtr > 0.0f ? fminf(gtr, 1.0f) : 0.0f;
        color += nd.w * local * ((1.0f - wr) * (1.0f - wt));
        if (gtr > 0.0f && sp < kMaxDeepBounces + 2) {
            const float ior = fmaxf(ior_at(S, m, h.uv), 1.0f);
            const float eta = nd.inside ? ior : 1.0f / ior;
            const float cosi = fmaxf(-dot(r.d, h.n), 1.0e-4f);
            const float k = 1.0f - eta * eta * (1.0f - cosi * cosi);
            const float3 td = k < 0.0f ? normalize(r.d + 2.0f * cosi * h.n)
                                       : normalize(eta * r.d + (eta * cosi - sqrtf(k)) * h.n);
            st[sp++] = Node{h.p + td * 0.002f, td, nd.w * gtr, nd.depth + 1, k < 0.0f ? nd.inside : !nd.inside};
        }
        if (wr > 0.0f && sp < kMaxDeepBounces + 2) {
            const float3 rd = normalize(r.d - h.n * (2.0f * dot(r.d, h.n)));
            st[sp++] = Node{h.p + h.n * 0.002f, rd, nd.w * (wr * (1.0f - wt)), nd.depth + 1, nd.inside};
        }
    }
    return color;
}

}  // namespace dev
}  // namespace sheen

