// shade.cuh -- surface shading pieces shared by the renderer forms.
//
// compute_lighting (render_kernel.cu:26-298) is split into independent
// steps so that the wavefront form can issue every shadow ray of a shading
// point as its own queue entry:
//   shade_prepare()  tangent frame, normal map, albedo, shininess
//   light_sample()   light position/direction, radiance, shadow-ray extent
//   brdf()           shade_direct (integrator/shading.h:158-175)
//   caustic_term()   photon-map gather (render_kernel.cu:286-296)
// The plain megakernel calls them in the reference's order.
#pragma once
#include "prims.cuh"

namespace sheen {
namespace dev {

// integrator/shading.h:20-22
__device__ __forceinline__ float tex_lod(const TextureRef& t, float uv_fp) {
    return log2f(fmaxf(uv_fp * (float)t.width, 1.0f));
}

// integrator/shading.h:26-58: bilinear RGB8 lookup in mip `lod` (rounded),
// repeat addressing, V flipped (image rows run top to bottom).
__device__ __forceinline__ float3 tex_fetch(const TextureRef& t, float2 uv, float lod) {
    int level = (int)floorf(lod + 0.5f);
    if (level < 0) level = 0;
    if (level >= t.mips) level = t.mips - 1;
    int w = t.width, h = t.height;
    size_t off = 0;
    for (int i = 0; i < level; i++) {
        off += (size_t)w * h * 3;
        w = w > 1 ? w / 2 : 1;
        h = h > 1 ? h / 2 : 1;
    }
    const unsigned char* base = t.pixels + off;
    float u = uv.x - floorf(uv.x);
    float v = 1.0f - (uv.y - floorf(uv.y));
    float fx = u * (float)(w - 1), fy = v * (float)(h - 1);
    int x0 = (int)fx, y0 = (int)fy;
    int x1 = (x0 + 1) % w, y1 = (y0 + 1) % h;
    float tx = fx - (float)x0, ty = fy - (float)y0;
    auto at = [&](int x, int y) {
        const unsigned char* p = base + (size_t)(y * w + x) * 3;
        return f3(p[0] / 255.0f, p[1] / 255.0f, p[2] / 255.0f);
    };
    float3 a = at(x0, y0) * (1.0f - tx) + at(x1, y0) * tx;
    float3 b = at(x0, y1) * (1.0f - tx) + at(x1, y1) * tx;
    return a * (1.0f - ty) + b * ty;
}

__device__ __forceinline__ bool has_mask(const DevScene& S, const Material& m) {
    return m.mask_id >= 0 && m.mask_id < S.num_textures;
}

// integrator/shading.h:92-108
__device__ __forceinline__ float transmission_at(const DevScene& S, const Material& m, float2 uv) {
    if (m.transmission <= 0.0f) return 0.0f;
    if (has_mask(S, m)) return m.transmission * tex_fetch(S.textures[m.mask_id], uv, 0.0f).x;
    return m.transmission;
}
__device__ __forceinline__ float ior_at(const DevScene& S, const Material& m, float2 uv) {
    if (has_mask(S, m)) return 1.0f + tex_fetch(S.textures[m.mask_id], uv, 0.0f).y;
    return m.ior;
}

// render_kernel.cu:328-334
__device__ __forceinline__ float3 sky(float3 d) {
    float t = 0.5f * (d.y + 1.0f);
    return f3((1.0f - t) * 1.0f + t * 0.5f, (1.0f - t) * 1.0f + t * 0.7f, (1.0f - t) * 1.0f + t * 1.0f);
}

// render_kernel.cu:13-24
__device__ __forceinline__ float3 sun_direction(const Light& l, uint32_t seed) {
    float3 base = -f3(l.direction);
    if (l.angle <= 0.0f) return base;
    float3 t1 = normalize(cross(base, up_for(base)));
    float3 t2 = cross(base, t1);
    float r = sqrtf(rand01(seed ^ 0x68e31da4u)) * tanf(l.angle);
    float phi = 6.2831853f * rand01(seed ^ 0xb5297a4du);
    return normalize(base + t1 * (cosf(phi) * r) + t2 * (sinf(phi) * r));
}

struct ShadePoint {
    float3 p;          // hit point
    float3 ng;         // normal of the hit record (faces the ray)
    float3 n;          // shading normal (normal map applied)
    float3 tan;
    float3 view;
    float2 uv;
    float uv_fp;
    float3 base;       // albedo
    float shin;
    int mat;
};

// Texture footprint scale and tangent frame of a triangle hit from its
// world edges and uv deltas (render_kernel.cu:82-114).
__device__ __forceinline__ void tri_lod(float3 e1, float3 e2, sheen_float2 uv0, sheen_float2 uv1, sheen_float2 uv2,
                                        float3 n, float footprint, float& uv_fp, float3& tu, float3& tv) {
    float2 d1 = make_float2(uv1.x - uv0.x, uv1.y - uv0.y);
    float2 d2 = make_float2(uv2.x - uv0.x, uv2.y - uv0.y);
    float w1 = sqrtf(dot(e1, e1)), w2 = sqrtf(dot(e2, e2));
    float u1 = sqrtf(d1.x * d1.x + d1.y * d1.y), u2 = sqrtf(d2.x * d2.x + d2.y * d2.y);
    float a1 = w1 > 1.0e-6f ? u1 / w1 : 0.0f, a2 = w2 > 1.0e-6f ? u2 / w2 : 0.0f;
    float dens = a1 > a2 ? a1 : a2;
    if (dens > 1.0e-6f) uv_fp = footprint * dens;
    float det = d1.x * d2.y - d2.x * d1.y;
    if (fabsf(det) > 1.0e-8f) {
        float3 du = (e1 * d2.y - e2 * d1.y) / det;
        float3 dv = (e2 * d1.x - e1 * d2.x) / det;
        du = du - n * dot(du, n);
        dv = dv - n * dot(dv, n);
        float lu = dot(du, du);
        if (lu > 1.0e-12f) {
            tu = du * rsqrtf(lu);
            dv = dv - tu * dot(dv, tu);
            float lv = dot(dv, dv);
            if (lv > 1.0e-12f) tv = dv * rsqrtf(lv);
        }
    }
}

// tri_lod of flattened triangle index ti when it is an instanced one
// (ti - num_tris among the instances' triangles, instance by instance):
// the mesh triangle's edges through the instance's object-to-world map.
static __device__ __noinline__ void inst_tri_lod(const DevScene& S, int ti, float3 n, float footprint, float& uv_fp,
                                                 float3& tu, float3& tv) {
    const int k = ti - S.num_tris;
    if (k < 0 || k >= S.inst_tri_total) return;
    int lo = 0, hi = S.num_instances - 1;   // last instance whose base <= k
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int4 m2 = __ldg(reinterpret_cast<const int4*>(S.inst_xf + (size_t)kInstRecord * mid + 7));
        if (m2.x <= k) lo = mid;
        else hi = mid - 1;
    }
    const float4* xf = S.inst_xf + (size_t)kInstRecord * lo;
    const int4 m2 = __ldg(reinterpret_cast<const int4*>(xf + 7));
    const Triangle& tr = S.inst_tris[m2.z + (k - m2.x)];
    const float4 fa = __ldg(&xf[3]), fb = __ldg(&xf[4]), fc = __ldg(&xf[5]);
    auto lin = [&](float3 d) {
        return f3(fa.x * d.x + fa.y * d.y + fa.z * d.z, fb.x * d.x + fb.y * d.y + fb.z * d.z,
                  fc.x * d.x + fc.y * d.y + fc.z * d.z);
    };
    tri_lod(lin(f3(tr.v1) - f3(tr.v0)), lin(f3(tr.v2) - f3(tr.v0)), tr.uv0, tr.uv1, tr.uv2, n, footprint, uv_fp, tu,
            tv);
}

// render_kernel.cu:67-150
__device__ __forceinline__ ShadePoint shade_prepare(const DevScene& S, const Hit& h, float3 view, float footprint) {
    ShadePoint sp;
    const Material& m = S.materials[h.mat];
    sp.p = h.p; sp.ng = h.n; sp.n = h.n; sp.tan = h.tan; sp.view = view; sp.uv = h.uv; sp.mat = h.mat;
    float uv_fp = footprint;
    float3 tu = f3(0.0f, 0.0f, 0.0f), tv = f3(0.0f, 0.0f, 0.0f);
    // Any negative object id is read as a triangle index when the scene has
    // triangles (render_kernel.cu:82-84); only texture LOD and normal maps
    // depend on it.
    if (h.obj < 0 && S.num_tris > 0) {
        int ti = -h.obj - 1;
        if (ti >= 0 && ti < S.num_tris) {
            const Triangle& tr = S.tris[ti];
            tri_lod(f3(tr.v1) - f3(tr.v0), f3(tr.v2) - f3(tr.v0), tr.uv0, tr.uv1, tr.uv2, h.n, footprint, uv_fp, tu,
                    tv);
        }
    }
    // instanced triangles: read as their flattened copies
    if (h.obj < 0 && S.num_instances > 0) inst_tri_lod(S, -h.obj - 1, h.n, footprint, uv_fp, tu, tv);
    sp.uv_fp = uv_fp;
    if (m.normal_id >= 0 && m.normal_id < S.num_textures) {
        const TextureRef& nt = S.textures[m.normal_id];
        float3 nm = tex_fetch(nt, sp.uv, tex_lod(nt, uv_fp));
        float nx = (nm.x * 2.0f - 1.0f) * m.normal_strength;
        float ny = (nm.y * 2.0f - 1.0f) * m.normal_strength;
        float3 n0 = sp.n, t1, t2;
        if (dot(tu, tu) > 0.5f && dot(tv, tv) > 0.5f) { t1 = tu; t2 = tv; }
        else { t1 = normalize(cross(up_for(n0), n0)); t2 = cross(n0, t1); }
        sp.n = normalize(n0 + t1 * nx + t2 * ny);
    }
    if (m.texture_id >= 0 && m.texture_id < S.num_textures) {
        const TextureRef& t = S.textures[m.texture_id];
        sp.base = tex_fetch(t, sp.uv, tex_lod(t, uv_fp));
    } else {
        sp.base = f3(m.diffuse_color);
    }
    sp.shin = m.shininess;
    if (has_mask(S, m)) {
        const TextureRef& mt = S.textures[m.mask_id];
        float r = tex_fetch(mt, sp.uv, tex_lod(mt, uv_fp)).z;
        float rr = fmaxf(r, 0.02f), r2 = rr * rr;
        sp.shin = fminf(fmaxf(2.0f / (r2 * r2) - 2.0f, 1.0f), 4096.0f);
    }
    return sp;
}

__device__ __forceinline__ float3 shade_emitted(const DevScene& S, const ShadePoint& sp) {
    const Material& m = S.materials[sp.mat];
    return sp.base * m.ambient + f3(m.emission_color) * m.emission;
}

struct LightSample {
    float3 L;          // direction to the light
    float3 radiance;
    float3 target;     // shadow-ray aim point
    float tmax;
};

// render_kernel.cu:152-235.  Returns false where the reference `continue`s
// before tracing (area light seen from behind, point outside a spot cone).
__device__ __forceinline__ bool light_sample(const DevScene& S, const ShadePoint& sp, int i, uint32_t seed,
                                             LightSample& ls) {
    const Light& l = S.lights[i];
    const uint32_t lseed = seed ^ (uint32_t)(i * 2654435761u);
    ls.tmax = 1e10f;
    if (l.type == 0) {
        ls.L = sun_direction(l, lseed);
        ls.radiance = f3(l.color) * l.intensity;
        ls.target = sp.p + ls.L * 1.0e6f;
        return true;
    }
    float3 pos = f3(l.position);
    if (l.type == 2) {
        float ru = rand01(lseed) * 2.0f - 1.0f;
        float rv = rand01(lseed ^ 0x9e3779b9u) * 2.0f - 1.0f;
        pos = f3(l.position) + f3(l.u_axis) * ru + f3(l.v_axis) * rv;
    }
    float3 tl = pos - sp.p;
    float d2 = fmaxf(dot(tl, tl), 1.0e-4f);
    float dist = sqrtf(d2);
    float3 L = tl / dist;
    if ((l.type == 1 || l.type == 3) && l.radius > 0.0f) {
        float3 t1 = normalize(cross(L, up_for(L)));
        float3 t2 = cross(L, t1);
        float r = sqrtf(rand01(lseed ^ 0x85ebca6bu)) * l.radius;
        float phi = 6.2831853f * rand01(lseed ^ 0xc2b2ae35u);
        pos = pos + t1 * (cosf(phi) * r) + t2 * (sinf(phi) * r);
        tl = pos - sp.p;
        d2 = fmaxf(dot(tl, tl), 1.0e-4f);
        dist = sqrtf(d2);
        L = tl / dist;
    }
    float att = l.intensity / (12.5663706f * d2);
    float3 gobo = f3(1.0f, 1.0f, 1.0f);
    if (l.type == 2) {
        float3 n = normalize(cross(f3(l.u_axis), f3(l.v_axis)));
        float c = dot(n, L);
        if (c <= 0.0f) return false;
        att *= c;
    } else if (l.type == 3) {
        float3 ts = normalize(sp.p - pos);
        float c = dot(ts, f3(l.direction));
        float ch = cosf(l.angle);
        if (c <= ch) return false;
        float bl = fminf(fmaxf(l.blend, 0.0f), 1.0f);
        float cs = cosf(l.angle * (1.0f - bl));
        if (cs > ch + 1.0e-4f) att *= fminf((c - ch) / (cs - ch), 1.0f);
        if (l.texture_id >= 0 && l.texture_id < S.num_textures) {
            float3 ax = f3(l.direction);
            float3 t1 = normalize(cross(ax, up_for(ax)));
            float3 t2 = cross(ax, t1);
            float th = tanf(fmaxf(l.angle, 1.0e-3f));
            float u = 0.5f + 0.5f * dot(ts, t1) / th;
            float v = 0.5f + 0.5f * dot(ts, t2) / th;
            gobo = tex_fetch(S.textures[l.texture_id], make_float2(u, v), 0.0f);
        }
    }
    ls.L = L;
    ls.radiance = f3(l.color) * att * gobo;
    ls.target = pos;
    ls.tmax = dist * 0.999f;
    return true;
}

// integrator/shading.h:112-175: Kajiya-Kay strands or Blinn-Phong.
__device__ __forceinline__ float3 brdf(const DevScene& S, const ShadePoint& sp, float3 L, float3 rad) {
    const Material& m = S.materials[sp.mat];
    if (m.anisotropy > 0.0f) {
        float3 T = sp.tan, N = sp.n, V = sp.view;
        float tl = dot(T, L);
        float sin_tl = sqrtf(fmaxf(1.0f - tl * tl, 0.0f));
        float back = fmaxf(-tl, 0.0f);
        float diffuse = sin_tl + m.hair_backlight * back * back;
        float3 res = f3(m.diffuse_color) * rad * diffuse * 0.75f;
        float wr = m.hair_spec_r, wt = m.hair_spec_t, er = m.hair_exp_r, et = m.hair_exp_t;
        if (wr <= 0.0f && wt <= 0.0f) { wr = m.specular; er = m.shininess; }
        float3 H = normalize(L + V);
        if (wr > 0.0f) {
            float3 Tr = normalize(T + m.hair_shift * N);
            float s = dot(Tr, H);
            res += rad * wr * powf(sqrtf(fmaxf(1.0f - s * s, 0.0f)), fmaxf(er, 1.0f));
        }
        if (wt > 0.0f) {
            float3 Tt = normalize(T - m.hair_shift * N);
            float s = dot(Tt, H);
            res += rad * wt * powf(sqrtf(fmaxf(1.0f - s * s, 0.0f)), fmaxf(et, 1.0f));
        }
        return res;
    }
    float diff = fmaxf(dot(sp.n, L), 0.0f);
    float3 res = sp.base * rad * diff;
    if (m.specular > 0.0f && diff > 0.0f) {
        float3 hv = normalize(L + sp.view);
        res += rad * m.specular * powf(fmaxf(dot(sp.n, hv), 0.0f), sp.shin);
    }
    return res;
}

// render_kernel.h:55-64
__device__ __forceinline__ int photon_cell(int ix, int iy, int iz, int num_cells) {
    unsigned h = ((unsigned)ix * 73856093u) ^ ((unsigned)iy * 19349663u) ^ ((unsigned)iz * 83492791u);
    h ^= h >> 16; h *= 0x7feb352du;
    h ^= h >> 15; h *= 0x846ca68bu;
    h ^= h >> 16;
    return (int)(h & (unsigned)(num_cells - 1));
}

// render_kernel.h:68-111: flux of the first `max_samples` photons found in
// the (<= 8 distinct) cells covering the ball, facing the query normal.
__device__ __forceinline__ float3 photon_gather(const PhotonMapView& m, float3 p, float3 n, float radius, int max_samples) {
    float3 acc = f3(0.0f, 0.0f, 0.0f);
    if (!m.pos || m.num_cells <= 0 || m.cell_size <= 0.0f) return acc;
    const int x0 = (int)floorf((p.x - radius) / m.cell_size), x1 = (int)floorf((p.x + radius) / m.cell_size);
    const int y0 = (int)floorf((p.y - radius) / m.cell_size), y1 = (int)floorf((p.y + radius) / m.cell_size);
    const int z0 = (int)floorf((p.z - radius) / m.cell_size), z1 = (int)floorf((p.z + radius) / m.cell_size);
    const float r2 = radius * radius;
    int cells[8], nc = 0, taken = 0;
    for (int iz = z0; iz <= z1; iz++)
        for (int iy = y0; iy <= y1; iy++)
            for (int ix = x0; ix <= x1; ix++) {
                int c = photon_cell(ix, iy, iz, m.num_cells);
                bool seen = false;
                for (int q = 0; q < nc; q++) seen |= (cells[q] == c);
                if (!seen && nc < 8) cells[nc++] = c;
            }
    for (int q = 0; q < nc && taken < max_samples; q++) {
        const int st = m.cell_start[cells[q]], cnt = m.cell_count[cells[q]];
        for (int k = 0; k < cnt && taken < max_samples; k++) {
            const float4 pp = __ldg(&m.pos[st + k]);
            float3 d = f3(pp.x, pp.y, pp.z) - p;
            if (dot(d, d) > r2) continue;
            const float4 pn = __ldg(&m.nrm[st + k]);
            if (dot(f3(pn.x, pn.y, pn.z), n) < 0.1f) continue;
            const float4 pf = __ldg(&m.flux[st + k]);
            acc += f3(pf.x, pf.y, pf.z);
            taken++;
        }
    }
    return acc;
}

// Extension (a scene created with "caustic.knn" = k, 1..64; the reference
// gathers the first <= 128 photons within r = cell / 2): the k nearest
// photons within r_max = cell / 2 facing the normal.  Pass 1 keeps the k
// smallest squared distances in a max-heap; pass 2 sums the flux of every
// photon within the k-th distance (ties included).  The radius of the
// estimate is that distance, or r_max when fewer than k photons are found;
// the flux goes through the reference's estimate flux / (pi^2 r^2).
constexpr int kKnnMax = 64;
__device__ __forceinline__ float3 photon_knn(const PhotonMapView& m, float3 p, float3 n, float rmax, int k,
                                                 float& r2_used) {
    float3 acc = f3(0.0f, 0.0f, 0.0f);
    r2_used = rmax * rmax;
    if (!m.pos || m.num_cells <= 0 || m.cell_size <= 0.0f || k <= 0) return acc;
    k = k > kKnnMax ? kKnnMax : k;
    const int x0 = (int)floorf((p.x - rmax) / m.cell_size), x1 = (int)floorf((p.x + rmax) / m.cell_size);
    const int y0 = (int)floorf((p.y - rmax) / m.cell_size), y1 = (int)floorf((p.y + rmax) / m.cell_size);
    const int z0 = (int)floorf((p.z - rmax) / m.cell_size), z1 = (int)floorf((p.z + rmax) / m.cell_size);
    int cells[27], nc = 0;
    for (int iz = z0; iz <= z1; iz++)
        for (int iy = y0; iy <= y1; iy++)
            for (int ix = x0; ix <= x1; ix++) {
                const int c = photon_cell(ix, iy, iz, m.num_cells);
                bool seen = false;
                for (int q = 0; q < nc; q++) seen |= (cells[q] == c);
                if (!seen && nc < 27) cells[nc++] = c;
            }
    float heap[kKnnMax];
    int hn = 0;
    const float rmax2 = rmax * rmax;
    for (int q = 0; q < nc; q++) {
        const int st = m.cell_start[cells[q]], cnt = m.cell_count[cells[q]];
        for (int j = 0; j < cnt; j++) {
            const float4 pp = __ldg(&m.pos[st + j]);
            const float3 d = f3(pp.x, pp.y, pp.z) - p;
            const float d2 = dot(d, d);
            if (d2 > rmax2) continue;
            const float4 pn = __ldg(&m.nrm[st + j]);
            if (dot(f3(pn.x, pn.y, pn.z), n) < 0.1f) continue;
            if (hn < k) {   // push, sift up
                int i = hn++;
                while (i > 0 && heap[(i - 1) / 2] < d2) { heap[i] = heap[(i - 1) / 2]; i = (i - 1) / 2; }
                heap[i] = d2;
            } else if (d2 < heap[0]) {   // replace the largest, sift down
                int i = 0;
                while (true) {
                    const int l = 2 * i + 1, r = l + 1;
                    int big = i;
                    float vb = d2;
                    if (l < hn && heap[l] > vb) { big = l; vb = heap[l]; }
                    if (r < hn && heap[r] > vb) { big = r; vb = heap[r]; }
                    if (big == i) break;
                    heap[i] = heap[big];
                    i = big;
                }
                heap[i] = d2;
            }
        }
    }
    const float r2 = hn < k ? rmax2 : heap[0];
    r2_used = r2;
    for (int q = 0; q < nc; q++) {
        const int st = m.cell_start[cells[q]], cnt = m.cell_count[cells[q]];
        for (int j = 0; j < cnt; j++) {
            const float4 pp = __ldg(&m.pos[st + j]);
            const float3 d = f3(pp.x, pp.y, pp.z) - p;
            if (dot(d, d) > r2) continue;
            const float4 pn = __ldg(&m.nrm[st + j]);
            if (dot(f3(pn.x, pn.y, pn.z), n) < 0.1f) continue;
            const float4 pf = __ldg(&m.flux[st + j]);
            acc += f3(pf.x, pf.y, pf.z);
        }
    }
    return acc;
}

__device__ __forceinline__ float3 caustic_term(const DevScene& S, const ShadePoint& sp) {
    if (!S.pmap.pos || S.caustics <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const float r = S.pmap.cell_size * 0.5f;
    if (S.caustic_knn > 0) {
        float r2 = r * r;
        const float3 flux = photon_knn(S.pmap, sp.p, sp.ng, r, S.caustic_knn, r2);
        return sp.base * flux * (S.caustics / (9.8696044f * r2));
    }
    float3 flux = photon_gather(S.pmap, sp.p, sp.ng, r, 128);
    return sp.base * flux * (S.caustics / (9.8696044f * r * r));
}

// render_kernel.cu:302-325
__device__ __forceinline__ bool medium_span(const Ray& r, float3 c, float3 hh, float& t0, float& t1) {
    t0 = -1.0e30f;
    t1 = 1.0e30f;
    const float o[3] = {r.o.x, r.o.y, r.o.z}, d[3] = {r.d.x, r.d.y, r.d.z};
    const float cc[3] = {c.x, c.y, c.z}, h[3] = {hh.x, hh.y, hh.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        if (fabsf(d[a]) < 1.0e-8f) {
            if (o[a] < cc[a] - h[a] || o[a] > cc[a] + h[a]) return false;
            continue;
        }
        float inv = 1.0f / d[a];
        float tn = (cc[a] - h[a] - o[a]) * inv, tf = (cc[a] + h[a] - o[a]) * inv;
        if (tn > tf) { float t = tn; tn = tf; tf = t; }
        t0 = fmaxf(t0, tn);
        t1 = fminf(t1, tf);
        if (t0 > t1) return false;
    }
    return true;
}

}  // namespace dev
}  // namespace sheen
