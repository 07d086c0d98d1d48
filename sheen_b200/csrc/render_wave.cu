// render_wave.cu -- wavefront form of the per-sample integrator
// (render_kernel.cu:487-809) over compacted ray queues.
//
// A frame runs as a fixed sequence of persistent kernels (one CUDA graph per
// frame shape, replayed):
//   primary   camera ray, closest hit, shading of the hit: writes the
//             sample's base term (ambient + emission, or sky), pushes one
//             shadow ray per light that passes the light's own tests, pushes
//             the mirror ray (reflect > 0) and the first refracted ray
//             (transmission > 0); records the blend weights
//   shadow    every queued shadow ray: up to three opaque-set queries with
//             glass passes, strand transmittance; writes its light slot
//   reflect   mirror rays: closest hit and shading (or sky) -> shadow queue
//   shadow
//   refract   refracted rays: up to three faces, then shading (or sky)
//   shadow
//   resolve   per pixel: every sample's color from its slots, averaged
// Each sample owns 3 segments (primary, mirror, refraction end) x (L + 2)
// RGB slots: base, one per light, caustic.  Slots are summed in the
// reference's order (base, light 0..L-1, caustic), then blended with the
// weights of render_kernel.cu:730-731 and 805, so no float atomics are
// needed and frames are bit-reproducible.  A segment whose weight is zero is
// never written nor read.
//
// Queues are filled with warp-aggregated appends (ballot + popc, one atomic
// per warp); persistent blocks claim 32-entry batches from an atomic head,
// so uneven work (glass, empty sky) balances across the SMs.
//
// Frames the queue pipeline does not cover -- visible spot beams, media, a
// material in the shadow-debug mode (shininess < 0), more than 16 lights,
// or reflect + refract recursion (an extension scene's max_depth > 1) --
// run on the BVH4 megakernel with identical results.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "dev/integrator.cuh"
#include "dev/trace_bvh4.cuh"
#include "engine.h"

namespace sheen {

namespace dev {

constexpr int kMaxWaveLights = 16;

enum CounterSlot {
    kShadowCount = 0, kShadowHead, kReflCount, kReflHead, kRefrCount, kRefrHead, kPrimHead, kPixHead,
    kRaysPrimary, kRaysShadow, kRaysSecondary, kCounterWords = 16
};

struct WaveView {
    float* slots;          // samples * 3 * (L + 2) * 3
    float* coef;           // samples * 3: weights of the primary / mirror / refraction segments
    float4* shq;           // shadow queue, 3 float4 per entry
    float4* rq;            // mirror queue, 2 float4 per entry
    float4* tq;            // refraction queue, 2 float4 per entry
    unsigned int* ctr;     // kCounterWords counters (queue sizes, batch heads, ray tallies)
    int L;                 // lights
    int ns;                // samples per pixel
    int W, H, x0, y0, rw, rh;
    int nsamples;          // rw * rh * ns
    float pix_angle;
    int count_rays;
    int tw_log2;           // log2 of the pixel tile's width (tiles of 128 pixels: 8x16, 16x8 or 32x4)
    // Multi-job launches (the MULTI kernels): the job table.  nsamples is
    // then the total over all jobs, npix the total of their padded pixels,
    // and the queues and counters above are shared; every per-frame field
    // is per job, in jobs[j].V, whose slots and coef point at the job's own
    // part and whose sample indices are local to the job.
    const struct JobDesc* jobs;
    int num_jobs;
    int npix;
};

// One region of one frame of one scene in a multi-job launch.
struct JobDesc {
    DevScene S;        // the job's scene
    WaveView V;        // its frame, slots and weights (job-local sample indices)
    float4* out;       // its image (V.W * V.H float4)
    int sample_base;   // its first sample in the launch's global sample order
    int pix_base;      // its first padded pixel in the launch's global pixel order
};

// Job of a global sample (pix = false) or padded pixel (pix = true) index:
// the last job whose base is at or below it.
__device__ __forceinline__ int job_of(const JobDesc* __restrict__ jobs, int n, int i, bool pix) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const int b = pix ? jobs[mid].pix_base : jobs[mid].sample_base;
        if (b <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Shadow queue entries carry their job and the strand flag in one word.
__device__ __forceinline__ float shadow_tag(int job, bool strands) {
    return __int_as_float((job << 1) | (strands ? 1 : 0));
}

__device__ __forceinline__ int seg_base(const WaveView& V, int sample, int seg) {
    return (sample * 3 + seg) * (V.L + 2);
}

__device__ __forceinline__ void put_slot(const WaveView& V, int slot, float3 c) {
    V.slots[3 * (size_t)slot] = c.x;
    V.slots[3 * (size_t)slot + 1] = c.y;
    V.slots[3 * (size_t)slot + 2] = c.z;
}

// Warp-aggregated append: every active lane with `want` gets a distinct
// index in [0, capacity); one atomicAdd per warp.
__device__ __forceinline__ unsigned int warp_append(unsigned int* counter, bool want) {
    const unsigned int active = __activemask();
    const unsigned int ballot = __ballot_sync(active, want);
    if (!ballot) return 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(ballot) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned int)__popc(ballot));
    base = __shfl_sync(active, base, leader);
    return want ? base + (unsigned int)__popc(ballot & ((1u << lane) - 1u)) : 0xffffffffu;
}

// Persistent batch claim: 32 consecutive items per warp.
__device__ __forceinline__ int claim_batch(unsigned int* head) {
    unsigned int b = 0;
    if ((threadIdx.x & 31) == 0) b = atomicAdd(head, 32u);
    return (int)__shfl_sync(0xffffffffu, b, 0);
}

// Sample index -> pixel and sample number.  Pixels are walked in tiles of
// 128 (16x8 by default; the "wave.tile_w" launch parameter picks 8x16 or
// 32x4) so a warp's primary rays are coherent.
__device__ __forceinline__ void sample_pixel(const WaveView& V, int i, int& x, int& y, int& s) {
    s = i % V.ns;
    const int p = i / V.ns;
    const int tw = 1 << V.tw_log2;
    const int tiles_x = (V.rw + tw - 1) >> V.tw_log2;
    const int tile = p >> 7, in = p & 127;
    const int tx = tile % tiles_x, ty = tile / tiles_x;
    x = V.x0 + tx * tw + (in & (tw - 1));
    y = V.y0 + ty * (128 >> V.tw_log2) + (in >> V.tw_log2);
}

__device__ __forceinline__ bool sample_valid(const WaveView& V, int x, int y) {
    return x < V.x0 + V.rw && y < V.y0 + V.rh;
}

__device__ __forceinline__ void tally(const WaveView& V, int word, unsigned int v) {
    if (!V.count_rays) return;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&V.ctr[word], v);
}

// Shading of a hit for segment `seg` of `sample`: the base term now, one
// queued shadow ray per light that passes its own tests (render_kernel.cu:
// 152-235), the caustic gather last.  Lights skipped before tracing get a
// zero slot.
__device__ __forceinline__ void shade_and_queue(const DevScene& S, const WaveView& V, const Hit& h, float3 view,
                                                float footprint, uint32_t seed, int sample, int seg, bool active,
                                                int job) {
    ShadePoint sp;
    int sb = 0;
    if (active) {
        sp = shade_prepare(S, h, view, footprint);
        sb = seg_base(V, sample, seg);
        put_slot(V, sb, shade_emitted(S, sp));
        put_slot(V, sb + V.L + 1, caustic_term(S, sp));
    }
    const bool strands = active && S.num_strands > 0 && S.materials[h.mat].anisotropy <= 0.0f;
    for (int i = 0; i < V.L; i++) {
        LightSample ls;
        bool want = false;
        float3 contrib = f3(0.0f, 0.0f, 0.0f);
        Ray sr;
        if (active) {
            want = light_sample(S, sp, i, seed, ls);
            if (want) {
                sr.o = sp.p + sp.ng * 0.002f;
                sr.d = normalize(ls.target - sr.o);
                sr.tmax = ls.tmax;
                contrib = brdf(S, sp, ls.L, ls.radiance);
            } else {
                put_slot(V, sb + 1 + i, f3(0.0f, 0.0f, 0.0f));
            }
        }
        const unsigned int q = warp_append(&V.ctr[kShadowCount], want);
        if (want) {
            V.shq[3 * (size_t)q] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.tmax);
            V.shq[3 * (size_t)q + 1] = make_float4(sr.d.x, sr.d.y, sr.d.z, __int_as_float(sb + 1 + i));
            V.shq[3 * (size_t)q + 2] = make_float4(contrib.x, contrib.y, contrib.z, shadow_tag(job, strands));
        }
    }
}

__device__ __forceinline__ float3 refract_dir(const DevScene& S, const Hit& gh, float3 d, bool entering,
                                              float& w) {
    const Material& sm = S.materials[gh.mat];
    const float ior = fmaxf(ior_at(S, sm, gh.uv), 1.0f);
    const float eta = entering ? 1.0f / ior : ior;
    const float cosi = fmaxf(-dot(d, gh.n), 1.0e-4f);
    const float k = 1.0f - eta * eta * (1.0f - cosi * cosi);
    const float3 td = k < 0.0f ? normalize(d + 2.0f * cosi * gh.n) : normalize(eta * d + (eta * cosi - sqrtf(k)) * gh.n);
    w *= transmission_at(S, sm, gh.uv);
    return td;
}

// One primary sample: local index i of the frame V (gi: its global index in
// a multi-job launch, which the secondary queues carry).
template <int F>
__device__ __forceinline__ void primary_item(const DevScene& S, const WaveView& V, int i, int gi, bool active,
                                             int job, Counters& c) {
    using T = FastTracer<false, F>;
    int x = 0, y = 0, s = 0;
    if (active) {
        sample_pixel(V, i, x, y, s);
        active = sample_valid(V, x, y);
    }
    Hit rec;
    Ray ray;
    bool hit = false;
    uint32_t seed = 0;
    if (active) {
        float pix;
        ray = camera_ray(S.cam, x, y, s, V.ns, V.W, V.H, pix, S.aa_centered);
        seed = sample_seed(x, y, s);
        hit = T::closest(S, ray, rec, c);
    }
    tally(V, kRaysPrimary, active ? 1u : 0u);
    float w = 0.0f, gtr = 0.0f;
    if (active) {
        if (!hit) {
            // sky: the segment's light and caustic slots are summed by the
            // resolve too, so they are cleared here
            const int sb = seg_base(V, i, 0);
            put_slot(V, sb, sky(ray.d));
            for (int l = 0; l < V.L + 1; l++) put_slot(V, sb + 1 + l, f3(0.0f, 0.0f, 0.0f));
            V.coef[3 * (size_t)i] = 1.0f;
            V.coef[3 * (size_t)i + 1] = 0.0f;
            V.coef[3 * (size_t)i + 2] = 0.0f;
        } else {
            const Material& pm = S.materials[rec.mat];
            w = pm.reflect > 0.0f ? fminf(pm.reflect, 1.0f) : 0.0f;
            gtr = transmission_at(S, pm, rec.uv);
            const float g = gtr > 0.0f ? 1.0f - fminf(gtr, 1.0f) : 1.0f;
            V.coef[3 * (size_t)i] = (1.0f - w) * g;
            V.coef[3 * (size_t)i + 1] = w * g;
            V.coef[3 * (size_t)i + 2] = 0.0f;   // set by the refraction stage
        }
    }
    shade_and_queue(S, V, rec, -ray.d, rec.t * V.pix_angle, seed, i, 0, active && hit, job);
    // mirror ray (render_kernel.cu:674-680)
    const bool want_r = active && hit && w > 0.0f;
    const unsigned int qr = warp_append(&V.ctr[kReflCount], want_r);
    if (want_r) {
        const float3 rd = normalize(ray.d - rec.n * (2.0f * dot(ray.d, rec.n)));
        const float3 ro = rec.p + rec.n * 0.002f;
        V.rq[2 * (size_t)qr] = make_float4(ro.x, ro.y, ro.z, __int_as_float(gi));
        V.rq[2 * (size_t)qr + 1] = make_float4(rd.x, rd.y, rd.z, 0.0f);
    }
    // first refraction face (render_kernel.cu:749-765 with b = 0)
    const bool want_t = active && hit && gtr > 0.0f;
    float wt = 1.0f;
    float3 td = f3(0.0f, 0.0f, 0.0f);
    if (want_t) td = refract_dir(S, rec, ray.d, true, wt);
    const unsigned int qt = warp_append(&V.ctr[kRefrCount], want_t);
    if (want_t) {
        const float3 to = rec.p + td * 0.002f;
        V.tq[2 * (size_t)qt] = make_float4(to.x, to.y, to.z, __int_as_float(gi));
        V.tq[2 * (size_t)qt + 1] = make_float4(td.x, td.y, td.z, wt);
    }
}

// MULTI: samples of every job in the launch's table (V0.jobs), one claim
// counter over their global order; otherwise the single frame S0 / V0.
template <int F, bool MULTI>
__global__ void __launch_bounds__(128, 8) wave_primary(const __grid_constant__ DevScene S0, WaveView V0) {
    Counters c;
    while (true) {
        const int base = claim_batch(&V0.ctr[kPrimHead]);
        if (base >= V0.nsamples) break;
        const int gi = base + (threadIdx.x & 31);
        const bool active = gi < V0.nsamples;
        if constexpr (MULTI) {
            const int j = job_of(V0.jobs, V0.num_jobs, active ? gi : V0.nsamples - 1, false);
            const JobDesc& J = V0.jobs[j];
            primary_item<F>(J.S, J.V, gi - J.sample_base, gi, active, j, c);
        } else {
            primary_item<F>(S0, V0, gi, gi, active, 0, c);
        }
    }
}

// One queued shadow ray (entry a, b, cc) of frame S / V: up to three
// opaque-set queries with glass passes, strand transmittance; writes its
// light slot.  Returns the queries issued.
template <int F>
__device__ __forceinline__ unsigned int shadow_item(const DevScene& S, const WaveView& V, float4 a, float4 b, float4 cc,
                                                    Counters& c) {
    using T = FastTracer<false, F>;
    unsigned int rays = 0;
    Ray r;
    r.o = f3(a.x, a.y, a.z);
    r.d = f3(b.x, b.y, b.z);
    r.tmin = 0.001f;
    r.tmax = a.w;
    const Ray first = r;
    bool blocked = false;
    for (int pass = 0; pass < 3; pass++) {
        rays++;
        ShadowHit sh;
        const int res = T::shadow(S, r, true, sh, c);
        if (res == kClear) break;
        if (res == kBlocked) { blocked = true; break; }
        r.o = sh.p + r.d * 0.002f;
    }
    float3 contrib = f3(0.0f, 0.0f, 0.0f);
    if (!blocked) {
        contrib = f3(cc.x, cc.y, cc.z);
        if (__float_as_int(cc.w) & 1) contrib = contrib * expf(-T::strand_depth(S, first, c));
    }
    put_slot(V, __float_as_int(b.w), contrib);
    return rays;
}

template <int F, bool MULTI>
__global__ void __launch_bounds__(128, 8) wave_shadow(const __grid_constant__ DevScene S0, WaveView V0) {
    Counters c;
    const unsigned int n = V0.ctr[kShadowCount];
    while (true) {
        const int base = claim_batch(&V0.ctr[kShadowHead]);
        if (base >= (int)n) break;
        const int q = base + (threadIdx.x & 31);
        unsigned int rays = 0;
        if (q < (int)n) {
            const float4 a = V0.shq[3 * (size_t)q], b = V0.shq[3 * (size_t)q + 1], cc = V0.shq[3 * (size_t)q + 2];
            if constexpr (MULTI) {
                const JobDesc& J = V0.jobs[__float_as_int(cc.w) >> 1];
                rays = shadow_item<F>(J.S, J.V, a, b, cc, c);
            } else {
                rays = shadow_item<F>(S0, V0, a, b, cc, c);
            }
        }
        tally(V0, kRaysShadow, rays);
    }
}

// Shadow stage with per-lane refill.  Same queries and results as
// wave_shadow, scheduled differently: every lane carries one shadow ray
// through a small state machine (sphere category -> closest walk over the
// passable triangles -> any-hit walk over the blocking ones -> the later
// categories -> next glass pass), and the warp steps all lanes' mesh walks
// together: inner nodes until every busy lane sits on a leaf, then one leaf
// each.  A lane whose ray is finished goes idle; once `refill_min` lanes are
// idle the warp claims that many new rays from the queue in one atomic, so
// long rays no longer hold 31 finished lanes hostage.  With `inner_min` > 0
// the inner-node phase also ends once fewer than inner_min lanes are still
// descending while some lane waits at a leaf: the descending lanes carry on
// in the next round (beside the refilled rays) instead of running the
// phase's tail with a few lanes.  The mesh walks are
// qmesh_trace's, step for step (same child order, same stack, same tests),
// so every ray's result is the one wave_shadow computes.
//
// SMEM_STACK places the node half of the traversal stack in shared memory
// (slot-major, [slot][thread]: the lanes of a warp touch 32 consecutive
// words, one per bank, whatever their stack depths) instead of per-thread
// local memory, whose scattered stores fill L1 with 32-byte sectors carrying
// 4 useful bytes; the entry distances (closest-hit walks of the passable set
// only) stay in local memory.  24 KB per 128-thread block.
template <int F, bool SMEM_STACK, bool MULTI>
__global__ void __launch_bounds__(128, 8) wave_shadow_refill(const __grid_constant__ DevScene S0, WaveView V0, int refill_min,
                                                             int inner_min) {
    using T = FastTracer<false, F>;
    constexpr unsigned int kFull = 0xffffffffu;
    constexpr uint32_t kLeafBit = 0x80000000u;
    // lane states: idle, walking the passable triangles (closest hit),
    // walking the blocking triangles (any hit), or waiting at the transition
    // site (a fresh ray, or a walk that has ended)
    enum { kIdle = 0, kWalkPass, kWalkBlock, kFresh, kEndPass, kEndBlock };
    Counters c;
    const unsigned int n = V0.ctr[kShadowCount];
    const int lane = threadIdx.x & 31;
    // the lane's job (MULTI): its scene and frame
    int job = 0;
    const DevScene* const s0 = &S0;
    auto scene = [&]() -> const DevScene& {
        if constexpr (MULTI) return V0.jobs[job].S;
        else return *s0;
    };
    auto view = [&]() -> const WaveView& {
        if constexpr (MULTI) return V0.jobs[job].V;
        else return V0;
    };

    // the lane's ray: q holds its current origin and direction
    QRay q{};
    float3 o_first = f3(0.0f, 0.0f, 0.0f), cc = o_first;
    float tmax = 0.0f;
    int slot = 0, pass = 0;
    bool strands = false;
    int state = kIdle;
    bool block_after_pass = false;
    int pass_tri = -1;
    float tp = 0.0f, up = 0.0f, vp = 0.0f;
    unsigned int rays = 0;
    // the lane's mesh walk
    const QNode4* wn = nullptr;
    const float4* wt = nullptr;
    uint32_t entry = 0;
    int sp = 0, wbest = -1;
    float t_best = 0.0f, wu = 0.0f, wv = 0.0f;
    uint32_t stack_e_local[SMEM_STACK ? 1 : kQStack];
    __shared__ uint32_t stack_e_shared[SMEM_STACK ? kQStack : 1][SMEM_STACK ? 128 : 1];
    float stack_t[kQStack];
    auto stack_e = [&](int i) -> uint32_t& {
        if constexpr (SMEM_STACK) return stack_e_shared[i][threadIdx.x];
        else return stack_e_local[i];
    };

    bool exhausted = false;
    for (;;) {
        // ---- refill idle lanes ------------------------------------------
        const unsigned int idle = __ballot_sync(kFull, state == kIdle);
        if (!exhausted && (idle == kFull || __popc(idle) >= refill_min)) {
            const unsigned int k = (unsigned int)__popc(idle);
            unsigned int b = 0;
            if (lane == 0) b = atomicAdd(&V0.ctr[kShadowHead], k);
            b = __shfl_sync(kFull, b, 0);
            if (b + k >= n) exhausted = true;
            if (state == kIdle) {
                const unsigned int item = b + (unsigned int)__popc(idle & ((1u << lane) - 1u));
                if (item < n) {
                    const float4 a = V0.shq[3 * (size_t)item], bb = V0.shq[3 * (size_t)item + 1],
                                 c4 = V0.shq[3 * (size_t)item + 2];
                    q.o = f3(a.x, a.y, a.z);
                    q.d = f3(bb.x, bb.y, bb.z);
                    o_first = q.o;
                    tmax = a.w;
                    slot = __float_as_int(bb.w);
                    cc = f3(c4.x, c4.y, c4.z);
                    strands = (__float_as_int(c4.w) & 1) != 0;
                    job = __float_as_int(c4.w) >> 1;
                    pass = 0;
                    state = kFresh;
                }
            }
        }
        // ---- transition site: start a pass, or settle an ended walk ---------
        if (state >= kFresh) {
            int res;
            ShadowHit sh{};
            Ray r;
            r.o = q.o; r.d = q.d; r.tmin = 0.001f; r.tmax = tmax;
            if (state == kFresh) {
                res = -2;   // start a pass
            } else if (state == kEndPass && scene().q_block.nodes) {
                // closest passable hit found; now any blocking hit strictly before it
                pass_tri = wbest; tp = t_best; up = wu; vp = wv;
                state = kWalkBlock; block_after_pass = true;
                wn = scene().q_block.nodes; wt = scene().q_block.tris;
                entry = 0; sp = 0; wbest = -1; t_best = tp;
                res = -3;   // keep walking
            } else {
                if (state == kEndPass) { pass_tri = wbest; tp = t_best; up = wu; vp = wv; }
                res = (state == kEndBlock && wbest >= 0) ? kBlocked : kClear;
                if (res == kClear && (state == kEndPass || block_after_pass) && pass_tri >= 0) {
                    Hit h;
                    tri_finish(r, scene().tris[pass_tri], tp, up, vp, h);
                    res = classify_shadow_hit(scene(), h, true, sh);
                }
                if (res == kClear) res = T::shadow_post_mesh(scene(), r, true, sh, c);
            }
            // settle: pass results and pass starts until the lane walks a
            // mesh or its ray is finished
            while (res != -3) {
                if (res == -2) {
                    rays++;
                    r.o = q.o;
                    res = T::shadow_pre_mesh(scene(), r, true, sh, c);
                    if (res >= 0) continue;
                    if ((F & kCatMesh) && scene().q_all.nodes) {
                        q = make_qray(r);
                        pass_tri = -1;
                        entry = 0; sp = 0; wbest = -1; t_best = tmax;
                        if (scene().q_pass.nodes) {
                            state = kWalkPass;
                            wn = scene().q_pass.nodes; wt = scene().q_pass.tris;
                        } else {
                            state = kWalkBlock; block_after_pass = false;
                            wn = scene().q_all.nodes; wt = scene().q_all.tris;
                        }
                        break;
                    }
                    res = T::shadow_post_mesh(scene(), r, true, sh, c);
                    continue;
                }
                if (res == kPass && ++pass < 3) {   // through the glass: next pass
                    q.o = sh.p + q.d * 0.002f;
                    res = -2;
                    continue;
                }
                // finished: blocked, clear, or three glass passes (lit)
                float3 contrib = f3(0.0f, 0.0f, 0.0f);
                if (res != kBlocked) {
                    contrib = cc;
                    if (strands) {
                        Ray first;
                        first.o = o_first; first.d = q.d; first.tmin = 0.001f; first.tmax = tmax;
                        contrib = contrib * expf(-T::strand_depth(scene(), first, c));
                    }
                }
                put_slot(view(), slot, contrib);
                state = kIdle;
                break;
            }
        }
        if (!__any_sync(kFull, state != kIdle)) {
            if (exhausted) break;
            continue;
        }
        // ---- inner nodes until every walking lane sits on a leaf ------------
        while (true) {
            const bool walking = state == kWalkPass || state == kWalkBlock;
            const bool inner = walking && !(entry & kLeafBit);
            const unsigned int descending = __ballot_sync(kFull, inner);
            if (!descending) break;
            if (__popc(descending) < inner_min && __any_sync(kFull, walking && (entry & kLeafBit))) break;
            if (!inner) continue;
            float tn[4];
            uint4 ch;
            const int mask = qnode_children(wn, (int)entry, q, t_best, tn, ch);
            const uint32_t cid[4] = {ch.x, ch.y, ch.z, ch.w};
            if (mask != 0) {
                if (state == kWalkBlock) {
                    int first = -1;
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        if (!(mask & (1 << i))) continue;
                        if (first < 0) first = i;
                        else if (sp < kQStack) stack_e(sp++) = cid[i];
                    }
                    entry = cid[first];
                } else {
                    uint32_t key[4];
                    int m = 0;
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        if (mask & (1 << i)) key[m++] = (__float_as_uint(fmaxf(tn[i], 0.0f)) & ~3u) | (uint32_t)i;
#define CSWAP(a, b) if (key[a] > key[b]) { uint32_t t_ = key[a]; key[a] = key[b]; key[b] = t_; }
                    if (m == 2) { CSWAP(0, 1) }
                    else if (m == 3) { CSWAP(0, 1) CSWAP(1, 2) CSWAP(0, 1) }
                    else if (m == 4) { CSWAP(0, 1) CSWAP(2, 3) CSWAP(0, 2) CSWAP(1, 3) CSWAP(1, 2) }
#undef CSWAP
                    for (int k = m - 1; k >= 1; k--) {
                        if (sp < kQStack) {
                            stack_e(sp) = cid[key[k] & 3u];
                            stack_t[sp] = tn[key[k] & 3u];
                            sp++;
                        }
                    }
                    entry = cid[key[0] & 3u];
                }
                continue;
            }
            // no child hit: pop (closest walks skip entries behind the hit)
            bool ended = true;
            while (sp > 0) {
                --sp;
                if (state == kWalkBlock || stack_t[sp] <= t_best) { entry = stack_e(sp); ended = false; break; }
            }
            if (ended) state = state == kWalkPass ? kEndPass : kEndBlock;
        }
        // ---- one leaf per walking lane at a leaf -----------------------------
        if ((state == kWalkPass || state == kWalkBlock) && (entry & kLeafBit)) {
            const int first = (int)((entry & 0x7fffffffu) >> 3);
            const int count = (int)(entry & 7u) + 1;
            bool ended = false;
            for (int k = 0; k < count; k++) {
                const int s = first + k;
                const float4 a = __ldg(&wt[3 * s]);
                const float4 b = __ldg(&wt[3 * s + 1]);
                const float4 c4 = __ldg(&wt[3 * s + 2]);
                float t, u, v;
                if (qtri_test<tri_of<F>()>(q, a, b, c4, q.tmin, tmax, t, u, v, scene().q_all.watertight) &&
                    t < t_best) {
                    t_best = t; wu = u; wv = v;
                    wbest = __float_as_int(a.w);
                    if (state == kWalkBlock) { ended = true; break; }
                }
            }
            if (!ended) {
                ended = true;
                while (sp > 0) {
                    --sp;
                    if (state == kWalkBlock || stack_t[sp] <= t_best) { entry = stack_e(sp); ended = false; break; }
                }
            }
            if (ended) state = state == kWalkPass ? kEndPass : kEndBlock;
        }
    }
    tally(V0, kRaysShadow, rays);
}

// One mirror ray (entry a, b; i = its job-local sample) of frame S / V.
template <int F>
__device__ __forceinline__ void reflect_item(const DevScene& S, const WaveView& V, float4 a, float4 b, int i,
                                             bool active, int job, Counters& c) {
    using T = FastTracer<false, F>;
    Ray rr;
    Hit rh;
    bool rhit = false;
    uint32_t seed = 0;
    if (active) {
        rr.o = f3(a.x, a.y, a.z);
        rr.d = f3(b.x, b.y, b.z);
        rr.tmin = 0.001f;
        rr.tmax = 1.0e10f;
        int x, y, s;
        sample_pixel(V, i, x, y, s);
        seed = sample_seed(x, y, s);
        rhit = T::closest(S, rr, rh, c);
        if (!rhit) {
            const int sb = seg_base(V, i, 1);
            put_slot(V, sb, sky(rr.d));
            for (int l = 0; l < V.L + 1; l++) put_slot(V, sb + 1 + l, f3(0.0f, 0.0f, 0.0f));
        }
    }
    tally(V, kRaysSecondary, active ? 1u : 0u);
    shade_and_queue(S, V, rh, -rr.d, rh.t * V.pix_angle, seed, i, 1, active && rhit, job);
}

template <int F, bool MULTI>
__global__ void __launch_bounds__(128, 8) wave_reflect(const __grid_constant__ DevScene S0, WaveView V0) {
    Counters c;
    const unsigned int n = V0.ctr[kReflCount];
    while (true) {
        const int base = claim_batch(&V0.ctr[kReflHead]);
        if (base >= (int)n) break;
        const int q = base + (threadIdx.x & 31);
        const bool active = q < (int)n;
        float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b = a;
        if (active) { a = V0.rq[2 * (size_t)q]; b = V0.rq[2 * (size_t)q + 1]; }
        const int gi = __float_as_int(a.w);
        if constexpr (MULTI) {
            const int j = job_of(V0.jobs, V0.num_jobs, gi, false);
            const JobDesc& J = V0.jobs[j];
            reflect_item<F>(J.S, J.V, a, b, gi - J.sample_base, active, j, c);
        } else {
            reflect_item<F>(S0, V0, a, b, gi, active, 0, c);
        }
    }
}

// One refracted ray (entry a, b; i = its job-local sample) of frame S / V:
// up to three faces, then shading (or sky).
template <int F>
__device__ __forceinline__ void refract_item(const DevScene& S, const WaveView& V, float4 a, float4 b, int i,
                                             bool active, int job, Counters& c) {
    using T = FastTracer<false, F>;
    Hit nh;
    bool shade = false;
    uint32_t seed = 0;
    float3 td = f3(0.0f, 0.0f, 0.0f);
    unsigned int rays = 0;
    if (active) {
        int x, y, s;
        sample_pixel(V, i, x, y, s);
        seed = sample_seed(x, y, s);
        Ray gr;
        gr.o = f3(a.x, a.y, a.z);
        gr.d = f3(b.x, b.y, b.z);
        gr.tmin = 0.001f;
        gr.tmax = 1.0e10f;
        float w = b.w;
        bool entering = true;
        float cT = 0.0f;
        const int sb = seg_base(V, i, 2);
        // render_kernel.cu:749-803: faces b = 0..2 (the first direction was
        // computed by the primary stage)
        for (int f = 0; f < 3; f++) {
            td = gr.d;
            rays++;
            if (!T::closest(S, gr, nh, c)) {
                put_slot(V, sb, sky(td));
                for (int l = 0; l < V.L + 1; l++) put_slot(V, sb + 1 + l, f3(0.0f, 0.0f, 0.0f));
                cT = w;
                break;
            }
            if (transmission_at(S, S.materials[nh.mat], nh.uv) > 0.0f) {
                entering = !entering;
                if (f == 2) break;   // the reference's loop ends here: no contribution
                const float3 nd = refract_dir(S, nh, gr.d, entering, w);
                gr.o = nh.p + nd * 0.002f;
                gr.d = nd;
                continue;
            }
            shade = true;
            cT = w;
            break;
        }
        V.coef[3 * (size_t)i + 2] = cT;
    }
    tally(V, kRaysSecondary, rays);
    shade_and_queue(S, V, nh, -td, nh.t * V.pix_angle, seed, i, 2, active && shade, job);
}

template <int F, bool MULTI>
__global__ void __launch_bounds__(128, 8) wave_refract(const __grid_constant__ DevScene S0, WaveView V0) {
    Counters c;
    const unsigned int n = V0.ctr[kRefrCount];
    while (true) {
        const int base = claim_batch(&V0.ctr[kRefrHead]);
        if (base >= (int)n) break;
        const int q = base + (threadIdx.x & 31);
        const bool active = q < (int)n;
        float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b = a;
        if (active) { a = V0.tq[2 * (size_t)q]; b = V0.tq[2 * (size_t)q + 1]; }
        const int gi = __float_as_int(a.w);
        if constexpr (MULTI) {
            const int j = job_of(V0.jobs, V0.num_jobs, gi, false);
            const JobDesc& J = V0.jobs[j];
            refract_item<F>(J.S, J.V, a, b, gi - J.sample_base, active, j, c);
        } else {
            refract_item<F>(S0, V0, a, b, gi, active, 0, c);
        }
    }
}

__device__ __forceinline__ float3 get_slot(const WaveView& V, int slot) {
    return f3(V.slots[3 * (size_t)slot], V.slots[3 * (size_t)slot + 1], V.slots[3 * (size_t)slot + 2]);
}

__device__ __forceinline__ float3 segment_value(const WaveView& V, int sb) {
    float3 v = get_slot(V, sb);
    for (int l = 0; l < V.L; l++) v += get_slot(V, sb + 1 + l);
    return v + get_slot(V, sb + V.L + 1);
}

// Pixel p (padded tile order of sample_pixel) of frame V: every sample's
// color from its slots, averaged.  Padding pixels fall outside the region
// and are skipped.
__device__ __forceinline__ void resolve_item(const WaveView& V, float4* __restrict__ out, int p) {
    int x, y, s;
    sample_pixel(V, p * V.ns, x, y, s);
    if (!sample_valid(V, x, y)) return;
    float3 acc = f3(0.0f, 0.0f, 0.0f);
    for (int k = 0; k < V.ns; k++) {
        const int i = p * V.ns + k;
        const float cP = V.coef[3 * (size_t)i], cR = V.coef[3 * (size_t)i + 1], cT = V.coef[3 * (size_t)i + 2];
        float3 col = segment_value(V, seg_base(V, i, 0)) * cP;
        if (cR != 0.0f) col += segment_value(V, seg_base(V, i, 1)) * cR;
        if (cT != 0.0f) col += segment_value(V, seg_base(V, i, 2)) * cT;
        acc += col;
    }
    const float inv = 1.0f / float(V.ns);
    out[(size_t)y * V.W + x] = make_float4(acc.x * inv, acc.y * inv, acc.z * inv, 1.0f);
}

template <bool MULTI>
__global__ void wave_resolve(WaveView V0, float4* __restrict__ out0) {
    const int gp = blockIdx.x * blockDim.x + threadIdx.x;
    if constexpr (MULTI) {
        if (gp >= V0.npix) return;
        const JobDesc& J = V0.jobs[job_of(V0.jobs, V0.num_jobs, gp, true)];
        resolve_item(J.V, J.out, gp - J.pix_base);
    } else {
        if (gp >= V0.nsamples / V0.ns) return;
        resolve_item(V0, out0, gp);
    }
}

// Copies the three ray counters into snap[3*k .. 3*k+2] (stage profiling).
__global__ void wave_snapshot(WaveView V, unsigned int* snap, int k) {
    snap[3 * k] = V.ctr[kRaysPrimary];
    snap[3 * k + 1] = V.ctr[kRaysShadow];
    snap[3 * k + 2] = V.ctr[kRaysSecondary];
}

__global__ void wave_tally_out(WaveView V, unsigned long long* tally) {
    tally[0] += V.ctr[kRaysPrimary];
    tally[1] += V.ctr[kRaysShadow];
    tally[2] += V.ctr[kRaysSecondary];
}

}  // namespace dev

// Queue and slot buffers of the wavefront form, carved from one device block,
// plus the frame graph.  A resident scene owns one for its own frames; the
// request loop carves one per in-flight request from memory it allocates, so
// concurrent requests on one scene never share scratch.
struct Wave {
    long long nsamples_cap = 0;
    int L = 0;
    float* slots = nullptr;
    float* coef = nullptr;
    float4* shq = nullptr;
    float4* rq = nullptr;
    float4* tq = nullptr;
    unsigned int* ctr = nullptr;
    void* block = nullptr;   // owned by this struct when it came from wave_reserve_into
    size_t bytes = 0;
    int sms = 148;
    // The frame's launch sequence captured once per frame shape and replayed.
    // The first frame of a shape is launched directly (a scene rendered once,
    // as by the one-call entry points, never pays for a capture); the graph
    // is captured when the same shape comes again.
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Key {
        int W, H, aa, x0, y0, x1, y1;
        const void* out;
        int tuning;   // tuning generation the graph was captured under
        bool operator==(const Key& o) const {
            return W == o.W && H == o.H && aa == o.aa && x0 == o.x0 && y0 == o.y0 && x1 == o.x1 && y1 == o.y1 &&
                   out == o.out && tuning == o.tuning;
        }
    } key{};
    Key direct{};              // shape of the last frame launched directly
    bool has_direct = false;
};

static constexpr size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Bytes of the queue and slot arrays for `nsamples` samples and L lights, as
// wave_carve lays them out (each array 256-byte aligned).
static constexpr size_t wave_scratch_bytes_for(int L, long long nsamples) {
    return align256((size_t)nsamples * 3 * (L + 2) * 3 * sizeof(float)) +
           align256((size_t)nsamples * 3 * sizeof(float)) +
           align256((size_t)nsamples * (L > 1 ? L : 1) * 3 * sizeof(float4)) +
           2 * align256((size_t)nsamples * 2 * sizeof(float4)) + align256(dev::kCounterWords * sizeof(unsigned int));
}

size_t wave_scratch_bytes(int L, long long nsamples) { return wave_scratch_bytes_for(L, nsamples); }

// Points w's arrays into [base, base + bytes) for `nsamples` samples and L
// lights (base 256-byte aligned).  False when the block is too small.
static bool wave_carve(Wave& w, void* base, size_t bytes, int L, long long nsamples) {
    if (wave_scratch_bytes(L, nsamples) > bytes) return false;
    const size_t n = (size_t)nsamples;
    char* p = static_cast<char*>(base);
    auto take = [&p](size_t b) {
        char* q = p;
        p += align256(b);
        return q;
    };
    w.slots = reinterpret_cast<float*>(take(n * 3 * (L + 2) * 3 * sizeof(float)));
    w.coef = reinterpret_cast<float*>(take(n * 3 * sizeof(float)));
    w.shq = reinterpret_cast<float4*>(take(n * std::max(L, 1) * 3 * sizeof(float4)));
    w.rq = reinterpret_cast<float4*>(take(n * 2 * sizeof(float4)));
    w.tq = reinterpret_cast<float4*>(take(n * 2 * sizeof(float4)));
    w.ctr = reinterpret_cast<unsigned int*>(take(dev::kCounterWords * sizeof(unsigned int)));
    w.nsamples_cap = nsamples;
    w.L = L;
    return true;
}

// SM count of the current device.
static int device_sms() {
    int dev_id = 0, n = 148;
    if (cudaGetDevice(&dev_id) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev_id);
    return n > 0 ? n : 148;
}

// Persistent grid: as many 128-thread blocks as fit on every SM.
template <class K>
static int persistent_grid(K kernel, int sms) {
    int b = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 128, 0);
    return sms * std::max(b, 1);
}

// Grid of the shadow stage: the tuned blocks per SM, capped by occupancy.
template <class K>
static int shadow_grid(K kernel, int sms, int per_sm) {
    const int full = persistent_grid(kernel, sms);
    return per_sm > 0 ? std::min(full, sms * per_sm) : full;
}

// Persistent grids of the primary, mirror and refraction kernels of one
// variant, per device: computed on a device's first frame under a lock, so
// threads that start frames at the same time, or on different GPU models,
// each see complete grids for their own device.
struct StageGrids {
    int sms = 0, primary = 0, reflect = 0, refract = 0;
};
constexpr int kGridDevices = 64;

template <int F, bool MULTI>
static StageGrids stage_grids() {
    static std::mutex mu;
    static StageGrids grids[kGridDevices];
    int d = 0;
    cudaGetDevice(&d);
    StageGrids g;
    if (d >= 0 && d < kGridDevices) {
        std::lock_guard<std::mutex> lk(mu);
        g = grids[d];
    }
    if (g.primary) return g;
    g.sms = device_sms();
    g.primary = persistent_grid(dev::wave_primary<F, MULTI>, g.sms);
    g.reflect = persistent_grid(dev::wave_reflect<F, MULTI>, g.sms);
    g.refract = persistent_grid(dev::wave_refract<F, MULTI>, g.sms);
    if (d >= 0 && d < kGridDevices) {
        std::lock_guard<std::mutex> lk(mu);
        grids[d] = g;
    }
    return g;
}

// The queue pipeline for category set F: one frame (S0 / V), or with MULTI
// every job of V.jobs (S0 unused; npad is then the total padded pixels).
// Stage profiling (not inside a graph): `ev` gets 8 events recorded at the
// stage boundaries (before primary, after primary, shadow, reflect, shadow,
// refract, shadow, resolve) and `snap` the ray counters after each of the 7
// kernels (3 words each).
template <int F, bool MULTI = false>
static cudaError_t run_pipeline(const dev::DevScene& S0, const dev::WaveView& V, int npad, float4* out,
                                cudaStream_t stream, unsigned long long* tally, cudaEvent_t* ev = nullptr,
                                unsigned int* snap = nullptr) {
    const StageGrids grids = stage_grids<F, MULTI>();
    const int sms = grids.sms, g_primary = grids.primary, g_reflect = grids.reflect, g_refract = grids.refract;
    const Tuning tu = tuning();
    // instanced meshes: the refill kernel walks the scene's own BVH4s lane by
    // lane and has no top level; such scenes take the per-ray shadow kernel
    // (batches group them apart)
    const bool refill = tu.shadow_kernel == 1 && S0.num_instances == 0;
    const bool smem = tu.shadow_stack == 1;
    const int g_shadow = !refill ? shadow_grid(dev::wave_shadow<F, MULTI>, sms, tu.shadow_blocks_per_sm)
                         : smem  ? shadow_grid(dev::wave_shadow_refill<F, true, MULTI>, sms, tu.shadow_blocks_per_sm)
                                 : shadow_grid(dev::wave_shadow_refill<F, false, MULTI>, sms, tu.shadow_blocks_per_sm);
    auto shadow = [&]() {
        if (!refill)
            dev::wave_shadow<F, MULTI><<<g_shadow, 128, 0, stream>>>(S0, V);
        else if (smem)
            dev::wave_shadow_refill<F, true, MULTI><<<g_shadow, 128, 0, stream>>>(S0, V, tu.refill_min, tu.inner_min);
        else
            dev::wave_shadow_refill<F, false, MULTI><<<g_shadow, 128, 0, stream>>>(S0, V, tu.refill_min,
                                                                                  tu.inner_min);
    };
    int mark = 0;
    auto stage_end = [&]() {
        if (snap) dev::wave_snapshot<<<1, 1, 0, stream>>>(V, snap, mark);
        if (ev) cudaEventRecord(ev[mark + 1], stream);
        mark++;
    };
    cudaError_t e;
    if ((e = cudaMemsetAsync(V.ctr, 0, dev::kCounterWords * sizeof(unsigned int), stream)) != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[0], stream);
    dev::wave_primary<F, MULTI><<<g_primary, 128, 0, stream>>>(S0, V);
    stage_end();
    shadow();
    stage_end();
    if ((e = cudaMemsetAsync(&V.ctr[dev::kShadowCount], 0, 2 * sizeof(unsigned int), stream)) != cudaSuccess) return e;
    dev::wave_reflect<F, MULTI><<<g_reflect, 128, 0, stream>>>(S0, V);
    stage_end();
    shadow();
    stage_end();
    if ((e = cudaMemsetAsync(&V.ctr[dev::kShadowCount], 0, 2 * sizeof(unsigned int), stream)) != cudaSuccess) return e;
    dev::wave_refract<F, MULTI><<<g_refract, 128, 0, stream>>>(S0, V);
    stage_end();
    shadow();
    stage_end();
    if (npad > 0) dev::wave_resolve<MULTI><<<(npad + 127) / 128, 128, 0, stream>>>(V, out);
    if (ev) cudaEventRecord(ev[7], stream);
    if (tally) dev::wave_tally_out<<<1, 1, 0, stream>>>(V, tally);
    return cudaGetLastError();
}

static void wave_free(Wave* w) {
    if (!w) return;
    if (w->exec) cudaGraphExecDestroy(w->exec);
    if (w->capture_stream) cudaStreamDestroy(w->capture_stream);
    dfree(w->block);
    delete w;
}

// A released scene's queue block is kept (one per device, the larger one)
// for the next scene that fits: the one-call entry points upload, render and
// release a scene per call, and a 4 GB pool allocation was measured at about
// 5 ms on a B200 even with the freed block in the pool.  The kept block goes
// back to the pool at sheen_cleanup, when the pool trims, before an
// allocation that ran out of memory is retried, and not at all with
// "mem.pool_keep_mb" 0.
namespace {
constexpr int kParkDevices = 64;
std::mutex g_park_mu;
Wave* g_parked[kParkDevices] = {};
}  // namespace

// The kept block of device `dev` when it holds at least `bytes` and `dev` is
// the current device (the block's memory belongs to it).
static Wave* take_parked(size_t bytes, int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != dev || dev < 0 || dev >= kParkDevices) return nullptr;
    std::lock_guard<std::mutex> lk(g_park_mu);
    Wave* w = g_parked[dev];
    if (!w || w->bytes < bytes) return nullptr;
    g_parked[dev] = nullptr;
    return w;
}

void release_parked_waves() {
    std::lock_guard<std::mutex> lk(g_park_mu);
    int cur = 0;
    cudaGetDevice(&cur);
    for (int d = 0; d < kParkDevices; d++) {
        if (!g_parked[d]) continue;
        cudaSetDevice(d);
        wave_free(g_parked[d]);
        g_parked[d] = nullptr;
    }
    cudaSetDevice(cur);
}

void wave_release(DeviceScene& s) {
    Wave* w = s.wave;
    s.wave = nullptr;
    if (!w) return;
    // kept under the scene's own device, and only when it is the current one
    // (the pool calls below act on the current device)
    const int dev = s.device;
    int cur = -1;
    if (tuning().pool_keep_mb <= 0 || cudaGetDevice(&cur) != cudaSuccess || cur != dev || dev < 0 ||
        dev >= kParkDevices) {
        wave_free(w);
        return;
    }
    cudaDeviceSynchronize();   // as a free: no frame of the released scene may still run
    if (w->exec) { cudaGraphExecDestroy(w->exec); w->exec = nullptr; }
    w->key = Wave::Key{};
    w->has_direct = false;
    std::lock_guard<std::mutex> lk(g_park_mu);
    Wave*& slot = g_parked[dev];
    if (slot && slot->bytes >= w->bytes) {
        wave_free(w);
    } else {
        wave_free(slot);
        slot = w;
    }
}

static bool wave_supported(const DeviceScene& s) {
    const dev::DevScene& v = s.view;
    if (v.num_media > 0 || v.num_lights > dev::kMaxWaveLights || v.bounces > 1) return false;
    return !s.wave_fallback;
}

// Makes the scene's own scratch hold at least `nsamples` samples for L
// lights: re-carves the block when it is large enough, else reallocates.
// A re-carve moves the arrays, so the captured frame graph is dropped.
static cudaError_t wave_reserve_into(Wave*& w, int L, long long nsamples, int dev) {
    if (w && w->nsamples_cap >= nsamples && w->L == L) return cudaSuccess;
    if (w && wave_scratch_bytes(L, nsamples) <= w->bytes) {
        if (w->exec) { cudaGraphExecDestroy(w->exec); w->exec = nullptr; }
        wave_carve(*w, w->block, w->bytes, L, nsamples);
        return cudaSuccess;
    }
    const size_t bytes = wave_scratch_bytes(L, nsamples);
    if (!w) {
        if (Wave* p = take_parked(bytes, dev)) {
            w = p;
            wave_carve(*w, w->block, w->bytes, L, nsamples);
            return cudaSuccess;
        }
    }
    wave_free(w);
    w = new Wave();
    cudaError_t e = dmalloc(&w->block, bytes);
    if (e != cudaSuccess) {
        delete w;
        w = nullptr;
        return e;
    }
    w->bytes = bytes;
    w->sms = device_sms();
    wave_carve(*w, w->block, bytes, L, nsamples);
    return cudaSuccess;
}

// The pixel tile of the sample order: log2 of its width (3, 4 or 5; tiles
// of 128 pixels), read once per frame from the launch parameters.
static int tile_log2() {
    const int w = tuning().tile_w;
    return w == 8 ? 3 : (w == 32 ? 5 : 4);
}

static long long region_padded(Region rg, int twl) {
    const long long tw = 1ll << twl, th = 128ll >> twl;
    const long long rw = rg.x1 - rg.x0, rh = rg.y1 - rg.y0;
    return (rw + tw - 1) / tw * tw * ((rh + th - 1) / th) * th;
}

static int clamp_spp(int aa) { return aa < 1 ? 1 : (aa > 64 ? 64 : aa); }

// Queue view of one frame region; the region's pixels are walked in whole
// tiles of 128 (sample_pixel), so its sample count is padded to them.
static dev::WaveView make_view(const DeviceScene& s, const Wave& w, int W, int H, int ns, Region rg, int twl) {
    dev::WaveView V;
    V.slots = w.slots; V.coef = w.coef; V.shq = w.shq; V.rq = w.rq; V.tq = w.tq; V.ctr = w.ctr;
    V.L = s.view.num_lights;
    V.ns = ns;
    V.W = W; V.H = H; V.x0 = rg.x0; V.y0 = rg.y0; V.rw = rg.x1 - rg.x0; V.rh = rg.y1 - rg.y0;
    V.nsamples = (int)(region_padded(rg, twl) * ns);
    V.tw_log2 = twl;
    const CameraData& cam = s.view.cam;
    float tan_x = 1.0f;
    if (cam.focal_length > 0.0f) {
        const float tan_h = 0.5f * cam.sensor_width / cam.focal_length;
        tan_x = (W >= H) ? tan_h : tan_h * float(W) / float(H);
    }
    V.pix_angle = 2.0f * tan_x / (float)W;
    V.count_rays = 1;
    V.jobs = nullptr;
    V.num_jobs = 0;
    V.npix = 0;
    return V;
}

// Calls fn(std::integral_constant<int, F>) with the queue kernels' template
// argument for a scene: its category set (triangles + spheres + planes only,
// or every category) and its triangle test (Moller-Trumbore or watertight).
template <class Fn>
static cudaError_t dispatch_variant(bool simple, bool watertight, Fn&& fn) {
    using dev::kCatAll;
    using dev::kCatSimple;
    using dev::kTriMT;
    using dev::kTriWT;
    if (simple)
        return watertight ? fn(std::integral_constant<int, kCatSimple | kTriWT>{})
                          : fn(std::integral_constant<int, kCatSimple | kTriMT>{});
    return watertight ? fn(std::integral_constant<int, kCatAll | kTriWT>{})
                      : fn(std::integral_constant<int, kCatAll | kTriMT>{});
}

static bool watertight_scene(const DeviceScene& s) { return s.view.q_all.watertight != 0; }

static bool simple_scene(const DeviceScene& s) {
    const dev::DevScene& sv = s.view;
    return sv.num_strands == 0 && sv.num_hfs == 0 && sv.num_ses == 0 && sv.num_lathes == 0 && sv.num_prisms == 0 &&
           sv.csg_root < 0 && sv.num_csg_roots == 0;
}

// Small frames run on the BVH4 megakernel: below wave.mega_samples samples
// (a quarter of that for scenes with triangles, whose megakernel carries the
// BVH4 walks and falls behind sooner) the fixed cost of the queue stages --
// eight launches, each a full-GPU persistent grid, and the slot traffic --
// outweighs the megakernel's divergence.  Same queries and shading; the
// image agrees with the queue pipeline's to the last bits of the float
// arithmetic.
static bool small_frame(const DeviceScene& s, long long nsamples) {
    const long long m = tuning().mega_samples;
    return m > 0 && nsamples <= (s.view.num_tris > 0 || s.view.num_instances > 0 ? m / 4 : m);
}

cudaError_t launch_wavefront(DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t stream,
                             bool count_nodes) {
    const int twl = tile_log2();
    if (!wave_supported(s) || count_nodes) return launch_mega_bvh4(s, W, H, aa, rg, out, stream, count_nodes);
    const int ns = clamp_spp(aa);
    const long long nsamples = region_padded(rg, twl) * ns;
    if (nsamples > (1ll << 30)) return cudaErrorInvalidValue;
    if (small_frame(s, nsamples)) return launch_mega_bvh4(s, W, H, aa, rg, out, stream, false);
    cudaError_t e = wave_reserve_into(s.wave, s.view.num_lights, nsamples, s.device);
    if (e != cudaSuccess) return e;
    Wave* w = s.wave;
    const dev::WaveView V = make_view(s, *w, W, H, ns, rg, twl);
    const int npad = (int)region_padded(rg, twl);
    const bool simple = simple_scene(s);
    // Replay the captured frame when the shape and output match.  A shape
    // seen for the first time is launched directly; on its second frame the
    // sequence is captured on the scene's own stream and instantiated.
    const Wave::Key key{W, H, aa, rg.x0, rg.y0, rg.x1, rg.y1, out, tuning_generation()};
    if ((!w->exec || !(w->key == key)) && !(w->has_direct && w->direct == key)) {
        w->direct = key;
        w->has_direct = true;
        return dispatch_variant(simple, watertight_scene(s), [&](auto f) {
            return run_pipeline<decltype(f)::value>(s.view, V, npad, out, stream, s.d_tally);
        });
    }
    if (!w->exec || !(w->key == key)) {
        if (w->exec) { cudaGraphExecDestroy(w->exec); w->exec = nullptr; }
        if (!w->capture_stream &&
            (e = cudaStreamCreateWithFlags(&w->capture_stream, cudaStreamNonBlocking)) != cudaSuccess)
            return e;
        if ((e = cudaStreamBeginCapture(w->capture_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
        cudaError_t le = dispatch_variant(simple, watertight_scene(s), [&](auto f) {
            return run_pipeline<decltype(f)::value>(s.view, V, npad, out, w->capture_stream, s.d_tally);
        });
        cudaGraph_t graph = nullptr;
        e = cudaStreamEndCapture(w->capture_stream, &graph);
        if (le != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return le; }
        if (e != cudaSuccess) return e;
        e = cudaGraphInstantiate(&w->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) { w->exec = nullptr; return e; }
        w->key = key;
    }
    return cudaGraphLaunch(w->exec, stream);
}

bool wave_pipeline_used(const DeviceScene& s) { return wave_supported(s); }

int frame_path(const DeviceScene& s, int W, int H, int aa) {
    if (s.form != SHEEN_FORM_WAVEFRONT) return SHEEN_PATH_PLAIN;
    if (!wave_supported(s)) return SHEEN_PATH_MEGAKERNEL;
    const long long nsamples = region_padded(Region{0, 0, W, H}, tile_log2()) * clamp_spp(aa);
    return small_frame(s, nsamples) ? SHEEN_PATH_MEGAKERNEL : SHEEN_PATH_QUEUES;
}

// Many frames, regions and scenes in one pass of the queue kernels: every
// stage is one persistent launch over the samples of all jobs, whose work
// the blocks claim from the same counters, so cheap jobs (sky, a small
// tile) and expensive ones (glass, a dense mesh) share the SMs.  Each job
// gets its own part of the slot and weight arrays (its light count decides
// its slot stride); the ray queues are shared and their entries carry the
// job.  Jobs run under the kernel variant their scene would use alone
// (scenes of triangles, spheres and planes only, or every category), one
// pass per variant, so every sample computes bit for bit what a single-frame
// render computes: the compiler rounds the two variants' shading arithmetic
// differently.  Scratch comes from the library's pool, ordered on `stream`.
template <int F>
static cudaError_t batch_pass(const std::vector<BatchItem>& items, cudaStream_t stream, unsigned long long* tally) {
    const int twl = tile_log2();
    const int n = (int)items.size();
    if (n == 0) return cudaSuccess;
    long long total_samples = 0, total_pix = 0, slot_floats = 0, shadow_entries = 0;
    for (const BatchItem& it : items) {
        const long long npad = region_padded(it.rg, twl), ns = clamp_spp(it.aa);
        const int L = it.s->view.num_lights;
        total_samples += npad * ns;
        total_pix += npad;
        slot_floats += npad * ns * 3 * (L + 2) * 3;
        shadow_entries += npad * ns * std::max(L, 1);
    }
    if (total_samples > (1ll << 30) || slot_floats > (1ll << 40)) return cudaErrorInvalidValue;
    const size_t b_jobs = align256((size_t)n * sizeof(dev::JobDesc));
    const size_t b_slots = align256((size_t)slot_floats * sizeof(float));
    const size_t b_coef = align256((size_t)total_samples * 3 * sizeof(float));
    const size_t b_shq = align256((size_t)shadow_entries * 3 * sizeof(float4));
    const size_t b_rq = align256((size_t)total_samples * 2 * sizeof(float4));
    const size_t b_ctr = align256(dev::kCounterWords * sizeof(unsigned int));
    char* block = nullptr;
    cudaError_t e = dmalloc_async(&block, b_jobs + b_slots + b_coef + b_shq + 2 * b_rq + b_ctr, stream);
    if (e != cudaSuccess) return e;
    dev::JobDesc* d_jobs = reinterpret_cast<dev::JobDesc*>(block);
    float* slots = reinterpret_cast<float*>(block + b_jobs);
    float* coef = reinterpret_cast<float*>(block + b_jobs + b_slots);
    float4* shq = reinterpret_cast<float4*>(block + b_jobs + b_slots + b_coef);
    float4* rq = reinterpret_cast<float4*>(block + b_jobs + b_slots + b_coef + b_shq);
    float4* tq = reinterpret_cast<float4*>(block + b_jobs + b_slots + b_coef + b_shq + b_rq);
    unsigned int* ctr = reinterpret_cast<unsigned int*>(block + b_jobs + b_slots + b_coef + b_shq + 2 * b_rq);
    std::vector<dev::JobDesc> jobs((size_t)n);
    long long sample_off = 0, pix_off = 0, slot_off = 0;
    for (int j = 0; j < n; j++) {
        const BatchItem& it = items[(size_t)j];
        const int ns = clamp_spp(it.aa);
        Wave w;
        w.slots = slots + slot_off;
        w.coef = coef + 3 * sample_off;
        w.shq = shq;
        w.rq = rq;
        w.tq = tq;
        w.ctr = ctr;
        dev::JobDesc& J = jobs[(size_t)j];
        std::memset(&J, 0, sizeof(J));
        J.S = it.s->view;
        J.V = make_view(*it.s, w, it.W, it.H, ns, it.rg, twl);
        J.out = it.out;
        J.sample_base = (int)sample_off;
        J.pix_base = (int)pix_off;
        const long long npad = region_padded(it.rg, twl);
        sample_off += npad * ns;
        pix_off += npad;
        slot_off += npad * ns * 3 * (it.s->view.num_lights + 2) * 3;
    }
    e = cudaMemcpyAsync(d_jobs, jobs.data(), (size_t)n * sizeof(dev::JobDesc), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
        dev::WaveView V0 = jobs[0].V;
        V0.slots = slots;
        V0.coef = coef;
        V0.nsamples = (int)total_samples;
        V0.npix = (int)total_pix;
        V0.jobs = d_jobs;
        V0.num_jobs = n;
        V0.count_rays = 1;
        e = run_pipeline<F, true>(items[0].s->view, V0, (int)total_pix, nullptr, stream, tally);
    }
    // the copy above reads `jobs` before returning (pageable host memory);
    // the block returns to the pool once the stream has finished with it
    dfree_async(block, stream);
    return e;
}

cudaError_t launch_wavefront_batch(const std::vector<BatchItem>& items, cudaStream_t stream,
                                   unsigned long long* tally) {
    // one pass per kernel variant: category set x triangle test, and scenes
    // with instanced meshes apart (their shadow stage is the per-ray kernel)
    std::vector<BatchItem> groups[8];
    for (const BatchItem& it : items) {
        if (!it.s || it.s->form != SHEEN_FORM_WAVEFRONT || !wave_supported(*it.s)) return cudaErrorInvalidValue;
        groups[(simple_scene(*it.s) ? 0 : 2) + (watertight_scene(*it.s) ? 1 : 0) +
               (it.s->view.num_instances > 0 ? 4 : 0)].push_back(it);
    }
    cudaError_t e = cudaSuccess;
    for (int g = 0; g < 8 && e == cudaSuccess; g++)
        if (!groups[g].empty())
            e = dispatch_variant((g & 2) == 0, (g & 1) != 0, [&](auto f) {
                return batch_pass<decltype(f)::value>(groups[g], stream, tally);
            });
    return e;
}

// One frame of the queue pipeline launched directly (no graph) with events
// at the stage boundaries and the ray counters read after every kernel.
cudaError_t profile_wavefront(DeviceScene& s, int W, int H, int aa, float4* out, cudaStream_t stream,
                              SheenStageProfile* prof) {
    const int twl = tile_log2();
    if (!wave_supported(s)) return cudaErrorNotSupported;
    const int ns = clamp_spp(aa);
    const Region rg{0, 0, W, H};
    const long long nsamples = region_padded(rg, twl) * ns;
    if (nsamples > (1ll << 30)) return cudaErrorInvalidValue;
    cudaError_t e = wave_reserve_into(s.wave, s.view.num_lights, nsamples, s.device);
    if (e != cudaSuccess) return e;
    const dev::WaveView V = make_view(s, *s.wave, W, H, ns, rg, twl);
    const int npad = (int)region_padded(rg, twl);
    cudaEvent_t ev[8] = {nullptr};
    unsigned int* snap = nullptr;
    for (int i = 0; i < 8 && e == cudaSuccess; i++) e = cudaEventCreate(&ev[i]);
    if (e == cudaSuccess) e = dmalloc(&snap, 21 * sizeof(unsigned int));
    if (e == cudaSuccess)
        e = dispatch_variant(simple_scene(s), watertight_scene(s), [&](auto f) {
            return run_pipeline<decltype(f)::value>(s.view, V, npad, out, stream, nullptr, ev, snap);
        });
    unsigned int h[21] = {0};
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess) e = cudaMemcpy(h, snap, sizeof(h), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
        float ms[7];
        for (int i = 0; i < 7; i++) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
        // stages in launch order: primary, shadow, reflect, shadow, refract, shadow, resolve
        prof->primary_ms = ms[0];
        prof->shadow_ms[0] = ms[1];
        prof->reflect_ms = ms[2];
        prof->shadow_ms[1] = ms[3];
        prof->refract_ms = ms[4];
        prof->shadow_ms[2] = ms[5];
        prof->resolve_ms = ms[6];
        float total = 0.0f;
        cudaEventElapsedTime(&total, ev[0], ev[7]);
        prof->total_ms = total;
        // rays issued by each kernel: differences of the counter snapshots
        unsigned int prev[3] = {0, 0, 0};
        unsigned long long rays[7];
        for (int k = 0; k < 7; k++) {
            rays[k] = 0;
            for (int j = 0; j < 3; j++) { rays[k] += h[3 * k + j] - prev[j]; prev[j] = h[3 * k + j]; }
        }
        prof->primary_rays = rays[0];
        prof->shadow_rays[0] = rays[1];
        prof->reflect_rays = rays[2];
        prof->shadow_rays[1] = rays[3];
        prof->refract_rays = rays[4];
        prof->shadow_rays[2] = rays[5];
    }
    for (int i = 0; i < 8; i++)
        if (ev[i]) cudaEventDestroy(ev[i]);
    dfree(snap);
    return e;
}

cudaError_t launch_wavefront_scratch(DeviceScene& s, void* scratch, size_t scratch_bytes, int W, int H, int aa,
                                     Region rg, float4* out, cudaStream_t stream, unsigned long long* tally) {
    const int twl = tile_log2();
    if (!wave_supported(s)) return launch_mega_bvh4(s, W, H, aa, rg, out, stream, false, tally);
    const int ns = clamp_spp(aa);
    const long long nsamples = region_padded(rg, twl) * ns;
    if (nsamples > (1ll << 30)) return cudaErrorInvalidValue;
    if (small_frame(s, nsamples)) return launch_mega_bvh4(s, W, H, aa, rg, out, stream, false, tally);
    Wave w;
    if (!wave_carve(w, scratch, scratch_bytes, s.view.num_lights, nsamples)) return cudaErrorInvalidValue;
    const dev::WaveView V = make_view(s, w, W, H, ns, rg, twl);
    const int npad = (int)region_padded(rg, twl);
    return dispatch_variant(simple_scene(s), watertight_scene(s), [&](auto f) {
        return run_pipeline<decltype(f)::value>(s.view, V, npad, out, stream, tally);
    });
}

// ---------------------------------------------------------------------
// Allocation-free rendering of a small region (sheen_scene_render_region_noalloc).
//
// Some callers cannot let the library allocate GPU memory while they draw:
// a real-time loop that reserves all of its device memory at start-up and
// treats any later allocation as a fault, or an embedding application whose
// memory manager must own every byte on the device.  The regular entry
// points allocate the wavefront queues on a scene's first frame (and again
// when a larger frame comes), so they cannot be used there.  This variant
// runs the same queue pipeline -- the same kernels, variant and launch
// parameters as a resident scene's own frames -- with its scratch (per-sample
// light slots, blend weights, the three ray queues and their counters)
// carved from one fixed array in the library's device globals instead.
//
// Limits: at most kNoAllocMaxSamples samples per call (the region's pixels
// rounded up to whole 128-pixel tiles, 16x8 by default, times the samples
// per pixel -- e.g. a
// 128x128 tile at 1 spp or 64x64 at 4 spp) and scenes with at most
// kNoAllocMaxLights lights.  The array (about 13 MB) is held on every GPU
// that loads the library until the process exits.  Every call uses the same
// array and each call clears the queue counters it starts from: calls that
// can overlap on the GPU (different streams, or threads issuing
// concurrently) race and must be serialised by the caller, e.g. by issuing
// them on one stream.
// ---------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxSamples = 16384;
constexpr int kNoAllocMaxLights = 8;
constexpr size_t kNoAllocBytes = wave_scratch_bytes_for(kNoAllocMaxLights, kNoAllocMaxSamples);

// The scratch itself.  Host code must not use this name as an address (on
// the host it names a stand-in, not device memory); noalloc_scratch() below
// resolves the device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device, looked up with
// cudaGetSymbolAddress on the first call on each device (and again after
// sheen_cleanup, which resets the device and forgets the addresses).
cudaError_t noalloc_scratch(unsigned char** out) {
    int dev_id = 0;
    cudaError_t e = cudaGetDevice(&dev_id);
    if (e != cudaSuccess) return e;
    if (dev_id < 0 || dev_id >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev_id]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev_id] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_ptr[dev_id];
    return cudaSuccess;
}

}  // namespace

void release_noalloc_scratch() {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    for (auto& p : g_noalloc_ptr) p = nullptr;
}

}  // namespace sheen

extern "C" int sheen_scene_render_region_noalloc(SheenDeviceScene h, int W, int H, int aa, int x0, int y0, int x1,
                                                 int y1, float* out_rgba_device, void* stream) {
    using namespace sheen;
    const int twl = tile_log2();
    auto* s = reinterpret_cast<DeviceScene*>(h);
    if (!s) { set_error("null scene handle"); return -1; }
    if (W <= 0 || H <= 0 || aa < 1 || aa > 64 || !out_rgba_device) { set_error("bad render params"); return -1; }
    if (x0 < 0 || y0 < 0 || x1 > W || y1 > H || x0 >= x1 || y0 >= y1) { set_error("bad render region"); return -1; }
    if (s->form != SHEEN_FORM_WAVEFRONT) {
        set_error("allocation-free rendering needs a scene created with SHEEN_FORM_WAVEFRONT");
        return -1;
    }
    const Region rg{x0, y0, x1, y1};
    const long long nsamples = region_padded(rg, twl) * aa;
    if (nsamples > kNoAllocMaxSamples) {
        set_error("region too large for allocation-free rendering: at most 16384 samples per call "
                  "(pixels rounded up to whole 128-pixel tiles, 16x8 by default, times samples per pixel)");
        return -1;
    }
    if (s->view.num_lights > kNoAllocMaxLights) {
        set_error("allocation-free rendering supports at most 8 lights");
        return -1;
    }
    unsigned char* base = nullptr;
    cudaError_t e = noalloc_scratch(&base);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return -1; }
    // Beams, media and the shadow-debug mode run on the BVH4 megakernel,
    // which needs no scratch; everything else runs the queue pipeline on the
    // carved array (launch_wavefront_scratch allocates nothing).
    e = launch_wavefront_scratch(*s, base, kNoAllocBytes, W, H, aa, rg, reinterpret_cast<float4*>(out_rgba_device),
                                 (cudaStream_t)stream, nullptr);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return -1; }
    return 0;
}
