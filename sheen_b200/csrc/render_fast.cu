// render_fast.cu -- the BVH4 megakernel: one thread per pixel running the
// shared integrator over FastTracer (BVH4 closest hit with culling, split
// any-hit shadow queries).  The wavefront form uses it for frames its queue
// pipeline does not cover, and it is a measurement point of its own.
#include "dev/integrator.cuh"
#include "dev/trace_bvh4.cuh"
#include "engine.h"

namespace sheen {
namespace dev {

__device__ __forceinline__ void warp_add_fast(unsigned long long* dst, unsigned long long v) {
    const unsigned mask = __activemask();
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(mask, v, o);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0) atomicAdd(dst, v);
}

// F: the scene's category set and triangle test (as the queue kernels'),
// so a scene of spheres, triangles and planes does not carry the other
// categories' code and registers.  Those smaller variants run 8 blocks of
// 128 threads per SM (64 registers): measured on a B200, the spheres frame
// 0.140 -> 0.126 ms and the mesh workload at depth 4 with instanced tori
// 119.1 -> 101.7 ms against the unbounded 168-register build.  The
// all-categories variant runs 4 blocks (128 registers): 640x360 1-spp
// frames of the analytic workload 2.59 -> 2.54 ms and of the caustics
// workload 6.63 -> 5.81 ms against its unbounded build.
template <bool COUNT, int F = kCatAll>
__global__ void __launch_bounds__(128, ((F & kCatAll) == kCatAll) ? 4 : 8) mega_bvh4_kernel(const __grid_constant__ DevScene S, float4* __restrict__ out, int W, int H, int aa,
                                                        int x0, int y0, int x1, int y1, unsigned long long* tally) {
    const int x = x0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int y = y0 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
    RayTally rt;
    Counters c;
    if (x < x1 && y < y1) {
        const int ns = aa < 1 ? 1 : (aa > 64 ? 64 : aa);
        float3 acc = f3(0.0f, 0.0f, 0.0f);
        if (S.bounces > 1) {   // extension: reflect + refract recursion
            for (int s = 0; s < ns; s++)
                acc += render_sample_deep<FastTracer<COUNT, F>, COUNT>(S, x, y, s, ns, W, H, rt, c);
        } else {
            for (int s = 0; s < ns; s++) acc += render_sample<FastTracer<COUNT, F>, COUNT>(S, x, y, s, ns, W, H, rt, c);
        }
        const float inv = 1.0f / float(ns);
        out[(size_t)y * W + x] = make_float4(acc.x * inv, acc.y * inv, acc.z * inv, 1.0f);
    }
    if (tally) {
        warp_add_fast(&tally[0], rt.primary);
        warp_add_fast(&tally[1], rt.shadow);
        warp_add_fast(&tally[2], rt.secondary);
        if (COUNT) {
            warp_add_fast(&tally[3], c.nodes);
            warp_add_fast(&tally[4], c.prims);
            warp_add_fast(&tally[5], c.shadow_nodes);
            warp_add_fast(&tally[6], c.shadow_prims);
        }
    }
}

__global__ void primary_hits_bvh4_kernel(const __grid_constant__ DevScene S, int W, int H, int ns, int* obj, int* mat, float* tt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    Counters c;
    for (int s = 0; s < ns; s++) {
        float pix;
        const Ray r = camera_ray(S.cam, x, y, s, ns, W, H, pix, S.aa_centered);
        Hit h;
        const size_t k = ((size_t)y * W + x) * ns + s;
        if (FastTracer<false>::closest(S, r, h, c)) { obj[k] = h.obj; mat[k] = h.mat; tt[k] = h.t; }
        else { obj[k] = (int)0x80000000; mat[k] = (int)0x80000000; tt[k] = -1.0f; }
    }
}

// Closest hits of arbitrary rays (sheen_scene_trace): rays[2i] = {origin,
// tmin}, rays[2i+1] = {direction, tmax}; T is the scene form's query policy.
template <class T>
__global__ void trace_rays_kernel(const __grid_constant__ DevScene S, const float4* __restrict__ rays, int n, int* obj, int* mat, float* tt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = rays[2 * (size_t)i], b = rays[2 * (size_t)i + 1];
    Ray r;
    r.o = f3(a.x, a.y, a.z);
    r.tmin = a.w;
    r.d = f3(b.x, b.y, b.z);
    r.tmax = b.w;
    Hit h;
    Counters c;
    if (T::closest(S, r, h, c)) { obj[i] = h.obj; mat[i] = h.mat; tt[i] = h.t; }
    else { obj[i] = (int)0x80000000; mat[i] = (int)0x80000000; tt[i] = -1.0f; }
}

}  // namespace dev

cudaError_t launch_trace_rays(const DeviceScene& s, const float4* rays, int n, int* obj, int* mat, float* t,
                              cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    if (s.form == SHEEN_FORM_PLAIN)
        dev::trace_rays_kernel<dev::RefTracer<false>><<<(n + 127) / 128, 128, 0, stream>>>(s.view, rays, n, obj, mat, t);
    else
        dev::trace_rays_kernel<dev::FastTracer<false>><<<(n + 127) / 128, 128, 0, stream>>>(s.view, rays, n, obj, mat, t);
    return cudaGetLastError();
}

cudaError_t launch_mega_bvh4(const DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t stream,
                             bool count_nodes,
                             unsigned long long* tally) {
    if (!tally) tally = s.d_tally;
    const dim3 block(16, 8);
    const dim3 grid((rg.x1 - rg.x0 + 15) / 16, (rg.y1 - rg.y0 + 7) / 8);
    const dev::DevScene& v = s.view;
    const bool simple = v.num_strands == 0 && v.num_hfs == 0 && v.num_ses == 0 && v.num_lathes == 0 &&
                        v.num_prisms == 0 && v.csg_root < 0 && v.num_csg_roots == 0;
    const bool wt = v.q_all.watertight != 0;
    const bool basic = simple && v.num_tris == 0 && v.num_instances == 0;
#define MEGA(C, F) dev::mega_bvh4_kernel<C, F><<<grid, block, 0, stream>>>(v, out, W, H, aa, rg.x0, rg.y0, rg.x1, \
                                                                          rg.y1, tally)
    if (count_nodes) MEGA(true, dev::kCatAll);
    else if (basic) MEGA(false, dev::kCatBasic);
    else if (simple && !wt) MEGA(false, dev::kCatSimple | dev::kTriMT);
    else if (simple) MEGA(false, dev::kCatSimple | dev::kTriWT);
    else if (!wt) MEGA(false, dev::kCatAll | dev::kTriMT);
    else MEGA(false, dev::kCatAll | dev::kTriWT);
#undef MEGA
    return cudaGetLastError();
}

cudaError_t launch_primary_hits_bvh4(const DeviceScene& s, int W, int H, int ns, int* obj, int* mat, float* t,
                                     cudaStream_t stream) {
    const dim3 block(16, 8);
    const dim3 grid((W + 15) / 16, (H + 7) / 8);
    dev::primary_hits_bvh4_kernel<<<grid, block, 0, stream>>>(s.view, W, H, ns, obj, mat, t);
    return cudaGetLastError();
}


}  // namespace sheen
