// render_plain.cu -- plain FP32 form: one thread per pixel, every sample of
// the pixel in that thread, reference-order BVH traversal (the drop-in for
// render_kernel, render_kernel.cu:438-814).
//
// Differences from the reference kernel that do not change results:
//   - no recursion and no 16 KB per-thread stack (CSG is iterative);
//   - BVH nodes are read as two 128-bit loads through the read-only path;
//   - triangle positions come from a 48-byte record, the 112-byte Triangle
//     only for the closest hit;
//   - 16x8 thread blocks;
//   - rays issued are counted (warp-aggregated atomics, one per warp).
#include "dev/integrator.cuh"
#include "engine.h"

namespace sheen {
namespace dev {

__device__ __forceinline__ void warp_add(unsigned long long* dst, unsigned long long v) {
    const unsigned mask = __activemask();
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(mask, v, o);
    if ((threadIdx.x + threadIdx.y * blockDim.x) % 32 == 0) atomicAdd(dst, v);
}

// 8 blocks of 128 threads per SM (64 registers): the kernel keeps its
// traversal stacks in local memory either way, and the latency of those
// and of the node fetches needs the warps.  Measured on a B200 (mesh
// frame, 1080p 4 spp): 135.8 ms at the default 168 registers (3 blocks),
// 113.0 ms at 4 blocks, 79.4 ms at 8.
template <bool COUNT>
__global__ void __launch_bounds__(128, 8) plain_kernel(const __grid_constant__ DevScene S, float4* __restrict__ out, int W, int H, int aa,
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
                acc += render_sample_deep<RefTracer<COUNT>, COUNT>(S, x, y, s, ns, W, H, rt, c);
        } else {
            for (int s = 0; s < ns; s++) acc += render_sample<RefTracer<COUNT>, COUNT>(S, x, y, s, ns, W, H, rt, c);
        }
        const float inv = 1.0f / float(ns);
        out[(size_t)y * W + x] = make_float4(acc.x * inv, acc.y * inv, acc.z * inv, 1.0f);
    }
    if (tally) {
        warp_add(&tally[0], rt.primary);
        warp_add(&tally[1], rt.shadow);
        warp_add(&tally[2], rt.secondary);
        if (COUNT) {
            warp_add(&tally[3], c.nodes);
            warp_add(&tally[4], c.prims);
            warp_add(&tally[5], c.shadow_nodes);
            warp_add(&tally[6], c.shadow_prims);
        }
    }
}

// Primary closest hit of every sample (camera ray of render_kernel.cu:491-518
// and scene_intersect), for hit-identity parity checks.
template <class T>
__global__ void primary_hits_kernel(const __grid_constant__ DevScene S, int W, int H, int ns, int* obj, int* mat, float* tt) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    Counters c;
    for (int s = 0; s < ns; s++) {
        float pix;
        const Ray r = camera_ray(S.cam, x, y, s, ns, W, H, pix, S.aa_centered);
        Hit h;
        const size_t k = ((size_t)y * W + x) * ns + s;
        if (T::closest(S, r, h, c)) { obj[k] = h.obj; mat[k] = h.mat; tt[k] = h.t; }
        else { obj[k] = (int)0x80000000; mat[k] = (int)0x80000000; tt[k] = -1.0f; }
    }
}

}  // namespace dev

cudaError_t launch_primary_hits_plain(const DeviceScene& s, int W, int H, int ns, int* obj, int* mat, float* t,
                                      cudaStream_t stream) {
    const dim3 block(16, 8);
    const dim3 grid((W + 15) / 16, (H + 7) / 8);
    dev::primary_hits_kernel<dev::RefTracer<false>><<<grid, block, 0, stream>>>(s.view, W, H, ns, obj, mat, t);
    return cudaGetLastError();
}

cudaError_t launch_plain(const DeviceScene& s, int W, int H, int aa, Region rg, float4* out, cudaStream_t stream,
                         bool count_nodes,
                         unsigned long long* tally) {
    if (!tally) tally = s.d_tally;
    const dim3 block(16, 8);
    const dim3 grid((rg.x1 - rg.x0 + 15) / 16, (rg.y1 - rg.y0 + 7) / 8);
    if (count_nodes)
        dev::plain_kernel<true><<<grid, block, 0, stream>>>(s.view, out, W, H, aa, rg.x0, rg.y0, rg.x1, rg.y1, tally);
    else
        dev::plain_kernel<false><<<grid, block, 0, stream>>>(s.view, out, W, H, aa, rg.x0, rg.y0, rg.x1, rg.y1, tally);
    return cudaGetLastError();
}

}  // namespace sheen
