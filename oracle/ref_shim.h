/*
 * ref_shim.h -- force-included (g++ -include) ahead of the reference's own
 * CUDA sources so that they compile as ordinary host C++.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or includes this:
 * it builds the reference renderer for the CPU into oracle/_ref/ so the
 * parity tests and the CPU baseline can run the reference's own per-pixel
 * code (render_kernel.cu:1-926) unchanged on the host cores.
 *
 * What it provides:
 *   - the CUDA vector types and launch-parameter declarations (the CUDA
 *     headers compile fine under g++);
 *   - rsqrtf, which the CUDA headers only declare for device code; here it
 *     is the exact 1/sqrt (the device instruction is an approximation, so
 *     host and device differ by a few ulp -- absorbed by the parity
 *     tolerances);
 *   - per-thread blockIdx/threadIdx/blockDim, set by the driver before each
 *     call of the kernel body;
 *   - __global__ / __launch_bounds__ as no-ops, so a kernel is a normal
 *     function with external linkage;
 *   - atomicAdd for the photon append counter, answered by the driver so the
 *     photon order is deterministic (slot = emission index);
 *   - printf muted: the reference prints one DEBUG line per caustic shade
 *     (render_kernel.cu:291-294), which would dominate a CPU run.
 */
#pragma once
#include <cstdio>
#include <cmath>
#include <cuda_runtime.h>
#include <device_launch_parameters.h>

inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }

extern thread_local uint3 sheen_ref_block_idx;
extern thread_local uint3 sheen_ref_thread_idx;
extern thread_local dim3 sheen_ref_block_dim;
#define blockIdx sheen_ref_block_idx
#define threadIdx sheen_ref_thread_idx
#define blockDim sheen_ref_block_dim

#undef __global__
#define __global__
#undef __launch_bounds__
#define __launch_bounds__(a, b)

unsigned int sheen_ref_atomic_add(unsigned int* p, unsigned int v);
inline unsigned int atomicAdd(unsigned int* p, unsigned int v) { return sheen_ref_atomic_add(p, v); }

#define printf(...) ((void)0)
