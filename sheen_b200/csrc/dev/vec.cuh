// vec.cuh -- float3 arithmetic for the device code.
//
// normalize() uses rsqrtf like the reference (types.h:314-317), so the plain
// form's directions match the reference kernel's to the bit where the
// compiler emits the same instructions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "sheen_types.h"

namespace sheen {
namespace dev {

__host__ __device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ float3 f3(const sheen_float3& a) { return make_float3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float s, float3 a) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float3& operator+=(float3& a, float3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize(float3 v) {
    float il = rsqrtf(dot(v, v));
    return make_float3(v.x * il, v.y * il, v.z * il);
}
__device__ __forceinline__ float3 up_for(float3 a) {
    return fabsf(a.y) < 0.9f ? make_float3(0.0f, 1.0f, 0.0f) : make_float3(1.0f, 0.0f, 0.0f);
}

// Counter-based RNG of the reference (sampling/aa.h:32-43).
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float rand01(uint32_t seed) {
    return float(hash32(seed) & 0xffffffu) / 16777216.0f;
}

// Sub-pixel sample position (sampling/aa.h:15-23, 45-71): n <= 4 uses the
// 2x2 cells with +-0.125 jitter (1 spp included), n > 4 a side x side grid
// with full-cell jitter.
__device__ __forceinline__ float2 sample_offset(int s, int n, int x, int y) {
    uint32_t seed = (uint32_t)(x * 73856093) ^ (uint32_t)(y * 19349663) ^ (uint32_t)(s * 83492791);
    if (n <= 4) {
        float cx = (s == 0 || s == 2) ? 0.25f : 0.75f;
        float cy = (s < 2) ? 0.25f : 0.75f;
        float jx = rand01(seed) - 0.5f;
        float jy = rand01(seed ^ 0x9e3779b9u) - 0.5f;
        return make_float2(cx + jx * 0.5f, cy + jy * 0.5f);
    }
    int side = 2;
    while (side * side < n) side++;
    float inv = 1.0f / (float)side;
    float jx = rand01(seed);
    float jy = rand01(seed ^ 0x9e3779b9u);
    return make_float2((float(s % side) + jx) * inv, (float(s / side) + jy) * inv);
}

// Sample positions without jitter (a scene created with "camera.centered"):
// the pixel centre at 1 spp, otherwise the centres of the same cells.
__device__ __forceinline__ float2 sample_offset_centered(int s, int n) {
    if (n <= 1) return make_float2(0.5f, 0.5f);
    if (n <= 4) return make_float2((s == 0 || s == 2) ? 0.25f : 0.75f, (s < 2) ? 0.25f : 0.75f);
    int side = 2;
    while (side * side < n) side++;
    const float inv = 1.0f / (float)side;
    return make_float2((float(s % side) + 0.5f) * inv, (float(s / side) + 0.5f) * inv);
}

}  // namespace dev
}  // namespace sheen
