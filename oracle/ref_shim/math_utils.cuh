// Stand-in for a helper header that the reference's UltraGauss sources include but that is
// absent from the reference tree (ops/ultragauss_renderer/setup.py:7 points at ../common).
// Only the three helpers those sources call are defined: a float3 dot product, float3
// subtraction and a 3-float copy. Used solely to compile the reference into oracle/_ref.
#pragma once
#include <cuda_runtime.h>

__device__ __forceinline__ float dot_prod(const float3 a, const float3 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

__device__ __forceinline__ float3 operator-(const float3 a, const float3 b) {
    return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}

__device__ __forceinline__ void vec3_copy(const float* src, float* dst) {
    dst[0] = src[0];
    dst[1] = src[1];
    dst[2] = src[2];
}

// float3 arithmetic used by the reference's UltraGray shader sources.
__device__ __forceinline__ float3 operator+(const float3 a, const float3 b) {
    return make_float3(a.x + b.x, a.y + b.y, a.z + b.z);
}

__device__ __forceinline__ float3 operator*(const float3 a, const float b) {
    return make_float3(a.x * b, a.y * b, a.z * b);
}
