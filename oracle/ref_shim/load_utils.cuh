// Stand-in for the reference's absent load_utils.cuh (included by its UltraGauss and
// UltraGray sources). Defines the one loader the UltraGray shader calls: xyz(float4).
// Used solely to compile the reference into oracle/_ref.
#pragma once
#include <cuda_runtime.h>

__device__ __forceinline__ float3 xyz(const float4 v) { return make_float3(v.x, v.y, v.z); }
