// Shared device/host helpers for the us3d_b200 library (sm_100a).
//
// Every C-ABI entry point returns an `int` status (US3D_OK etc.) and records a message
// retrievable through us3d_last_error(). No entry point synchronises the stream it is
// given unless its documentation says so; all launches go to the caller's stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/us3d_b200.h"

namespace us3d {

// Thread-local last-error message (defined in status.cu).
void set_error(const char* fmt, ...);

// Benchmark instrumentation (status.cu): a process-wide count of this library's kernel
// launches, and optional CUDA-event brackets around one named stage.
void count_launches(int n);
int prof_begin(const char* stage, cudaStream_t stream);
void prof_end(int slot, cudaStream_t stream);

#define US3D_CHECK_ARG(cond, ...)                 \
    do {                                          \
        if (!(cond)) {                            \
            ::us3d::set_error(__VA_ARGS__);       \
            return US3D_INVALID_ARG;              \
        }                                         \
    } while (0)

#define US3D_CHECK_LAUNCH(name)                                                        \
    do {                                                                               \
        cudaError_t _e = cudaGetLastError();                                           \
        if (_e != cudaSuccess) {                                                       \
            ::us3d::set_error("%s launch failed: %s", name, cudaGetErrorString(_e));   \
            return US3D_CUDA_ERROR;                                                    \
        }                                                                              \
    } while (0)

#define US3D_CHECK_CUDA(call)                                                          \
    do {                                                                               \
        cudaError_t _e = (call);                                                       \
        if (_e != cudaSuccess) {                                                       \
            ::us3d::set_error("%s failed: %s", #call, cudaGetErrorString(_e));         \
            return US3D_CUDA_ERROR;                                                    \
        }                                                                              \
    } while (0)

static inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Bump allocator that carves one caller-provided workspace into 256-byte aligned slices.
struct Carver {
    char* base;
    size_t off;
    explicit Carver(void* b) : base(static_cast<char*>(b)), off(0) {}
    template <typename T>
    T* take(size_t count) {
        off = align_up(off, 256);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
};

// ---- small float3 helpers (device) ----
__device__ __forceinline__ float3 f3_sub(const float3 a, const float3 b) {
    return make_float3(a.x - b.x, a.y - b.y, a.z - b.z);
}
// Dot product in the operand order x, y, z (the order every parity-critical window test uses).
__device__ __forceinline__ float f3_dot(const float3 a, const float3 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}

// float -> uint32 conversion with the saturating semantics of the PTX cvt.rzi.u32.f32
// instruction (negative and NaN -> 0, too large -> 0xFFFFFFFF). Written out so the host
// oracle can state the same rule.
__device__ __forceinline__ uint32_t f32_to_u32_sat(float x) { return (uint32_t)x; }

// Logistic function of a raw (logit) parameter, computed in double and rounded once, so that it
// does not depend on the fast single-precision exponential this library is compiled with.
__device__ __forceinline__ float sigmoid_logit(float x) { return (float)(1.0 / (1.0 + exp(-(double)x))); }

}  // namespace us3d
