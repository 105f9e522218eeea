// Stand-in for the reference's absent covariance.cuh (included by its UltraGray shader,
// ops/ultragray_renderer/src/shader/{forward,backward}.cu:1). The four functions the shader
// calls are defined here from the mathematics their call sites imply; the reference's own
// versions are not available, so these pieces are not pinned to the reference:
//   compute_rot_from_quat        R (row-major) of the normalised (w,x,y,z) quaternion stored
//                                in (q.x, q.y, q.z, q.w); columns are the Gaussian's axes, as
//                                include/shader/shared.cuh:38-47 uses R^T (x - mu).
//   compute_cov3d_from_scale_rot the precision R diag(1/s^2) R^T (its result is used as
//                                SigmaInv by compute_gaussian_weight).
//   transform_grads_sigma_to_R_S adds dL/dR = (G + G^T) R D and dL/ds_k = -2 (R^T G R)_kk / s_k^3
//                                for G = dL/dSigmaInv, D = diag(1/s^2).
//   transform_grads_R_to_Quat    dL/dq through R(q/|q|), written (not accumulated).
// Used solely to compile the reference into oracle/_ref.
#pragma once
#include <cuda_runtime.h>

__device__ __forceinline__ void compute_rot_from_quat(const float4 q, float* R) {
    const float n = rsqrtf(fmaxf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w, 1e-12f));
    const float w = q.x * n, x = q.y * n, y = q.z * n, z = q.w * n;
    R[0] = 1.f - 2.f * (y * y + z * z);
    R[1] = 2.f * (x * y - w * z);
    R[2] = 2.f * (x * z + w * y);
    R[3] = 2.f * (x * y + w * z);
    R[4] = 1.f - 2.f * (x * x + z * z);
    R[5] = 2.f * (y * z - w * x);
    R[6] = 2.f * (x * z - w * y);
    R[7] = 2.f * (y * z + w * x);
    R[8] = 1.f - 2.f * (x * x + y * y);
}

__device__ __forceinline__ void compute_cov3d_from_scale_rot(const float3 s, const float* R, float* P) {
    const float d0 = 1.f / (s.x * s.x), d1 = 1.f / (s.y * s.y), d2 = 1.f / (s.z * s.z);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            P[r * 3 + c] = R[r * 3 + 0] * d0 * R[c * 3 + 0] + R[r * 3 + 1] * d1 * R[c * 3 + 1] +
                           R[r * 3 + 2] * d2 * R[c * 3 + 2];
}

__device__ __forceinline__ void transform_grads_sigma_to_R_S(const float3 s, const float* R, const float* G,
                                                             float* dL_dR, float3& dL_dS) {
    const float d[3] = {1.f / (s.x * s.x), 1.f / (s.y * s.y), 1.f / (s.z * s.z)};
    float Gs[9];
    for (int i = 0; i < 9; ++i) Gs[i] = G[i] + G[(i % 3) * 3 + i / 3];
    for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k)
            dL_dR[r * 3 + k] += (Gs[r * 3 + 0] * R[0 * 3 + k] + Gs[r * 3 + 1] * R[1 * 3 + k] + Gs[r * 3 + 2] * R[2 * 3 + k]) * d[k];
    float acc[3];
    for (int k = 0; k < 3; ++k) {
        float a = 0.f;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) a += R[i * 3 + k] * G[i * 3 + j] * R[j * 3 + k];
        acc[k] = a;
    }
    dL_dS.x += -2.f * acc[0] * d[0] / s.x;
    dL_dS.y += -2.f * acc[1] * d[1] / s.y;
    dL_dS.z += -2.f * acc[2] * d[2] / s.z;
}

__device__ __forceinline__ void transform_grads_R_to_Quat(const float4 q, const float* g, float4& dq) {
    const float len = sqrtf(fmaxf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w, 1e-12f));
    const float n = 1.f / len;
    const float w = q.x * n, x = q.y * n, y = q.z * n, z = q.w * n;
    const float gw = 2.f * (-z * g[1] + y * g[2] + z * g[3] - x * g[5] - y * g[6] + x * g[7]);
    const float gx = 2.f * (y * g[1] + z * g[2] + y * g[3] - 2.f * x * g[4] - w * g[5] + z * g[6] + w * g[7] - 2.f * x * g[8]);
    const float gy = 2.f * (-2.f * y * g[0] + x * g[1] + w * g[2] + x * g[3] + z * g[5] - w * g[6] + z * g[7] - 2.f * y * g[8]);
    const float gz = 2.f * (-2.f * z * g[0] - w * g[1] + x * g[2] + w * g[3] - 2.f * z * g[4] + y * g[5] + x * g[6] + y * g[7]);
    const float dot = w * gw + x * gx + y * gy + z * gz;
    dq = make_float4((gw - w * dot) * n, (gx - x * dot) * n, (gy - y * dot) * n, (gz - z * dot) * n);
}
