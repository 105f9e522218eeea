// Slice-adapted 3DGS projection: 3D Gaussians -> kept 2D splats for the bounded additive
// splat, fused into one pass per Gaussian plus an order-preserving compaction, and its
// hand-written vector-Jacobian product.
//
// Reference behaviour restated here (KevinWCCC/ultrasound-3d-reconstruction,
// baselines/slice_adapted_3dgs/render.py): view transform of the means (:67-68, :132-135),
// camera-space covariance R diag(s^2) R^T seen through the view rotation (:157-163), slice
// distance and thickness sigma (:69-74), cull |z| <= cull_std sigma thickness_scale (:76),
// 2x2 inverse with the clamped determinant (:89-94), weights o exp(-z^2 / 2 sigma^2) /
// sqrt(det) (:96-98); the kept subset in index order (:81-87). The reference runs this as
// about thirty PyTorch operations and boolean-mask gathers per frame.
#include "us3d_common.cuh"
#include "scan.cuh"

namespace us3d {
namespace sap {

struct ProjParams {
    const float* means;
    const float* scales;
    const float* quats;
    const float* opac;
    const float* colors;
    const float* view;  // 4x4 row-major, points as row vectors: cam = [p, 1] @ view
    float focal_depth, thickness, cull_std, thickness_scale, min_cov;
    int normalize;
};

struct Proj {
    float cam[3];
    float C[3][3];  // camera-space covariance
    float c2[2][2]; // + min_cov I
    float R[3][3], qn[4], qlen, s[3];
    float rel_z, var_z_raw, sigma_z, det_raw, det, E, w;
    bool keep;
};

__device__ __forceinline__ void project(const ProjParams& p, int g, Proj& o) {
    const float* V = p.view;
    const float px = p.means[3 * g], py = p.means[3 * g + 1], pz = p.means[3 * g + 2];
#pragma unroll
    for (int j = 0; j < 3; ++j) o.cam[j] = px * V[j] + py * V[4 + j] + pz * V[8 + j] + V[12 + j];
    o.rel_z = o.cam[2] - p.focal_depth;
    // normalised quaternion (w, x, y, z), q / max(|q|, 1e-8)
    const float q0 = p.quats[4 * g], q1 = p.quats[4 * g + 1], q2 = p.quats[4 * g + 2], q3 = p.quats[4 * g + 3];
    o.qlen = sqrtf(q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3);
    const float inv = 1.0f / fmaxf(o.qlen, 1e-8f);
    const float w = q0 * inv, x = q1 * inv, y = q2 * inv, z = q3 * inv;
    o.qn[0] = w; o.qn[1] = x; o.qn[2] = y; o.qn[3] = z;
    o.R[0][0] = 1 - 2 * (y * y + z * z); o.R[0][1] = 2 * (x * y - z * w); o.R[0][2] = 2 * (x * z + y * w);
    o.R[1][0] = 2 * (x * y + z * w); o.R[1][1] = 1 - 2 * (x * x + z * z); o.R[1][2] = 2 * (y * z - x * w);
    o.R[2][0] = 2 * (x * z - y * w); o.R[2][1] = 2 * (y * z + x * w); o.R[2][2] = 1 - 2 * (x * x + y * y);
#pragma unroll
    for (int k = 0; k < 3; ++k) o.s[k] = p.scales[3 * g + k];
    // Sigma_world = R diag(s^2) R^T ; C = r_wc^T Sigma_world r_wc with r_wc = view[:3,:3]
    float S[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            S[i][j] = o.R[i][0] * (o.s[0] * o.s[0]) * o.R[j][0] + o.R[i][1] * (o.s[1] * o.s[1]) * o.R[j][1] +
                      o.R[i][2] * (o.s[2] * o.s[2]) * o.R[j][2];
    float SV[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int b = 0; b < 3; ++b) SV[i][b] = S[i][0] * V[b] + S[i][1] * V[4 + b] + S[i][2] * V[8 + b];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) o.C[a][b] = V[a] * SV[0][b] + V[4 + a] * SV[1][b] + V[8 + a] * SV[2][b];
    o.c2[0][0] = o.C[0][0] + p.min_cov;
    o.c2[0][1] = o.C[0][1];
    o.c2[1][0] = o.C[1][0];
    o.c2[1][1] = o.C[1][1] + p.min_cov;
    o.var_z_raw = o.C[2][2];
    const float var_z = fmaxf(o.var_z_raw, p.min_cov);
    o.sigma_z = sqrtf(var_z + p.thickness * p.thickness);
    o.keep = fabsf(o.rel_z) <= p.cull_std * o.sigma_z * p.thickness_scale;
    o.det_raw = o.c2[0][0] * o.c2[1][1] - o.c2[0][1] * o.c2[1][0];
    o.det = fmaxf(o.det_raw, p.min_cov);
    const float u = o.rel_z / fmaxf(o.sigma_z, 1e-6f);
    o.E = __expf(-0.5f * (u * u));
    o.w = p.opac[g] * o.E;
    if (p.normalize) o.w = o.w / sqrtf(o.det);
}

__global__ void __launch_bounds__(256) flags_kernel(ProjParams p, int G, int* __restrict__ flags) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    Proj o;
    project(p, g, o);
    flags[g] = o.keep ? 1 : 0;
}

__global__ void __launch_bounds__(256)
compact_kernel(ProjParams p, int G, const int* __restrict__ flags, const int* __restrict__ offsets,
               float* __restrict__ means2d, float* __restrict__ inv2d, float* __restrict__ weights,
               float* __restrict__ colors, int* __restrict__ keep_idx, uint8_t* __restrict__ keep_mask) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    if (keep_mask) keep_mask[g] = (uint8_t)flags[g];
    if (!flags[g]) return;
    Proj o;
    project(p, g, o);
    const int i = offsets[g];
    means2d[2 * i] = o.cam[0];
    means2d[2 * i + 1] = o.cam[1];
    inv2d[4 * i] = o.c2[1][1] / o.det;
    inv2d[4 * i + 1] = -o.c2[0][1] / o.det;
    inv2d[4 * i + 2] = -o.c2[1][0] / o.det;
    inv2d[4 * i + 3] = o.c2[0][0] / o.det;
    weights[i] = o.w;
    colors[3 * i] = p.colors[3 * g];
    colors[3 * i + 1] = p.colors[3 * g + 1];
    colors[3 * i + 2] = p.colors[3 * g + 2];
    keep_idx[i] = g;
}

__global__ void zero_kernel(int G, float* __restrict__ dm, float* __restrict__ ds, float* __restrict__ dq,
                            float* __restrict__ dop, float* __restrict__ dc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dm[3 * g + k] = 0.f;
        ds[3 * g + k] = 0.f;
        dc[3 * g + k] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) dq[4 * g + k] = 0.f;
    dop[g] = 0.f;
}

// Vector-Jacobian product of the projection for each kept Gaussian (clamps pass gradient
// where their input is at or above the bound, as torch.clamp does).
__global__ void __launch_bounds__(256)
project_backward_kernel(ProjParams p, int N, const int* __restrict__ keep_idx, const float* __restrict__ d_means2d,
                        const float* __restrict__ d_inv2d, const float* __restrict__ d_weights,
                        const float* __restrict__ d_colors_kept, float* __restrict__ dm, float* __restrict__ ds,
                        float* __restrict__ dq, float* __restrict__ dop, float* __restrict__ dc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int g = keep_idx[i];
    Proj o;
    project(p, g, o);
    const float* V = p.view;
#pragma unroll
    for (int k = 0; k < 3; ++k) dc[3 * g + k] = d_colors_kept[3 * i + k];
    const float dw = d_weights[i];
    const float szc = fmaxf(o.sigma_z, 1e-6f);
    const float u = o.rel_z / szc;
    const float nd = p.normalize ? 1.0f / sqrtf(o.det) : 1.0f;
    dop[g] = dw * o.E * nd;
    const float du = -dw * o.w * u;
    float d_relz = du / szc;
    const float d_szc = -du * u / szc;
    const float d_sigma = (o.sigma_z >= 1e-6f) ? d_szc : 0.f;
    float d_det = p.normalize ? -0.5f * dw * o.w / o.det : 0.f;
    // inverse
    const float di00 = d_inv2d[4 * i], di01 = d_inv2d[4 * i + 1], di10 = d_inv2d[4 * i + 2], di11 = d_inv2d[4 * i + 3];
    const float inv_det = 1.0f / o.det;
    float dc00 = di11 * inv_det, dc11 = di00 * inv_det, dc01 = -di01 * inv_det, dc10 = -di10 * inv_det;
    d_det -= (di00 * o.c2[1][1] - di01 * o.c2[0][1] - di10 * o.c2[1][0] + di11 * o.c2[0][0]) * inv_det * inv_det;
    if (o.det_raw >= p.min_cov) {
        dc00 += d_det * o.c2[1][1];
        dc11 += d_det * o.c2[0][0];
        dc01 -= d_det * o.c2[1][0];
        dc10 -= d_det * o.c2[0][1];
    }
    float dC[3][3] = {{dc00, dc01, 0.f}, {dc10, dc11, 0.f}, {0.f, 0.f, 0.f}};
    const float dvar = d_sigma * 0.5f / o.sigma_z;
    if (o.var_z_raw >= p.min_cov) dC[2][2] = dvar;
    // camera position: means2d = cam[0:2], rel_z = cam[2] - focal
    const float dcam[3] = {d_means2d[2 * i], d_means2d[2 * i + 1], d_relz};
#pragma unroll
    for (int k = 0; k < 3; ++k) dm[3 * g + k] = V[4 * k] * dcam[0] + V[4 * k + 1] * dcam[1] + V[4 * k + 2] * dcam[2];
    // C = r^T S r  ->  dS = r dC r^T  (r[i][a] = V[4 i + a])
    float t[3][3], dS[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int j = 0; j < 3; ++j) t[a][j] = dC[a][0] * V[4 * j] + dC[a][1] * V[4 * j + 1] + dC[a][2] * V[4 * j + 2];
#pragma unroll
    for (int ii = 0; ii < 3; ++ii)
#pragma unroll
        for (int j = 0; j < 3; ++j) dS[ii][j] = V[4 * ii] * t[0][j] + V[4 * ii + 1] * t[1][j] + V[4 * ii + 2] * t[2][j];
    // S = R D R^T, D = diag(s^2)
    const float Dd[3] = {o.s[0] * o.s[0], o.s[1] * o.s[1], o.s[2] * o.s[2]};
    float dR[3][3];
#pragma unroll
    for (int ii = 0; ii < 3; ++ii)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float a = 0.f;
#pragma unroll
            for (int j = 0; j < 3; ++j) a += (dS[ii][j] + dS[j][ii]) * o.R[j][k];
            dR[ii][k] = a * Dd[k];
        }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float a = 0.f;
#pragma unroll
        for (int ii = 0; ii < 3; ++ii)
#pragma unroll
            for (int j = 0; j < 3; ++j) a += o.R[ii][k] * dS[ii][j] * o.R[j][k];
        ds[3 * g + k] = 2.f * o.s[k] * a;
    }
    // R(qn) -> qn
    const float w = o.qn[0], x = o.qn[1], y = o.qn[2], z = o.qn[3];
    const float gw = 2.f * (-z * dR[0][1] + y * dR[0][2] + z * dR[1][0] - x * dR[1][2] - y * dR[2][0] + x * dR[2][1]);
    const float gx = 2.f * (y * dR[0][1] + z * dR[0][2] + y * dR[1][0] - 2.f * x * dR[1][1] - w * dR[1][2] + z * dR[2][0] +
                            w * dR[2][1] - 2.f * x * dR[2][2]);
    const float gy = 2.f * (-2.f * y * dR[0][0] + x * dR[0][1] + w * dR[0][2] + x * dR[1][0] + z * dR[1][2] -
                            w * dR[2][0] + z * dR[2][1] - 2.f * y * dR[2][2]);
    const float gz = 2.f * (-2.f * z * dR[0][0] - w * dR[0][1] + x * dR[0][2] + w * dR[1][0] - 2.f * z * dR[1][1] +
                            y * dR[1][2] + x * dR[2][0] + y * dR[2][1]);
    // qn = q / max(|q|, eps)
    if (o.qlen > 1e-8f) {
        const float dot = w * gw + x * gx + y * gy + z * gz;
        const float il = 1.0f / o.qlen;
        dq[4 * g] = (gw - w * dot) * il;
        dq[4 * g + 1] = (gx - x * dot) * il;
        dq[4 * g + 2] = (gy - y * dot) * il;
        dq[4 * g + 3] = (gz - z * dot) * il;
    } else {
        dq[4 * g] = gw * 1e8f;
        dq[4 * g + 1] = gx * 1e8f;
        dq[4 * g + 2] = gy * 1e8f;
        dq[4 * g + 3] = gz * 1e8f;
    }
}

}  // namespace sap
}  // namespace us3d

using namespace us3d;
using namespace us3d::sap;

struct SapWorkspace {
    long long* total;
    int* flags;
    int* offsets;
    long long* bs;
    size_t bytes;
};

static SapWorkspace sap_carve(void* base, int64_t G) {
    Carver c(base);
    SapWorkspace w;
    w.total = c.take<long long>(2);
    w.flags = c.take<int>((size_t)G);
    w.offsets = c.take<int>((size_t)G + 1);
    w.bs = c.take<long long>((size_t)scan_num_blocks(G) + 1);
    w.bytes = align_up(c.off, 256);
    return w;
}

static ProjParams sap_params(const float* means, const float* scales, const float* quats, const float* opac,
                             const float* colors, const float* view, float focal_depth, float thickness,
                             float cull_std, float thickness_scale, float min_cov, int32_t normalize) {
    ProjParams p;
    p.means = means; p.scales = scales; p.quats = quats; p.opac = opac; p.colors = colors; p.view = view;
    p.focal_depth = focal_depth; p.thickness = thickness; p.cull_std = cull_std; p.thickness_scale = thickness_scale;
    p.min_cov = min_cov; p.normalize = normalize ? 1 : 0;
    return p;
}

extern "C" size_t us3d_sa_project_workspace_bytes(int64_t n_gauss) {
    if (n_gauss < 0) return 0;
    return sap_carve(nullptr, n_gauss).bytes;
}

extern "C" int us3d_sa_project(void* workspace, size_t workspace_bytes, int64_t n_gauss, const float* means,
                               const float* scales, const float* quats, const float* opacities, const float* colors,
                               const float* viewmatrix, float focal_depth, float slice_thickness, float cull_std,
                               float thickness_scale, float min_covariance, int32_t normalize_by_footprint,
                               float* out_means2d, float* out_inv2d, float* out_weights, float* out_colors,
                               int32_t* out_keep_idx, uint8_t* out_keep_mask, int64_t* out_kept, void* stream_) {
    US3D_CHECK_ARG(n_gauss >= 0 && n_gauss <= 0x7fffffffLL, "n_gauss out of range");
    US3D_CHECK_ARG(workspace && viewmatrix, "NULL pointer argument");
    US3D_CHECK_ARG(n_gauss == 0 || (means && scales && quats && opacities && colors && out_means2d && out_inv2d &&
                                    out_weights && out_colors && out_keep_idx),
                   "NULL Gaussian pointer");
    const SapWorkspace w = sap_carve(workspace, n_gauss);
    US3D_CHECK_ARG(workspace_bytes >= w.bytes, "workspace too small");
    cudaStream_t stream = (cudaStream_t)stream_;
    const ProjParams p = sap_params(means, scales, quats, opacities, colors, viewmatrix, focal_depth, slice_thickness,
                                    cull_std, thickness_scale, min_covariance, normalize_by_footprint);
    const unsigned gb = (unsigned)((n_gauss + 255) / 256);
    if (n_gauss > 0) flags_kernel<<<gb, 256, 0, stream>>>(p, (int)n_gauss, w.flags);
    US3D_CHECK_CUDA(exclusive_scan(w.flags, n_gauss, w.offsets, w.bs, w.total, stream));
    if (n_gauss > 0)
        compact_kernel<<<gb, 256, 0, stream>>>(p, (int)n_gauss, w.flags, w.offsets, out_means2d, out_inv2d,
                                               out_weights, out_colors, out_keep_idx, out_keep_mask);
    US3D_CHECK_LAUNCH("sa project");
    count_launches(3 + 2 * (n_gauss > 0));
    if (out_kept) {
        long long k = 0;
        US3D_CHECK_CUDA(cudaMemcpyAsync(&k, w.total, sizeof(k), cudaMemcpyDeviceToHost, stream));
        US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
        *out_kept = k;
    }
    return US3D_OK;
}

extern "C" int us3d_sa_project_backward(int64_t n_gauss, int64_t n_kept, const int32_t* keep_idx, const float* means,
                                        const float* scales, const float* quats, const float* opacities,
                                        const float* viewmatrix, float focal_depth, float slice_thickness,
                                        float cull_std, float thickness_scale, float min_covariance,
                                        int32_t normalize_by_footprint, const float* d_means2d, const float* d_inv2d,
                                        const float* d_weights, const float* d_colors_kept, float* d_means,
                                        float* d_scales, float* d_quats, float* d_opacities, float* d_colors,
                                        void* stream_) {
    US3D_CHECK_ARG(n_gauss >= 0 && n_kept >= 0 && n_kept <= n_gauss && n_gauss <= 0x7fffffffLL, "bad sizes");
    US3D_CHECK_ARG(n_gauss == 0 || (means && scales && quats && opacities && viewmatrix && d_means && d_scales &&
                                    d_quats && d_opacities && d_colors),
                   "NULL pointer argument");
    US3D_CHECK_ARG(n_kept == 0 || (keep_idx && d_means2d && d_inv2d && d_weights && d_colors_kept),
                   "NULL gradient pointer");
    cudaStream_t stream = (cudaStream_t)stream_;
    const ProjParams p = sap_params(means, scales, quats, opacities, nullptr, viewmatrix, focal_depth, slice_thickness,
                                    cull_std, thickness_scale, min_covariance, normalize_by_footprint);
    if (n_gauss > 0)
        zero_kernel<<<(unsigned)((n_gauss + 255) / 256), 256, 0, stream>>>((int)n_gauss, d_means, d_scales, d_quats,
                                                                           d_opacities, d_colors);
    if (n_kept > 0)
        project_backward_kernel<<<(unsigned)((n_kept + 255) / 256), 256, 0, stream>>>(
            p, (int)n_kept, keep_idx, d_means2d, d_inv2d, d_weights, d_colors_kept, d_means, d_scales, d_quats,
            d_opacities, d_colors);
    US3D_CHECK_LAUNCH("sa project backward");
    count_launches((n_gauss > 0) + (n_kept > 0));
    return US3D_OK;
}
