// GaussianPile projected-slice ("us_focus") additive splatting: binning, forward, backward.
//
// Reference behaviour restated here (paths inside KevinWCCC/ultrasound-3d-reconstruction,
// ops/gaussianplie_renderer):
//   include/shader/us_focus_device.cuh:88-316     conditional footprint of a 3D Gaussian on
//                                                 the slice under an elevational beam PSF
//   include/shader/plane_cond2d_device.cuh:14-98  world covariance, probe-frame covariance
//   include/shader/shared.cuh:6-34                quaternion -> rotation, normalisation
//   src/mapper/core_tile.cu:25-234                tile rectangles, keys, ranges
//   src/shader/forward.cu:27-210                  per-tile additive forward
//   src/shader/us_focus.cu:129-803, 805-966       sufficient-statistics backward, per-Gaussian
//                                                 finalize with finite-difference shape grads
//
// B200 design: each Gaussian's footprint is computed once per call and cached (the reference
// recomputes it in the mapper, once per tile in the forward and again per tile in the
// backward); instances are bucketed per tile and ordered in shared memory like the UltraGauss
// path; the backward writes one partial record per (tile, Gaussian) instance and a
// per-Gaussian pass reduces them in a fixed order (the reference adds ~35 float atomics per
// instance into a per-Gaussian workspace) before the finalize.
//
// Arithmetic that decides integer outputs or that the forward image depends on (footprint,
// rectangles, window test, weights) uses the reference's operations in the reference's
// order, so that with the same --use_fast_math flags rectangles, sorted ids and tile ranges
// are bit-exact and images match to rounding of the summation.
#include <algorithm>

#include "us3d_common.cuh"
#include "scan.cuh"
#include "binning.cuh"

namespace us3d {
namespace gp {

// Slice grid pack layout (reference include/shader/slice_grid_geometry.cuh:4-16).
enum { SG_PROBE_TYPE = 0, SG_H = 1, SG_W = 2, SG_DELTA_LAT_MM = 3, SG_DELTA_AX_MM = 4, SG_NEAR_MM = 5,
       SG_LAT_COL_OFFSET = 6, SG_CENTER_LATERAL = 7 };
// us_focus parameter vector layout (reference include/shader/us_focus_device.cuh:9-23).
enum { UF_SIGMA_ELE_0 = 0, UF_SIGMA_ELE_1 = 1, UF_SIGMA_ELE_MIN = 2, UF_SIGMA_ELE_MAX = 3, UF_SIGMA_LAT_0 = 4,
       UF_SIGMA_LAT_1 = 5, UF_SIGMA_LAT_MIN = 6, UF_SIGMA_LAT_MAX = 7, UF_DET_GAMMA = 8, UF_DET_EPS = 9,
       UF_WEIGHT_MIN = 10, UF_USE_LATERAL_FOCUS = 11, UF_INFLATE_LAT_MM = 12, UF_INFLATE_AX_MM = 13 };

constexpr int FWD_BATCH = 256;
constexpr int PARTIAL_F4 = 5;  // per-instance partial record: 20 floats
constexpr float GRAD_CLAMP = 1e3f;

struct Workspace {
    long long* header;
    int4* rects;        // G
    uint32_t* dkey;     // G
    int* touched;       // G
    int* inst_offset;   // G + 1
    long long* bs_g;
    int* tile_count;    // T
    int* tile_start;    // T + 1
    int* tile_cursor;   // T
    long long* bs_t;
    float4* cand;       // G x 3: (base_weight, intensity, mu2_lat, mu2_ax) (inv00, inv01, inv11, r_lat) (r_ax, valid)
    float4* bfp;        // G x 4, what the backward needs of the forward's footprint:
                        // (mu2_lat, mu2_ax, r_lat (< 0: no footprint), r_ax) (inv00, inv01, inv11, bno_const)
                        // (s2_00, s2_01, s2_11, 1 / det_norm) (mu_ele, 1 / denom_ele, dsigma_ele/dax, sigma_ele)
    unsigned long long* keys;
    int* slot_inst;
    int* sorted_gid;
    int* sorted_inst;
    size_t bytes;
};

static Workspace carve(void* base, int64_t G, int64_t T, int64_t cap) {
    Carver c(base);
    Workspace w;
    w.header = c.take<long long>(H_WORDS);
    w.rects = c.take<int4>((size_t)G);
    w.dkey = c.take<uint32_t>((size_t)G);
    w.touched = c.take<int>((size_t)G);
    w.inst_offset = c.take<int>((size_t)G + 1);
    w.bs_g = c.take<long long>((size_t)scan_num_blocks(G) + 1);
    w.tile_count = c.take<int>((size_t)T);
    w.tile_start = c.take<int>((size_t)T + 1);
    w.tile_cursor = c.take<int>((size_t)T);
    w.bs_t = c.take<long long>((size_t)scan_num_blocks(T) + 1);
    w.cand = c.take<float4>((size_t)G * 3);
    w.bfp = c.take<float4>((size_t)G * 4);
    w.keys = c.take<unsigned long long>((size_t)cap);
    w.slot_inst = c.take<int>((size_t)cap);
    w.sorted_gid = c.take<int>((size_t)cap);
    w.sorted_inst = c.take<int>((size_t)cap);
    w.bytes = align_up(c.off, 256);
    return w;
}

// ---- geometry helpers (reference include/shader/shared.cuh:6-34) ----

__device__ __forceinline__ float3 normalize3(const float3 v) {
    const float n = sqrtf(fmaxf(1e-12f, f3_dot(v, v)));
    return make_float3(v.x / n, v.y / n, v.z / n);
}

// Probe axes are the normalised columns of the 4x4 pose, the origin its translation column.
struct Axes {
    float3 raw_lat, raw_ax, raw_ele, lat, ax, ele, origin;
};

__device__ __forceinline__ Axes axes_from_pose(const float* __restrict__ pose) {
    Axes a;
    a.raw_lat = make_float3(pose[0], pose[4], pose[8]);
    a.raw_ax = make_float3(pose[1], pose[5], pose[9]);
    a.raw_ele = make_float3(pose[2], pose[6], pose[10]);
    a.lat = normalize3(a.raw_lat);
    a.ax = normalize3(a.raw_ax);
    a.ele = normalize3(a.raw_ele);
    a.origin = make_float3(pose[3], pose[7], pose[11]);
    return a;
}

// Rotation from a (w, x, y, z) quaternion normalised with rsqrt.
__device__ __forceinline__ void quat_rot(const float q0, const float q1, const float q2, const float q3, float R[9]) {
    const float nq = rsqrtf(fmaxf(1e-12f, q0 * q0 + q1 * q1 + q2 * q2 + q3 * q3));
    const float w = q0 * nq, x = q1 * nq, y = q2 * nq, z = q3 * nq;
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xy = x * y, xz = x * z, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    R[0] = 1.f - 2.f * (yy + zz);
    R[1] = 2.f * (xy - wz);
    R[2] = 2.f * (xz + wy);
    R[3] = 2.f * (xy + wz);
    R[4] = 1.f - 2.f * (xx + zz);
    R[5] = 2.f * (yz - wx);
    R[6] = 2.f * (xz - wy);
    R[7] = 2.f * (yz + wx);
    R[8] = 1.f - 2.f * (xx + yy);
}

// Sigma_w = R diag(s^2) R^T (reference plane_cond2d_device.cuh:48-69).
__device__ __forceinline__ void sigma_world(float sx, float sy, float sz, const float R[9], float S[9]) {
    float M[9];
    M[0] = R[0] * sx * sx; M[1] = R[1] * sy * sy; M[2] = R[2] * sz * sz;
    M[3] = R[3] * sx * sx; M[4] = R[4] * sy * sy; M[5] = R[5] * sz * sz;
    M[6] = R[6] * sx * sx; M[7] = R[7] * sy * sy; M[8] = R[8] * sz * sz;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) S[i * 3 + j] = M[i * 3 + 0] * R[j] + M[i * 3 + 1] * R[3 + j] + M[i * 3 + 2] * R[6 + j];
}

// Sc = A^T Sigma_w A with A = [lat ax ele] (reference plane_cond2d_device.cuh:71-98).
__device__ __forceinline__ void sigma_probe(const float S[9], float3 a0, float3 a1, float3 a2, float Sc[9]) {
    const float3 c0 = make_float3(S[0] * a0.x + S[1] * a0.y + S[2] * a0.z, S[3] * a0.x + S[4] * a0.y + S[5] * a0.z,
                                  S[6] * a0.x + S[7] * a0.y + S[8] * a0.z);
    const float3 c1 = make_float3(S[0] * a1.x + S[1] * a1.y + S[2] * a1.z, S[3] * a1.x + S[4] * a1.y + S[5] * a1.z,
                                  S[6] * a1.x + S[7] * a1.y + S[8] * a1.z);
    const float3 c2 = make_float3(S[0] * a2.x + S[1] * a2.y + S[2] * a2.z, S[3] * a2.x + S[4] * a2.y + S[5] * a2.z,
                                  S[6] * a2.x + S[7] * a2.y + S[8] * a2.z);
    Sc[0] = a0.x * c0.x + a0.y * c0.y + a0.z * c0.z;
    Sc[1] = a0.x * c1.x + a0.y * c1.y + a0.z * c1.z;
    Sc[2] = a0.x * c2.x + a0.y * c2.y + a0.z * c2.z;
    Sc[3] = a1.x * c0.x + a1.y * c0.y + a1.z * c0.z;
    Sc[4] = a1.x * c1.x + a1.y * c1.y + a1.z * c1.z;
    Sc[5] = a1.x * c2.x + a1.y * c2.y + a1.z * c2.z;
    Sc[6] = a2.x * c0.x + a2.y * c0.y + a2.z * c0.z;
    Sc[7] = a2.x * c1.x + a2.y * c1.y + a2.z * c1.z;
    Sc[8] = a2.x * c2.x + a2.y * c2.y + a2.z * c2.z;
}

// Adjugate inverse of a 3x3 matrix; false unless det > 1e-12 and finite
// (reference us_focus_device.cuh:115-151).
__device__ __forceinline__ bool inv3(const float M[9], float Mi[9]) {
    const float a00 = M[0], a01 = M[1], a02 = M[2], a10 = M[3], a11 = M[4], a12 = M[5], a20 = M[6], a21 = M[7],
                a22 = M[8];
    const float c00 = a11 * a22 - a12 * a21;
    const float c01 = a02 * a21 - a01 * a22;
    const float c02 = a01 * a12 - a02 * a11;
    const float c10 = a12 * a20 - a10 * a22;
    const float c11 = a00 * a22 - a02 * a20;
    const float c12 = a02 * a10 - a00 * a12;
    const float c20 = a10 * a21 - a11 * a20;
    const float c21 = a01 * a20 - a00 * a21;
    const float c22 = a00 * a11 - a01 * a10;
    const float det = a00 * c00 + a01 * c10 + a02 * c20;
    if (!(det > 1e-12f) || !isfinite(det)) return false;
    const float id = 1.f / det;
    Mi[0] = c00 * id; Mi[1] = c01 * id; Mi[2] = c02 * id;
    Mi[3] = c10 * id; Mi[4] = c11 * id; Mi[5] = c12 * id;
    Mi[6] = c20 * id; Mi[7] = c21 * id; Mi[8] = c22 * id;
    return true;
}

__device__ __forceinline__ float det_norm_factor(float d, float gamma) {
    if (gamma == 0.f) return 1.f;
    if (fabsf(gamma - 0.25f) < 1e-7f) return 1.f / sqrtf(sqrtf(d));
    if (fabsf(gamma - 0.5f) < 1e-7f) return 1.f / sqrtf(d);
    if (fabsf(gamma - 1.f) < 1e-7f) return 1.f / d;
    return powf(d, -gamma);
}

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

struct Footprint {
    float mu2_lat, mu2_ax, s2_00, s2_01, s2_11, inv00, inv01, inv11, det2;
    float sigma_ele, sigma_lat, mu_lat, mu_ax, mu_ele, sc22;
    float Lc[9], Se[9];
    float r_lat, r_ax;
};

// Elevational-PSF conditional footprint (reference us_focus_device.cuh:179-316):
// Sc = A^T Sigma_w A + 1e-6 I, Lc = Sc^-1, Le = Lc + diag(lat focus, 0, 1/sigma_ele^2),
// Se = Le^-1, mu_e = Se Lc mu_c, Sigma_2 = Se[0:2, 0:2] (symmetrised), radii from it.
__device__ __forceinline__ bool footprint(const float m0, const float m1, const float m2, const float s0,
                                          const float s1, const float s2, const float q0, const float q1,
                                          const float q2, const float q3, const Axes& A, float near_mm, float k_sigma,
                                          const float* __restrict__ P, Footprint& F) {
    const float3 d = make_float3(m0 - A.origin.x, m1 - A.origin.y, m2 - A.origin.z);
    F.mu_lat = f3_dot(d, A.lat);
    F.mu_ax = f3_dot(d, A.ax);
    F.mu_ele = f3_dot(d, A.ele);
    float R[9];
    quat_rot(q0, q1, q2, q3, R);
    const float sx = fmaxf(s0, 1e-6f), sy = fmaxf(s1, 1e-6f), sz = fmaxf(s2, 1e-6f);
    float Sw[9], Sc[9];
    sigma_world(sx, sy, sz, R, Sw);
    sigma_probe(Sw, A.lat, A.ax, A.ele, Sc);
    Sc[0] += 1e-6f;
    Sc[4] += 1e-6f;
    Sc[8] += 1e-6f;
    if (!inv3(Sc, F.Lc)) return false;
    const float depth = fmaxf(F.mu_ax - near_mm, 0.f);
    F.sigma_ele = clampf(P[UF_SIGMA_ELE_0] + P[UF_SIGMA_ELE_1] * depth, P[UF_SIGMA_ELE_MIN], P[UF_SIGMA_ELE_MAX]);
    F.sigma_lat = clampf(P[UF_SIGMA_LAT_0] + P[UF_SIGMA_LAT_1] * depth, P[UF_SIGMA_LAT_MIN], P[UF_SIGMA_LAT_MAX]);
    float Le[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) Le[i] = F.Lc[i];
    if (P[UF_USE_LATERAL_FOCUS] != 0.f) Le[0] += 1.f / fmaxf(F.sigma_lat * F.sigma_lat, 1e-12f);
    Le[8] += 1.f / fmaxf(F.sigma_ele * F.sigma_ele, 1e-12f);
    if (!inv3(Le, F.Se)) return false;
    const float mc[3] = {F.mu_lat, F.mu_ax, F.mu_ele};
    const float t0 = F.Lc[0] * mc[0] + F.Lc[1] * mc[1] + F.Lc[2] * mc[2];
    const float t1 = F.Lc[3] * mc[0] + F.Lc[4] * mc[1] + F.Lc[5] * mc[2];
    const float t2 = F.Lc[6] * mc[0] + F.Lc[7] * mc[1] + F.Lc[8] * mc[2];
    F.mu2_lat = F.Se[0] * t0 + F.Se[1] * t1 + F.Se[2] * t2;
    F.mu2_ax = F.Se[3] * t0 + F.Se[4] * t1 + F.Se[5] * t2;
    const float il = fmaxf(P[UF_INFLATE_LAT_MM], 0.f), ia = fmaxf(P[UF_INFLATE_AX_MM], 0.f);
    F.s2_00 = F.Se[0] + il * il;
    F.s2_01 = 0.5f * (F.Se[1] + F.Se[3]);
    F.s2_11 = F.Se[4] + ia * ia;
    F.det2 = F.s2_00 * F.s2_11 - F.s2_01 * F.s2_01;
    if (!(F.det2 > P[UF_DET_EPS]) || !isfinite(F.det2)) return false;
    const float idet = 1.f / F.det2;
    F.inv00 = F.s2_11 * idet;
    F.inv01 = -F.s2_01 * idet;
    F.inv11 = F.s2_00 * idet;
    F.sc22 = Sc[8];
    const float cross = fabsf(F.s2_01);
    F.r_lat = k_sigma * sqrtf(fmaxf(F.s2_00 + cross, 1e-12f));
    F.r_ax = k_sigma * sqrtf(fmaxf(F.s2_11 + cross, 1e-12f));
    return true;
}

// ------------------------------------------------------------------------------------
// Binning
// ------------------------------------------------------------------------------------

__global__ void init_kernel(int64_t T, int* __restrict__ tile_count, int* __restrict__ tile_cursor,
                            long long* __restrict__ header, int64_t cap, int64_t G) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < H_WORDS) {
        long long v = 0;
        if (threadIdx.x == H_CAP) v = cap;
        if (threadIdx.x == H_G) v = G;
        if (threadIdx.x == H_T) v = T;
        header[threadIdx.x] = v;
    }
    if (t >= T) return;
    tile_count[t] = 0;
    tile_cursor[t] = 0;
}

// Footprint, tile rectangle, depth key and forward candidate of every Gaussian
// (reference src/mapper/core_tile.cu:25-174 and src/shader/forward.cu:27-86).
__global__ void __launch_bounds__(256)
preprocess_kernel(int64_t G, int H, int W, int tile, int tiles_x, int tiles_y, float lat_mm, float ax_mm,
                  float near_mm, float k_sigma, int sort_by_v, const float* __restrict__ means,
                  const float* __restrict__ scales, const float* __restrict__ quats, const float* __restrict__ opac,
                  const float* __restrict__ inten, const float* __restrict__ pose, const float* __restrict__ grid,
                  const float* __restrict__ params, int4* __restrict__ rects, uint32_t* __restrict__ dkey,
                  int* __restrict__ touched, int* __restrict__ tile_count, float4* __restrict__ cand,
                  float4* __restrict__ bfp) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const Axes A = axes_from_pose(pose);
    const float* m = means + 3 * g;
    const float* s = scales + 3 * g;
    const float* q = quats + 4 * g;
    Footprint F;
    rects[g] = make_int4(0, 0, 0, 0);
    touched[g] = 0;
    dkey[g] = 0;
    if (!footprint(m[0], m[1], m[2], s[0], s[1], s[2], q[0], q[1], q[2], q[3], A, near_mm, k_sigma, params, F)) return;
    const float u_pix = F.mu2_lat / lat_mm + grid[SG_LAT_COL_OFFSET];
    const float v_pix = (F.mu2_ax - near_mm) / ax_mm;
    const float r_lat_pix = fmaxf(1.0f, F.r_lat / fmaxf(1e-8f, lat_mm));
    const float r_ax_pix = fmaxf(1.0f, F.r_ax / fmaxf(1e-8f, ax_mm));
    const float ts = (float)tile;
    int x0 = (int)floorf((u_pix - r_lat_pix) / ts);
    int y0 = (int)floorf((v_pix - r_ax_pix) / ts);
    int x1 = (int)ceilf((u_pix + r_lat_pix) / ts);
    int y1 = (int)ceilf((v_pix + r_ax_pix) / ts);
    x0 = max(0, x0);
    y0 = max(0, y0);
    x1 = min(tiles_x, x1);
    y1 = min(tiles_y, y1);
    (void)H;
    (void)W;
    if (x0 >= x1 || y0 >= y1) return;
    rects[g] = make_int4(x0, y0, x1, y1);
    dkey[g] = sort_by_v ? f32_to_u32_sat((v_pix + 500.0f) * 1000.0f) : 0u;
    touched[g] = (x1 - x0) * (y1 - y0);
    (void)tile_count;  // counted per block by rect_count_kernel
    // Forward candidate, computed with the forward's own near plane (the grid pack's);
    // the mapper's footprint is reused when the two near planes agree.
    Footprint Ff = F;
    bool okf = true;
    if (grid[SG_NEAR_MM] != near_mm)
        okf = footprint(m[0], m[1], m[2], s[0], s[1], s[2], q[0], q[1], q[2], q[3], A, grid[SG_NEAR_MM], k_sigma,
                        params, Ff);
    float bw = 0.f;
    bool valid = okf;
    if (okf) {
        const float det_eps = params[UF_DET_EPS];
        const float denom_ele = fmaxf(Ff.sc22 + Ff.sigma_ele * Ff.sigma_ele + det_eps, 1e-12f);
        const float slice_response = expf(-0.5f * Ff.mu_ele * Ff.mu_ele / denom_ele);
        const float norm = det_norm_factor(Ff.det2 + det_eps, params[UF_DET_GAMMA]);
        bw = opac[g] * slice_response * norm;
        valid = isfinite(bw);
    }
    cand[3 * g + 0] = make_float4(bw, inten[g], Ff.mu2_lat, Ff.mu2_ax);
    cand[3 * g + 1] = make_float4(Ff.inv00, Ff.inv01, Ff.inv11, Ff.r_lat);
    cand[3 * g + 2] = make_float4(Ff.r_ax, valid ? 1.f : 0.f, 0.f, 0.f);
    // The backward's per-Gaussian factors (reference us_focus.cu:398-477), with the grid's near
    // plane as the backward uses it.
    {
        const float det_eps = params[UF_DET_EPS], det_gamma = params[UF_DET_GAMMA];
        const float near_b = grid[SG_NEAR_MM];
        const float denom_ele = fmaxf(Ff.sc22 + Ff.sigma_ele * Ff.sigma_ele + det_eps, 1e-12f);
        const float slice_response = expf(-0.5f * Ff.mu_ele * Ff.mu_ele / denom_ele);
        const float norm = det_norm_factor(Ff.det2 + det_eps, det_gamma);
        const float depth = fmaxf(Ff.mu_ax - near_b, 0.f);
        const float se_raw = params[UF_SIGMA_ELE_0] + params[UF_SIGMA_ELE_1] * depth;
        const float dse_dax = (Ff.mu_ax > near_b && se_raw > params[UF_SIGMA_ELE_MIN] &&
                               se_raw < params[UF_SIGMA_ELE_MAX]) ? params[UF_SIGMA_ELE_1] : 0.f;
        bfp[4 * g + 0] = make_float4(Ff.mu2_lat, Ff.mu2_ax, okf ? Ff.r_lat : -1.f, Ff.r_ax);
        bfp[4 * g + 1] = make_float4(Ff.inv00, Ff.inv01, Ff.inv11, slice_response * norm);
        bfp[4 * g + 2] = make_float4(Ff.s2_00, Ff.s2_01, Ff.s2_11, 1.f / fmaxf(Ff.det2 + det_eps, 1e-12f));
        bfp[4 * g + 3] = make_float4(Ff.mu_ele, 1.f / denom_ele, dse_dax, Ff.sigma_ele);
    }
}

__global__ void check_kernel(long long* __restrict__ header, int64_t cap) {
    const long long tg = header[H_SCAN_G], tt = header[H_SCAN_T];
    long long flags = header[H_FLAGS];
    if (tg != tt) flags |= FLAG_TABLE;
    if (tg > cap || tg > 0x7fffffffLL) flags |= FLAG_OVERFLOW;
    header[H_TOTAL] = tg;
    header[H_FLAGS] = flags;
}


// ------------------------------------------------------------------------------------
// Forward
// ------------------------------------------------------------------------------------

// One block per tile, or per 1/SPLIT of a tile, with PARTS threads per pixel (the block's
// pixels rounded up to whole warps, times PARTS); candidates of the tile list are staged in
// shared memory. The sum over a pixel's candidates is split by Gaussian index into four classes
// (g mod 4), each summed in list order, and the class sums are added as ((c0 + c1) + c2) + c3;
// thread part p of a pixel owns the classes congruent to p mod PARTS. The grouping depends on
// neither PARTS, SPLIT nor the tile size, so the image does not either (the reference sums the
// whole list in order, src/shader/forward.cu:88-210: the results agree up to rounding). SPLIT
// > 1 serves small frames: a 256x256 slice has 256 tiles, under two 1024-thread blocks per SM,
// while quarter tiles give 1024 blocks of 256 threads that the SMs can balance.
template <int PARTS, int SPLIT>
__global__ void forward_kernel(int H, int W, int tile, int tiles_x, const float* __restrict__ grid,
                               const float* __restrict__ params, const int* __restrict__ tile_start,
                               const int* __restrict__ sorted_gid, const long long* __restrict__ header,
                               const float4* __restrict__ cand, float* __restrict__ image) {
    constexpr int PER = 4 / PARTS;  // classes per thread
    __shared__ float4 sc0[FWD_BATCH], sc1[FWD_BATCH];
    __shared__ float2 sc2[FWD_BATCH];
    __shared__ unsigned char s_cls[FWD_BATCH];
    __shared__ float s_class_sum[4 * 1024 / PARTS];
    if (header[H_FLAGS] != 0) return;
    const int t = blockIdx.x / SPLIT, sub = blockIdx.x % SPLIT;
    const int tx = t % tiles_x, ty = t / tiles_x;
    // pixel slots per part (whole warps); with SPLIT > 1 the host guarantees tile^2 / SPLIT is
    // a multiple of 32, so the sub-blocks partition the tile
    const int npix = SPLIT == 1 ? (tile * tile + 31) / 32 * 32 : tile * tile / SPLIT;
    const int slot = threadIdx.x % npix + sub * npix, part = threadIdx.x / npix;
    const int lx = slot % tile, ly = slot / tile;
    const int x = tx * tile + lx, y = ty * tile + ly;
    // the extra slots of the last warp own no pixel
    const bool valid = slot < tile * tile && (x < W) && (y < H);
    const float weight_min = params[UF_WEIGHT_MIN];
    float xi_lat = 0.f, xi_ax = 0.f;
    if (valid) {
        xi_lat = (static_cast<float>(x) - grid[SG_LAT_COL_OFFSET]) * grid[SG_DELTA_LAT_MM];
        xi_ax = static_cast<float>(y) * grid[SG_DELTA_AX_MM] + grid[SG_NEAR_MM];
    }
    const int s0 = tile_start[t], n = tile_start[t + 1] - s0;
    float acc[PER];
#pragma unroll
    for (int c = 0; c < PER; ++c) acc[c] = 0.f;
    const int nthreads = blockDim.x;
    // The warp's pixel extent in mm: a candidate whose box misses it (with a margin for the
    // rounding of the per-pixel test) is skipped by the whole warp.
    const int lane = threadIdx.x & 31;
    float lat_lo = valid ? xi_lat : 3.0e38f, lat_hi = valid ? xi_lat : -3.0e38f;
    float ax_lo = valid ? xi_ax : 3.0e38f, ax_hi = valid ? xi_ax : -3.0e38f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lat_lo = fminf(lat_lo, __shfl_xor_sync(0xffffffffu, lat_lo, o));
        lat_hi = fmaxf(lat_hi, __shfl_xor_sync(0xffffffffu, lat_hi, o));
        ax_lo = fminf(ax_lo, __shfl_xor_sync(0xffffffffu, ax_lo, o));
        ax_hi = fmaxf(ax_hi, __shfl_xor_sync(0xffffffffu, ax_hi, o));
    }
    for (int b0 = 0; b0 < n; b0 += FWD_BATCH) {
        const int nb = min(FWD_BATCH, n - b0);
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += nthreads) {
            const int g = sorted_gid[s0 + b0 + j];
            sc0[j] = cand[3 * g];
            sc1[j] = cand[3 * g + 1];
            const float4 c2 = cand[3 * g + 2];
            sc2[j] = make_float2(c2.x, c2.y);
            s_cls[j] = (unsigned char)(g & 3);
        }
        __syncthreads();
        for (int jc = 0; jc < nb; jc += 32) {
            bool near = false;
            const int jl = jc + lane;
            if (jl < nb && (PARTS == 1 || (int)(s_cls[jl] % PARTS) == part)) {
                const float2 c2 = sc2[jl];
                const float4 c0 = sc0[jl];
                const float rl = sc1[jl].w;
                const float ml = 1e-5f * (fabsf(c0.z) + rl + fabsf(lat_lo) + fabsf(lat_hi)) + 1e-30f;
                const float ma = 1e-5f * (fabsf(c0.w) + c2.x + fabsf(ax_lo) + fabsf(ax_hi)) + 1e-30f;
                near = c2.y != 0.f && lat_hi >= c0.z - rl - ml && lat_lo <= c0.z + rl + ml &&
                       ax_hi >= c0.w - c2.x - ma && ax_lo <= c0.w + c2.x + ma;
            }
            unsigned bits = __ballot_sync(0xffffffffu, near);
            if (!valid) continue;
            while (bits != 0u) {
                const int j = jc + __ffs(bits) - 1;
                bits &= bits - 1u;
                const float2 c2 = sc2[j];
                const float4 c0 = sc0[j];
                const float4 c1 = sc1[j];
                if (fabsf(xi_lat - c0.z) > c1.w || fabsf(xi_ax - c0.w) > c2.x) continue;
                const float dlat = xi_lat - c0.z;
                const float dax = xi_ax - c0.w;
                const float qlat = c1.x * dlat + c1.y * dax;
                const float qax = c1.y * dlat + c1.z * dax;
                const float quad = dlat * qlat + dax * qax;
                if (!(quad >= 0.f) || !isfinite(quad)) continue;
                const float weight = c0.x * expf(-0.5f * quad);
                if (!isfinite(weight) || weight < weight_min) continue;
                const float v = c0.y * weight;
                if (PER == 1) {
                    acc[0] += v;
                } else {
                    const int k = s_cls[j] / PARTS;  // this thread's class index
#pragma unroll
                    for (int c = 0; c < PER; ++c)
                        if (c == k) acc[c] += v;
                }
            }
        }
    }
    // class c's sum sits in part c % PARTS, slot c / PARTS of its accumulators
    const int ls = slot - sub * npix;  // the slot within this block
#pragma unroll
    for (int c = 0; c < PER; ++c) s_class_sum[(c * PARTS + part) * npix + ls] = acc[c];
    __syncthreads();
    if (part != 0 || !valid) return;
    float total = s_class_sum[ls];
#pragma unroll
    for (int c = 1; c < 4; ++c) total += s_class_sum[c * npix + ls];
    image[y * W + x] = total;
}

// ------------------------------------------------------------------------------------
// Backward
// ------------------------------------------------------------------------------------

// Per-instance partial record (20 floats); only the sufficient statistics that can be
// non-zero for the additive us_focus footprint are kept (the reference's 35-float
// workspace carries structurally zero entries).
enum { P_MU_PROBE1 = 0, P_MU_PROBE2, P_SC22, P_MU_E0, P_MU_E1, P_SE00, P_SE01, P_SE11, P_OPACITY, P_INTENSITY,
       P_FP_MU2_LAT, P_FP_MU2_AX, P_FP_INV00, P_FP_INV01, P_FP_INV11, P_FP_DET2, P_FP_MU_ELE, P_FP_SC22,
       P_FP_SIGMA_ELE, P_COUNT };

// One warp per instance of the sorted instance list (tile by tile): the lanes share the
// pixels of the footprint's bounding box within the instance's tile and accumulate the
// per-pixel adjoint of the footprint (reference src/shader/us_focus.cu:398-477, 805-966); the
// 19 sums are then reduced over the warp in a fixed order. The footprints are the forward's
// (cached per Gaussian by the preprocess).
constexpr int BWD_WARPS = 8;  // warps per CTA

__global__ void __launch_bounds__(BWD_WARPS * 32, 4)
backward_inst_kernel(int T, int W, int tile, int tiles_x, const float* __restrict__ opac,
                     const float* __restrict__ inten, const float4* __restrict__ bfp,
                     const float* __restrict__ grid, const float* __restrict__ params,
                     const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                     const int* __restrict__ sorted_inst, const long long* __restrict__ header,
                     const float* __restrict__ grad_image, float* __restrict__ partial, int H) {
    if (header[H_FLAGS] != 0) return;
    const int lane = threadIdx.x & 31;
    const int64_t total = tile_start[T];
    const float det_gamma = params[UF_DET_GAMMA];
    const float weight_min = params[UF_WEIGHT_MIN];
    const float lat_delta = grid[SG_DELTA_LAT_MM], ax_delta = grid[SG_DELTA_AX_MM];
    const float col_off = grid[SG_LAT_COL_OFFSET], near_mm = grid[SG_NEAR_MM];
    // Each warp owns a contiguous run of instances, so the instance's tile (the last t with
    // tile_start[t] <= k; empty tiles share a start) is found by one binary search per warp and
    // then followed forward as k advances.
    const int64_t n_warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t chunk = (total + n_warps - 1) / n_warps;
    const int64_t k_begin = wid * chunk, k_end = min(total, k_begin + chunk);
    int t = 0;
    if (k_begin < k_end) {
        int lo = 0, hi = T;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (tile_start[mid] <= k_begin) lo = mid; else hi = mid;
        }
        t = lo;
    }
    for (int64_t k = k_begin; k < k_end; ++k) {
        while (t + 1 < T && tile_start[t + 1] <= k) ++t;
        const int tx = t % tiles_x, ty = t / tiles_x;
        const int x0 = tx * tile, y0 = ty * tile;
        const int x1 = min(W, (tx + 1) * tile), y1 = min(H, (ty + 1) * tile);
        const int g = sorted_gid[k];
        const float4 f0 = bfp[4 * (int64_t)g], f1 = bfp[4 * (int64_t)g + 1];
        const float4 f2 = bfp[4 * (int64_t)g + 2], f3 = bfp[4 * (int64_t)g + 3];
        const float mu2_lat = f0.x, mu2_ax = f0.y, r_lat = f0.z, r_ax = f0.w;
        const float inv00 = f1.x, inv01 = f1.y, inv11 = f1.z, bno_const = f1.w;
        const float s2_00 = f2.x, s2_01 = f2.y, s2_11 = f2.z, inv_det_norm = f2.w;
        const float mu_ele = f3.x, inv_de = f3.y, dse_dax = f3.z, sigma_ele = f3.w;
        // Every term of the per-instance partial is a fixed combination of nine sums over the
        // contributing pixels of ub = up * bno (bno = the weight without the opacity) times 1,
        // q_lat, q_ax, q_lat^2, q_lat q_ax, q_ax^2 (q = inv2 d) and dlat^2, dlat dax, dax^2: the
        // lanes accumulate those and the terms are formed once. The q-weighted sums are taken
        // per pixel, not expanded from moments of d: for an elongated footprint q nearly
        // cancels along the long axis, and the expansion inv00^2 S(dlat^2) + 2 inv00 inv01
        // S(dlat dax) + ... loses in fp32 the digits that the chain through Se and Lc (with
        // entries in the hundreds for such footprints) then amplifies.
        float m0 = 0.f, sl = 0.f, sa = 0.f, sll = 0.f, sla = 0.f, saa = 0.f, mxx = 0.f, mxy = 0.f, myy = 0.f;
        float o = 0.f, c = 0.f;
        if (r_lat >= 0.f) {
            const int cx0 = max(x0, (int)ceilf((mu2_lat - r_lat) / lat_delta + col_off));
            const int cx1 = min(x1, (int)floorf((mu2_lat + r_lat) / lat_delta + col_off) + 1);
            const int cy0 = max(y0, (int)ceilf((mu2_ax - r_ax - near_mm) / ax_delta));
            const int cy1 = min(y1, (int)floorf((mu2_ax + r_ax - near_mm) / ax_delta) + 1);
            const int bw = cx1 - cx0, npx = bw > 0 && cy1 > cy0 ? bw * (cy1 - cy0) : 0;
            o = opac[g];
            c = inten[g];
            // pixel pi = lane + 32 i of the box, row-major: (row, column) stepped without divisions
            int ry = bw > 0 ? lane / bw : 0, rx = lane - ry * bw;
            const int step_y = bw > 0 ? 32 / bw : 0, step_x = 32 - step_y * bw;
            for (int pi = lane; pi < npx; pi += 32) {
                const int x = cx0 + rx, y = cy0 + ry;
                rx += step_x;
                ry += step_y;
                if (rx >= bw) {
                    rx -= bw;
                    ++ry;
                }
                const float xi_ax = static_cast<float>(y) * ax_delta + near_mm;
                const float xi_lat = (static_cast<float>(x) - col_off) * lat_delta;
                if (fabsf(xi_lat - mu2_lat) > r_lat || fabsf(xi_ax - mu2_ax) > r_ax) continue;
                const float dlat = xi_lat - mu2_lat;
                const float dax = xi_ax - mu2_ax;
                const float qlat = inv00 * dlat + inv01 * dax;
                const float qax = inv01 * dlat + inv11 * dax;
                const float quad = dlat * qlat + dax * qax;
                if (!(quad >= 0.f) || !isfinite(quad)) continue;
                const float phi = expf(-0.5f * quad);
                const float bno = bno_const * phi;
                const float weight = o * bno;
                if (!isfinite(weight) || weight < weight_min) continue;
                const float ub = grad_image[y * W + x] * bno;
                const float ul = ub * qlat, ua = ub * qax;
                const float ux = ub * dlat, uy = ub * dax;
                m0 += ub;
                sl += ul;
                sa += ua;
                sll += ul * qlat;
                sla += ul * qax;
                saa += ua * qax;
                mxx += ux * dlat;
                mxy += ux * dax;
                myy += uy * dax;
            }
        }
        // Transposed warp reduction of the nine sums (padded to 16): each exchange halves the
        // values a lane carries, so after four exchanges lanes 2j and 2j + 1 hold partial sums
        // of value j over 16 lanes, the fifth completes them, and every lane then reads the
        // nine totals from lanes 0, 2, ..., 16 (25 shuffles instead of 45; fixed order).
        {
            const unsigned FULL = 0xffffffffu;
            const float v[16] = {m0, sl, sa, sll, sla, saa, mxx, mxy, myy, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            float a8[8], b4[4], c2[2];
            const bool h16 = lane & 16, h8 = lane & 8, h4 = lane & 4, h2 = lane & 2;
#pragma unroll
            for (int i = 0; i < 8; ++i)
                a8[i] = (h16 ? v[8 + i] : v[i]) + __shfl_xor_sync(FULL, h16 ? v[i] : v[8 + i], 16);
#pragma unroll
            for (int i = 0; i < 4; ++i)
                b4[i] = (h8 ? a8[4 + i] : a8[i]) + __shfl_xor_sync(FULL, h8 ? a8[i] : a8[4 + i], 8);
#pragma unroll
            for (int i = 0; i < 2; ++i)
                c2[i] = (h4 ? b4[2 + i] : b4[i]) + __shfl_xor_sync(FULL, h4 ? b4[i] : b4[2 + i], 4);
            float d = (h2 ? c2[1] : c2[0]) + __shfl_xor_sync(FULL, h2 ? c2[0] : c2[1], 2);
            d += __shfl_xor_sync(FULL, d, 1);
            // value j = bits 4..1 of the lane (bit 4 selected the upper eight, bit 3 the upper four, ...)
            m0 = __shfl_sync(FULL, d, 0);
            sl = __shfl_sync(FULL, d, 2);
            sa = __shfl_sync(FULL, d, 4);
            sll = __shfl_sync(FULL, d, 6);
            sla = __shfl_sync(FULL, d, 8);
            saa = __shfl_sync(FULL, d, 10);
            mxx = __shfl_sync(FULL, d, 12);
            mxy = __shfl_sync(FULL, d, 14);
            myy = __shfl_sync(FULL, d, 16);
        }
        // The terms of reference us_focus.cu:398-477 (per pixel: up * weight, up c bno and
        // cm = up c weight times the footprint derivatives) from the six moments.
        float acc[P_COUNT];
        {
            const float co = c * o;  // cm = co * up * bno
            const float ql = sl, qa = sa, qll = sll, qla = sla, qaa = saa;
            const float ele2 = mu_ele * mu_ele * inv_de * inv_de;
            acc[P_INTENSITY] = o * m0;
            acc[P_OPACITY] = c * m0;
            acc[P_MU_E0] = co * ql;
            acc[P_MU_E1] = co * qa;
            acc[P_FP_MU2_LAT] = co * ql;
            acc[P_FP_MU2_AX] = co * qa;
            acc[P_FP_INV00] = co * (-0.5f * mxx);
            acc[P_FP_INV01] = co * (-mxy);
            acc[P_FP_INV11] = co * (-0.5f * myy);
            acc[P_FP_DET2] = co * m0 * (-det_gamma * inv_det_norm);
            acc[P_SE00] = co * (0.5f * qll - det_gamma * s2_11 * inv_det_norm * m0);
            acc[P_SE01] = 0.5f * co * (qla + 2.f * det_gamma * s2_01 * inv_det_norm * m0);
            acc[P_SE11] = co * (0.5f * qaa - det_gamma * s2_00 * inv_det_norm * m0);
            acc[P_MU_PROBE2] = co * m0 * (-mu_ele * inv_de);
            acc[P_SC22] = co * m0 * (0.5f * ele2);
            acc[P_MU_PROBE1] = co * m0 * (ele2 * dse_dax);
            acc[P_FP_MU_ELE] = co * m0 * (-mu_ele * inv_de);
            acc[P_FP_SC22] = co * m0 * (0.5f * ele2);
            acc[P_FP_SIGMA_ELE] = co * m0 * (ele2 * sigma_ele);
        }
        float4* out = reinterpret_cast<float4*>(partial) + (int64_t)PARTIAL_F4 * sorted_inst[k];
        if (lane == 0) {
            out[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
            out[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
            out[2] = make_float4(acc[8], acc[9], acc[10], acc[11]);
            out[3] = make_float4(acc[12], acc[13], acc[14], acc[15]);
            out[4] = make_float4(acc[16], acc[17], acc[18], 0.f);
        }
    }
}

__device__ __forceinline__ float sanitize(float g) {
    if (!isfinite(g)) return 0.f;
    if (fabsf(g) > GRAD_CLAMP) return copysignf(GRAD_CLAMP, g);
    return g;
}

// g_M -= Inv^T g_Inv Inv^T: adjoint of a 3x3 inverse (reference us_focus.cu:375-396).
__device__ __forceinline__ void inv3_bwd(const float Inv[9], const float gInv[9], float gM[9]) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float acc = 0.f;
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int b = 0; b < 3; ++b) acc += Inv[a * 3 + r] * gInv[a * 3 + b] * Inv[c * 3 + b];
            gM[r * 3 + c] -= acc;
        }
}

struct FpAdjoint {
    float mu2_lat, mu2_ax, inv00, inv01, inv11, det2, mu_ele, sc22, sigma_ele;
};

__device__ __forceinline__ float fp_dot(const Footprint& F, const FpAdjoint& a) {
    return a.mu2_lat * F.mu2_lat + a.mu2_ax * F.mu2_ax + a.inv00 * F.inv00 + a.inv01 * F.inv01 +
           a.inv11 * F.inv11 + a.det2 * F.det2 + a.mu_ele * F.mu_ele + a.sc22 * F.sc22 + a.sigma_ele * F.sigma_ele;
}

// Central difference (step eps) of the footprint/adjoint dot product with respect to one
// scale or quaternion component (reference us_focus.cu:313-373).
__device__ float shape_fd(const float* m, const float* s, const float* q, bool is_quat, int idx, float eps,
                          const Axes& A, float near_mm, float k_sigma, const float* P, const FpAdjoint& a) {
    float sp[3] = {s[0], s[1], s[2]}, sm[3] = {s[0], s[1], s[2]};
    float qp[4] = {q[0], q[1], q[2], q[3]}, qm[4] = {q[0], q[1], q[2], q[3]};
    if (is_quat) {
        qp[idx] += eps;
        qm[idx] -= eps;
    } else {
        sp[idx] += eps;
        sm[idx] -= eps;
    }
    Footprint Fp, Fm;
    const bool okp = footprint(m[0], m[1], m[2], sp[0], sp[1], sp[2], qp[0], qp[1], qp[2], qp[3], A, near_mm, k_sigma, P, Fp);
    const bool okm = footprint(m[0], m[1], m[2], sm[0], sm[1], sm[2], qm[0], qm[1], qm[2], qm[3], A, near_mm, k_sigma, P, Fm);
    const float lp = okp ? fp_dot(Fp, a) : 0.f;
    const float lm = okm ? fp_dot(Fm, a) : 0.f;
    return (lp - lm) / (2.f * eps);
}

// Exact shape gradient (analytic mode; the reference has only the central differences
// above): the adjoint of the probe-frame covariance, g_Sc (from the same chain through Se and
// Lc that gives the mean and pose gradients), is carried back through Sc = A^T Sigma_w A +
// 1e-6 I (Sc_ij = a_i^T Sigma_w a_j), the world covariance exactly as sigma_world forms it,
// Sigma_w = R D R with D = diag(s^2) (the reference's product, R from quat_rot), and
// R = rot(q / |q|):
//   G = dL/dSigma_w = sum_ij g_Sc[i][j] a_i a_j^T,
//   dL/ds_k = 2 s_k sum_ij G_ij R_ik R_kj (0 where the 1e-6 floor of the scale is active),
//   dL/dR = G R^T D + D R^T G, and dL/dq through the rotation of the normalised quaternion and
//   the normalisation.
__device__ void shape_analytic(const float* s, const float* q, const Axes& A, const float g_Sc[9], float d_s[3],
                               float d_q[4]) {
    const float3 ax[3] = {A.lat, A.ax, A.ele};
    float G[9];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float acc = 0.f;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const float ai = r == 0 ? ax[i].x : (r == 1 ? ax[i].y : ax[i].z);
                    const float aj = c == 0 ? ax[j].x : (c == 1 ? ax[j].y : ax[j].z);
                    acc += g_Sc[i * 3 + j] * ai * aj;
                }
            G[r * 3 + c] = acc;
        }
    float R[9];
    quat_rot(q[0], q[1], q[2], q[3], R);
    const float sv[3] = {s[0], s[1], s[2]};
    float D[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float sk = fmaxf(sv[k], 1e-6f);
        D[k] = sk * sk;
        float acc = 0.f;  // sum_ij G_ij R_ik R_kj
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) acc += G[i * 3 + j] * R[i * 3 + k] * R[k * 3 + j];
        d_s[k] = sv[k] > 1e-6f ? 2.f * sk * acc : 0.f;
    }
    float gR[9];  // dL/dR = G R^T D + D R^T G
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            float u = 0.f, v = 0.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                u += G[a * 3 + c] * R[b * 3 + c];
                v += R[c * 3 + a] * G[c * 3 + b];
            }
            gR[a * 3 + b] = u * D[b] + D[a] * v;
        }
    // R of the unit quaternion (w, x, y, z) as in quat_rot; derivative per component
    const float n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    const float nq = rsqrtf(fmaxf(1e-12f, n2));
    const float w = q[0] * nq, x = q[1] * nq, y = q[2] * nq, z = q[3] * nq;
    const float gw = 2.f * (-z * gR[1] + y * gR[2] + z * gR[3] - x * gR[5] - y * gR[6] + x * gR[7]);
    const float gx = 2.f * (y * gR[1] + z * gR[2] + y * gR[3] - 2.f * x * gR[4] - w * gR[5] + z * gR[6] + w * gR[7] -
                            2.f * x * gR[8]);
    const float gy = 2.f * (-2.f * y * gR[0] + x * gR[1] + w * gR[2] + x * gR[3] + z * gR[5] - w * gR[6] + z * gR[7] -
                            2.f * y * gR[8]);
    const float gz = 2.f * (-2.f * z * gR[0] - w * gR[1] + x * gR[2] + w * gR[3] - 2.f * z * gR[4] + y * gR[5] +
                            x * gR[6] + y * gR[7]);
    // through the normalisation u = q / |q| (no normalisation term where the 1e-12 floor is active)
    const float dot = (n2 > 1e-12f) ? (w * gw + x * gx + y * gy + z * gz) : 0.f;
    d_q[0] = nq * (gw - w * dot);
    d_q[1] = nq * (gx - x * dot);
    d_q[2] = nq * (gy - y * dot);
    d_q[3] = nq * (gz - z * dot);
}

__device__ __forceinline__ float3 normalize3_bwd(const float3 raw, const float3 n, const float3 g) {
    const float len = sqrtf(fmaxf(1e-12f, f3_dot(raw, raw)));
    const float il = 1.f / len;
    const float dn = f3_dot(n, g);
    return make_float3((g.x - n.x * dn) * il, (g.y - n.y * dn) * il, (g.z - n.z * dn) * il);
}

// Per-Gaussian sums of its instances' partial records, in instance order, written over its first
// instance's record: PARTIAL_F4 threads per Gaussian, thread f summing float4 column f, so that
// the threads of a Gaussian read each 80-byte record together and many Gaussians' loads are in
// flight (the sums are the ones a thread summing all columns would form).
constexpr int REDUCE_THREADS = 32 * PARTIAL_F4;  // 32 Gaussians per block
__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_partials_kernel(int64_t G, const int* __restrict__ inst_offset, const long long* __restrict__ header,
                       float4* __restrict__ partial) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g = t / PARTIAL_F4;
    const int f = (int)(t % PARTIAL_F4);
    if (g >= G || header[H_FLAGS] != 0) return;
    const int i0 = inst_offset[g], i1 = inst_offset[g + 1];
    if (i1 <= i0) return;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    int i = i0;
    for (; i + 4 <= i1; i += 4) {  // four instances' loads in flight
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = partial[(int64_t)PARTIAL_F4 * (i + u) + f];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            acc.x += v[u].x;
            acc.y += v[u].y;
            acc.z += v[u].z;
            acc.w += v[u].w;
        }
    }
    for (; i < i1; ++i) {
        const float4 v = partial[(int64_t)PARTIAL_F4 * i + f];
        acc.x += v.x;
        acc.y += v.y;
        acc.z += v.z;
        acc.w += v.w;
    }
    partial[(int64_t)PARTIAL_F4 * i0 + f] = acc;
}

// Per Gaussian: its instance partials summed by reduce_partials_kernel, then the chain rule
// through Se and Lc, finite-difference shape gradients, sanitising, and the pose contribution
// (reference us_focus.cu:479-803).
__global__ void __launch_bounds__(128)
finalize_kernel(int64_t G, float k_sigma, const int* __restrict__ inst_offset, const int4* __restrict__ rects,
                const float* __restrict__ means, const float* __restrict__ scales, const float* __restrict__ quats,
                const float* __restrict__ pose, const float* __restrict__ grid, const float* __restrict__ params,
                const long long* __restrict__ header, const float* __restrict__ partial, int pose_grad,
                int shape_analytic_mode, float* __restrict__ d_means, float* __restrict__ d_scales, float* __restrict__ d_quats,
                float* __restrict__ d_opac, float* __restrict__ d_inten, float* __restrict__ pose_partial) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    float* pp = pose_grad ? pose_partial + 12 * g : nullptr;
    if (pp) {
#pragma unroll
        for (int i = 0; i < 12; ++i) pp[i] = 0.f;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        d_means[3 * g + i] = 0.f;
        d_scales[3 * g + i] = 0.f;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) d_quats[4 * g + i] = 0.f;
    d_opac[g] = 0.f;
    d_inten[g] = 0.f;
    if (header[H_FLAGS] != 0) return;
    if ((int)(grid[SG_PROBE_TYPE] + 0.5f) != 0) return;  // linear probes only, as the reference
    const int4 rect = rects[g];
    if (rect.x >= rect.z || rect.y >= rect.w) return;
    const Axes A = axes_from_pose(pose);
    const float near_mm = grid[SG_NEAR_MM];
    const float* m = means + 3 * g;
    const float* s = scales + 3 * g;
    const float* q = quats + 4 * g;
    Footprint F;
    if (!footprint(m[0], m[1], m[2], s[0], s[1], s[2], q[0], q[1], q[2], q[3], A, near_mm, k_sigma, params, F)) return;

    float acc[P_COUNT];
#pragma unroll
    for (int i = 0; i < P_COUNT; ++i) acc[i] = 0.f;
    if (inst_offset[g + 1] > inst_offset[g]) {  // the sums reduce_partials_kernel left in the first record
        const float4* r = reinterpret_cast<const float4*>(partial) + (int64_t)PARTIAL_F4 * inst_offset[g];
        const float4 a = r[0], b = r[1], c = r[2], d = r[3], e = r[4];
        acc[0] = a.x; acc[1] = a.y; acc[2] = a.z; acc[3] = a.w;
        acc[4] = b.x; acc[5] = b.y; acc[6] = b.z; acc[7] = b.w;
        acc[8] = c.x; acc[9] = c.y; acc[10] = c.z; acc[11] = c.w;
        acc[12] = d.x; acc[13] = d.y; acc[14] = d.z; acc[15] = d.w;
        acc[16] = e.x; acc[17] = e.y; acc[18] = e.z;
    }

    const float depth = fmaxf(F.mu_ax - near_mm, 0.f);
    const bool depth_active = F.mu_ax > near_mm;
    const float se_raw = params[UF_SIGMA_ELE_0] + params[UF_SIGMA_ELE_1] * depth;
    const float sl_raw = params[UF_SIGMA_LAT_0] + params[UF_SIGMA_LAT_1] * depth;
    const bool use_lat = params[UF_USE_LATERAL_FOCUS] != 0.f;
    const float dse = (depth_active && se_raw > params[UF_SIGMA_ELE_MIN] && se_raw < params[UF_SIGMA_ELE_MAX])
                          ? params[UF_SIGMA_ELE_1] : 0.f;
    const float dsl = (use_lat && depth_active && sl_raw > params[UF_SIGMA_LAT_MIN] && sl_raw < params[UF_SIGMA_LAT_MAX])
                          ? params[UF_SIGMA_LAT_1] : 0.f;
    const float dlam_ele = -2.f * dse / fmaxf(F.sigma_ele * F.sigma_ele * F.sigma_ele, 1e-12f);
    const float dlam_lat = use_lat ? -2.f * dsl / fmaxf(F.sigma_lat * F.sigma_lat * F.sigma_lat, 1e-12f) : 0.f;

    const float mu_c[3] = {F.mu_lat, F.mu_ax, F.mu_ele};
    const float* Lc = F.Lc;
    const float* Se = F.Se;
    float g_mu_probe[3] = {0.f, acc[P_MU_PROBE1], acc[P_MU_PROBE2]};
    float g_Sc[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, acc[P_SC22]};
    const float g_mu_e[3] = {acc[P_MU_E0], acc[P_MU_E1], 0.f};
    float g_Se[9] = {acc[P_SE00], acc[P_SE01], 0.f, acc[P_SE01], acc[P_SE11], 0.f, 0.f, 0.f, 0.f};
    const float y_lc[3] = {Lc[0] * mu_c[0] + Lc[1] * mu_c[1] + Lc[2] * mu_c[2],
                           Lc[3] * mu_c[0] + Lc[4] * mu_c[1] + Lc[5] * mu_c[2],
                           Lc[6] * mu_c[0] + Lc[7] * mu_c[1] + Lc[8] * mu_c[2]};
    const float g_y[3] = {Se[0] * g_mu_e[0] + Se[3] * g_mu_e[1] + Se[6] * g_mu_e[2],
                          Se[1] * g_mu_e[0] + Se[4] * g_mu_e[1] + Se[7] * g_mu_e[2],
                          Se[2] * g_mu_e[0] + Se[5] * g_mu_e[1] + Se[8] * g_mu_e[2]};
    float g_Lc[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) g_Lc[i * 3 + j] = g_y[i] * mu_c[j];
    g_mu_probe[0] += Lc[0] * g_y[0] + Lc[3] * g_y[1] + Lc[6] * g_y[2];
    g_mu_probe[1] += Lc[1] * g_y[0] + Lc[4] * g_y[1] + Lc[7] * g_y[2];
    g_mu_probe[2] += Lc[2] * g_y[0] + Lc[5] * g_y[1] + Lc[8] * g_y[2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) g_Se[i * 3 + j] += g_mu_e[i] * y_lc[j];
    float g_Le[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    inv3_bwd(Se, g_Se, g_Le);
#pragma unroll
    for (int i = 0; i < 9; ++i) g_Lc[i] += g_Le[i];
    g_mu_probe[1] += g_Le[0] * dlam_lat + g_Le[8] * dlam_ele;
    inv3_bwd(Lc, g_Lc, g_Sc);

    d_inten[g] = sanitize(acc[P_INTENSITY]);
    d_opac[g] = sanitize(acc[P_OPACITY]);
    const FpAdjoint adj = {acc[P_FP_MU2_LAT], acc[P_FP_MU2_AX], acc[P_FP_INV00], acc[P_FP_INV01], acc[P_FP_INV11],
                           acc[P_FP_DET2], acc[P_FP_MU_ELE], acc[P_FP_SC22], acc[P_FP_SIGMA_ELE]};
    if (shape_analytic_mode) {
        float ds[3], dq[4];
        shape_analytic(s, q, A, g_Sc, ds, dq);
        for (int k = 0; k < 3; ++k) d_scales[3 * g + k] = sanitize(ds[k]);
        for (int k = 0; k < 4; ++k) d_quats[4 * g + k] = sanitize(dq[k]);
    } else {
        for (int k = 0; k < 3; ++k)
            d_scales[3 * g + k] = sanitize(shape_fd(m, s, q, false, k, 1e-3f, A, near_mm, k_sigma, params, adj));
        for (int k = 0; k < 4; ++k)
            d_quats[4 * g + k] = sanitize(shape_fd(m, s, q, true, k, 1e-3f, A, near_mm, k_sigma, params, adj));
    }
    const float3 g_delta = make_float3(g_mu_probe[0] * A.lat.x + g_mu_probe[1] * A.ax.x + g_mu_probe[2] * A.ele.x,
                                       g_mu_probe[0] * A.lat.y + g_mu_probe[1] * A.ax.y + g_mu_probe[2] * A.ele.y,
                                       g_mu_probe[0] * A.lat.z + g_mu_probe[1] * A.ax.z + g_mu_probe[2] * A.ele.z);
    d_means[3 * g + 0] = sanitize(g_delta.x);
    d_means[3 * g + 1] = sanitize(g_delta.y);
    d_means[3 * g + 2] = sanitize(g_delta.z);
    if (!pp) return;

    // Pose contribution of this Gaussian (reference us_focus.cu:754-802); reduced over
    // Gaussians by pose_reduce_kernel instead of float atomics.
    float R[9];
    quat_rot(q[0], q[1], q[2], q[3], R);
    const float sx = fmaxf(s[0], 1e-6f), sy = fmaxf(s[1], 1e-6f), sz = fmaxf(s[2], 1e-6f);
    float Sw[9];
    sigma_world(sx, sy, sz, R, Sw);
    const float3 axes[3] = {A.lat, A.ax, A.ele};
    float3 ga[3] = {make_float3(0.f, 0.f, 0.f), make_float3(0.f, 0.f, 0.f), make_float3(0.f, 0.f, 0.f)};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const float gij = g_Sc[i * 3 + j];
            const float3 ai = axes[i], aj = axes[j];
            const float3 Sai = make_float3(Sw[0] * ai.x + Sw[1] * ai.y + Sw[2] * ai.z, Sw[3] * ai.x + Sw[4] * ai.y + Sw[5] * ai.z,
                                           Sw[6] * ai.x + Sw[7] * ai.y + Sw[8] * ai.z);
            const float3 Saj = make_float3(Sw[0] * aj.x + Sw[1] * aj.y + Sw[2] * aj.z, Sw[3] * aj.x + Sw[4] * aj.y + Sw[5] * aj.z,
                                           Sw[6] * aj.x + Sw[7] * aj.y + Sw[8] * aj.z);
            ga[i].x += gij * Saj.x; ga[i].y += gij * Saj.y; ga[i].z += gij * Saj.z;
            ga[j].x += gij * Sai.x; ga[j].y += gij * Sai.y; ga[j].z += gij * Sai.z;
        }
    const float3 dw = make_float3(m[0] - A.origin.x, m[1] - A.origin.y, m[2] - A.origin.z);
    const float3 g_lat = normalize3_bwd(A.raw_lat, A.lat, make_float3(g_mu_probe[0] * dw.x + ga[0].x, g_mu_probe[0] * dw.y + ga[0].y, g_mu_probe[0] * dw.z + ga[0].z));
    const float3 g_ax = normalize3_bwd(A.raw_ax, A.ax, make_float3(g_mu_probe[1] * dw.x + ga[1].x, g_mu_probe[1] * dw.y + ga[1].y, g_mu_probe[1] * dw.z + ga[1].z));
    const float3 g_ele = normalize3_bwd(A.raw_ele, A.ele, make_float3(g_mu_probe[2] * dw.x + ga[2].x, g_mu_probe[2] * dw.y + ga[2].y, g_mu_probe[2] * dw.z + ga[2].z));
    // 4x4 row-major pose indices: column 0 = lateral, 1 = axial, 2 = elevational, 3 = origin.
    pp[0] = g_lat.x; pp[1] = g_lat.y; pp[2] = g_lat.z;
    pp[3] = g_ax.x; pp[4] = g_ax.y; pp[5] = g_ax.z;
    pp[6] = g_ele.x; pp[7] = g_ele.y; pp[8] = g_ele.z;
    pp[9] = -g_delta.x; pp[10] = -g_delta.y; pp[11] = -g_delta.z;
}

// Sums the per-Gaussian pose contributions in a fixed order, in two launches: block b of
// POSE_BLOCKS reduces the contiguous chunk b of Gaussians and leaves its 12 sums in the chunk's
// first slot of pose_partial; one block then adds the chunk sums in block order.
constexpr int POSE_BLOCKS = 512;

// The pose gradient is a sum over all Gaussians of terms with long lever arms that largely
// cancel, so the sums run in double: per-Gaussian float contributions, chunk sums and the final
// sum accumulate in double (fixed order), and the chunk sums stay in double (two float slots
// each, in the chunk's own first Gaussians' slots; chunks hold at least two Gaussians).
__device__ __forceinline__ void pose_block_sum(double a[12]) {
    __shared__ double red[256][13];
#pragma unroll
    for (int i = 0; i < 12; ++i) red[threadIdx.x][i] = a[i];
    __syncthreads();
    for (int stride = 128; stride > 0; stride >>= 1) {
        if (threadIdx.x < stride)
#pragma unroll
            for (int i = 0; i < 12; ++i) red[threadIdx.x][i] += red[threadIdx.x + stride][i];
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) a[i] = red[0][i];
}

__global__ void __launch_bounds__(256)
pose_chunk_kernel(int64_t G, int64_t chunk, float* __restrict__ pose_partial) {
    const int64_t g0 = (int64_t)blockIdx.x * chunk;
    if (g0 >= G) return;
    const int64_t g1 = g0 + chunk < G ? g0 + chunk : G;
    double a[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) a[i] = 0.0;
    for (int64_t g = g0 + threadIdx.x; g < g1; g += blockDim.x)
#pragma unroll
        for (int i = 0; i < 12; ++i) a[i] += (double)pose_partial[12 * g + i];
    pose_block_sum(a);  // ends with every read of the chunk done
    double* out = reinterpret_cast<double*>(pose_partial + 12 * g0);
    if (threadIdx.x < 12) out[threadIdx.x] = a[threadIdx.x];
}

__global__ void __launch_bounds__(256)
pose_final_kernel(int64_t G, int64_t chunk, const float* __restrict__ pose_partial, float* __restrict__ d_pose) {
    const int nb = (int)((G + chunk - 1) / chunk);
    double a[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) a[i] = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const double* in = reinterpret_cast<const double*>(pose_partial + 12 * (int64_t)b * chunk);
#pragma unroll
        for (int i = 0; i < 12; ++i) a[i] += in[i];
    }
    pose_block_sum(a);
    if (threadIdx.x == 0) {
        const int idx[12] = {0, 4, 8, 1, 5, 9, 2, 6, 10, 3, 7, 11};
        for (int i = 0; i < 16; ++i) d_pose[i] = 0.f;
        for (int i = 0; i < 12; ++i) d_pose[idx[i]] = (float)a[i];
    }
}

__global__ void export_kernel(int T, const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                              int* __restrict__ out_ids, int* __restrict__ rs, int* __restrict__ re) {
    const int t = blockIdx.x;
    if (t >= T) return;
    const int s0 = tile_start[t], s1 = tile_start[t + 1];
    if (threadIdx.x == 0) {
        rs[t] = (s1 > s0) ? s0 : -1;
        re[t] = (s1 > s0) ? s1 : -1;
    }
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) out_ids[s] = sorted_gid[s];
}

}  // namespace gp
}  // namespace us3d

using namespace us3d;
using namespace us3d::gp;

static bool g_gp_sort_attr[128];

static int gp_sizes(int H, int W, int tile, int* tx, int* ty) {
    US3D_CHECK_ARG(H > 0 && W > 0, "H/W must be positive");
    US3D_CHECK_ARG(tile > 0 && tile * tile <= 1024, "tile_size_px must be in [1, 32]");
    *tx = (W + tile - 1) / tile;
    *ty = (H + tile - 1) / tile;
    return US3D_OK;
}

extern "C" size_t us3d_gp_workspace_bytes(int64_t n_gauss, int32_t H, int32_t W, int32_t tile, int64_t cap) {
    if (n_gauss < 0 || cap < 0 || H <= 0 || W <= 0 || tile <= 0) return 0;
    const int64_t T = (int64_t)((W + tile - 1) / tile) * ((H + tile - 1) / tile);
    return carve(nullptr, n_gauss, T, cap).bytes;
}

extern "C" size_t us3d_gp_backward_scratch_bytes(int64_t n_gauss, int64_t cap) {
    if (n_gauss < 0 || cap < 0) return 0;
    // + 2 Gaussians' pose slots: a chunk's double sums span two slots, also for a last chunk of one
    return (size_t)cap * PARTIAL_F4 * sizeof(float4) + (size_t)(n_gauss + 2) * 12 * sizeof(float) + 256;
}

extern "C" int us3d_gp_forward(void* workspace, size_t workspace_bytes, int64_t n_gauss, const float* means,
                               const float* scales, const float* quats, const float* opacities,
                               const float* intensities, const float* pose, const float* grid_pack,
                               const float* focus_params, int32_t H, int32_t W, float lateral_spacing,
                               float axial_spacing, float axial_near, int32_t tile_size, float k_sigma,
                               int32_t sort_by_v, int64_t cap, float* out_image, void* stream_) {
    int tx, ty;
    int st = gp_sizes(H, W, tile_size, &tx, &ty);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace && out_image && pose && grid_pack && focus_params, "NULL pointer argument");
    US3D_CHECK_ARG(n_gauss >= 0 && n_gauss <= 0x7fffffffLL, "n_gauss out of range");
    US3D_CHECK_ARG(n_gauss == 0 || (means && scales && quats && opacities && intensities), "NULL parameter pointer");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(lateral_spacing > 0.f && axial_spacing > 0.f, "pixel spacing must be > 0");
    const int64_t T = (int64_t)tx * ty;
    const Workspace w = carve(workspace, n_gauss, T, cap);
    US3D_CHECK_ARG(workspace_bytes >= w.bytes, "workspace too small: %zu < %zu", workspace_bytes, w.bytes);
    cudaStream_t stream = (cudaStream_t)stream_;
    const int prof = prof_begin("gp_forward", stream);
    init_kernel<<<(unsigned)((T + 255) / 256), 256, 0, stream>>>(T, w.tile_count, w.tile_cursor, w.header, cap, n_gauss);
    const unsigned gb = (unsigned)((n_gauss + 255) / 256);
    if (n_gauss > 0)
        preprocess_kernel<<<gb, 256, 0, stream>>>(n_gauss, H, W, tile_size, tx, ty, lateral_spacing, axial_spacing,
                                                  axial_near, k_sigma, sort_by_v, means, scales, quats, opacities,
                                                  intensities, pose, grid_pack, focus_params, w.rects, w.dkey,
                                                  w.touched, w.tile_count, w.cand, w.bfp);
    US3D_CHECK_LAUNCH("gp preprocess");
    US3D_CHECK_CUDA(launch_rect_count(n_gauss, tx, T, RectOf4{w.rects}, w.tile_count, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.touched, n_gauss, w.inst_offset, w.bs_g, w.header + H_SCAN_G, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.tile_count, T, w.tile_start, w.bs_t, w.header + H_SCAN_T, stream));
    check_kernel<<<1, 1, 0, stream>>>(w.header, cap);
    US3D_CHECK_CUDA(launch_rect_scatter(n_gauss, tx, T, RectOf4{w.rects}, w.dkey, w.inst_offset, w.tile_start,
                                        w.tile_cursor, w.header, w.keys, w.slot_inst, stream));
    US3D_CHECK_CUDA(launch_tile_sort(T, n_gauss, w.tile_start, w.header, w.keys, w.slot_inst, w.sorted_gid, w.sorted_inst,
                                     g_gp_sort_attr, stream));
    // up to four threads per pixel (a whole-warp pixel block of at most 1024 threads); frames
    // with fewer than four tiles per SM split each tile over four blocks when it divides into
    // whole warps
    const int npix = (tile_size * tile_size + 31) / 32 * 32;
    auto launch = [&](auto kernel, int parts, int split) {
        kernel<<<(unsigned)(T * split), npix / split * parts, 0, stream>>>(
            H, W, tile_size, tx, grid_pack, focus_params, w.tile_start, w.sorted_gid, w.header, w.cand, out_image);
    };
    const bool split4 = T < 4 * 148 && (tile_size * tile_size) % 128 == 0;
    if (npix <= 256)
        split4 ? launch(forward_kernel<4, 4>, 4, 4) : launch(forward_kernel<4, 1>, 4, 1);
    else if (npix <= 512)
        split4 ? launch(forward_kernel<2, 4>, 2, 4) : launch(forward_kernel<2, 1>, 2, 1);
    else
        split4 ? launch(forward_kernel<1, 4>, 1, 4) : launch(forward_kernel<1, 1>, 1, 1);
    US3D_CHECK_LAUNCH("gp forward");
    prof_end(prof, stream);
    count_launches(1 + (n_gauss > 0) * 3 + 6 + 1 + tile_sort_launches(n_gauss) + 1);
    return US3D_OK;
}

extern "C" int us3d_gp_read_status(const void* workspace, int64_t* total, int32_t* flags, void* stream_) {
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    long long hdr[H_WORDS];
    cudaStream_t stream = (cudaStream_t)stream_;
    US3D_CHECK_CUDA(cudaMemcpyAsync(hdr, workspace, sizeof(hdr), cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
    if (total) *total = hdr[H_TOTAL];
    if (flags) *flags = (int32_t)hdr[H_FLAGS];
    return US3D_OK;
}

extern "C" int us3d_gp_backward(void* workspace, int64_t n_gauss, const float* means, const float* scales,
                                const float* quats, const float* opacities, const float* intensities,
                                const float* pose, const float* grid_pack, const float* focus_params, int32_t H,
                                int32_t W, int32_t tile_size, float k_sigma, int64_t cap, const float* grad_image,
                                int32_t grad_flags, void* scratch, size_t scratch_bytes, float* d_means,
                                float* d_scales, float* d_quats, float* d_opacities, float* d_intensities,
                                float* d_pose, void* stream_) {
    US3D_CHECK_ARG((grad_flags & ~(US3D_GP_GRAD_POSE | US3D_GP_GRAD_SHAPE_ANALYTIC)) == 0,
                   "unknown gradient flags 0x%x", (unsigned)grad_flags);
    const int pose_grad = (grad_flags & US3D_GP_GRAD_POSE) ? 1 : 0;
    const int shape_analytic_mode = (grad_flags & US3D_GP_GRAD_SHAPE_ANALYTIC) ? 1 : 0;
    int tx, ty;
    int st = gp_sizes(H, W, tile_size, &tx, &ty);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace && grad_image && pose && grid_pack && focus_params, "NULL pointer argument");
    US3D_CHECK_ARG(n_gauss >= 0 && n_gauss <= 0x7fffffffLL, "n_gauss out of range");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(scratch_bytes >= us3d_gp_backward_scratch_bytes(n_gauss, cap), "backward scratch too small");
    US3D_CHECK_ARG(n_gauss == 0 || (means && scales && quats && opacities && intensities && d_means && d_scales &&
                                    d_quats && d_opacities && d_intensities), "NULL gradient/parameter pointer");
    US3D_CHECK_ARG(!pose_grad || d_pose, "d_pose is NULL");
    const int64_t T = (int64_t)tx * ty;
    const Workspace w = carve(workspace, n_gauss, T, cap);
    float* partial = reinterpret_cast<float*>(scratch);
    float* pose_partial = partial + (size_t)cap * PARTIAL_F4 * 4;
    pose_partial = reinterpret_cast<float*>(align_up(reinterpret_cast<uintptr_t>(pose_partial), 256));
    cudaStream_t stream = (cudaStream_t)stream_;
    const int prof = prof_begin("gp_backward", stream);
    int launches = 0;
    if (T > 0) {
        backward_inst_kernel<<<148 * 8, BWD_WARPS * 32, 0, stream>>>(
            (int)T, W, tile_size, tx, opacities, intensities, w.bfp, grid_pack, focus_params, w.tile_start,
            w.sorted_gid, w.sorted_inst, w.header, grad_image, partial, H);
        US3D_CHECK_LAUNCH("gp backward instances");
        launches = 1;
    }
    if (n_gauss > 0) {
        reduce_partials_kernel<<<(unsigned)((n_gauss * PARTIAL_F4 + REDUCE_THREADS - 1) / REDUCE_THREADS),
                                 REDUCE_THREADS, 0, stream>>>(n_gauss, w.inst_offset, w.header,
                                                              reinterpret_cast<float4*>(partial));
        ++launches;
        finalize_kernel<<<(unsigned)((n_gauss + 127) / 128), 128, 0, stream>>>(
            n_gauss, k_sigma, w.inst_offset, w.rects, means, scales, quats, pose, grid_pack, focus_params, w.header,
            partial, pose_grad, shape_analytic_mode, d_means, d_scales, d_quats, d_opacities, d_intensities,
            pose_partial);
        US3D_CHECK_LAUNCH("gp finalize");
        ++launches;
    }
    if (pose_grad) {
        const int64_t chunk = std::max<int64_t>(2, (n_gauss + POSE_BLOCKS - 1) / POSE_BLOCKS);
        if (n_gauss > 0) {
            pose_chunk_kernel<<<(unsigned)((n_gauss + chunk - 1) / chunk), 256, 0, stream>>>(n_gauss, chunk,
                                                                                             pose_partial);
            ++launches;
        }
        pose_final_kernel<<<1, 256, 0, stream>>>(n_gauss, chunk, pose_partial, d_pose);
        US3D_CHECK_LAUNCH("gp pose reduce");
        ++launches;
    }
    prof_end(prof, stream);
    count_launches(launches);
    return US3D_OK;
}

extern "C" int us3d_gp_export_bins(const void* workspace, int64_t n_gauss, int32_t H, int32_t W, int32_t tile_size,
                                   int64_t cap, int32_t* out_sorted_ids, int32_t* out_range_start,
                                   int32_t* out_range_end, int32_t* out_rects, void* stream_) {
    int tx, ty;
    int st = gp_sizes(H, W, tile_size, &tx, &ty);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace && out_range_start && out_range_end, "NULL pointer argument");
    const int64_t T = (int64_t)tx * ty;
    const Workspace w = carve(const_cast<void*>(workspace), n_gauss, T, cap);
    cudaStream_t stream = (cudaStream_t)stream_;
    export_kernel<<<(unsigned)T, 256, 0, stream>>>((int)T, w.tile_start, w.sorted_gid, out_sorted_ids,
                                                   out_range_start, out_range_end);
    if (out_rects && n_gauss > 0)
        US3D_CHECK_CUDA(cudaMemcpyAsync(out_rects, w.rects, sizeof(int4) * n_gauss, cudaMemcpyDeviceToDevice, stream));
    US3D_CHECK_LAUNCH("gp export");
    count_launches(1);
    return US3D_OK;
}
