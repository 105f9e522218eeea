// UltraGray scanline ray-integral B-mode renderer: ray binning, forward, backward.
//
// Reference behaviour restated here (paths inside KevinWCCC/ultrasound-3d-reconstruction,
// ops/ultragray_renderer):
//   src/mapper/core.cu:3-129           probe-frame projection, near / elevational culls, ray
//                                      range, (ray, depth) keys, per-ray CSR, sorted depths
//   include/shader/shared.cuh:5-85     Gaussian weight, degree-1 SH echo, 3-point
//                                      Gauss-Legendre ray-Gaussian attenuation integral
//   src/shader/forward.cu:22-119       per pixel: transmission product over shallower
//                                      Gaussians, echo over nearby ones, B = T * gamma * E
//   src/shader/backward.cu:26-325      adjoint (integral and weight VJPs)
// The reference tree lacks the header defining the quaternion rotation, the precision
// R diag(1/s^2) R^T and their gradients; they are defined here from the mathematics their
// call sites imply (normalised (w,x,y,z) quaternion, row-major R with the Gaussian's axes
// as columns).
//
// B200 design: rays are binned like tiles (bucket per ray + in-shared-memory ordering by
// (depth key, Gaussian)); every Gaussian's rotation, precision and sigmoid attenuation are
// computed once per call into a 112-byte record; the forward stages a ray's records in
// shared memory and gives each thread one pixel of the ray, in list order (the reference's
// multiplication order); it saves (T, sum I w, sum w) per pixel so the backward needs no
// recompute pass. The backward gives each thread one (ray, Gaussian) instance, sweeps the
// ray's pixels (whose adjoint coefficients sit in shared memory) and accumulates that
// instance's gradient in registers, including dL/dR and dL/dSigma^-1, which are mapped to
// quaternion and scale gradients once per instance; partials are reduced per Gaussian in a
// fixed order (the reference issues 16 float atomics per pair).
#include "us3d_common.cuh"
#include "scan.cuh"
#include "binning.cuh"

namespace us3d {
namespace ugr {

constexpr int BATCH = 128;       // records staged per shared-memory batch
constexpr int REC_F4 = 7;        // 112-byte Gaussian record
constexpr int PARTIAL_F4 = 4;    // 16-float per-instance partial
constexpr int PIX_CHUNK = 256;   // pixels of a ray staged at once by the backward

struct Workspace {
    long long* header;
    int2* ray_range;    // G
    uint32_t* dkey;     // G
    int* touched;       // G
    int* inst_offset;   // G + 1
    long long* bs_g;
    int* ray_count;     // W
    int* ray_start;     // W + 1
    int* ray_cursor;    // W
    long long* bs_t;
    float4* rec;        // G x 7
    unsigned long long* keys;
    int* slot_inst;
    int* sorted_gid;
    int* sorted_inst;
    float4* pixel_state;  // P: T_final, sum I w, sum w, t_pixel
    // Transmittance checkpoints (quadrature window radius > 0, full transmission):
    float* t_pix;         // P: sample depth t along its ray (ray-major)
    int* mono;            // W: 1 if the ray's sample depths never decrease
    float4* aux;          // cap: per instance (t_gauss, echo radius, far factor F, first far sample)
    long long* far_log;   // P: fixed-point sum of log F of the instances whose far zone starts at the
                          //    sample, then (in place) its prefix along the ray
    float* t_far;         // P: product of the far factors of every instance settled at the sample
    float4* b_pos;        // P: backward: sample position, t
    float4* b_coef;       // P: backward: dL/dT, T, dL/dnum, dL/dw (zero for skipped samples)
    float* b_suffix;      // P: backward: sum over the ray's samples y' >= y of dL/dT * T
    size_t bytes;
};

static Workspace carve(void* base, int64_t G, int64_t W, int64_t P, int64_t cap) {
    Carver c(base);
    Workspace w;
    w.header = c.take<long long>(H_WORDS);
    w.ray_range = c.take<int2>((size_t)G);
    w.dkey = c.take<uint32_t>((size_t)G);
    w.touched = c.take<int>((size_t)G);
    w.inst_offset = c.take<int>((size_t)G + 1);
    w.bs_g = c.take<long long>((size_t)scan_num_blocks(G) + 1);
    w.ray_count = c.take<int>((size_t)W);
    w.ray_start = c.take<int>((size_t)W + 1);
    w.ray_cursor = c.take<int>((size_t)W);
    w.bs_t = c.take<long long>((size_t)scan_num_blocks(W) + 1);
    w.rec = c.take<float4>((size_t)G * REC_F4);
    w.keys = c.take<unsigned long long>((size_t)cap);
    w.slot_inst = c.take<int>((size_t)cap);
    w.sorted_gid = c.take<int>((size_t)cap);
    w.sorted_inst = c.take<int>((size_t)cap);
    w.pixel_state = c.take<float4>((size_t)P);
    w.t_pix = c.take<float>((size_t)P);
    w.mono = c.take<int>((size_t)W);
    w.aux = c.take<float4>((size_t)cap);
    w.far_log = c.take<long long>((size_t)P);
    w.t_far = c.take<float>((size_t)P);
    w.b_pos = c.take<float4>((size_t)P);
    w.b_coef = c.take<float4>((size_t)P);
    w.b_suffix = c.take<float>((size_t)P);
    w.bytes = align_up(c.off, 256);
    return w;
}

// float3 helpers written as the reference's operators so the compiler contracts them the same way.
__device__ __forceinline__ float3 v_add(const float3 a, const float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 v_sub(const float3 a, const float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 v_mul(const float3 a, const float b) { return make_float3(a.x * b, a.y * b, a.z * b); }
__device__ __forceinline__ float v_dot(const float3 a, const float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Rotation of the normalised (w,x,y,z) quaternion stored as (q.x, q.y, q.z, q.w).
__device__ __forceinline__ void quat_rot(const float4 q, float* R) {
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

// Precision R diag(1/s^2) R^T.
__device__ __forceinline__ void precision(const float3 s, const float* R, float* P) {
    const float d0 = 1.f / (s.x * s.x), d1 = 1.f / (s.y * s.y), d2 = 1.f / (s.z * s.z);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            P[r * 3 + c] = R[r * 3 + 0] * d0 * R[c * 3 + 0] + R[r * 3 + 1] * d1 * R[c * 3 + 1] + R[r * 3 + 2] * d2 * R[c * 3 + 2];
}

// dL/dq of R(q/|q|) for the (w,x,y,z) quaternion stored as (q.x, q.y, q.z, q.w), given dL/dR.
__device__ __forceinline__ float4 quat_grad(const float4 q, const float* g) {
    const float len = sqrtf(fmaxf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w, 1e-12f));
    const float n = 1.f / len;
    const float w = q.x * n, x = q.y * n, y = q.z * n, z = q.w * n;
    const float gw = 2.f * (-z * g[1] + y * g[2] + z * g[3] - x * g[5] - y * g[6] + x * g[7]);
    const float gx = 2.f * (y * g[1] + z * g[2] + y * g[3] - 2.f * x * g[4] - w * g[5] + z * g[6] + w * g[7] - 2.f * x * g[8]);
    const float gy = 2.f * (-2.f * y * g[0] + x * g[1] + w * g[2] + x * g[3] + z * g[5] - w * g[6] + z * g[7] - 2.f * y * g[8]);
    const float gz = 2.f * (-2.f * z * g[0] - w * g[1] + x * g[2] + w * g[3] - 2.f * z * g[4] + y * g[5] + x * g[6] + y * g[7]);
    const float dot = w * gw + x * gx + y * gy + z * gz;
    return make_float4((gw - w * dot) * n, (gx - x * dot) * n, (gy - y * dot) * n, (gz - z * dot) * n);
}

// Gauss-Legendre (3 points) integral of the canonical Gaussian along the ray over [0, l],
// restricted to a window of radius wr around the closest approach (reference shared.cuh:27-85).
// With wr > 0 the integral ends at min(l, tc + wr): for every pixel depth l >= tc + wr it is
// one value per (ray, Gaussian), which *tcw_out (if not NULL) receives as tc + wr.
__device__ __forceinline__ float ray_integral(const float3 ro, const float3 rd, const float3 mu, const float3 s,
                                              const float* R, float l, float wr, float* tcw_out = nullptr) {
    if (l <= 0.0f) return 0.0f;
    const float3 diff = v_sub(ro, mu);
    float3 ol, dl;
    ol.x = R[0] * diff.x + R[3] * diff.y + R[6] * diff.z;
    ol.y = R[1] * diff.x + R[4] * diff.y + R[7] * diff.z;
    ol.z = R[2] * diff.x + R[5] * diff.y + R[8] * diff.z;
    dl.x = R[0] * rd.x + R[3] * rd.y + R[6] * rd.z;
    dl.y = R[1] * rd.x + R[4] * rd.y + R[7] * rd.z;
    dl.z = R[2] * rd.x + R[5] * rd.y + R[8] * rd.z;
    const float3 og = make_float3(ol.x / s.x, ol.y / s.y, ol.z / s.z);
    const float3 dg = make_float3(dl.x / s.x, dl.y / s.y, dl.z / s.z);
    const float dg2 = v_dot(dg, dg);
    const float tc = -v_dot(og, dg) / (dg2 + 1e-8f);
    float t0s = 0.0f, t1s = l;
    if (wr > 0.0f) {
        t0s = fmaxf(0.0f, tc - wr);
        t1s = fminf(l, tc + wr);
        if (tcw_out) *tcw_out = tc + wr;
    }
    if (t1s <= t0s) return 0.0f;
    const float half = 0.5f * (t1s - t0s);
    const float c = 0.5f * (t1s + t0s);
    const float ta = half * -0.7745966692f + c;
    const float tb = half * 0.0f + c;
    const float tz = half * 0.7745966692f + c;
    const float3 xa = v_add(og, v_mul(dg, ta));
    const float3 xb = v_add(og, v_mul(dg, tb));
    const float3 xz = v_add(og, v_mul(dg, tz));
    const float fa = __expf(-0.5f * v_dot(xa, xa));
    const float fb = __expf(-0.5f * v_dot(xb, xb));
    const float fz = __expf(-0.5f * v_dot(xz, xz));
    return half * (0.5555555556f * fa + 0.8888888889f * fb + 0.5555555556f * fz);
}

// Record layout (7 float4): (mu, tau) (s, max s) (R0..R3) (R4..R7) (R8, P00, P01, P02) (P11, P12, P22, -) (sh)
struct Rec {
    float3 mu, s;
    float tau, smax;
    float R[9];
    float P[9];
    float4 sh;
};

__device__ __forceinline__ void load_rec(const float4* __restrict__ r, Rec& o) {
    const float4 a = r[0], b = r[1], c = r[2], d = r[3], e = r[4], f = r[5];
    o.mu = make_float3(a.x, a.y, a.z);
    o.tau = a.w;
    o.s = make_float3(b.x, b.y, b.z);
    o.smax = b.w;
    o.R[0] = c.x; o.R[1] = c.y; o.R[2] = c.z; o.R[3] = c.w;
    o.R[4] = d.x; o.R[5] = d.y; o.R[6] = d.z; o.R[7] = d.w;
    o.R[8] = e.x;
    o.P[0] = e.y; o.P[1] = e.z; o.P[2] = e.w;
    o.P[3] = e.z; o.P[4] = f.x; o.P[5] = f.y;
    o.P[6] = e.w; o.P[7] = f.y; o.P[8] = f.z;
    o.sh = r[6];
}

// Reference Gaussian weight: exp(-0.5 * d^T P d) with the full 9-entry form (shared.cuh:5-19).
__device__ __forceinline__ float gauss_weight(const float3 p, const float3 mu, const float* P) {
    const float dx = p.x - mu.x, dy = p.y - mu.y, dz = p.z - mu.z;
    const float power = -0.5f * ((P[0] * dx + P[1] * dy + P[2] * dz) * dx + (P[3] * dx + P[4] * dy + P[5] * dz) * dy +
                                 (P[6] * dx + P[7] * dy + P[8] * dz) * dz);
    return __expf(power);
}

// ------------------------------------------------------------------------------------
// Binning
// ------------------------------------------------------------------------------------

__global__ void init_kernel(int64_t W, int* __restrict__ ray_count, int* __restrict__ ray_cursor,
                            long long* __restrict__ header, int64_t cap, int64_t G, int64_t P) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < H_WORDS) {
        long long v = 0;
        if (threadIdx.x == H_CAP) v = cap;
        if (threadIdx.x == H_G) v = G;
        if (threadIdx.x == H_T) v = W;
        if (threadIdx.x == H_P) v = P;
        header[threadIdx.x] = v;
    }
    if (t >= W) return;
    ray_count[t] = 0;
    ray_cursor[t] = 0;
}

// Projection, culls, ray range and depth key (reference src/mapper/core.cu:3-96) plus the
// per-Gaussian record.
__global__ void __launch_bounds__(256)
preprocess_kernel(int64_t G, int W, float pixel_spacing, float col_off, float near_mm, float elev_cut, float k_sigma,
                  const float* __restrict__ means, const float* __restrict__ scales, const float* __restrict__ quats,
                  const float* __restrict__ attens, const float* __restrict__ sh, const float* __restrict__ origin,
                  const float* __restrict__ a_lat, const float* __restrict__ a_ele, const float* __restrict__ a_ax,
                  int2* __restrict__ ray_range, uint32_t* __restrict__ dkey, int* __restrict__ touched,
                  int* __restrict__ ray_count, float4* __restrict__ rec) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const float3 o = make_float3(origin[0], origin[1], origin[2]);
    const float3 u = make_float3(a_lat[0], a_lat[1], a_lat[2]);
    const float3 v = make_float3(a_ele[0], a_ele[1], a_ele[2]);
    const float3 w = make_float3(a_ax[0], a_ax[1], a_ax[2]);
    const float3 mu = make_float3(means[3 * g], means[3 * g + 1], means[3 * g + 2]);
    const float3 s = make_float3(scales[3 * g], scales[3 * g + 1], scales[3 * g + 2]);
    // record
    const float4 q = make_float4(quats[4 * g], quats[4 * g + 1], quats[4 * g + 2], quats[4 * g + 3]);
    float R[9], P[9];
    quat_rot(q, R);
    precision(s, R, P);
    const float tau = 1.0f / (1.0f + __expf(-attens[g]));
    const float smax = fmaxf(s.x, fmaxf(s.y, s.z));
    float4* r = rec + REC_F4 * g;
    r[0] = make_float4(mu.x, mu.y, mu.z, tau);
    r[1] = make_float4(s.x, s.y, s.z, smax);
    r[2] = make_float4(R[0], R[1], R[2], R[3]);
    r[3] = make_float4(R[4], R[5], R[6], R[7]);
    r[4] = make_float4(R[8], P[0], P[1], P[2]);
    r[5] = make_float4(P[4], P[5], P[8], 0.f);
    r[6] = make_float4(sh[4 * g], sh[4 * g + 1], sh[4 * g + 2], sh[4 * g + 3]);
    // mapper
    touched[g] = 0;
    ray_range[g] = make_int2(0, -1);
    dkey[g] = 0;
    const float3 diff = v_sub(mu, o);
    const float px = v_dot(diff, u), py = v_dot(diff, v), pz = v_dot(diff, w);
    const float radius_safe = smax * k_sigma;
    if (pz + radius_safe < near_mm) return;
    if (fabsf(py) > (radius_safe + elev_cut)) return;
    const float centre = (px / pixel_spacing) + col_off;
    const float rad = radius_safe / pixel_spacing;
    int r0 = (int)floorf(centre - rad);
    int r1 = (int)ceilf(centre + rad);
    r0 = max(0, r0);
    r1 = min(W - 1, r1);
    if (r0 > r1) return;
    touched[g] = r1 - r0 + 1;
    ray_range[g] = make_int2(r0, r1);
    dkey[g] = f32_to_u32_sat(fmaxf(0.0f, pz) * 1000.0f);
    (void)ray_count;  // counted per block by rect_count_kernel
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

// Local transmission window: the reference walks the depth-sorted ray list from the lower
// bound of t_pixel - max_win and stops past t_pixel + max_win (forward.cu:71-79); on a
// sorted list that is exactly this per-entry test.
__device__ __forceinline__ bool in_local_window(float depth, float t_pixel, float max_win) {
    return !(depth < t_pixel - max_win) && !(depth > t_pixel + max_win);
}

struct RayGeo {
    float3 o, d;
};

__device__ __forceinline__ RayGeo ray_geo(int x, const float* __restrict__ ray_o, const float* __restrict__ ray_d,
                                          const float* __restrict__ a_ele, const float* __restrict__ pert) {
    RayGeo r;
    const float3 ele = make_float3(a_ele[0], a_ele[1], a_ele[2]);
    r.o = v_add(make_float3(ray_o[3 * x], ray_o[3 * x + 1], ray_o[3 * x + 2]), v_mul(ele, pert[x]));
    r.d = make_float3(ray_d[3 * x], ray_d[3 * x + 1], ray_d[3 * x + 2]);
    return r;
}

// Block (x, y) shades samples [FWD_SAMPLES y, FWD_SAMPLES (y + 1)) of ray x, one per thread;
// the ray's instances are staged in shared memory and walked in list order (reference
// forward.cu:22-119).
#ifndef US3D_UGR_FWD_SAMPLES
#define US3D_UGR_FWD_SAMPLES 64
#endif
constexpr int FWD_SAMPLES = US3D_UGR_FWD_SAMPLES;
__global__ void __launch_bounds__(FWD_SAMPLES)
forward_kernel(int W, int H, const int* __restrict__ ray_start, const int* __restrict__ sorted_gid,
               const long long* __restrict__ header, const float4* __restrict__ rec,
               const float* __restrict__ pixels, const float* __restrict__ ray_o, const float* __restrict__ ray_d,
               const float* __restrict__ a_ele, const float* __restrict__ pert, const uint32_t* __restrict__ dkey,
               float k_sigma, float wr, int local_only, float max_win, const int* __restrict__ ckpt_rays,
               float* __restrict__ image, float4* __restrict__ pixel_state) {
    __shared__ float4 s_rec[BATCH * REC_F4];
    __shared__ float s_tg[BATCH];
    __shared__ float s_depth[BATCH];
    __shared__ float s_tcw[BATCH];   // window end tc + wr of the transmission integral (+inf: none)
    __shared__ float s_far[BATCH];   // its factor tau + (1 - tau) exp(-psi) for pixels at or past it
    if (header[H_FLAGS] != 0) return;
    const int x = blockIdx.x;
    if (ckpt_rays && ckpt_rays[x]) return;  // rendered by the checkpointed path
    const int s0 = ray_start[x], n = ray_start[x + 1] - s0;
    const RayGeo rg = ray_geo(x, ray_o, ray_d, a_ele, pert);
    // blockIdx.y: which blockDim.x samples of the ray this block shades
    for (int y0 = blockIdx.y * blockDim.x; y0 < H; y0 += gridDim.y * blockDim.x) {
        const int y = y0 + threadIdx.x;
        const bool valid = y < H;
        float3 p = make_float3(0.f, 0.f, 0.f);
        if (valid) {
            const float* pp = pixels + ((int64_t)x * H + y) * 3;
            p = make_float3(pp[0], pp[1], pp[2]);
        }
        const float t_pixel = fmaxf(0.0f, v_dot(v_sub(p, rg.o), rg.d));
        float trans = 1.0f, num = 0.0f, den = 0.0f, sacc = 0.0f;
        for (int b0 = 0; b0 < n; b0 += BATCH) {
            const int nb = min(BATCH, n - b0);
            __syncthreads();
            for (int j = threadIdx.x; j < nb * REC_F4; j += blockDim.x) {
                const int k = j / REC_F4, f = j - k * REC_F4;
                s_rec[j] = rec[(int64_t)REC_F4 * sorted_gid[s0 + b0 + k] + f];
            }
            __syncthreads();
            for (int k = threadIdx.x; k < nb; k += blockDim.x) {
                const float4 a = s_rec[k * REC_F4];
                s_tg[k] = v_dot(v_sub(make_float3(a.x, a.y, a.z), rg.o), rg.d);
                s_depth[k] = (float)dkey[sorted_gid[s0 + b0 + k]] * 0.001f;
                float tcw = 3.0e38f, far = 1.0f;
                if (wr > 0.0f) {
                    Rec r;
                    load_rec(s_rec + k * REC_F4, r);
                    const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, 3.0e38f, wr, &tcw);
                    far = r.tau + (1.0f - r.tau) * __expf(-psi);
                }
                s_tcw[k] = tcw;
                s_far[k] = far;
            }
            __syncthreads();
            if (!valid || n == 0) continue;
            for (int k = 0; k < nb; ++k) {
                if (local_only && !in_local_window(s_depth[k], t_pixel, max_win)) continue;
                const float t_gauss = s_tg[k];
                const float smax = s_rec[k * REC_F4 + 1].w;
                const float depth_radius = smax * k_sigma;
                bool need_t = t_gauss < t_pixel;
                if (local_only) need_t = need_t && ((t_pixel - t_gauss) <= depth_radius + wr);
                const bool need_e = fabsf(t_gauss - t_pixel) <= depth_radius;
                if (!need_t && !need_e) continue;
                // past the window end the factor is the ray's per-Gaussian constant
                if (need_t && !need_e && t_pixel > 0.0f && t_pixel >= s_tcw[k]) {
                    trans *= s_far[k];
                    continue;
                }
                Rec r;
                load_rec(s_rec + k * REC_F4, r);
                if (need_t) {
                    if (t_pixel > 0.0f && t_pixel >= s_tcw[k]) {
                        trans *= s_far[k];
                    } else {
                        const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, t_pixel, wr);
                        trans *= r.tau + (1.0f - r.tau) * __expf(-psi);
                    }
                }
                if (need_e) {
                    const float wgt = gauss_weight(p, r.mu, r.P);
                    const float I = r.sh.x + r.sh.y * rg.d.x + r.sh.z * rg.d.y + r.sh.w * rg.d.z;
                    num += I * wgt;
                    den += wgt;
                    sacc += wgt;
                }
            }
        }
        if (!valid) continue;
        float out = 0.0f;
        if (n > 0) {
            const float gamma = 1.0f - __expf(-sacc);
            const float echo = num / (den + 1e-6f);
            out = trans * (gamma * echo);
        }
        image[(int64_t)y * W + x] = out;
        pixel_state[(int64_t)x * H + y] = make_float4(trans, num, den, sacc);
    }
}

// ------------------------------------------------------------------------------------
// Transmittance checkpoints (quadrature window radius wr > 0, full transmission)
// ------------------------------------------------------------------------------------
//
// With wr > 0 the transmission factor of instance k at a sample of depth t no longer depends on
// t once t >= tcw_k = tc_k + wr (and t > t_gauss, t > 0): it is the instance's far factor F_k
// (the reference evaluates the same integral, over the same window, at every such sample).
// Along a ray whose sample depths never decrease, instance k is therefore "settled" from its
// first far sample y_far(k) on. The product of the settled factors at every sample is a
// checkpoint: log F_k is added, in 2^-32 fixed point (exact, order-free integer sums), at
// y_far(k), a prefix sum along the ray gives each sample's sum, and T_far = exp(sum) (double).
// A sample's transmittance is then T_far times the factors of the instances it is still inside
// the window of (t_gauss < t < tcw), evaluated as the reference does, in list order; the
// forward of a tile of samples walks only the instances near or echoing in that tile. The
// backward reads the same checkpoints: the far part of an instance's gradient is the suffix
// sum over the ray's samples of dL/dT * T divided by F_k, and only the samples inside its
// window or echo range are visited. Rays whose sample depths decrease somewhere keep the
// per-sample path above.

constexpr double FAR_LOG_SCALE = 4294967296.0;  // 2^32
constexpr double FAR_LOG_MIN = -1000.0;          // log F below this (F < 1e-434) counts as -1000

// Sample depths of every ray (as the forward computes them) and whether they never decrease.
__global__ void __launch_bounds__(256)
ray_depth_kernel(int W, int H, const long long* __restrict__ header, const float* __restrict__ pixels,
                 const float* __restrict__ ray_o, const float* __restrict__ ray_d, const float* __restrict__ a_ele,
                 const float* __restrict__ pert, float* __restrict__ t_pix, int* __restrict__ mono) {
    const int x = blockIdx.x;
    if (x >= W) return;
    const RayGeo rg = ray_geo(x, ray_o, ray_d, a_ele, pert);
    for (int y = threadIdx.x; y < H; y += blockDim.x) {
        const float* pp = pixels + ((int64_t)x * H + y) * 3;
        const float3 p = make_float3(pp[0], pp[1], pp[2]);
        t_pix[(int64_t)x * H + y] = fmaxf(0.0f, v_dot(v_sub(p, rg.o), rg.d));
    }
    __syncthreads();
    int ok = 1;
    for (int y = threadIdx.x + 1; y < H; y += blockDim.x)
        ok &= t_pix[(int64_t)x * H + y] >= t_pix[(int64_t)x * H + y - 1];
    ok = __syncthreads_and(ok);
    if (threadIdx.x == 0) mono[x] = (header[H_FLAGS] == 0 && ok) ? 1 : 0;
}

// First sample index in [0, H) of a nondecreasing depth array whose depth satisfies pred
// (monotone in the index), H if none.
template <typename Pred>
__device__ __forceinline__ int first_sample(const float* __restrict__ t, int H, Pred pred) {
    int lo = 0, hi = H;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (pred(t[mid])) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// Per instance of a checkpointed ray: depth, echo radius, far factor and first far sample;
// the fixed-point log of the far factor is added to that sample's slot.
__global__ void __launch_bounds__(128)
far_prep_kernel(int W, int H, const int* __restrict__ ray_start, const int* __restrict__ sorted_gid,
                const long long* __restrict__ header, const float4* __restrict__ rec,
                const float* __restrict__ ray_o, const float* __restrict__ ray_d, const float* __restrict__ a_ele,
                const float* __restrict__ pert, const int* __restrict__ mono, const float* __restrict__ t_pix,
                float k_sigma, float wr, float4* __restrict__ aux, long long* __restrict__ far_log) {
    if (header[H_FLAGS] != 0) return;
    const int x = blockIdx.x;
    if (!mono[x]) return;
    const int s0 = ray_start[x], n = ray_start[x + 1] - s0;
    const RayGeo rg = ray_geo(x, ray_o, ray_d, a_ele, pert);
    const float* t = t_pix + (int64_t)x * H;
    for (int k = blockIdx.y * blockDim.x + threadIdx.x; k < n; k += gridDim.y * blockDim.x) {
        Rec r;
        load_rec(rec + (int64_t)REC_F4 * sorted_gid[s0 + k], r);
        const float t_gauss = v_dot(v_sub(r.mu, rg.o), rg.d);
        float tcw = 3.0e38f;
        const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, 3.0e38f, wr, &tcw);
        const float F = r.tau + (1.0f - r.tau) * __expf(-psi);
        const int y_far = first_sample(t, H, [&](float tp) { return tp > 0.0f && tp > t_gauss && tp >= tcw; });
        aux[s0 + k] = make_float4(t_gauss, r.smax * k_sigma, F, __int_as_float(y_far));
        if (y_far < H) {
            const double lf = F > 0.0f ? fmax(log((double)F), FAR_LOG_MIN) : FAR_LOG_MIN;
            atomicAdd(reinterpret_cast<unsigned long long*>(far_log + (int64_t)x * H + y_far),
                      (unsigned long long)llrint(lf * FAR_LOG_SCALE));
        }
    }
}

// Prefix of the fixed-point far logs along each checkpointed ray (one warp per ray) and the
// far transmittance of every sample.
__global__ void __launch_bounds__(32)
far_prefix_kernel(int W, int H, const long long* __restrict__ header, const int* __restrict__ mono,
                  long long* __restrict__ far_log, float* __restrict__ t_far) {
    const int x = blockIdx.x;
    if (x >= W || header[H_FLAGS] != 0 || !mono[x]) return;
    const int lane = threadIdx.x;
    long long carry = 0;
    for (int y0 = 0; y0 < H; y0 += 32) {
        const int y = y0 + lane;
        long long v = y < H ? far_log[(int64_t)x * H + y] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
        }
        v += carry;
        if (y < H) {
            far_log[(int64_t)x * H + y] = v;
            t_far[(int64_t)x * H + y] = (float)exp((double)v / FAR_LOG_SCALE);
        }
        carry = __shfl_sync(0xffffffffu, v, 31);
    }
}

// Forward of a checkpointed ray: block (x, y) shades samples [FWD_SAMPLES y, ...) of ray x.
// The ray's instances that are still inside their window somewhere in the tile, or echo in it,
// are listed in list order (chunks of LIST_CAP), their records staged, and every sample
// multiplies its checkpoint T_far by the window factors of the listed instances it has passed
// but not left (t_gauss < t < tcw) and adds their echo terms, as the reference does.
constexpr int LIST_CAP = 192;
constexpr int SCAN_ROUND = 4;  // chunks of FWD_SAMPLES instances listed per block barrier

__global__ void __launch_bounds__(FWD_SAMPLES)
forward_ckpt_kernel(int W, int H, const int* __restrict__ ray_start, const int* __restrict__ sorted_gid,
                    const long long* __restrict__ header, const float4* __restrict__ rec,
                    const float* __restrict__ pixels, const float* __restrict__ ray_o, const float* __restrict__ ray_d,
                    const float* __restrict__ a_ele, const float* __restrict__ pert, const int* __restrict__ mono,
                    const float* __restrict__ t_pix, const float4* __restrict__ aux, const float* __restrict__ t_far,
                    float wr, float* __restrict__ image, float4* __restrict__ pixel_state) {
    __shared__ float4 s_rec[LIST_CAP * REC_F4];
    __shared__ float4 s_aux[LIST_CAP];
    constexpr int NW = FWD_SAMPLES / 32;
    __shared__ int s_list[LIST_CAP + SCAN_ROUND * FWD_SAMPLES];
    __shared__ int s_cnt[2][SCAN_ROUND * NW];  // kept instances per (chunk, warp), double-buffered
    if (header[H_FLAGS] != 0) return;
    const int x = blockIdx.x;
    if (!mono[x]) return;
    const int y0 = blockIdx.y * FWD_SAMPLES;
    if (y0 >= H) return;
    const int y1 = min(H, y0 + FWD_SAMPLES);
    const int s0 = ray_start[x], n = ray_start[x + 1] - s0;
    const float* t = t_pix + (int64_t)x * H;
    const float t_lo = t[y0], t_hi = t[y1 - 1];
    const RayGeo rg = ray_geo(x, ray_o, ray_d, a_ele, pert);
    const int y = y0 + threadIdx.x;
    const bool valid = y < H;
    float3 p = make_float3(0.f, 0.f, 0.f);
    float t_pixel = 0.f, trans = 1.0f;
    if (valid) {
        const float* pp = pixels + ((int64_t)x * H + y) * 3;
        p = make_float3(pp[0], pp[1], pp[2]);
        t_pixel = t[y];
        trans = t_far[(int64_t)x * H + y];
    }
    float num = 0.0f, den = 0.0f, sacc = 0.0f;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    int nl = 0, par = 0;  // listed instances (the same in every thread), s_cnt buffer
    for (int k0 = 0; k0 < n; k0 += SCAN_ROUND * FWD_SAMPLES) {
        // list the instances of these chunks that matter to the tile (order kept): each chunk's
        // warps count by ballot, one barrier publishes the counts, every thread then knows the
        // offset of its own (chunk, warp) and the new list length
        bool keep[SCAN_ROUND];
        unsigned bits[SCAN_ROUND];
#pragma unroll
        for (int u = 0; u < SCAN_ROUND; ++u) {
            const int k = k0 + u * FWD_SAMPLES + threadIdx.x;
            keep[u] = false;
            if (k < n) {
                const float4 a = aux[s0 + k];
                const int y_far = __float_as_int(a.w);
                keep[u] = (y_far > y0 && a.x < t_hi) || (a.x + a.y >= t_lo && a.x - a.y <= t_hi);
            }
            bits[u] = __ballot_sync(0xffffffffu, keep[u]);
            if (lane == 0) s_cnt[par][u * NW + warp] = __popc(bits[u]);
        }
        __syncthreads();
        int off = nl;
#pragma unroll
        for (int u = 0; u < SCAN_ROUND; ++u) {
            int base = off;
            for (int w2 = 0; w2 < NW; ++w2) {
                const int c = s_cnt[par][u * NW + w2];
                if (w2 < warp) base += c;
                off += c;
            }
            if (keep[u]) s_list[base + __popc(bits[u] & lt_mask)] = k0 + u * FWD_SAMPLES + threadIdx.x;
        }
        nl = off;
        par ^= 1;
        const bool last = k0 + SCAN_ROUND * FWD_SAMPLES >= n;
        if (nl < LIST_CAP && !last) continue;
        __syncthreads();  // the list entries are written
        // stage and shade the listed instances (at most LIST_CAP at a time, in list order)
        for (int b0 = 0; b0 < nl; b0 += LIST_CAP) {
            const int nb = min(LIST_CAP, nl - b0);
            for (int j = threadIdx.x; j < nb * REC_F4; j += blockDim.x) {
                const int e = j / REC_F4, f = j - e * REC_F4;
                s_rec[j] = rec[(int64_t)REC_F4 * sorted_gid[s0 + s_list[b0 + e]] + f];
            }
            for (int e = threadIdx.x; e < nb; e += blockDim.x) s_aux[e] = aux[s0 + s_list[b0 + e]];
            __syncthreads();
            if (valid) {
                for (int e = 0; e < nb; ++e) {
                    const float4 a = s_aux[e];
                    const float t_gauss = a.x;
                    const bool need_t = t_gauss < t_pixel && y < __float_as_int(a.w);  // passed, not yet far
                    const bool need_e = fabsf(t_gauss - t_pixel) <= a.y;
                    if (!need_t && !need_e) continue;
                    Rec r;
                    load_rec(s_rec + e * REC_F4, r);
                    if (need_t) {
                        const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, t_pixel, wr);
                        trans *= r.tau + (1.0f - r.tau) * __expf(-psi);
                    }
                    if (need_e) {
                        const float wgt = gauss_weight(p, r.mu, r.P);
                        const float I = r.sh.x + r.sh.y * rg.d.x + r.sh.z * rg.d.y + r.sh.w * rg.d.z;
                        num += I * wgt;
                        den += wgt;
                        sacc += wgt;
                    }
                }
            }
            __syncthreads();
        }
        nl = 0;
    }
    if (!valid) return;
    float out = 0.0f;
    if (n > 0) {
        const float gamma = 1.0f - __expf(-sacc);
        const float echo = num / (den + 1e-6f);
        out = trans * (gamma * echo);
    }
    image[(int64_t)y * W + x] = out;
    pixel_state[(int64_t)x * H + y] = make_float4(trans, num, den, sacc);
}

// VJP of ray_integral w.r.t. the Gaussian (mean, scales, rotation), the quadrature nodes held
// fixed (reference backward.cu:26-108), accumulated into ds, dmu, dR; l is the pixel depth.
// With wr > 0, *tcw_out (if not NULL) receives the window end tc + wr it uses.
__device__ __forceinline__ void psi_vjp(const RayGeo& rg, const Rec& r, float t_pixel, float wr, float dpsi,
                                        float ds[3], float dmu[3], float dR[9], float* tcw_out = nullptr) {
    if (t_pixel > 0.0f) {
        const float3 diff = v_sub(rg.o, r.mu);
        float3 ol, dl;
        ol.x = r.R[0] * diff.x + r.R[3] * diff.y + r.R[6] * diff.z;
        ol.y = r.R[1] * diff.x + r.R[4] * diff.y + r.R[7] * diff.z;
        ol.z = r.R[2] * diff.x + r.R[5] * diff.y + r.R[8] * diff.z;
        dl.x = r.R[0] * rg.d.x + r.R[3] * rg.d.y + r.R[6] * rg.d.z;
        dl.y = r.R[1] * rg.d.x + r.R[4] * rg.d.y + r.R[7] * rg.d.z;
        dl.z = r.R[2] * rg.d.x + r.R[5] * rg.d.y + r.R[8] * rg.d.z;
        const float3 is = make_float3(1.0f / r.s.x, 1.0f / r.s.y, 1.0f / r.s.z);
        const float3 og = make_float3(ol.x * is.x, ol.y * is.y, ol.z * is.z);
        const float3 dg = make_float3(dl.x * is.x, dl.y * is.y, dl.z * is.z);
        const float dg2 = v_dot(dg, dg);
        const float tc = -v_dot(og, dg) / (dg2 + 1e-8f);
        float ta0 = 0.0f, ta1 = t_pixel;
        if (wr > 0.0f) {
            ta0 = fmaxf(0.0f, tc - wr);
            ta1 = fminf(t_pixel, tc + wr);
            if (tcw_out) *tcw_out = tc + wr;
        }
        if (ta1 > ta0 && dpsi != 0.0f) {
            const float half = 0.5f * (ta1 - ta0), c = 0.5f * (ta1 + ta0);
            const float tn[3] = {half * -0.7745966692f + c, half * 0.0f + c, half * 0.7745966692f + c};
            const float wn[3] = {0.5555555556f, 0.8888888889f, 0.5555555556f};
            const float coeff = dpsi * half;
            float3 gog = make_float3(0.f, 0.f, 0.f), gdg = make_float3(0.f, 0.f, 0.f);
#pragma unroll
            for (int qn = 0; qn < 3; ++qn) {
                const float3 xq = v_add(og, v_mul(dg, tn[qn]));
                const float f = __expf(-0.5f * v_dot(xq, xq));
                gog = v_add(gog, v_mul(xq, -coeff * wn[qn] * f));
                gdg = v_add(gdg, v_mul(xq, -coeff * wn[qn] * f * tn[qn]));
            }
            const float3 gol = make_float3(gog.x * is.x, gog.y * is.y, gog.z * is.z);
            const float3 gdl = make_float3(gdg.x * is.x, gdg.y * is.y, gdg.z * is.z);
            ds[0] += gog.x * (-og.x * is.x) + gdg.x * (-dg.x * is.x);
            ds[1] += gog.y * (-og.y * is.y) + gdg.y * (-dg.y * is.y);
            ds[2] += gog.z * (-og.z * is.z) + gdg.z * (-dg.z * is.z);
            dmu[0] += -(r.R[0] * gol.x + r.R[1] * gol.y + r.R[2] * gol.z);
            dmu[1] += -(r.R[3] * gol.x + r.R[4] * gol.y + r.R[5] * gol.z);
            dmu[2] += -(r.R[6] * gol.x + r.R[7] * gol.y + r.R[8] * gol.z);
            const float dv[3] = {diff.x, diff.y, diff.z}, rv[3] = {rg.d.x, rg.d.y, rg.d.z};
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) {
                dR[rr * 3 + 0] += gol.x * dv[rr] + gdl.x * rv[rr];
                dR[rr * 3 + 1] += gol.y * dv[rr] + gdl.y * rv[rr];
                dR[rr * 3 + 2] += gol.z * dv[rr] + gdl.z * rv[rr];
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// Backward
// ------------------------------------------------------------------------------------

// End of an instance's backward: the far-field VJP applied once with the summed scalar adjoint
// far_dT, dL/dP (symmetric sum over pixels) -> dL/dR, dL/ds, dL/dR -> dL/dq, and the partial.
__device__ __forceinline__ void instance_epilogue(const RayGeo& rg, const Rec& r, float wr, float far_dT, float far_exp,
                                                  float dP[9], float dR[9], float ds[3], float dmu[3], float dtau_raw,
                                                  const float dsh[4], const float* __restrict__ quats, int g,
                                                  float4* __restrict__ out) {
    if (far_dT != 0.0f) {
        dtau_raw += far_dT * (1.0f - far_exp) * (r.tau * (1.0f - r.tau));
        psi_vjp(rg, r, 3.0e38f, wr, far_dT * (1.0f - r.tau) * far_exp * (-1.0f), ds, dmu, dR);
    }
    dP[3] = dP[1];
    dP[6] = dP[2];
    dP[7] = dP[5];
    {
        const float d[3] = {1.f / (r.s.x * r.s.x), 1.f / (r.s.y * r.s.y), 1.f / (r.s.z * r.s.z)};
#pragma unroll
        for (int rr = 0; rr < 3; ++rr)
#pragma unroll
            for (int kk = 0; kk < 3; ++kk)
                dR[rr * 3 + kk] += 2.0f * (dP[rr * 3 + 0] * r.R[kk] + dP[rr * 3 + 1] * r.R[3 + kk] + dP[rr * 3 + 2] * r.R[6 + kk]) * d[kk];
        const float sv[3] = {r.s.x, r.s.y, r.s.z};
#pragma unroll
        for (int kk = 0; kk < 3; ++kk) {
            float a = 0.f;
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) a += r.R[i * 3 + kk] * dP[i * 3 + j] * r.R[j * 3 + kk];
            ds[kk] += -2.f * a * d[kk] / sv[kk];
        }
    }
    const float4 q = make_float4(quats[4 * (int64_t)g], quats[4 * (int64_t)g + 1], quats[4 * (int64_t)g + 2],
                                 quats[4 * (int64_t)g + 3]);
    const float4 dq = quat_grad(q, dR);
    out[0] = make_float4(dmu[0], dmu[1], dmu[2], dtau_raw);
    out[1] = make_float4(ds[0], ds[1], ds[2], dsh[0]);
    out[2] = make_float4(dsh[1], dsh[2], dsh[3], 0.f);
    out[3] = dq;
}

// One instance's transmission term at a sample inside its window, and its echo term.
__device__ __forceinline__ void near_terms(const RayGeo& rg, const Rec& r, float wr, const float4 pt, const float4 cf,
                                           bool need_t, bool need_e, float dP[9], float dR[9], float ds[3],
                                           float dmu[3], float& dtau_raw, float dsh[4]) {
    const float t_pixel = pt.w;
    if (need_t) {
        const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, t_pixel, wr);
        const float exp_psi = __expf(-psi);
        const float T_i = r.tau + (1.0f - r.tau) * exp_psi;
        float dTi = 0.0f;
        if (T_i > 1e-6f) dTi = cf.x * (cf.y / T_i);
        dtau_raw += dTi * (1.0f - exp_psi) * (r.tau * (1.0f - r.tau));
        const float dpsi = dTi * (1.0f - r.tau) * exp_psi * (-1.0f);
        psi_vjp(rg, r, t_pixel, wr, dpsi, ds, dmu, dR);
    }
    if (need_e) {
        const float3 p = make_float3(pt.x, pt.y, pt.z);
        const float wgt = gauss_weight(p, r.mu, r.P);
        const float I = r.sh.x + r.sh.y * rg.d.x + r.sh.z * rg.d.y + r.sh.w * rg.d.z;
        const float a = cf.z * wgt;
        dsh[0] += a;
        dsh[1] += a * rg.d.x;
        dsh[2] += a * rg.d.y;
        dsh[3] += a * rg.d.z;
        const float dw = (cf.z * I) + cf.w;
        const float dQ = dw * wgt * (-0.5f);
        const float dx = p.x - r.mu.x, dy = p.y - r.mu.y, dz = p.z - r.mu.z;
        const float v0 = r.P[0] * dx + r.P[1] * dy + r.P[2] * dz;
        const float v1 = r.P[3] * dx + r.P[4] * dy + r.P[5] * dz;
        const float v2 = r.P[6] * dx + r.P[7] * dy + r.P[8] * dz;
        dmu[0] += dQ * (-2.0f * v0);
        dmu[1] += dQ * (-2.0f * v1);
        dmu[2] += dQ * (-2.0f * v2);
        const float ux = dQ * dx, uy = dQ * dy, uz = dQ * dz;
        dP[0] += ux * dx; dP[1] += ux * dy; dP[2] += ux * dz;
        dP[4] += uy * dy; dP[5] += uy * dz;
        dP[8] += uz * dz;
    }
}

// Backward of a checkpointed ray, per sample: the adjoint coefficients the per-sample path
// stages (zero for samples whose |dL/dB| < 1e-6, which the reference skips), and the suffix sums
// along the ray of dL/dT * T (in double, fixed order; one warp per ray).
__global__ void __launch_bounds__(32)
ckpt_coef_kernel(int W, int H, const long long* __restrict__ header, const int* __restrict__ mono,
                 const float* __restrict__ pixels, const float* __restrict__ t_pix,
                 const float4* __restrict__ pixel_state, const float* __restrict__ grad_image,
                 float4* __restrict__ b_pos, float4* __restrict__ b_coef, float* __restrict__ b_suffix) {
    const int x = blockIdx.x;
    if (x >= W || header[H_FLAGS] != 0 || !mono[x]) return;
    const int lane = threadIdx.x;
    double carry = 0.0;
    const int nchunks = (H + 31) / 32;
    for (int c = nchunks - 1; c >= 0; --c) {  // from the deepest samples up: suffix sums
        const int y = c * 32 + lane;
        double v = 0.0;
        if (y < H) {
            const int64_t pi = (int64_t)x * H + y;
            const float* pp = pixels + pi * 3;
            const float gB = grad_image[(int64_t)y * W + x];
            const float4 st = pixel_state[pi];  // T, num, den, S
            const float gamma = 1.0f - __expf(-st.w);
            const float eps = 1e-6f;
            const float e_raw = st.y / (st.z + eps);
            const float e_val = gamma * e_raw;
            const float dT = gB * e_val;
            const float dE = gB * st.x;
            const float dgam = dE * e_raw;
            const float de_raw = dE * gamma;
            const float dS = dgam * __expf(-st.w);
            const float dnum = de_raw * (1.0f / (st.z + eps));
            const float dden = de_raw * (-st.y / ((st.z + eps) * (st.z + eps)));
            const bool active = !(fabsf(gB) < 1e-6f);
            b_pos[pi] = make_float4(pp[0], pp[1], pp[2], t_pix[pi]);
            b_coef[pi] = active ? make_float4(dT, st.x, dnum, dden + dS) : make_float4(0.f, 0.f, 0.f, 0.f);
            v = active ? (double)dT * (double)st.x : 0.0;
        }
        // inclusive suffix within the chunk: lane l sums lanes l..31
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double u = __shfl_down_sync(0xffffffffu, v, o);
            if (lane + o < 32) v += u;
        }
        v += carry;
        if (y < H) b_suffix[(int64_t)x * H + y] = (float)v;
        carry = __shfl_sync(0xffffffffu, v, 0);
    }
}

// Thread per instance of a checkpointed ray: the far part of its gradient from the suffix sum at
// its first far sample, the samples inside its window [first sample past t_gauss, first far
// sample) and its echo range |t - t_gauss| <= radius visited in sample order. The ray's
// instances go out in chunks of CKPT_CHUNK; a block first finds each instance's sample range and
// then hands the instances to its threads in order of that range's length (a counting sort on
// CKPT_BINS classes), so that the lanes of a warp sweep similar numbers of samples. Which thread
// computes an instance does not change its partial.
constexpr int CKPT_CHUNK = 512;
constexpr int CKPT_BINS = 32;  // classes of 8 samples
__global__ void __launch_bounds__(128)
backward_ckpt_kernel(int W, int H, const int* __restrict__ ray_start, const int* __restrict__ sorted_gid,
                     const int* __restrict__ sorted_inst, const long long* __restrict__ header,
                     const float4* __restrict__ rec, const float* __restrict__ quats, const float* __restrict__ ray_o,
                     const float* __restrict__ ray_d, const float* __restrict__ a_ele, const float* __restrict__ pert,
                     const int* __restrict__ mono, const float* __restrict__ t_pix, const float4* __restrict__ aux,
                     const float4* __restrict__ b_pos, const float4* __restrict__ b_coef,
                     const float* __restrict__ b_suffix, float wr, float4* __restrict__ partial) {
    __shared__ int s_key[CKPT_CHUNK];  // length class << 16 | rank within the class
    __shared__ int s_ord[CKPT_CHUNK];  // chunk positions ordered by class
    __shared__ int s_yt[CKPT_CHUNK], s_ya[CKPT_CHUNK], s_yb[CKPT_CHUNK];
    __shared__ int s_bin[CKPT_BINS];
    if (header[H_FLAGS] != 0) return;
    const int x = blockIdx.x;
    if (!mono[x]) return;
    const int s0 = ray_start[x], n = ray_start[x + 1] - s0;
    const RayGeo rg = ray_geo(x, ray_o, ray_d, a_ele, pert);
    const float* t = t_pix + (int64_t)x * H;
    const int64_t row = (int64_t)x * H;
    for (int k0 = blockIdx.y * CKPT_CHUNK; k0 < n; k0 += gridDim.y * CKPT_CHUNK) {
        const int nc = min(CKPT_CHUNK, n - k0);
        __syncthreads();  // the previous chunk's arrays are read to the end
        if (threadIdx.x < CKPT_BINS) s_bin[threadIdx.x] = 0;
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            const float4 a = aux[s0 + k0 + j];
            const float t_gauss = a.x, radius = a.y;
            const int y_far = __float_as_int(a.w);
            const int y_t = first_sample(t, H, [&](float tp) { return tp > t_gauss; });
            const int y_e0 = first_sample(t, H, [&](float tp) { return tp >= t_gauss - radius; });
            const int y_e1 = first_sample(t, H, [&](float tp) { return tp > t_gauss + radius; });
            const int ya = min(y_t, y_e0), yb = max(y_far, y_e1);
            s_yt[j] = y_t;
            s_ya[j] = ya;
            s_yb[j] = yb;
            const int bin = min(CKPT_BINS - 1, max(yb - ya, 0) >> 3);
            s_key[j] = (bin << 16) | atomicAdd(&s_bin[bin], 1);
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // exclusive scan of the class counts in one warp
            const int v = s_bin[threadIdx.x];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)threadIdx.x >= o) incl += u;
            }
            s_bin[threadIdx.x] = incl - v;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            const int key = s_key[j];
            s_ord[s_bin[key >> 16] + (key & 0xffff)] = j;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < nc; q += blockDim.x) {
            const int j = s_ord[q], k = k0 + j;
            Rec r;
            const int g = sorted_gid[s0 + k];
            load_rec(rec + (int64_t)REC_F4 * g, r);
            const float4 a = aux[s0 + k];
            const float t_gauss = a.x, radius = a.y;
            const int y_far = __float_as_int(a.w);
            float dmu[3] = {0.f, 0.f, 0.f}, ds[3] = {0.f, 0.f, 0.f}, dR[9], dP[9], dtau_raw = 0.f;
            float dsh[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                dR[i] = 0.f;
                dP[i] = 0.f;
            }
            // the far factor, as the per-sample path evaluates it
            const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, 3.0e38f, wr);
            const float far_exp = __expf(-psi);
            const float far_T = r.tau + (1.0f - r.tau) * far_exp;
            const int y_t = s_yt[j], ya = s_ya[j], yb = s_yb[j];
            for (int y = ya; y < yb; ++y) {
                const float4 cf = b_coef[row + y];
                if (cf.x == 0.0f && cf.z == 0.0f && cf.w == 0.0f) continue;  // skipped sample: every term is zero
                const float4 pt = b_pos[row + y];
                const bool need_t = y >= y_t && y < y_far;
                const bool need_e = fabsf(t_gauss - pt.w) <= radius;
                if (need_t || need_e) near_terms(rg, r, wr, pt, cf, need_t, need_e, dP, dR, ds, dmu, dtau_raw, dsh);
            }
            float far_dT = 0.0f;
            if (y_far < H && far_T > 1e-6f) far_dT = b_suffix[row + y_far] / far_T;
            instance_epilogue(rg, r, wr, far_dT, far_exp, dP, dR, ds, dmu, dtau_raw, dsh, quats, g,
                              partial + (int64_t)PARTIAL_F4 * sorted_inst[s0 + k]);
        }
    }
}

// Blocks (x, *) share ray x's instances; a thread owns one instance at a time and sweeps
// the ray's pixels in chunks whose adjoint coefficients are staged in shared memory
// (reference backward.cu:138-325).
__global__ void __launch_bounds__(128)
backward_kernel(int W, int H, const int* __restrict__ ray_start, const int* __restrict__ sorted_gid,
                const int* __restrict__ sorted_inst, const long long* __restrict__ header,
                const float4* __restrict__ rec, const float* __restrict__ quats, const float* __restrict__ pixels,
                const float* __restrict__ ray_o, const float* __restrict__ ray_d, const float* __restrict__ a_ele,
                const float* __restrict__ pert, const uint32_t* __restrict__ dkey,
                const float4* __restrict__ pixel_state, const float* __restrict__ grad_image, float k_sigma,
                float wr, int local_only, float max_win, const int* __restrict__ ckpt_rays,
                float4* __restrict__ partial) {
    __shared__ float4 s_p[PIX_CHUNK];   // pixel position, t_pixel
    __shared__ float4 s_c[PIX_CHUNK];   // dL/dT, T_final, dL/dnum, dL/dw_common (den + gamma terms)
    __shared__ int s_active[PIX_CHUNK];
    if (header[H_FLAGS] != 0) return;
    const int x = blockIdx.x;
    if (ckpt_rays && ckpt_rays[x]) return;  // differentiated by the checkpointed path
    const int s0 = ray_start[x], n = ray_start[x + 1] - s0;
    if (n <= 0) return;
    const RayGeo rg = ray_geo(x, ray_o, ray_d, a_ele, pert);
    // blocks (x, y) share ray x's instances: block y takes rounds y, y + gridDim.y, ...
    for (int kb = blockIdx.y * blockDim.x; kb < n; kb += gridDim.y * blockDim.x) {
        const int k = kb + threadIdx.x;
        const bool own = k < n;
        Rec r;
        float dmu[3] = {0.f, 0.f, 0.f}, ds[3] = {0.f, 0.f, 0.f}, dR[9], dP[9], dtau_raw = 0.f;
        float dsh[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            dR[i] = 0.f;
            dP[i] = 0.f;
        }
        float t_gauss = 0.f, depth_radius = -1.f, depth = 0.f;
        // far field (wr > 0, pixel past both window ends): constant factor and VJP
        float far_tcw = 3.0e38f, far_tcw_vjp = 3.0e38f, far_T = 1.0f, far_exp = 1.0f, far_dT = 0.0f;
        if (own) {
            const int gk = sorted_gid[s0 + k];
            load_rec(rec + (int64_t)REC_F4 * gk, r);
            depth = (float)dkey[gk] * 0.001f;
            t_gauss = v_dot(v_sub(r.mu, rg.o), rg.d);
            depth_radius = r.smax * k_sigma;
            if (wr > 0.0f) {
                const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, 3.0e38f, wr, &far_tcw);
                far_exp = __expf(-psi);
                far_T = r.tau + (1.0f - r.tau) * far_exp;
                psi_vjp(rg, r, 3.0e38f, wr, 0.0f, ds, dmu, dR, &far_tcw_vjp);
            }
        }
        for (int y0 = 0; y0 < H; y0 += PIX_CHUNK) {
            const int ny = min(PIX_CHUNK, H - y0);
            __syncthreads();
            for (int j = threadIdx.x; j < ny; j += blockDim.x) {
                const int y = y0 + j;
                const float* pp = pixels + ((int64_t)x * H + y) * 3;
                const float3 p = make_float3(pp[0], pp[1], pp[2]);
                const float t_pixel = fmaxf(0.0f, v_dot(v_sub(p, rg.o), rg.d));
                const float gB = grad_image[(int64_t)y * W + x];
                const float4 st = pixel_state[(int64_t)x * H + y];  // T, num, den, S
                const float gamma = 1.0f - __expf(-st.w);
                const float eps = 1e-6f;
                const float e_raw = st.y / (st.z + eps);
                const float e_val = gamma * e_raw;
                const float dT = gB * e_val;
                const float dE = gB * st.x;
                const float dgam = dE * e_raw;
                const float de_raw = dE * gamma;
                const float dS = dgam * __expf(-st.w);
                const float dnum = de_raw * (1.0f / (st.z + eps));
                const float dden = de_raw * (-st.y / ((st.z + eps) * (st.z + eps)));
                s_p[j] = make_float4(p.x, p.y, p.z, t_pixel);
                s_c[j] = make_float4(dT, st.x, dnum, dden + dS);
                s_active[j] = !(fabsf(gB) < 1e-6f);
            }
            __syncthreads();
            if (!own) continue;
            for (int j = 0; j < ny; ++j) {
                if (!s_active[j]) continue;
                const float4 pt = s_p[j];
                const float t_pixel = pt.w;
                if (local_only && !in_local_window(depth, t_pixel, max_win)) continue;
                bool need_t = t_gauss < t_pixel;
                if (local_only) need_t = need_t && ((t_pixel - t_gauss) <= depth_radius + wr);
                const bool need_e = fabsf(t_gauss - t_pixel) <= depth_radius;
                if (!need_t && !need_e) continue;
                const float4 cf = s_c[j];
                if (need_t && t_pixel > 0.0f && t_pixel >= far_tcw && t_pixel >= far_tcw_vjp) {
                    // past both window ends: the factor and its VJP are the instance's constants,
                    // so only the scalar adjoint is summed here (applied once after the sweep)
                    if (far_T > 1e-6f) far_dT += cf.x * (cf.y / far_T);
                } else if (need_t) {
                    const float psi = ray_integral(rg.o, rg.d, r.mu, r.s, r.R, t_pixel, wr);
                    const float exp_psi = __expf(-psi);
                    const float T_i = r.tau + (1.0f - r.tau) * exp_psi;
                    float dTi = 0.0f;
                    if (T_i > 1e-6f) dTi = cf.x * (cf.y / T_i);
                    dtau_raw += dTi * (1.0f - exp_psi) * (r.tau * (1.0f - r.tau));
                    const float dpsi = dTi * (1.0f - r.tau) * exp_psi * (-1.0f);
                    // integral VJP with the quadrature nodes held fixed (reference backward.cu:26-108)
                    psi_vjp(rg, r, t_pixel, wr, dpsi, ds, dmu, dR);
                }
                if (need_e) {
                    const float3 p = make_float3(pt.x, pt.y, pt.z);
                    const float wgt = gauss_weight(p, r.mu, r.P);
                    const float I = r.sh.x + r.sh.y * rg.d.x + r.sh.z * rg.d.y + r.sh.w * rg.d.z;
                    const float a = cf.z * wgt;
                    dsh[0] += a;
                    dsh[1] += a * rg.d.x;
                    dsh[2] += a * rg.d.y;
                    dsh[3] += a * rg.d.z;
                    const float dw = (cf.z * I) + cf.w;
                    const float dQ = dw * wgt * (-0.5f);
                    const float dx = p.x - r.mu.x, dy = p.y - r.mu.y, dz = p.z - r.mu.z;
                    const float v0 = r.P[0] * dx + r.P[1] * dy + r.P[2] * dz;
                    const float v1 = r.P[3] * dx + r.P[4] * dy + r.P[5] * dz;
                    const float v2 = r.P[6] * dx + r.P[7] * dy + r.P[8] * dz;
                    dmu[0] += dQ * (-2.0f * v0);
                    dmu[1] += dQ * (-2.0f * v1);
                    dmu[2] += dQ * (-2.0f * v2);
                    const float ux = dQ * dx, uy = dQ * dy, uz = dQ * dz;
                    dP[0] += ux * dx; dP[1] += ux * dy; dP[2] += ux * dz;
                    dP[4] += uy * dy; dP[5] += uy * dz;
                    dP[8] += uz * dz;
                }
            }
        }
        if (!own) continue;
        instance_epilogue(rg, r, wr, far_dT, far_exp, dP, dR, ds, dmu, dtau_raw, dsh, quats, sorted_gid[s0 + k],
                          partial + (int64_t)PARTIAL_F4 * sorted_inst[s0 + k]);
    }
}

// Per-Gaussian gradient: the sum of its instances' partial records in instance order.
// REDUCE_COLS threads per Gaussian, thread f summing float4 column f, so that a Gaussian's
// threads read each record together and many Gaussians' loads are in flight; the sums are the
// ones a thread summing all columns would form.
constexpr int REDUCE_COLS = 4;
constexpr int REDUCE_THREADS = 64 * REDUCE_COLS;  // 64 Gaussians per block
__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_kernel(int64_t G, const int* __restrict__ inst_offset, const long long* __restrict__ header,
              const float4* __restrict__ partial, float* __restrict__ d_means, float* __restrict__ d_scales,
              float* __restrict__ d_quats, float* __restrict__ d_attens, float* __restrict__ d_sh) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g = t / REDUCE_COLS;
    const int f = (int)(t % REDUCE_COLS);
    if (g >= G) return;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    if (header[H_FLAGS] == 0) {
        const int i1 = inst_offset[g + 1];
        int i = inst_offset[g];
        for (; i + 4 <= i1; i += 4) {  // four instances' loads in flight, summed in order
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = partial[(int64_t)PARTIAL_F4 * (i + u) + f];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a.x += v[u].x; a.y += v[u].y; a.z += v[u].z; a.w += v[u].w;
            }
        }
        for (; i < i1; ++i) {
            const float4 v = partial[(int64_t)PARTIAL_F4 * i + f];
            a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
        }
    }
    if (f == 0) {
        d_means[3 * g] = a.x; d_means[3 * g + 1] = a.y; d_means[3 * g + 2] = a.z;
        d_attens[g] = a.w;
    } else if (f == 1) {
        d_scales[3 * g] = a.x; d_scales[3 * g + 1] = a.y; d_scales[3 * g + 2] = a.z;
        d_sh[4 * g] = a.w;
    } else if (f == 2) {
        d_sh[4 * g + 1] = a.x; d_sh[4 * g + 2] = a.y; d_sh[4 * g + 3] = a.z;
    } else {
        d_quats[4 * g] = a.x; d_quats[4 * g + 1] = a.y; d_quats[4 * g + 2] = a.z; d_quats[4 * g + 3] = a.w;
    }
}

// Reference-format CSR of the ray binning (MapperForwardCUDA outputs, wrapper_mapper.cu:119-127).
__global__ void export_kernel(int W, const int* __restrict__ ray_start, const unsigned long long* __restrict__ keys,
                              const int* __restrict__ sorted_gid, int* __restrict__ counts, int* __restrict__ offsets,
                              int* __restrict__ indices, float* __restrict__ depths) {
    const int x = blockIdx.x;
    if (x >= W) return;
    const int s0 = ray_start[x], s1 = ray_start[x + 1];
    if (threadIdx.x == 0) {
        counts[x] = s1 - s0;
        offsets[x] = (s1 > s0) ? s0 : 0;
    }
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        indices[s] = sorted_gid[s];
        depths[s] = ((float)(uint32_t)(keys[s] >> 32)) * 0.001f;
    }
}

}  // namespace ugr
}  // namespace us3d

using namespace us3d;
using namespace us3d::ugr;

static bool g_ugr_sort_attr[128];

// The transmittance checkpoints apply with a quadrature window (its far factor is constant) and
// full transmission (the local-window mode bounds the product differently); forward and
// backward take the same decision from the same arguments.
static inline bool uses_checkpoints(int H, float wr, int local_only) { return H > 0 && wr > 0.0f && !local_only; }

// Blocks per ray for the per-instance kernels: enough to give every SM several (a frame has few rays).
static inline unsigned per_ray_blocks(int W) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(64, (148 * 8 + W - 1) / std::max<int64_t>(W, 1)));
}

extern "C" size_t us3d_ugr_workspace_bytes(int64_t n_gauss, int32_t W, int32_t H, int64_t cap) {
    if (n_gauss < 0 || W <= 0 || H < 0 || cap < 0) return 0;
    return carve(nullptr, n_gauss, W, (int64_t)W * H, cap).bytes;
}

extern "C" size_t us3d_ugr_backward_scratch_bytes(int64_t cap) {
    return cap < 0 ? 0 : (size_t)cap * PARTIAL_F4 * sizeof(float4);
}

extern "C" int us3d_ugr_forward(void* workspace, size_t workspace_bytes, int64_t n_gauss, const float* means,
                                const float* scales, const float* quats, const float* attenuations,
                                const float* sh_coeffs, const float* pixel_positions, const float* ray_origins,
                                const float* ray_dirs, const float* origin, const float* axis_lat,
                                const float* axis_ele, const float* axis_ax, const float* ray_perturbations,
                                int32_t W, int32_t H, float width_mm, float near_mm, float lateral_col_offset,
                                float elev_cutoff_mm, float k_sigma, float quadrature_window_radius_mm,
                                int32_t local_window_only, float local_max_window_mm, int64_t cap,
                                float* out_image, void* stream_) {
    US3D_CHECK_ARG(W > 0 && H >= 0, "image_width/image_height must be positive");
    US3D_CHECK_ARG(width_mm > 0.f && k_sigma > 0.f, "width_mm and k_sigma must be > 0");
    US3D_CHECK_ARG(n_gauss >= 0 && n_gauss <= 0x7fffffffLL, "n_gauss out of range");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(workspace && out_image && ray_origins && ray_dirs && origin && axis_lat && axis_ele && axis_ax &&
                   ray_perturbations && (H == 0 || pixel_positions), "NULL pointer argument");
    US3D_CHECK_ARG(n_gauss == 0 || (means && scales && quats && attenuations && sh_coeffs), "NULL parameter pointer");
    const int64_t P = (int64_t)W * H;
    const Workspace w = carve(workspace, n_gauss, W, P, cap);
    US3D_CHECK_ARG(workspace_bytes >= w.bytes, "workspace too small: %zu < %zu", workspace_bytes, w.bytes);
    cudaStream_t stream = (cudaStream_t)stream_;
    const int prof = prof_begin("ugr_forward", stream);
    init_kernel<<<(unsigned)((W + 255) / 256), 256, 0, stream>>>(W, w.ray_count, w.ray_cursor, w.header, cap, n_gauss, P);
    const unsigned gb = (unsigned)((n_gauss + 255) / 256);
    const float spacing = width_mm / (float)W;
    if (n_gauss > 0)
        preprocess_kernel<<<gb, 256, 0, stream>>>(n_gauss, W, spacing, lateral_col_offset, near_mm, elev_cutoff_mm,
                                                  k_sigma, means, scales, quats, attenuations, sh_coeffs, origin,
                                                  axis_lat, axis_ele, axis_ax, w.ray_range, w.dkey, w.touched,
                                                  w.ray_count, w.rec);
    US3D_CHECK_LAUNCH("ugr preprocess");
    US3D_CHECK_CUDA(launch_rect_count(n_gauss, W, W, RangeOf2{w.ray_range}, w.ray_count, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.touched, n_gauss, w.inst_offset, w.bs_g, w.header + H_SCAN_G, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.ray_count, W, w.ray_start, w.bs_t, w.header + H_SCAN_T, stream));
    check_kernel<<<1, 1, 0, stream>>>(w.header, cap);
    US3D_CHECK_CUDA(launch_rect_scatter(n_gauss, W, W, RangeOf2{w.ray_range}, w.dkey, w.inst_offset, w.ray_start,
                                        w.ray_cursor, w.header, w.keys, w.slot_inst, stream));
    US3D_CHECK_CUDA(launch_tile_sort(W, n_gauss, w.ray_start, w.header, w.keys, w.slot_inst, w.sorted_gid, w.sorted_inst,
                                     g_ugr_sort_attr, stream));
    const unsigned tiles_y = (unsigned)((H + FWD_SAMPLES - 1) / FWD_SAMPLES);
    const int* ckpt_rays = nullptr;
    int launches = 1 + 3 * (n_gauss > 0) + 6 + 1 + tile_sort_launches(n_gauss) + 1;
    if (uses_checkpoints(H, quadrature_window_radius_mm, local_window_only)) {
        const unsigned by = per_ray_blocks(W);
        ray_depth_kernel<<<(unsigned)W, 256, 0, stream>>>(W, H, w.header, pixel_positions, ray_origins, ray_dirs,
                                                          axis_ele, ray_perturbations, w.t_pix, w.mono);
        US3D_CHECK_CUDA(cudaMemsetAsync(w.far_log, 0, sizeof(long long) * (size_t)P, stream));
        far_prep_kernel<<<dim3((unsigned)W, by), 128, 0, stream>>>(W, H, w.ray_start, w.sorted_gid, w.header, w.rec,
                                                                  ray_origins, ray_dirs, axis_ele, ray_perturbations,
                                                                  w.mono, w.t_pix, k_sigma, quadrature_window_radius_mm,
                                                                  w.aux, w.far_log);
        far_prefix_kernel<<<(unsigned)W, 32, 0, stream>>>(W, H, w.header, w.mono, w.far_log, w.t_far);
        forward_ckpt_kernel<<<dim3((unsigned)W, tiles_y), FWD_SAMPLES, 0, stream>>>(
            W, H, w.ray_start, w.sorted_gid, w.header, w.rec, pixel_positions, ray_origins, ray_dirs, axis_ele,
            ray_perturbations, w.mono, w.t_pix, w.aux, w.t_far, quadrature_window_radius_mm, out_image,
            w.pixel_state);
        US3D_CHECK_LAUNCH("ugr checkpointed forward");
        ckpt_rays = w.mono;
        launches += 4;
    }
    forward_kernel<<<dim3((unsigned)W, tiles_y), FWD_SAMPLES, 0, stream>>>(W, H, w.ray_start, w.sorted_gid, w.header, w.rec, pixel_positions,
                                                    ray_origins, ray_dirs, axis_ele, ray_perturbations, w.dkey,
                                                    k_sigma, quadrature_window_radius_mm, local_window_only ? 1 : 0,
                                                    local_max_window_mm, ckpt_rays, out_image, w.pixel_state);
    US3D_CHECK_LAUNCH("ugr forward");
    prof_end(prof, stream);
    count_launches(launches);
    return US3D_OK;
}

extern "C" int us3d_ugr_read_status(const void* workspace, int64_t* total, int32_t* flags, void* stream_) {
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    long long hdr[H_WORDS];
    cudaStream_t stream = (cudaStream_t)stream_;
    US3D_CHECK_CUDA(cudaMemcpyAsync(hdr, workspace, sizeof(hdr), cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
    if (total) *total = hdr[H_TOTAL];
    if (flags) *flags = (int32_t)hdr[H_FLAGS];
    return US3D_OK;
}

extern "C" int us3d_ugr_backward(void* workspace, int64_t n_gauss, const float* quats, const float* pixel_positions,
                                 const float* ray_origins, const float* ray_dirs, const float* axis_ele,
                                 const float* ray_perturbations, int32_t W, int32_t H, float k_sigma,
                                 float quadrature_window_radius_mm, int32_t local_window_only,
                                 float local_max_window_mm, int64_t cap, const float* grad_image,
                                 void* scratch, size_t scratch_bytes, float* d_means, float* d_scales, float* d_quats,
                                 float* d_attenuations, float* d_sh, void* stream_) {
    US3D_CHECK_ARG(W > 0 && H >= 0 && n_gauss >= 0 && cap >= 0, "bad sizes");
    US3D_CHECK_ARG(workspace && grad_image && ray_origins && ray_dirs && axis_ele && ray_perturbations,
                   "NULL pointer argument");
    US3D_CHECK_ARG(scratch_bytes >= us3d_ugr_backward_scratch_bytes(cap), "backward scratch too small");
    US3D_CHECK_ARG(n_gauss == 0 || (quats && d_means && d_scales && d_quats && d_attenuations && d_sh),
                   "NULL gradient pointer");
    const int64_t P = (int64_t)W * H;
    const Workspace w = carve(workspace, n_gauss, W, P, cap);
    cudaStream_t stream = (cudaStream_t)stream_;
    float4* partial = reinterpret_cast<float4*>(scratch);
    const int prof = prof_begin("ugr_backward", stream);
    const unsigned by = per_ray_blocks(W);
    const int* ckpt_rays = nullptr;
    int launches = 1 + (n_gauss > 0);
    if (uses_checkpoints(H, quadrature_window_radius_mm, local_window_only)) {
        ckpt_coef_kernel<<<(unsigned)W, 32, 0, stream>>>(W, H, w.header, w.mono, pixel_positions, w.t_pix,
                                                         w.pixel_state, grad_image, w.b_pos, w.b_coef, w.b_suffix);
        backward_ckpt_kernel<<<dim3((unsigned)W, by), 128, 0, stream>>>(
            W, H, w.ray_start, w.sorted_gid, w.sorted_inst, w.header, w.rec, quats, ray_origins, ray_dirs, axis_ele,
            ray_perturbations, w.mono, w.t_pix, w.aux, w.b_pos, w.b_coef, w.b_suffix, quadrature_window_radius_mm,
            partial);
        US3D_CHECK_LAUNCH("ugr checkpointed backward");
        ckpt_rays = w.mono;
        launches += 2;
    }
    backward_kernel<<<dim3((unsigned)W, by), 128, 0, stream>>>(W, H, w.ray_start, w.sorted_gid, w.sorted_inst, w.header, w.rec,
                                                     quats, pixel_positions, ray_origins, ray_dirs, axis_ele,
                                                     ray_perturbations, w.dkey, w.pixel_state, grad_image, k_sigma,
                                                     quadrature_window_radius_mm, local_window_only ? 1 : 0,
                                                     local_max_window_mm, ckpt_rays, partial);
    if (n_gauss > 0)
        reduce_kernel<<<(unsigned)((n_gauss * REDUCE_COLS + REDUCE_THREADS - 1) / REDUCE_THREADS), REDUCE_THREADS, 0,
                        stream>>>(n_gauss, w.inst_offset, w.header, partial, d_means, d_scales, d_quats,
                                  d_attenuations, d_sh);
    US3D_CHECK_LAUNCH("ugr backward");
    prof_end(prof, stream);
    count_launches(launches);
    return US3D_OK;
}

extern "C" int us3d_ugr_export_csr(const void* workspace, int64_t n_gauss, int32_t W, int32_t H, int64_t cap,
                                   int32_t* out_counts, int32_t* out_offsets, int32_t* out_indices,
                                   float* out_sorted_depths, void* stream_) {
    US3D_CHECK_ARG(workspace && out_counts && out_offsets && W > 0, "bad argument");
    const Workspace w = carve(const_cast<void*>(workspace), n_gauss, W, (int64_t)W * H, cap);
    export_kernel<<<(unsigned)W, 256, 0, (cudaStream_t)stream_>>>(W, w.ray_start, w.keys, w.sorted_gid, out_counts,
                                                                  out_offsets, out_indices, out_sorted_depths);
    US3D_CHECK_LAUNCH("ugr export");
    count_launches(1);
    return US3D_OK;
}
