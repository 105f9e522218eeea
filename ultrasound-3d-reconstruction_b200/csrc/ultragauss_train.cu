// The training step around the UltraGauss renderer: the per-frame image loss of the
// reference's training loop (L1 + global SSIM, pipeline_god_file.py:606-637) reduced per frame
// into the coefficients of its gradient (consumed inside the backward kernel), and one
// multi-tensor Adam launch with the logistic activation's chain rule fused in
// (torch.optim.Adam over GaussianParameters, pipeline_god_file.py:740,764).
#include <algorithm>
#include <cmath>

#include "us3d_common.cuh"

namespace us3d {
namespace train {

constexpr int LOSS_BLOCKS = 64;     // partial-sum blocks per frame (fixed: deterministic order)
constexpr int LOSS_THREADS = 256;
constexpr int LOSS_TERMS = 6;       // sum x, sum y, sum x^2, sum y^2, sum xy, sum |x - y|

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block (b, f): partial sums over the pixels b, b + LOSS_BLOCKS * LOSS_THREADS, ... of frame f,
// in a fixed order (thread stride, then warp shuffles, then warps in order).
__global__ void __launch_bounds__(LOSS_THREADS)
loss_partial_kernel(const us3d_slice_frame* __restrict__ frames, int64_t P, const float* __restrict__ image,
                    const float* __restrict__ target, double* __restrict__ partial) {
    __shared__ double s[LOSS_THREADS / 32][LOSS_TERMS];
    const int f = blockIdx.y;
    const int64_t off = frames[f].pixel_offset;
    const int64_t n = (int64_t)frames[f].height * frames[f].width;
    double a[LOSS_TERMS] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int64_t i = (int64_t)blockIdx.x * LOSS_THREADS + threadIdx.x; i < n; i += (int64_t)LOSS_BLOCKS * LOSS_THREADS) {
        const int64_t p = off + i;
        if (p >= P) break;
        const double x = image[p], y = target[p];
        a[0] += x;
        a[1] += y;
        a[2] += x * x;
        a[3] += y * y;
        a[4] += x * y;
        a[5] += fabs(x - y);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < LOSS_TERMS; ++k) {
        const double v = warp_sum(a[k]);
        if (lane == 0) s[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < LOSS_TERMS) {
        double v = 0.0;
        for (int w = 0; w < LOSS_THREADS / 32; ++w) v += s[w][threadIdx.x];
        partial[((int64_t)f * LOSS_BLOCKS + blockIdx.x) * LOSS_TERMS + threadIdx.x] = v;
    }
}

// One thread per frame: the frame's statistics, loss and gradient coefficients.
__global__ void loss_final_kernel(const us3d_slice_frame* __restrict__ frames, int F, float l1_weight,
                                  float ssim_weight, const double* __restrict__ partial, double* __restrict__ stats,
                                  float4* __restrict__ coef) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    double t[LOSS_TERMS] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < LOSS_BLOCKS; ++b)
        for (int k = 0; k < LOSS_TERMS; ++k) t[k] += partial[((int64_t)f * LOSS_BLOCKS + b) * LOSS_TERMS + k];
    const double n = (double)frames[f].height * frames[f].width;
    const double c1 = 0.01 * 0.01, c2 = 0.03 * 0.03;
    double mx = 0.0, my = 0.0, vx = 0.0, vy = 0.0, vxy = 0.0, l1 = 0.0, ssim = 1.0;
    double a = 0.0, b0 = 0.0, cx = 0.0, cy = 0.0;
    if (n > 0.0) {
        mx = t[0] / n;
        my = t[1] / n;
        vx = fmax(t[2] / n - mx * mx, 0.0);
        vy = fmax(t[3] / n - my * my, 0.0);
        vxy = t[4] / n - mx * my;
        l1 = t[5] / n;
        const double A = 2.0 * mx * my + c1, B = 2.0 * vxy + c2, C = mx * mx + my * my + c1, D = vx + vy + c2;
        ssim = (A * B) / (C * D);
        // dSSIM/dx_i = SSIM * 2/n * [my/A - mx/C + (y_i - my)/B - (x_i - mx)/D]
        a = (double)l1_weight / n;
        if (ssim_weight != 0.0f) {
            const double k = -(double)ssim_weight * ssim * 2.0 / n;
            b0 = k * (my / A - mx / C - my / B + mx / D);
            cy = k / B;
            cx = -k / D;
        }
    }
    double* o = stats + 8 * (int64_t)f;
    o[0] = mx;
    o[1] = my;
    o[2] = vx;
    o[3] = vy;
    o[4] = vxy;
    o[5] = l1;
    o[6] = ssim;
    o[7] = (double)l1_weight * l1 + (double)ssim_weight * (1.0 - ssim);
    coef[f] = make_float4((float)a, (float)b0, (float)cx, (float)cy);
}

// Densification statistics: importance[g] += |dL/dmean_g|, visits[g] += 1 if that gradient is
// non-zero (the Gaussian reached a pixel of the step's frames).
__global__ void __launch_bounds__(256)
refine_stats_kernel(int64_t G, const float* __restrict__ grad_means, float* __restrict__ importance,
                    int* __restrict__ visits) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const float x = grad_means[3 * g], y = grad_means[3 * g + 1], z = grad_means[3 * g + 2];
    const float n = sqrtf(x * x + y * y + z * z);
    if (n > 0.0f) {
        importance[g] += n;
        visits[g] += 1;
    }
}

struct AdamTable {
    us3d_adam_tensor t[US3D_ADAM_MAX_TENSORS];
    int64_t start[US3D_ADAM_MAX_TENSORS + 1];
    int n;
};

// torch.optim.Adam's element update (foreach form): lerp for the first moment, mul + addcmul
// for the second, denominator sqrt(v) / sqrt(bias_correction2) + eps, addcdiv with
// -lr / bias_correction1. Division and square root are the correctly rounded ones.
__global__ void __launch_bounds__(256)
adam_kernel(const AdamTable tab, float w1, float beta2, float w2, float eps, float step_size, float bc2_sqrt) {
    const int64_t total = tab.start[tab.n];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int k = 0;
        while (k + 1 < tab.n && i >= tab.start[k + 1]) ++k;
        const us3d_adam_tensor& T = tab.t[k];
        const int64_t j = i - tab.start[k];
        const float p = T.param[j];
        float g = T.grad[j];
        if (T.activation == US3D_ADAM_LOGISTIC) {
            const float s = sigmoid_logit(p);
            g = g * (1.0f - s) * s;
        }
        float m = T.exp_avg[j];
        m = (w1 < 0.5f) ? m + w1 * (g - m) : g - (g - m) * (1.0f - w1);
        float v = T.exp_avg_sq[j] * beta2;
        v = v + w2 * g * g;
        const float denom = __fdiv_rn(__fsqrt_rn(v), bc2_sqrt) + eps;
        T.exp_avg[j] = m;
        T.exp_avg_sq[j] = v;
        T.param[j] = p + (-step_size) * __fdiv_rn(m, denom);
    }
}

}  // namespace train
}  // namespace us3d

using namespace us3d;
using namespace us3d::train;

extern "C" size_t us3d_ug_loss_scratch_bytes(int32_t n_frames) {
    if (n_frames < 0) return 0;
    return (size_t)n_frames * LOSS_BLOCKS * LOSS_TERMS * sizeof(double);
}

extern "C" int us3d_ug_loss(const us3d_slice_frame* frames, int32_t n_frames, int64_t n_pixels, const float* image,
                            const float* target, float l1_weight, float ssim_weight, void* scratch,
                            size_t scratch_bytes, double* out_stats, float* out_coef, void* stream_) {
    US3D_CHECK_ARG(n_frames >= 0 && n_pixels >= 0, "negative size");
    US3D_CHECK_ARG(n_frames <= 65535, "at most 65535 frames per call");
    if (n_frames == 0) return US3D_OK;
    US3D_CHECK_ARG(frames != nullptr, "frames table is NULL");
    US3D_CHECK_ARG(n_pixels == 0 || (image && target), "image or target is NULL");
    US3D_CHECK_ARG(out_stats && out_coef, "output pointer is NULL");
    US3D_CHECK_ARG((reinterpret_cast<uintptr_t>(out_coef) & 15) == 0, "out_coef must be 16-byte aligned");
    US3D_CHECK_ARG(scratch != nullptr && scratch_bytes >= us3d_ug_loss_scratch_bytes(n_frames),
                   "loss scratch too small: %zu < %zu", scratch_bytes, us3d_ug_loss_scratch_bytes(n_frames));
    cudaStream_t stream = (cudaStream_t)stream_;
    double* partial = reinterpret_cast<double*>(scratch);
    loss_partial_kernel<<<dim3(LOSS_BLOCKS, (unsigned)n_frames), LOSS_THREADS, 0, stream>>>(frames, n_pixels, image,
                                                                                          target, partial);
    loss_final_kernel<<<(unsigned)((n_frames + 63) / 64), 64, 0, stream>>>(frames, n_frames, l1_weight, ssim_weight,
                                                                          partial, out_stats,
                                                                          reinterpret_cast<float4*>(out_coef));
    US3D_CHECK_LAUNCH("ug loss");
    count_launches(2);
    return US3D_OK;
}

extern "C" int us3d_adam_step(const us3d_adam_tensor* tensors, int32_t n_tensors, double lr, double beta1,
                              double beta2, double eps, int64_t step, void* stream_) {
    US3D_CHECK_ARG(n_tensors >= 0 && n_tensors <= US3D_ADAM_MAX_TENSORS, "n_tensors must be in [0, %d]",
                   US3D_ADAM_MAX_TENSORS);
    US3D_CHECK_ARG(n_tensors == 0 || tensors != nullptr, "tensor table is NULL");
    US3D_CHECK_ARG(step >= 1, "step counts from 1");
    US3D_CHECK_ARG(beta1 >= 0.0 && beta1 < 1.0 && beta2 >= 0.0 && beta2 < 1.0, "betas must be in [0, 1)");
    AdamTable tab;
    tab.n = n_tensors;
    tab.start[0] = 0;
    for (int k = 0; k < n_tensors; ++k) {
        const us3d_adam_tensor& T = tensors[k];
        US3D_CHECK_ARG(T.numel >= 0, "tensor %d: negative size", k);
        US3D_CHECK_ARG(T.numel == 0 || (T.param && T.grad && T.exp_avg && T.exp_avg_sq), "tensor %d: NULL pointer", k);
        US3D_CHECK_ARG(T.activation == US3D_ADAM_IDENTITY || T.activation == US3D_ADAM_LOGISTIC,
                       "tensor %d: unknown activation %d", k, T.activation);
        tab.t[k] = T;
        tab.start[k + 1] = tab.start[k] + T.numel;
    }
    const int64_t total = tab.start[n_tensors];
    if (total == 0) return US3D_OK;
    // scalars in double on the host and rounded to float once, as torch does with its
    // Python-float hyper-parameters
    const double bc1 = 1.0 - std::pow(beta1, (double)step);
    const double bc2 = 1.0 - std::pow(beta2, (double)step);
    const float step_size = (float)(lr / bc1);
    const float bc2_sqrt = (float)std::sqrt(bc2);
    const int64_t blocks = std::min<int64_t>((total + 255) / 256, 148 * 8);
    adam_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream_>>>(tab, (float)(1.0 - beta1), (float)beta2,
                                                                     (float)(1.0 - beta2), (float)eps, step_size,
                                                                     bc2_sqrt);
    US3D_CHECK_LAUNCH("adam");
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_ug_refine_stats(const float* grad_means, int64_t n_gauss, float* importance, int32_t* visits,
                                    void* stream_) {
    US3D_CHECK_ARG(n_gauss >= 0, "negative size");
    if (n_gauss == 0) return US3D_OK;
    US3D_CHECK_ARG(grad_means && importance && visits, "pointer is NULL");
    refine_stats_kernel<<<(unsigned)((n_gauss + 255) / 256), 256, 0, (cudaStream_t)stream_>>>(n_gauss, grad_means,
                                                                                              importance, visits);
    US3D_CHECK_LAUNCH("refine stats");
    count_launches(1);
    return US3D_OK;
}
