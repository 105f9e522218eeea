// Frame batches assembled on the device from a dataset that lives in HBM: the frame records
// of a batch of dataset indices, their pixel centre positions (gathered, or generated from the
// frame geometry exactly as the reference's dataset does) and their target images (with the
// reference's 8-bit scaling). Replaces the per-frame host work of NpzUltrasoundDataset.get_frame
// (pipeline_god_file.py:178-245, 292-306) for the batched training step.
#include <algorithm>

#include "us3d_common.cuh"

namespace us3d {
namespace frames {

constexpr int TILE = 16;
constexpr int THREADS = 256;

// The reference's generated pixel grid (pipeline_god_file.py:299-306): lateral = (u - centre)
// * delta_lateral, axial = near + v * delta_axial, p = (origin + lateral * lat) + axial * ax,
// each operation rounded to float on its own (PyTorch evaluates them as separate kernels).
__device__ __forceinline__ void grid_pixel(const us3d_slice_frame& fr, int u, int v, float* out) {
    const float lat_mm = __fmul_rn(__fsub_rn((float)u, fr.lateral_col_offset), fr.lateral_spacing);
    const float ax_mm = __fadd_rn(__fmul_rn((float)v, fr.axial_spacing), fr.axial_near);
#pragma unroll
    for (int c = 0; c < 3; ++c)
        out[c] = __fadd_rn(__fadd_rn(fr.origin[c], __fmul_rn(lat_mm, fr.axis_lat[c])), __fmul_rn(ax_mm, fr.axis_ax[c]));
}

__global__ void __launch_bounds__(THREADS)
gather_kernel(const us3d_slice_frame* __restrict__ all, int64_t n_all, const int64_t* __restrict__ indices, int H,
              int W, const float* __restrict__ all_pixels, const void* __restrict__ images, int image_format,
              us3d_slice_frame* __restrict__ out_frames, float* __restrict__ out_pixels,
              float* __restrict__ out_targets, int* __restrict__ status) {
    const int f = blockIdx.y;
    const int64_t hw = (int64_t)H * W;
    int64_t k = indices[f];
    if (k < 0 || k >= n_all) {  // reported, and the slot takes frame 0 so that nothing is read out of range
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, 1);
        k = 0;
    }
    const us3d_slice_frame fr = all[k];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        us3d_slice_frame o = fr;
        o.height = H;
        o.width = W;
        o.tiles_x = (W + TILE - 1) / TILE;
        o.tiles_y = (H + TILE - 1) / TILE;
        o.pixel_offset = (int32_t)(f * hw);
        o.tile_offset = f * o.tiles_x * o.tiles_y;
        out_frames[f] = o;
    }
    const int64_t i = (int64_t)blockIdx.x * THREADS + threadIdx.x;
    if (i >= hw) return;
    const int64_t dst = (int64_t)f * hw + i;
    float p[3];
    if (all_pixels) {
        const float* src = all_pixels + 3 * (k * hw + i);
        p[0] = src[0];
        p[1] = src[1];
        p[2] = src[2];
    } else {
        grid_pixel(fr, (int)(i % W), (int)(i / W), p);
    }
    out_pixels[3 * dst + 0] = p[0];
    out_pixels[3 * dst + 1] = p[1];
    out_pixels[3 * dst + 2] = p[2];
    float y;
    if (image_format == US3D_IMAGES_U8 || image_format == US3D_IMAGES_U8_DIV255)
        y = (float)static_cast<const uint8_t*>(images)[k * hw + i];
    else
        y = static_cast<const float*>(images)[k * hw + i];
    if (image_format == US3D_IMAGES_U8_DIV255 || image_format == US3D_IMAGES_F32_DIV255) y = __fdiv_rn(y, 255.0f);
    out_targets[dst] = y;
}

// Scanline and pose geometry of a batch of frames (reference pipeline_god_file.py:308-336):
// ray origin u = origin + ((u - centre) * delta_lateral) * lat, each operation rounded on its
// own as PyTorch's separate kernels do; ray direction = the axial axis; world-to-probe pose
// [R | -R origin] with R's rows the lateral, axial and elevational axes.
__global__ void __launch_bounds__(THREADS)
geometry_kernel(const us3d_slice_frame* __restrict__ all, int64_t n_all, const int64_t* __restrict__ indices, int W,
                const float* __restrict__ all_origins, const float* __restrict__ all_dirs,
                const float* __restrict__ all_poses, float* __restrict__ out_origins, float* __restrict__ out_dirs,
                float* __restrict__ out_pose, int* __restrict__ status) {
    const int f = blockIdx.y;
    int64_t k = indices[f];
    if (k < 0 || k >= n_all) {
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, 1);
        k = 0;
    }
    const us3d_slice_frame fr = all[k];
    const int u = blockIdx.x * THREADS + threadIdx.x;
    if (u < W) {
        const int64_t dst = 3 * ((int64_t)f * W + u);
        const int64_t src = 3 * (k * W + u);
        if (all_origins) {
            out_origins[dst] = all_origins[src];
            out_origins[dst + 1] = all_origins[src + 1];
            out_origins[dst + 2] = all_origins[src + 2];
        } else {
            const float lat_mm = __fmul_rn(__fsub_rn((float)u, fr.lateral_col_offset), fr.lateral_spacing);
#pragma unroll
            for (int c = 0; c < 3; ++c) out_origins[dst + c] = __fadd_rn(fr.origin[c], __fmul_rn(lat_mm, fr.axis_lat[c]));
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) out_dirs[dst + c] = all_dirs ? all_dirs[src + c] : fr.axis_ax[c];
    }
    if (blockIdx.x == 0 && threadIdx.x < 16) {
        const int r = threadIdx.x / 4, c = threadIdx.x % 4;
        float v;
        if (all_poses) {
            v = all_poses[16 * k + threadIdx.x];
        } else if (r == 3) {
            v = c == 3 ? 1.0f : 0.0f;
        } else {
            const float* row = r == 0 ? fr.axis_lat : (r == 1 ? fr.axis_ax : fr.axis_ele);
            v = c < 3 ? row[c]
                      : -__fadd_rn(__fadd_rn(__fmul_rn(row[0], fr.origin[0]), __fmul_rn(row[1], fr.origin[1])),
                                   __fmul_rn(row[2], fr.origin[2]));
        }
        out_pose[16 * (int64_t)f + threadIdx.x] = v;
    }
}

}  // namespace frames
}  // namespace us3d

using namespace us3d;

extern "C" int us3d_frames_gather(const us3d_slice_frame* all_frames, int64_t n_all, const int64_t* indices,
                                  int32_t n_batch, int32_t height, int32_t width, const float* all_pixel_positions,
                                  const void* images, int32_t image_format, us3d_slice_frame* out_frames,
                                  float* out_pixel_positions, float* out_targets, int32_t* status, void* stream_) {
    US3D_CHECK_ARG(n_all >= 0 && n_batch >= 0 && height >= 0 && width >= 0, "negative size");
    US3D_CHECK_ARG(n_batch <= 65535, "at most 65535 frames per batch");
    US3D_CHECK_ARG((int64_t)n_batch * height * width <= 0x7fffffffLL, "batch pixel count must fit in int32");
    US3D_CHECK_ARG(image_format >= US3D_IMAGES_F32 && image_format <= US3D_IMAGES_U8_DIV255,
                   "unknown image format %d", image_format);
    if (n_batch == 0) return US3D_OK;
    US3D_CHECK_ARG(n_all > 0, "the dataset has no frames");
    US3D_CHECK_ARG(all_frames && indices && images && out_frames && out_pixel_positions && out_targets && status,
                   "pointer is NULL");
    const int64_t hw = (int64_t)height * width;
    if (hw == 0) return US3D_OK;
    const dim3 grid((unsigned)((hw + frames::THREADS - 1) / frames::THREADS), (unsigned)n_batch);
    frames::gather_kernel<<<grid, frames::THREADS, 0, (cudaStream_t)stream_>>>(
        all_frames, n_all, indices, height, width, all_pixel_positions, images, image_format, out_frames,
        out_pixel_positions, out_targets, status);
    US3D_CHECK_LAUNCH("frames gather");
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_frames_geometry(const us3d_slice_frame* all_frames, int64_t n_all, const int64_t* indices,
                                    int32_t n_batch, int32_t width, const float* all_ray_origins,
                                    const float* all_ray_dirs, const float* all_poses, float* out_ray_origins,
                                    float* out_ray_dirs, float* out_pose, int32_t* status, void* stream_) {
    US3D_CHECK_ARG(n_all >= 0 && n_batch >= 0 && width >= 0, "negative size");
    US3D_CHECK_ARG(n_batch <= 65535, "at most 65535 frames per batch");
    if (n_batch == 0) return US3D_OK;
    US3D_CHECK_ARG(n_all > 0, "the dataset has no frames");
    US3D_CHECK_ARG(all_frames && indices && out_pose && status && (width == 0 || (out_ray_origins && out_ray_dirs)),
                   "pointer is NULL");
    const dim3 grid((unsigned)std::max<int64_t>(1, ((int64_t)width + frames::THREADS - 1) / frames::THREADS),
                    (unsigned)n_batch);
    frames::geometry_kernel<<<grid, frames::THREADS, 0, (cudaStream_t)stream_>>>(
        all_frames, n_all, indices, width, all_ray_origins, all_ray_dirs, all_poses, out_ray_origins, out_ray_dirs,
        out_pose, status);
    US3D_CHECK_LAUNCH("frames geometry");
    count_launches(1);
    return US3D_OK;
}
