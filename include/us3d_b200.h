/*
 * us3d_b200 — C ABI of the B200-native Gaussian rasterisation library for freehand 3D
 * ultrasound (sm_100a). Plain pointers and sizes only: every pointer argument named
 * `*_dev` or documented as "device" is CUDA device memory owned by the caller; `stream`
 * is a cudaStream_t passed as void*. No entry point allocates device memory or
 * synchronises `stream` unless its comment says so.
 *
 * Status codes: every function returns US3D_OK (0) or an error code; the message of the
 * last error on the calling thread is available from us3d_last_error().
 *
 * Reference interfaces replaced (paths inside the reference project
 * KevinWCCC/ultrasound-3d-reconstruction):
 *   GaussianPile: ops/gaussianplie_renderer/src/bindings.cpp:5-8
 *                (ProjectedSliceForwardCUDA, ProjectedSliceBackwardCUDA)
 *   slice-adapted 3DGS: ops/slice_adapted_3dgs_renderer/src/bindings.cpp:46-91
 *                (forward, backward, bounded_forward, bounded_backward)
 *   UltraGauss:  ops/ultragauss_renderer/src/bindings.cpp:6-10
 *                (MapperForwardCUDA  -> src/mapper/wrapper_mapper.cu:35-206,
 *                 ShaderForwardCUDA  -> src/shader/wrapper_shader.cu:17-66,
 *                 ShaderBackwardCUDA -> src/shader/wrapper_shader.cu:68-122)
 *   UltraGray:   ops/ultragray_renderer/src/bindings.cpp:6-10
 *                (MapperForwardCUDA, ShaderForwardCUDA, ShaderBackwardCUDA)
 *   UltraGS baseline: ops/ultrags_baseline_renderer/ext.cpp:14-18
 *                (rasterize_gaussians, rasterize_gaussians_backward, mark_visible)
 *   slice-adapted adapter projection: baselines/slice_adapted_3dgs/render.py:66-98,132-163
 */
#ifndef US3D_B200_H
#define US3D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define US3D_API __attribute__((visibility("default")))
#else
#define US3D_API
#endif

#define US3D_OK 0
#define US3D_INVALID_ARG 1
#define US3D_CAPACITY_OVERFLOW 2
#define US3D_CUDA_ERROR 3
#define US3D_TIMEOUT 4

/* Message of the last failed call on this thread ("" if none). */
US3D_API const char* us3d_last_error(void);
/* Library ABI version (major*10000 + minor*100 + patch). */
US3D_API int us3d_version(void);
/* Makes `device` current for this library's calls on the calling thread (cudaSetDevice). */
US3D_API int us3d_set_device(int device);

/* Benchmark instrumentation. us3d_launch_count: number of kernels this library has
 * launched in this process. us3d_profile_stage: from now on, bracket up to max_launches
 * executions of the named stage ("ug_bin", "ug_forward", "ug_backward") with CUDA events
 * on the launching stream (NULL or 0 disables); us3d_profile_collect waits for them and
 * returns how many ran and their summed duration, then resets the count. */
US3D_API long long us3d_launch_count(void);
US3D_API int us3d_profile_stage(const char* stage, int max_launches);
US3D_API int us3d_profile_collect(int* n_launches, double* total_ms);

/*
 * One planar probe slice ("frame"). The library reads an array of these from DEVICE
 * memory, so one launch can render many frames of different sizes. Pixel (row y, col x)
 * of frame f is pixel index `pixel_offset + y*width + x` of the concatenated pixel arrays;
 * its 16x16 tile (tx, ty) is tile `tile_offset + ty*tiles_x + tx` of the concatenated tile
 * numbering. tiles_x = ceil(width/16), tiles_y = ceil(height/16).
 * Axes and spacings have the meaning of the reference's UltraGaussRenderConfig /
 * SliceGeometry (ops/ultragauss_renderer/ultragauss_renderer/types.py:6-40).
 */
typedef struct us3d_slice_frame {
    float origin[3];
    float axis_lat[3];
    float axis_ax[3];
    float axis_ele[3];
    float lateral_spacing;    /* mm per pixel (lateral)          */
    float axial_spacing;      /* mm per pixel (axial / depth)    */
    float axial_near;         /* depth of pixel row 0, mm        */
    float lateral_col_offset; /* column of lateral coordinate 0  */
    int32_t height;
    int32_t width;
    int32_t tiles_x;
    int32_t tiles_y;
    int32_t pixel_offset;
    int32_t tile_offset;
    int32_t gauss_offset;     /* with US3D_UG_BIN_GAUSSIAN_SETS: first Gaussian of this */
    int32_t gauss_count;      /* frame's set and its size (otherwise 0, 0: all of them) */
} us3d_slice_frame; /* 96 bytes */

/* ------------------------------------------------------------------------------------
 * UltraGauss probe-plane slice splatting.
 *
 * Gaussian parameters (device, fp32, contiguous): means (G,3) world mm; precision_tril
 * (G,6) raw lower-Cholesky factor of the precision in the order l11,l12,l13,l22,l23,l33
 * with diagonal entries raw^2 + diag_beta; opacities (G); intensities (G).
 * Pixels (device, fp32): pixel_positions (n_pixels,3) world mm, frames concatenated.
 *
 * Workspace: one caller-allocated device buffer of us3d_ug_workspace_bytes() bytes,
 * which holds the binning of the last us3d_ug_bin() call; keep it alive (unchanged)
 * between us3d_ug_bin, us3d_ug_forward and us3d_ug_backward of the same frames, and pass
 * every call the same sizes and instance_capacity (they locate the arrays inside it).
 * ---------------------------------------------------------------------------------- */

/* Bytes of workspace for G Gaussians, n_frames frames with n_tiles tiles and n_pixels
 * pixels in total, and room for `instance_capacity` (tile, Gaussian) instances. */
US3D_API size_t us3d_ug_workspace_bytes(int64_t n_gauss, int32_t n_frames, int64_t n_tiles,
                               int64_t n_pixels, int64_t instance_capacity);

/* Bytes of the backward scratch buffer (per-instance partial gradients). */
US3D_API size_t us3d_ug_backward_scratch_bytes(int64_t instance_capacity);

/*
 * Mapper: per-Gaussian probe-frame projection, chi-square window radii, elevational cull,
 * 16x16 tile rectangles, (tile, depth) keys, per-tile stable ordering and tile ranges.
 * Replaces MapperForwardCUDA (ops/ultragauss_renderer/src/mapper/wrapper_mapper.cu:35-206)
 * up to the tile ranges; the per-pixel candidate lists are produced by us3d_ug_forward
 * (counts) and us3d_ug_pixel_csr (indices). Never synchronises: the instance total and
 * an overflow flag stay on the device (read them with us3d_ug_read_status).
 */
US3D_API int us3d_ug_bin(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames_dev,
                int32_t n_frames, int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                const float* means, const float* precision_tril, const float* opacities,
                const float* intensities, float chi2_threshold, float diag_beta,
                int32_t sort_by_depth, int64_t instance_capacity, void* stream);

/*
 * us3d_ug_bin with options. flags = US3D_UG_BIN_SLICE_CULL keeps a (tile, Gaussian)
 * instance only if the Gaussian's chi-square quadratic, restricted to the frame's pixel grid,
 * can reach chi2_threshold inside the tile (exact test in double precision with margins for
 * the pixels' distance from the grid, measured from pixel_positions (n_pixels,3), and for
 * float rounding). Images, alpha, depth and gradients are identical to those of a full
 * binning (the kept lists are order-preserving subsequences and the dropped instances have no
 * contributing pixel); the per-pixel window-test counts, the candidate lists
 * (us3d_ug_pixel_csr) and us3d_ug_export_bins describe the reference's full binning only,
 * so after a culled binning us3d_ug_forward leaves out_counts unwritten and
 * us3d_ug_pixel_csr writes nothing. No counterpart in the reference (its mapper always bins
 * the full window rectangle).
 */
#define US3D_UG_BIN_SLICE_CULL 1
/*
 * flags |= US3D_UG_BIN_LOGIT_ATTRIBUTES: `opacities` and `intensities` are raw logits and the
 * binning activates them with the logistic function (the reference's training
 * parameterisation, GaussianParameters.opacities()/intensities() in pipeline_god_file.py:
 * 368-372, torch.sigmoid), so that a training step needs no separate activation pass.
 */
#define US3D_UG_BIN_LOGIT_ATTRIBUTES 2
/*
 * flags |= US3D_UG_BIN_GAUSSIAN_SETS: every frame renders only its own Gaussians, the range
 * [gauss_offset, gauss_offset + gauss_count) of the parameter arrays, so that independent
 * sweeps with their own Gaussian sets (of any sizes, with frames of any sizes) bin, shade and
 * differentiate in one launch sequence over the concatenated parameters. The frames of one
 * set must be contiguous in the table and the sets must appear in increasing gauss_offset
 * order without overlapping (each Gaussian then belongs to at most one set; gradients of a
 * Gaussian sum over its set's frames). No counterpart in the reference (one frame and one
 * parameter set per call).
 */
#define US3D_UG_BIN_GAUSSIAN_SETS 4
US3D_API int us3d_ug_bin_ex(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames_dev,
                            int32_t n_frames, int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                            const float* means, const float* precision_tril, const float* opacities,
                            const float* intensities, float chi2_threshold, float diag_beta,
                            int32_t sort_by_depth, int64_t instance_capacity, const float* pixel_positions,
                            int32_t flags, void* stream);

/* Copies the instance total and overflow flag of the last us3d_ug_bin to the host.
 * SYNCHRONISES `stream`. */
US3D_API int us3d_ug_read_status(const void* workspace, int64_t* total_instances, int32_t* overflow,
                        void* stream);

/*
 * Forward shading: per pixel, the candidates that pass the reference's lateral/axial
 * window test, then q <= chi2, alpha_hat = o*exp(-q/2) (skipped if <= 1e-8);
 * image = clamp01((sum a*c + bg_a*bg_i) / max(sum a + bg_a, 1e-8)), alpha = sum a + bg_a,
 * depth = sum a*((mean-origin).ele) / max(sum a, 1e-8). Also writes the per-pixel
 * candidate count (the reference's pixel_gauss_counts) and the no-skip sums that the
 * backward needs. Replaces ShaderForwardCUDA (src/shader/wrapper_shader.cu:17-66,
 * kernel src/shader/forward.cu:17-76). out_counts may be NULL.
 */
US3D_API int us3d_ug_forward(void* workspace, const us3d_slice_frame* frames_dev, int32_t n_frames,
                    int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                    int64_t instance_capacity, const float* pixel_positions, float chi2_threshold, float diag_beta,
                    float bg_alpha, float bg_intensity, float* out_image, float* out_alpha,
                    float* out_depth, int32_t* out_counts, void* stream);

/*
 * Backward (adjoint): gradients of (image, alpha, depth) w.r.t. means (G,3),
 * precision_tril (G,6), opacities (G) and intensities (G), summed over all frames of the
 * last bin. Deterministic: per (tile, Gaussian) partials are reduced per Gaussian in a
 * fixed order (no float atomics). Overwrites the four gradient arrays. Replaces
 * ShaderBackwardCUDA (src/shader/wrapper_shader.cu:68-122, kernel
 * src/shader/backward.cu:17-131).
 */
US3D_API int us3d_ug_backward(void* workspace, const us3d_slice_frame* frames_dev, int32_t n_frames,
                     int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                     int64_t instance_capacity, const float* pixel_positions, const float* d_image,
                     const float* d_alpha, const float* d_depth, const float* saved_alpha,
                     float chi2_threshold, float diag_beta, float bg_alpha,
                     float bg_intensity, void* scratch, size_t scratch_bytes,
                     float* d_means, float* d_precision_tril, float* d_opacities,
                     float* d_intensities, void* stream);

/*
 * Launch shapes of the UltraGauss shading kernels, process-wide (read at every launch; set
 * them before capturing a CUDA graph): Gaussians staged per forward batch (128, 256 or 512)
 * and threads per backward CTA (128 or 256). Results do not depend on them. The defaults
 * (512, 256) are the fastest measured on the headline scene; us3d_b200.batch.autotune_launch
 * times every pair on a caller's workload and keeps the fastest. No counterpart in the
 * reference (its kernels have fixed launch shapes).
 */
US3D_API int us3d_ug_set_launch_config(int32_t forward_batch, int32_t backward_threads);
US3D_API int us3d_ug_get_launch_config(int32_t* forward_batch, int32_t* backward_threads);

/* Backward kernel variant of the UltraGauss shading adjoint (process-wide, read at every
 * launch): 0 = one pixel per FP32 instruction, 1 = two pixels per packed FP32 instruction
 * (sm_100 f32x2; same pair selection, each lane rounding as the scalar instruction, sums
 * of even and odd pixels kept apart and added once per instance). Both are deterministic;
 * they differ in summation order only. Default 0. No counterpart in the reference. */
US3D_API int us3d_ug_set_backward_variant(int32_t variant);
US3D_API int us3d_ug_get_backward_variant(int32_t* variant);

/* Forward kernel variant of the UltraGauss shading (process-wide, read at every launch): 0 =
 * one pixel per thread and FP32 instruction, 1 = two pixels per thread and packed FP32
 * instruction (sm_100 f32x2; 128-thread blocks whose warps own 8x8 quadrants, at most 256
 * staged Gaussians per batch (a forward batch of 512 runs as 256); each lane
 * rounds as the scalar kernel, so images, alpha, depth and the saved sums are bit-identical).
 * The windowed case (diag_beta < 1e-10) always uses variant 0. Default 0. No counterpart in
 * the reference. */
US3D_API int us3d_ug_set_forward_variant(int32_t variant);
US3D_API int us3d_ug_get_forward_variant(int32_t* variant);

/*
 * Per-frame image loss of the reference's training step (image_loss in
 * pipeline_god_file.py:606-617 with simple_ssim at :627-637): for each frame f of the table,
 * loss_f = l1_weight * mean|x - y| + ssim_weight * (1 - SSIM_f), SSIM_f the global SSIM of
 * the frame's image x against its target y (means, population variances and covariance over
 * the frame's H*W pixels; c1 = 0.01^2, c2 = 0.03^2). Writes out_stats (n_frames x 8 doubles:
 * mean x, mean y, var x, var y, cov xy, mean |x - y|, SSIM, loss) and out_coef (n_frames x 4
 * floats, 16-byte aligned): the per-frame coefficients (a, b, c, d) of dL_f/dx_i =
 * a*sign(x_i - y_i) + b + c*x_i + d*y_i, which us3d_ug_backward_loss uses. A batch of frames
 * is trained on the sum of its frames' losses, so every frame keeps the gradient of a
 * single-frame step. scratch: us3d_ug_loss_scratch_bytes(n_frames) bytes. Deterministic
 * (fixed-order double-precision reductions); never synchronises. No counterpart in the
 * reference's CUDA (its loss is PyTorch code).
 */
US3D_API size_t us3d_ug_loss_scratch_bytes(int32_t n_frames);
US3D_API int us3d_ug_loss(const us3d_slice_frame* frames_dev, int32_t n_frames, int64_t n_pixels,
                          const float* image, const float* target, float l1_weight, float ssim_weight,
                          void* scratch, size_t scratch_bytes, double* out_stats, float* out_coef, void* stream);

/*
 * us3d_ug_backward with dL/dimage fused in from the per-frame loss of us3d_ug_loss (image,
 * target, and its coefficients `loss_coef`), and dL/dalpha = dL/ddepth = 0. Same gradients as
 * us3d_ug_backward given the loss gradient image, without materialising it. No counterpart
 * in the reference (there ShaderBackwardCUDA receives the autograd gradient of the PyTorch
 * loss).
 */
US3D_API int us3d_ug_backward_loss(void* workspace, const us3d_slice_frame* frames_dev, int32_t n_frames,
                                   int64_t n_tiles, int64_t n_pixels, int64_t n_gauss, int64_t instance_capacity,
                                   const float* pixel_positions, const float* image, const float* target,
                                   const float* loss_coef, const float* saved_alpha, float chi2_threshold,
                                   float diag_beta, float bg_alpha, float bg_intensity, void* scratch,
                                   size_t scratch_bytes, float* d_means, float* d_precision_tril,
                                   float* d_opacities, float* d_intensities, void* stream);

/*
 * One Adam step over up to US3D_ADAM_MAX_TENSORS parameter tensors in a single launch,
 * with torch.optim.Adam's update (defaults: no weight decay, no amsgrad; the optimiser the
 * reference's training loop uses, pipeline_god_file.py:740,764): m = lerp(m, g, 1 - beta1),
 * v = beta2 v + (1 - beta2) g^2, p -= lr / (1 - beta1^step) * m / (sqrt(v) / sqrt(1 -
 * beta2^step) + eps), `step` counted from 1. A tensor with activation
 * US3D_ADAM_LOGISTIC holds logits whose gradient was taken w.r.t. their logistic
 * activation: the chain rule g * (1 - s) * s, s = sigmoid(p), is applied first (the
 * backward of torch.sigmoid). The hyper-parameters are rounded to float once, like torch's
 * Python-float ones. Never synchronises.
 */
#define US3D_ADAM_MAX_TENSORS 8
#define US3D_ADAM_IDENTITY 0
#define US3D_ADAM_LOGISTIC 1
typedef struct us3d_adam_tensor {
    float* param;
    const float* grad;
    float* exp_avg;
    float* exp_avg_sq;
    int64_t numel;
    int32_t activation;
    int32_t reserved;
} us3d_adam_tensor;
US3D_API int us3d_adam_step(const us3d_adam_tensor* tensors, int32_t n_tensors, double lr, double beta1,
                            double beta2, double eps, int64_t step, void* stream);

/*
 * A batch of frames assembled on the device from a dataset held in device memory (the
 * batched replacement of NpzUltrasoundDataset.get_frame, pipeline_god_file.py:212-245): for
 * each of the n_batch dataset indices (device int64; an index outside [0, n_all) sets bit 0
 * of *status and takes frame 0), the frame record of all_frames (n_all records of height x
 * width frames) with this batch's pixel and tile offsets; its pixel centre positions, gathered
 * from all_pixel_positions (n_all x height*width x 3) or, if that is NULL, generated from the
 * record exactly as the reference does (pipeline_god_file.py:299-306: lateral = (u -
 * lateral_col_offset) * lateral_spacing, axial = axial_near + v * axial_spacing, p = (origin +
 * lateral * axis_lat) + axial * axis_ax, float operations rounded one by one); and its target
 * image from `images` (n_all x height*width) in `image_format`. The _DIV255 formats apply the
 * reference's scaling of images whose maximum exceeds 1.5 (pipeline_god_file.py:184-186):
 * float(x) / 255. Outputs: out_frames (n_batch records), out_pixel_positions (n_batch*H*W x
 * 3), out_targets (n_batch*H*W). Never synchronises.
 */
#define US3D_IMAGES_F32 0
#define US3D_IMAGES_F32_DIV255 1
#define US3D_IMAGES_U8 2
#define US3D_IMAGES_U8_DIV255 3
US3D_API int us3d_frames_gather(const us3d_slice_frame* all_frames, int64_t n_all, const int64_t* indices,
                                int32_t n_batch, int32_t height, int32_t width, const float* all_pixel_positions,
                                const void* images, int32_t image_format, us3d_slice_frame* out_frames,
                                float* out_pixel_positions, float* out_targets, int32_t* status, void* stream);

/*
 * Scanline and pose geometry of a batch of dataset frames, replacing the per-frame host work
 * of NpzUltrasoundDataset._ray_origins / _ray_dirs / _pose_world_to_probe
 * (pipeline_god_file.py:308-336). For each of the n_batch dataset indices: `width` ray origins
 * origin + ((u - lateral_col_offset) * lateral_spacing) * axis_lat, u = 0..width-1 (or
 * all_ray_origins[k], (n_all, width, 3)), `width` ray directions axis_ax (or
 * all_ray_dirs[k]), and the row-major 4x4 world-to-probe pose [R | -R origin] with R's rows
 * axis_lat, axis_ax, axis_ele (or all_poses[k], (n_all, 16)). The stored arrays may be NULL.
 * Outputs: out_ray_origins / out_ray_dirs (n_batch, width, 3), out_pose (n_batch, 16). An
 * index outside [0, n_all) sets *status bit 0 and takes frame 0. Never synchronises.
 */
US3D_API int us3d_frames_geometry(const us3d_slice_frame* all_frames, int64_t n_all, const int64_t* indices,
                                  int32_t n_batch, int32_t width, const float* all_ray_origins,
                                  const float* all_ray_dirs, const float* all_poses, float* out_ray_origins,
                                  float* out_ray_dirs, float* out_pose, int32_t* status, void* stream);

/*
 * Densification statistics of a training step (the refinement the UltraG-Ray paper
 * describes, absent from the reference's code): for each of the n_gauss Gaussians,
 * importance[g] += |dL/dmean_g| (Euclidean norm of its row of grad_means, (G,3)) and
 * visits[g] += 1 when that norm is non-zero. Never synchronises. No counterpart in the
 * reference.
 */
US3D_API int us3d_ug_refine_stats(const float* grad_means, int64_t n_gauss, float* importance, int32_t* visits,
                                  void* stream);

/*
 * Per-pixel candidate lists in the reference's CSR layout (pixel_gauss_indices of
 * MapperForwardCUDA, src/mapper/core.cu:237-287): for each pixel, in tile-list order,
 * the Gaussians passing the window test. `offsets` is the exclusive scan of the counts
 * written by us3d_ug_forward (n_pixels entries); `out_indices` must hold the total.
 */
US3D_API int us3d_ug_pixel_csr(void* workspace, const us3d_slice_frame* frames_dev, int32_t n_frames,
                      int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                      int64_t instance_capacity, const float* pixel_positions, float chi2_threshold, float diag_beta,
                      const int32_t* offsets, int32_t* out_indices, void* stream);

/*
 * Sorted keys, values and tile ranges of one frame in the reference's format
 * (key = (tile << 32) | depth_key, value = Gaussian index; empty tiles have start = end
 * = -1; src/mapper/core.cu:118-164). out_keys/out_values hold the frame's instances
 * (in tile order); out_range_start/out_range_end hold tiles_x*tiles_y entries.
 */
US3D_API int us3d_ug_export_bins(const void* workspace, int64_t n_tiles, int32_t frame_tile_offset,
                        int32_t frame_n_tiles, int64_t* out_keys, int32_t* out_values,
                        int32_t* out_range_start, int32_t* out_range_end, void* stream);

/* Instance offset of a frame's first tile and its instance count (device -> host copy;
 * SYNCHRONISES `stream`). */
US3D_API int us3d_ug_frame_instances(const void* workspace, int64_t n_tiles, int32_t frame_tile_offset,
                            int32_t frame_n_tiles, int64_t* first, int64_t* count,
                            void* stream);

/* ------------------------------------------------------------------------------------
 * GaussianPile projected-slice ("us_focus") additive splatting, one slice per call.
 *
 * Gaussians (device, fp32): means (G,3), scales (G,3), quats (G,4) as (w,x,y,z),
 * opacities (G), intensities (G). pose (16 floats, row-major 4x4; probe axes are its
 * normalised columns 0..2 and the origin its column 3), grid_pack (16 floats, the
 * reference's slice grid layout), focus_params (14 floats, the reference's us_focus
 * parameter layout) are device arrays. The reference passes the same values as these
 * scalar arguments and as the pack; both are taken here so that each computation reads
 * the one the reference reads.
 * ---------------------------------------------------------------------------------- */

US3D_API size_t us3d_gp_workspace_bytes(int64_t n_gauss, int32_t height, int32_t width, int32_t tile_size,
                                        int64_t instance_capacity);
US3D_API size_t us3d_gp_backward_scratch_bytes(int64_t n_gauss, int64_t instance_capacity);

/* Mapper + forward: footprints, tile rectangles, keys, per-tile order, ranges and the
 * additive image (H,W). Replaces ProjectedSliceForwardCUDA
 * (ops/gaussianplie_renderer/src/shader/wrapper_shader.cu:49-217) for the us_focus shader
 * with the tile mapper and additive compositing. Never synchronises. */
US3D_API int us3d_gp_forward(void* workspace, size_t workspace_bytes, int64_t n_gauss, const float* means,
                             const float* scales, const float* quats, const float* opacities,
                             const float* intensities, const float* pose, const float* grid_pack,
                             const float* focus_params, int32_t height, int32_t width, float lateral_spacing,
                             float axial_spacing, float axial_near, int32_t tile_size, float k_sigma,
                             int32_t sort_by_v, int64_t instance_capacity, float* out_image, void* stream);

/* Instance total and flags of the last us3d_gp_forward (SYNCHRONISES `stream`). */
US3D_API int us3d_gp_read_status(const void* workspace, int64_t* total_instances, int32_t* overflow,
                                 void* stream);

/* Backward: gradients w.r.t. means (G,3), scales (G,3), quats (G,4), opacities,
 * intensities and, with US3D_GP_GRAD_POSE in grad_flags, the pose (4x4). Scale and
 * quaternion gradients are, by default, the reference's central differences (step 1e-3) of
 * the footprint/adjoint dot product; with US3D_GP_GRAD_SHAPE_ANALYTIC they are the exact
 * derivative instead (the probe-frame covariance adjoint carried through R diag(s^2) R^T
 * and the quaternion normalisation; no counterpart in the reference). Gradients are
 * NaN-sanitised and clamped to +-1e3 as in the reference. Deterministic.
 * Replaces ProjectedSliceBackwardCUDA (wrapper_shader.cu:218-416; kernels
 * src/shader/us_focus.cu:479-966). */
#define US3D_GP_GRAD_POSE 1
#define US3D_GP_GRAD_SHAPE_ANALYTIC 2
US3D_API int us3d_gp_backward(void* workspace, int64_t n_gauss, const float* means, const float* scales,
                              const float* quats, const float* opacities, const float* intensities,
                              const float* pose, const float* grid_pack, const float* focus_params,
                              int32_t height, int32_t width, int32_t tile_size, float k_sigma,
                              int64_t instance_capacity, const float* grad_image, int32_t grad_flags,
                              void* scratch, size_t scratch_bytes, float* d_means, float* d_scales,
                              float* d_quats, float* d_opacities, float* d_intensities, float* d_pose,
                              void* stream);

/* Sorted Gaussian ids (instance total entries), tile ranges (-1 for empty tiles) and
 * per-Gaussian tile rectangles (G x int4, may be NULL) in the reference's format
 * (OursTileGaussMapperCUDA, src/mapper/core_tile.cu:238-379). */
US3D_API int us3d_gp_export_bins(const void* workspace, int64_t n_gauss, int32_t height, int32_t width,
                                 int32_t tile_size, int64_t instance_capacity, int32_t* out_sorted_ids,
                                 int32_t* out_range_start, int32_t* out_range_end, int32_t* out_rects,
                                 void* stream);

/* ------------------------------------------------------------------------------------
 * slice-adapted 3DGS: bounded additive splatting of projected 2D Gaussians.
 *
 * Inputs (device, fp32): means2d (N,2) in slice-plane mm, inv2d (N,2,2) inverse 2D
 * covariances, weights (N), colors (N,3). Pixel (x, y) sits at
 * (-half_width + 2 half_width x/(W-1), -half_height + 2 half_height y/(H-1)).
 * Outputs: image (H*W, 3) RGB and alpha (H*W) weight sums, as the reference returns them.
 * ---------------------------------------------------------------------------------- */

US3D_API size_t us3d_sa_workspace_bytes(int64_t n, int32_t height, int32_t width, int64_t instance_capacity);
US3D_API size_t us3d_sa_backward_scratch_bytes(int64_t instance_capacity);

/* Replaces bounded_forward (ops/slice_adapted_3dgs_renderer/src/render.cu:836-921) for
 * every N (the reference scatters with atomics below 16384 Gaussians and bins above;
 * results agree up to summation order). Never synchronises. */
US3D_API int us3d_sa_bounded_forward(void* workspace, size_t workspace_bytes, int64_t n, int32_t height,
                                     int32_t width, float half_width, float half_height, const float* means2d,
                                     const float* inv2d, const float* weights, const float* colors,
                                     float radius_sigma, int64_t instance_capacity, float* out_image,
                                     float* out_alpha, void* stream);
US3D_API int us3d_sa_read_status(const void* workspace, int64_t* total_instances, int32_t* overflow,
                                 void* stream);
/* Replaces bounded_backward (render.cu:923-1013): gradients w.r.t. means2d (N,2),
 * inv2d (N,2,2), weights (N) and colors (N,3). Deterministic. */
US3D_API int us3d_sa_bounded_backward(void* workspace, int64_t n, int32_t height, int32_t width, float half_width,
                                      float half_height, const float* means2d, const float* inv2d,
                                      const float* weights, const float* colors, const float* grad_image,
                                      const float* grad_alpha, float radius_sigma, int64_t instance_capacity,
                                      void* scratch, size_t scratch_bytes, float* d_means2d, float* d_inv2d,
                                      float* d_weights, float* d_colors, void* stream);
/* Sorted Gaussian ids and tile ranges (-1 for empty tiles) of the 16x16 binning
 * (reference build_tile_binning, render.cu:673-760). */
US3D_API int us3d_sa_export_bins(const void* workspace, int64_t n, int32_t height, int32_t width,
                                 int64_t instance_capacity, int32_t* out_sorted_ids, int32_t* out_range_start,
                                 int32_t* out_range_end, void* stream);
/* Unbounded splat over arbitrary pixel coordinates (P,2): replaces forward / backward
 * (render.cu:41-153, the package's additive_splat). */
US3D_API int us3d_sa_dense_forward(int64_t n_pixels, int64_t n, const float* pixels, const float* means2d,
                                   const float* inv2d, const float* weights, const float* colors,
                                   float* out_image, float* out_alpha, void* stream);
US3D_API int us3d_sa_dense_backward(int64_t n_pixels, int64_t n, const float* pixels, const float* means2d,
                                    const float* inv2d, const float* weights, const float* colors,
                                    const float* grad_image, const float* grad_alpha, float* d_means2d,
                                    float* d_inv2d, float* d_weights, float* d_colors, void* stream);

/* Fused slice projection of 3D Gaussians for the bounded splat: replaces the PyTorch
 * projection of the slice-adapted adapter (baselines/slice_adapted_3dgs/render.py:66-98,
 * 132-163). Inputs: means (G,3), scales (G,3), quats (G,4) (w,x,y,z), opacities (G),
 * colors (G,3), viewmatrix (4,4 row-major, points as row vectors). Writes the kept
 * Gaussians, in index order, to the first n_kept rows of means2d (G,2), inv2d (G,2,2),
 * weights (G), colors (G,3) and keep_idx (G); keep_mask (G, may be NULL) flags every
 * Gaussian. If out_kept is not NULL, synchronises `stream` and returns the count there. */
US3D_API size_t us3d_sa_project_workspace_bytes(int64_t n_gauss);
US3D_API int us3d_sa_project(void* workspace, size_t workspace_bytes, int64_t n_gauss, const float* means,
                             const float* scales, const float* quats, const float* opacities, const float* colors,
                             const float* viewmatrix, float focal_depth, float slice_thickness, float cull_std,
                             float thickness_scale, float min_covariance, int32_t normalize_by_footprint,
                             float* out_means2d, float* out_inv2d, float* out_weights, float* out_colors,
                             int32_t* out_keep_idx, uint8_t* out_keep_mask, int64_t* out_kept, void* stream);
/* Vector-Jacobian product of us3d_sa_project: gradients of the kept rows in, gradients of
 * means, scales, quats, opacities and colors (all G rows written; zero for culled) out. */
US3D_API int us3d_sa_project_backward(int64_t n_gauss, int64_t n_kept, const int32_t* keep_idx, const float* means,
                                      const float* scales, const float* quats, const float* opacities,
                                      const float* viewmatrix, float focal_depth, float slice_thickness,
                                      float cull_std, float thickness_scale, float min_covariance,
                                      int32_t normalize_by_footprint, const float* d_means2d, const float* d_inv2d,
                                      const float* d_weights, const float* d_colors_kept, float* d_means,
                                      float* d_scales, float* d_quats, float* d_opacities, float* d_colors,
                                      void* stream);

/* ------------------------------------------------------------------------------------
 * UltraGray: scanline B-mode rendering by ray-Gaussian attenuation integrals.
 *
 * Inputs (device, fp32, contiguous): means (G,3), scales (G,3), quats (G,4) (w,x,y,z),
 * attenuations (G) (raw, sigmoid applied inside), sh_coeffs (G,4) degree-1 echo terms,
 * pixel_positions (W,H,3), ray_origins (W,3), ray_dirs (W,3), probe origin and axes (3
 * each), ray_perturbations (W) elevational offsets in mm. W rays (image columns), H
 * samples per ray. Output image (H,W). The workspace keeps the ray binning and, per
 * pixel, the forward's (transmission, echo numerator, echo denominator, weight sum) so
 * the backward needs no recompute pass.
 * ---------------------------------------------------------------------------------- */

US3D_API size_t us3d_ugr_workspace_bytes(int64_t n_gauss, int32_t width, int32_t height,
                                         int64_t instance_capacity);
US3D_API size_t us3d_ugr_backward_scratch_bytes(int64_t instance_capacity);

/* Replaces MapperForwardCUDA followed by ShaderForwardCUDA
 * (ops/ultragray_renderer/src/mapper/wrapper_mapper.cu:7-128,
 * src/shader/wrapper_shader.cu:7-58). Never synchronises; an instance total above
 * instance_capacity sets the overflow flag read by us3d_ugr_read_status and leaves the
 * image unwritten. */
US3D_API int us3d_ugr_forward(void* workspace, size_t workspace_bytes, int64_t n_gauss, const float* means,
                              const float* scales, const float* quats, const float* attenuations,
                              const float* sh_coeffs, const float* pixel_positions, const float* ray_origins,
                              const float* ray_dirs, const float* origin, const float* axis_lateral,
                              const float* axis_elevational, const float* axis_axial,
                              const float* ray_perturbations, int32_t width, int32_t height, float width_mm,
                              float near_mm, float lateral_col_offset, float elev_cutoff_mm, float k_sigma,
                              float quadrature_window_radius_mm, int32_t local_transmission_window_only,
                              float local_transmission_max_window_mm, int64_t instance_capacity,
                              float* out_image, void* stream);
/* Synchronises `stream`: instance total and overflow flags of the last us3d_ugr_forward. */
US3D_API int us3d_ugr_read_status(const void* workspace, int64_t* total_instances, int32_t* overflow,
                                  void* stream);
/* Replaces ShaderBackwardCUDA (src/shader/wrapper_shader.cu:60-123): gradients w.r.t.
 * means (G,3), scales (G,3), quats (G,4), attenuations (G) and sh_coeffs (G,4), every
 * entry written. Deterministic (fixed-order per-Gaussian reduction). */
US3D_API int us3d_ugr_backward(void* workspace, int64_t n_gauss, const float* quats, const float* pixel_positions,
                               const float* ray_origins, const float* ray_dirs, const float* axis_elevational,
                               const float* ray_perturbations, int32_t width, int32_t height, float k_sigma,
                               float quadrature_window_radius_mm, int32_t local_transmission_window_only,
                               float local_transmission_max_window_mm, int64_t instance_capacity,
                               const float* grad_image, void* scratch, size_t scratch_bytes, float* d_means,
                               float* d_scales, float* d_quats, float* d_attenuations, float* d_sh_coeffs,
                               void* stream);
/* The ray binning in MapperForwardCUDA's output format: ray_counts (W), ray_offsets (W,
 * 0 for empty rays), ray_indices and sorted_depths (instance total entries). */
US3D_API int us3d_ugr_export_csr(const void* workspace, int64_t n_gauss, int32_t width, int32_t height,
                                 int64_t instance_capacity, int32_t* out_ray_counts, int32_t* out_ray_offsets,
                                 int32_t* out_ray_indices, float* out_sorted_depths, void* stream);

/* ------------------------------------------------------------------------------------
 * UltraGS baseline: 2D-Gaussian-surfel rasterisation with auxiliary maps.
 *
 * Inputs (device, fp32, contiguous): means3D (P,3); exactly one of shs (P,M,3) with
 * sh_degree/sh_coeffs or colors_precomp (P,3); opacities (P); exactly one of scales (P,2)
 * + rotations (P,4) (w,x,y,z) or transmat_precomp (P,9); viewmatrix, projmatrix (4,4) in
 * the reference's row-vector layout; campos (3) (SH only); background (3). NULL stands for
 * an absent optional input. Outputs: color (3,H,W), others (7,H,W: depth, alpha, normal x3,
 * median depth, distortion) and radii (P). The workspace keeps the binning, the records and
 * the per-pixel compositing state for the backward.
 * ---------------------------------------------------------------------------------- */

US3D_API size_t us3d_gs_workspace_bytes(int64_t n_gauss, int32_t width, int32_t height, int64_t instance_capacity);
US3D_API size_t us3d_gs_backward_scratch_bytes(int64_t instance_capacity);

/* Replaces RasterizeGaussiansCUDA
 * (ops/ultrags_baseline_renderer/rasterize_points.cu:41-133). Never synchronises; an
 * instance total above instance_capacity, or a Gaussian failing the near test while
 * `prefiltered` is set (the reference traps the GPU there), sets a flag read by
 * us3d_gs_read_status and leaves the outputs unwritten. */
US3D_API int us3d_gs_forward(void* workspace, size_t workspace_bytes, int64_t n_gauss, int32_t sh_degree,
                             int32_t sh_coeffs, const float* background, int32_t width, int32_t height,
                             const float* means3D, const float* shs, const float* colors_precomp,
                             const float* opacities, const float* scales, float scale_modifier,
                             const float* rotations, const float* transmat_precomp, const float* viewmatrix,
                             const float* projmatrix, const float* campos, int32_t prefiltered,
                             int64_t instance_capacity, float* out_color, float* out_others, int32_t* out_radii,
                             void* stream);
/* Synchronises `stream`: instance total and flags (1 overflow, 2 table, 4 prefiltered). */
US3D_API int us3d_gs_read_status(const void* workspace, int64_t* total_instances, int32_t* flags, void* stream);
/* Replaces RasterizeGaussiansBackwardCUDA (rasterize_points.cu:135-233). Gradient outputs
 * (every entry written): means2D (P,3), colors (P,3), opacity (P), means3D (P,3),
 * transmat (P,9), sh (P,M,3) when shs is given, scales (P,2) and rotations (P,4) when
 * given (may be NULL otherwise). Deterministic. */
US3D_API int us3d_gs_backward(void* workspace, int64_t n_gauss, int32_t sh_degree, int32_t sh_coeffs,
                              const float* background, int32_t width, int32_t height, const float* means3D,
                              const float* shs, const float* colors_precomp, const float* scales,
                              float scale_modifier, const float* rotations, const float* transmat_precomp,
                              const float* viewmatrix, const float* projmatrix, const float* campos, float tan_fovx,
                              float tan_fovy, const int32_t* radii, int64_t instance_capacity,
                              const float* dL_dcolor, const float* dL_dothers, void* scratch, size_t scratch_bytes,
                              float* d_means2D, float* d_colors, float* d_opacity, float* d_means3D,
                              float* d_transmat, float* d_sh, float* d_scales, float* d_rotations, void* stream);
/* The binning and compositing state in the reference's formats: point_list (instance
 * total), keys (tile << 32 | depth bits; may be NULL), tile ranges (T,2; 0,0 for empty
 * tiles), n_contrib (2,H,W), accum (3,H,W: final T, M1, M2) and the 80-byte records (P,20)
 * (may be NULL). */
US3D_API int us3d_gs_export(const void* workspace, int64_t n_gauss, int32_t width, int32_t height,
                            int64_t instance_capacity, uint32_t* out_point_list, uint64_t* out_keys,
                            uint32_t* out_ranges, uint32_t* out_n_contrib, float* out_accum, float* out_records,
                            void* stream);
/* Replaces markVisible (rasterize_points.cu:235-254): view-space depth > 0.2. */
US3D_API int us3d_gs_mark_visible(int64_t n_gauss, const float* means3D, const float* viewmatrix,
                                  uint8_t* out_present, void* stream);

/*
 * UltraGauss forward render without any device allocation. No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc (an application that owns
 * the device memory pool, or a real-time pipeline that must not allocate or stall while
 * it runs). Does us3d_ug_bin + us3d_ug_forward with the workspace taken from one
 * file-scope device array of US3D_UG_NOALLOC_BYTES bytes that every GPU loading this
 * library holds until exit. Sizes whose workspace does not fit are rejected
 * (US3D_INVALID_ARG) before anything is launched. The rest of the array is split between
 * (Gaussian, frame) pairs surviving the cull and (tile, Gaussian) instances; more of
 * either than fits returns US3D_CAPACITY_OVERFLOW and writes no output. SYNCHRONISES
 * `stream` once (twice on an overflow) to read the instance total, also returned in
 * *out_instances if not NULL; when the surviving pairs overflowed first, the instances
 * were not counted and *out_instances is the number of pairs, a lower bound of the
 * instance total. The first call on a device resolves the array's address and should
 * come before any stream capture on that device (a call failing with US3D_CUDA_ERROR
 * forgets it, so the next call resolves it again). All calls on a device share the array
 * and keep the last call's contents there: calls that overlap on one GPU race.
 */
#define US3D_UG_NOALLOC_BYTES (32 * 1024 * 1024)
US3D_API int us3d_ug_render_noalloc(const us3d_slice_frame* frames_dev, int32_t n_frames, int64_t n_tiles,
                                    int64_t n_pixels, int64_t n_gauss, const float* means,
                                    const float* precision_tril, const float* opacities,
                                    const float* intensities, const float* pixel_positions,
                                    float chi2_threshold, float diag_beta, int32_t sort_by_depth,
                                    float bg_alpha, float bg_intensity, float* out_image, float* out_alpha,
                                    float* out_depth, int32_t* out_counts, int64_t* out_instances, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* US3D_B200_H */
