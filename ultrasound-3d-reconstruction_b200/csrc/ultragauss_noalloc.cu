// UltraGauss forward render (binning + shading) that allocates no device memory.
//
// Some callers cannot call cudaMalloc: an application that owns the whole device memory
// pool (a scanner's real-time imaging pipeline or a host framework with its own allocator
// that forbids raw allocations after start-up), or code that must not allocate while it
// runs (cudaMalloc can synchronise the device and stall a real-time stream). For them this
// entry point takes its scratch memory from one file-scope device array of fixed size
// instead of a caller-provided workspace. The caller still passes all inputs and outputs.
//
// The array is US3D_UG_NOALLOC_BYTES (32 MiB) on every GPU that loads this library, held
// until the process exits. All calls on one device share it and it keeps the last call's
// contents: calls that overlap on that GPU (two streams or two host threads) race on it
// and must be serialised by the caller. Nothing in it needs to start at zero: the binning
// clears the counters it uses at the start of every call.
#include "us3d_common.cuh"

#include <mutex>

// Scratch of the no-allocation entry point. In host code this name is a host-side
// stand-in, not a device address: the address is taken once per device with
// cudaGetSymbolAddress and only that pointer is handed to the kernels.
static __device__ __align__(256) unsigned char g_ug_noalloc_scratch[US3D_UG_NOALLOC_BYTES];

namespace {

constexpr int kMaxDevices = 128;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Set-up, once per device with that device current: resolve the device address of the
// scratch array. Runs on the first call made on each device; that call should therefore
// happen before any stream capture on the device.
int scratch_for_current_device(void** out) {
    int dev = 0;
    US3D_CHECK_CUDA(cudaGetDevice(&dev));
    US3D_CHECK_ARG(dev >= 0 && dev < kMaxDevices, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_ug_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            us3d::set_error("cudaGetSymbolAddress(no-allocation scratch) failed on device %d: %s", dev,
                            cudaGetErrorString(e));
            return US3D_CUDA_ERROR;
        }
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return US3D_OK;
}

}  // namespace

extern "C" int us3d_ug_render_noalloc(const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles,
                                      int64_t n_pixels, int64_t n_gauss, const float* means,
                                      const float* precision_tril, const float* opacities,
                                      const float* intensities, const float* pixel_positions, float chi2_threshold,
                                      float diag_beta, int32_t sort_by_depth, float bg_alpha, float bg_intensity,
                                      float* out_image, float* out_alpha, float* out_depth, int32_t* out_counts,
                                      int64_t* out_instances, void* stream) {
    US3D_CHECK_ARG(n_gauss >= 0 && n_tiles >= 0 && n_pixels >= 0 && n_frames >= 0, "negative size");
    // Largest instance capacity whose workspace fits the fixed array for these sizes.
    const size_t base = us3d_ug_workspace_bytes(n_gauss, n_frames, n_tiles, n_pixels, 0);
    US3D_CHECK_ARG(base > 0 && base + 4096 <= (size_t)US3D_UG_NOALLOC_BYTES,
                   "sizes exceed the no-allocation scratch (%zu bytes needed before any instance, %d available): "
                   "G=%lld tiles=%lld pixels=%lld",
                   base, (int)US3D_UG_NOALLOC_BYTES, (long long)n_gauss, (long long)n_tiles, (long long)n_pixels);
    int64_t cap = (int64_t)(((size_t)US3D_UG_NOALLOC_BYTES - base) / 20);
    while (cap > 0 && us3d_ug_workspace_bytes(n_gauss, n_frames, n_tiles, n_pixels, cap) > (size_t)US3D_UG_NOALLOC_BYTES)
        cap -= 64;
    US3D_CHECK_ARG(cap > 0, "no room for instances in the no-allocation scratch");

    void* ws = nullptr;
    int st = scratch_for_current_device(&ws);
    if (st != US3D_OK) return st;
    st = us3d_ug_bin(ws, US3D_UG_NOALLOC_BYTES, frames, n_frames, n_tiles, n_pixels, n_gauss, means, precision_tril,
                     opacities, intensities, chi2_threshold, diag_beta, sort_by_depth, cap, stream);
    if (st != US3D_OK) return st;
    int64_t total = 0;
    int32_t flags = 0;
    st = us3d_ug_read_status(ws, &total, &flags, stream);  // synchronises `stream`
    if (st != US3D_OK) return st;
    if (out_instances) *out_instances = total;
    if (flags != 0) {
        us3d::set_error("no-allocation render: %lld (tile, Gaussian) instances exceed the %lld that fit in the "
                        "%d-byte scratch (flags=%d)",
                        (long long)total, (long long)cap, (int)US3D_UG_NOALLOC_BYTES, (int)flags);
        return US3D_CAPACITY_OVERFLOW;
    }
    return us3d_ug_forward(ws, frames, n_frames, n_tiles, n_pixels, n_gauss, cap, pixel_positions, chi2_threshold,
                           diag_beta, bg_alpha, bg_intensity, out_image, out_alpha, out_depth, out_counts, stream);
}
