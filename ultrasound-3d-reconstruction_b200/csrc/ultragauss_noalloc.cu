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

#include <algorithm>
#include <mutex>

// Scratch of the no-allocation entry point. In host code this name is a host-side
// stand-in, not a device address: the address is taken once per device with
// cudaGetSymbolAddress and only that pointer is handed to the kernels.
static __device__ __align__(256) unsigned char g_ug_noalloc_scratch[US3D_UG_NOALLOC_BYTES];

namespace us3d {
namespace ug {
// Internal to the library (ultragauss.cu): binning with an explicit (Gaussian, frame) task
// capacity, its workspace size, and the task count of the last binning.
size_t workspace_bytes_with_tasks(int64_t n_gauss, int64_t n_tiles, int64_t n_pixels, int64_t cap, int64_t tc);
int read_task_count(const void* workspace, int64_t* n_tasks, void* stream);
int bin_with_task_capacity(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames, int32_t n_frames,
                           int64_t n_tiles, int64_t n_pixels, int64_t n_gauss, const float* means, const float* tril,
                           const float* opac, const float* inten, float chi2, float beta, int32_t sort_by_depth,
                           int64_t cap, int64_t task_cap, const float* pixels, int32_t flags, void* stream_);
}  // namespace ug
}  // namespace us3d

namespace {

constexpr int kMaxDevices = 128;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Set-up, once per device with that device current: resolve the device address of the
// scratch array. Runs on the first call made on each device; that call should therefore
// happen before any stream capture on the device. A call that fails with a CUDA error
// forgets the address (forget_scratch), so that a device that was reset and given a new
// context resolves it again on its next call.
int scratch_for_current_device(void** out, int* dev_out) {
    int dev = 0;
    US3D_CHECK_CUDA(cudaGetDevice(&dev));
    US3D_CHECK_ARG(dev >= 0 && dev < kMaxDevices, "device index %d out of range", dev);
    *dev_out = dev;
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

void forget_scratch(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev >= 0 && dev < kMaxDevices) g_scratch_ptr[dev] = nullptr;
}

// Splits the array between (Gaussian, frame) tasks and (tile, Gaussian) instances. A full
// binning gives every task at least one instance, so there are never more tasks than
// instances nor more than n_gauss * n_frames: the task capacity is the smaller of
// n_gauss * n_frames and the instance capacity, and the instance capacity is the largest
// that fits with it. A task overflow then always comes with an instance overflow, and no
// input is refused for its tasks while its instances would fit. The layout is monotonic
// in both capacities, so a bisection finds the largest instance capacity.
bool split_scratch(int64_t G, int64_t F, int64_t T, int64_t P, int64_t* cap_out, int64_t* tc_out) {
    const size_t limit = (size_t)US3D_UG_NOALLOC_BYTES;
    const int64_t pairs = G * F;
    auto fits = [&](int64_t cap) {
        const int64_t tc = std::min<int64_t>(pairs, cap);
        const size_t b = us3d::ug::workspace_bytes_with_tasks(G, T, P, cap, tc);
        return b > 0 && b <= limit;
    };
    if (!fits(1)) return false;
    int64_t lo = 1, hi = (int64_t)(limit / 8);  // every instance takes more than 8 bytes
    while (lo < hi) {
        const int64_t mid = lo + (hi - lo + 1) / 2;
        if (fits(mid)) lo = mid; else hi = mid - 1;
    }
    *cap_out = lo;
    *tc_out = std::min<int64_t>(pairs, lo);
    return true;
}

int render(const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
           const float* means, const float* precision_tril, const float* opacities, const float* intensities,
           const float* pixel_positions, float chi2_threshold, float diag_beta, int32_t sort_by_depth, float bg_alpha,
           float bg_intensity, float* out_image, float* out_alpha, float* out_depth, int32_t* out_counts,
           int64_t* out_instances, void* stream, int* dev) {
    US3D_CHECK_ARG(n_gauss >= 0 && n_tiles >= 0 && n_pixels >= 0 && n_frames >= 0, "negative size");
    int64_t cap = 0, tc = 0;
    const size_t base = us3d_ug_workspace_bytes(n_gauss, n_frames, n_tiles, n_pixels, 0);
    US3D_CHECK_ARG(split_scratch(n_gauss, n_frames, n_tiles, n_pixels, &cap, &tc),
                   "sizes exceed the no-allocation scratch (%zu bytes needed before any instance, %d available): "
                   "G=%lld tiles=%lld pixels=%lld",
                   base, (int)US3D_UG_NOALLOC_BYTES, (long long)n_gauss, (long long)n_tiles, (long long)n_pixels);

    void* ws = nullptr;
    int st = scratch_for_current_device(&ws, dev);
    if (st != US3D_OK) return st;
    st = us3d::ug::bin_with_task_capacity(ws, US3D_UG_NOALLOC_BYTES, frames, n_frames, n_tiles, n_pixels, n_gauss,
                                          means, precision_tril, opacities, intensities, chi2_threshold, diag_beta,
                                          sort_by_depth, cap, tc, nullptr, 0, stream);
    if (st != US3D_OK) return st;
    int64_t total = 0, n_tasks = 0;
    int32_t flags = 0;
    st = us3d_ug_read_status(ws, &total, &flags, stream);  // synchronises `stream`
    if (st != US3D_OK) return st;
    if (flags != 0) {
        st = us3d::ug::read_task_count(ws, &n_tasks, stream);
        if (st != US3D_OK) return st;
        if (n_tasks > tc) {
            // the instances were never counted; each task has at least one
            if (out_instances) *out_instances = n_tasks;
            us3d::set_error("no-allocation render: %lld (Gaussian, frame) pairs survive the cull, more than the %lld "
                            "(tile, Gaussian) instances that fit in the %d-byte scratch (each pair has at least one "
                            "instance; the instance total was not counted)",
                            (long long)n_tasks, (long long)cap, (int)US3D_UG_NOALLOC_BYTES);
            return US3D_CAPACITY_OVERFLOW;
        }
    }
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

}  // namespace

extern "C" int us3d_ug_render_noalloc(const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles,
                                      int64_t n_pixels, int64_t n_gauss, const float* means,
                                      const float* precision_tril, const float* opacities,
                                      const float* intensities, const float* pixel_positions, float chi2_threshold,
                                      float diag_beta, int32_t sort_by_depth, float bg_alpha, float bg_intensity,
                                      float* out_image, float* out_alpha, float* out_depth, int32_t* out_counts,
                                      int64_t* out_instances, void* stream) {
    int dev = -1;
    const int st = render(frames, n_frames, n_tiles, n_pixels, n_gauss, means, precision_tril, opacities, intensities,
                          pixel_positions, chi2_threshold, diag_beta, sort_by_depth, bg_alpha, bg_intensity, out_image,
                          out_alpha, out_depth, out_counts, out_instances, stream, &dev);
    if (st == US3D_CUDA_ERROR) forget_scratch(dev);
    return st;
}
