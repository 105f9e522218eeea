// Error-message plumbing for the C ABI.
#include <stdarg.h>
#include <stdio.h>

#include "us3d_common.cuh"

namespace us3d {

static thread_local char g_last_error[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

}  // namespace us3d

extern "C" const char* us3d_last_error(void) { return us3d::g_last_error; }

extern "C" int us3d_version(void) { return 100; }

extern "C" int us3d_set_device(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        us3d::set_error("cudaSetDevice(%d) failed: %s", device, cudaGetErrorString(e));
        return US3D_CUDA_ERROR;
    }
    return US3D_OK;
}

// ---- launch counter and stage timing (benchmark instrumentation) ----
#include <atomic>
#include <mutex>
#include <string.h>
#include <vector>

namespace us3d {

static std::atomic<long long> g_launches{0};

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

struct StageProfile {
    char name[64] = {0};
    std::vector<cudaEvent_t> start, stop;
    int used = 0;
    bool enabled = false;
};

static std::mutex g_prof_mu;
static StageProfile g_prof;

// Records the "start" event of the next bracket if `name` is the profiled stage.
int prof_begin(const char* name, cudaStream_t stream) {
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_prof.enabled || strcmp(name, g_prof.name) != 0 || g_prof.used >= (int)g_prof.start.size()) return -1;
    cudaEventRecord(g_prof.start[g_prof.used], stream);
    return g_prof.used++;
}

void prof_end(int slot, cudaStream_t stream) {
    if (slot < 0) return;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    cudaEventRecord(g_prof.stop[slot], stream);
}

}  // namespace us3d

extern "C" long long us3d_launch_count(void) { return us3d::g_launches.load(); }

extern "C" int us3d_profile_stage(const char* stage, int max_launches) {
    std::lock_guard<std::mutex> lk(us3d::g_prof_mu);
    auto& p = us3d::g_prof;
    for (size_t i = 0; i < p.start.size(); ++i) {
        cudaEventDestroy(p.start[i]);
        cudaEventDestroy(p.stop[i]);
    }
    p.start.clear();
    p.stop.clear();
    p.used = 0;
    p.enabled = false;
    if (stage == nullptr || max_launches <= 0) return US3D_OK;
    snprintf(p.name, sizeof(p.name), "%s", stage);
    p.start.resize(max_launches);
    p.stop.resize(max_launches);
    for (int i = 0; i < max_launches; ++i) {
        if (cudaEventCreate(&p.start[i]) != cudaSuccess || cudaEventCreate(&p.stop[i]) != cudaSuccess) {
            us3d::set_error("cudaEventCreate failed");
            return US3D_CUDA_ERROR;
        }
    }
    p.enabled = true;
    return US3D_OK;
}

extern "C" int us3d_profile_collect(int* n_launches, double* total_ms) {
    std::lock_guard<std::mutex> lk(us3d::g_prof_mu);
    auto& p = us3d::g_prof;
    double tot = 0.0;
    for (int i = 0; i < p.used; ++i) {
        if (cudaEventSynchronize(p.stop[i]) != cudaSuccess) {
            us3d::set_error("cudaEventSynchronize failed");
            return US3D_CUDA_ERROR;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, p.start[i], p.stop[i]);
        tot += ms;
    }
    if (n_launches) *n_launches = p.used;
    if (total_ms) *total_ms = tot;
    p.used = 0;
    return US3D_OK;
}
