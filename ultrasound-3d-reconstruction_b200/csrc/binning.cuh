// Tile binning shared by the renderers: header words of a binned workspace, and the
// per-tile ordering of bucketed instances by their 64-bit (depth key << 32 | Gaussian) key.
// Everything here has internal linkage so that each renderer's translation unit carries
// its own copy of the kernels.
#pragma once

#include "us3d_common.cuh"

namespace us3d {

constexpr int SORT_THREADS = 512;
constexpr int SORT_SMEM_CAP = 8192;  // keys sorted in shared memory per tile (96 KB)

// Header words at the start of a binned workspace.
enum { H_TOTAL = 0, H_FLAGS = 1, H_SCAN_G = 2, H_SCAN_T = 3, H_CAP = 4, H_G = 5, H_T = 6, H_P = 7, H_MODE = 8, H_NTASK = 9, H_WORDS = 16 };
enum { FLAG_OVERFLOW = 1, FLAG_TABLE = 2 };

static __device__ __forceinline__ void cswap(unsigned long long* k, int* v, int a, int b) {
    const unsigned long long ka = k[a], kb = k[b];
    if (kb < ka) {
        k[a] = kb;
        k[b] = ka;
        const int t = v[a];
        v[a] = v[b];
        v[b] = t;
    }
}

// Ascending bitonic sort of n (not necessarily a power of two) keys with payload, in the
// "mirror" formulation where every compare-exchange puts the smaller key at the lower
// index; positions >= n act as +infinity and are never touched.
static __device__ void bitonic_sort(unsigned long long* k, int* v, int n) {
    int npow = 1;
    while (npow < n) npow <<= 1;
    const int half_n = npow >> 1;
    for (int size = 2; size <= npow; size <<= 1) {
        const int hs = size >> 1;
        for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
            const int blk = i / hs, off = i - blk * hs;
            const int a = blk * size + off, b = blk * size + size - 1 - off;
            if (b < n) cswap(k, v, a, b);
        }
        __syncthreads();
        for (int h = hs >> 1; h >= 1; h >>= 1) {
            for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
                const int blk = i / h, off = i - blk * h;
                const int a = blk * 2 * h + off, b = a + h;
                if (b < n) cswap(k, v, a, b);
            }
            __syncthreads();
        }
    }
}

// One block per tile: order the tile's bucket by (depth key, Gaussian index), which is the
// order the reference's stable radix sort of (tile << 32 | depth key) over instances
// enumerated Gaussian by Gaussian produces (src/mapper/wrapper_mapper.cu:134-146).
static __global__ void __launch_bounds__(SORT_THREADS)
tile_sort_kernel(int64_t T, const int* __restrict__ tile_start, const long long* __restrict__ header,
                 unsigned long long* __restrict__ keys, int* __restrict__ slot_inst,
                 int* __restrict__ sorted_gid, int* __restrict__ sorted_inst) {
    extern __shared__ unsigned long long s_keys[];
    int* s_idx = reinterpret_cast<int*>(s_keys + SORT_SMEM_CAP);
    const int64_t t = blockIdx.x;
    if (t >= T || header[H_FLAGS] != 0) return;
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    if (n <= 0) return;
    if (n <= SORT_SMEM_CAP) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            s_keys[i] = keys[s0 + i];
            s_idx[i] = i;
        }
        __syncthreads();
        bitonic_sort(s_keys, s_idx, n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long k = s_keys[i];
            sorted_gid[s0 + i] = (int)(uint32_t)(k & 0xffffffffull);
            sorted_inst[s0 + i] = slot_inst[s0 + s_idx[i]];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) keys[s0 + i] = s_keys[i];
    } else {
        // Oversized bucket: same network directly on global memory (one block owns it).
        bitonic_sort(keys + s0, slot_inst + s0, n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            sorted_gid[s0 + i] = (int)(uint32_t)(keys[s0 + i] & 0xffffffffull);
            sorted_inst[s0 + i] = slot_inst[s0 + i];
        }
    }
}


// Raises the sort kernel's dynamic shared-memory limit once per device for the calling
// translation unit's copy of the kernel.
static inline cudaError_t ensure_tile_sort_smem(bool* done_per_device, int n_devices) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < n_devices && done_per_device[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(tile_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             SORT_SMEM_CAP * (int)(sizeof(unsigned long long) + sizeof(int)));
    if (e == cudaSuccess && dev >= 0 && dev < n_devices) done_per_device[dev] = true;
    return e;
}

static inline size_t tile_sort_smem_bytes() { return SORT_SMEM_CAP * (sizeof(unsigned long long) + sizeof(int)); }

}  // namespace us3d
