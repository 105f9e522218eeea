// Device-wide exclusive prefix sum of int32 counts (three launches, no spin-waits).
//
//   1. scan_reduce:     each 4096-element block reduces its counts to an int64 sum;
//   2. scan_blocksums:  one block scans the block sums in place and stores the total;
//   3. scan_downsweep:  each block scans its counts again and adds its block prefix.
//
// out[i] = sum(in[0..i)) for i in [0, n], out[n] = total (int32, valid while the total
// fits; the int64 total is also stored for overflow checks by the caller).
#pragma once

#include "us3d_common.cuh"

namespace us3d {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

static inline int scan_num_blocks(int64_t n) { return (int)((n + SCAN_TILE - 1) / SCAN_TILE); }

// Inclusive warp scan of a 64-bit value.
static __device__ __forceinline__ long long warp_inclusive_scan(long long v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan (blockDim.x == SCAN_THREADS); returns the block total in *total.
static __device__ __forceinline__ long long block_exclusive_scan(long long v, long long* total) {
    __shared__ long long warp_sums[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    long long inc = warp_inclusive_scan(v);
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        long long s = (lane < SCAN_THREADS / 32) ? warp_sums[lane] : 0;
        long long si = warp_inclusive_scan(s);
        if (lane < SCAN_THREADS / 32) warp_sums[lane] = si - s;
    }
    __syncthreads();
    long long excl = inc - v + warp_sums[warp];
    // Total = exclusive prefix of the last thread + its value.
    __shared__ long long s_total;
    if (threadIdx.x == SCAN_THREADS - 1) s_total = excl + v;
    __syncthreads();
    *total = s_total;
    return excl;
}

static __device__ __forceinline__ void load_items(const int* in, int64_t n, int64_t base, int (&x)[SCAN_ITEMS]) {
    if (base + SCAN_ITEMS <= n && ((reinterpret_cast<uintptr_t>(in + base) & 15) == 0)) {
        const int4* p = reinterpret_cast<const int4*>(in + base);
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS / 4; ++k) {
            int4 v = p[k];
            x[4 * k + 0] = v.x; x[4 * k + 1] = v.y; x[4 * k + 2] = v.z; x[4 * k + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; ++k) x[k] = (base + k < n) ? in[base + k] : 0;
    }
}

static __global__ void __launch_bounds__(SCAN_THREADS)
scan_reduce_kernel(const int* __restrict__ in, int64_t n, long long* __restrict__ block_sums) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int x[SCAN_ITEMS];
    load_items(in, n, base, x);
    long long s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) s += x[k];
    long long total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(SCAN_THREADS)
scan_blocksums_kernel(long long* __restrict__ block_sums, int nb, long long* __restrict__ total_out) {
    long long carry = 0;
    for (int base = 0; base < nb; base += SCAN_THREADS) {
        const int i = base + threadIdx.x;
        long long v = (i < nb) ? block_sums[i] : 0;
        long long tot;
        long long ex = block_exclusive_scan(v, &tot);
        if (i < nb) block_sums[i] = carry + ex;
        carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total_out = carry;
}

static __global__ void __launch_bounds__(SCAN_THREADS)
scan_downsweep_kernel(const int* __restrict__ in, int64_t n, const long long* __restrict__ block_sums,
                      const long long* __restrict__ total, int* __restrict__ out) {
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int x[SCAN_ITEMS];
    load_items(in, n, base, x);
    long long s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) s += x[k];
    long long btot;
    long long run = block_exclusive_scan(s, &btot) + block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = (int)run;
        run += x[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        long long t = *total;
        out[n] = (t > 0x7fffffffLL) ? 0x7fffffff : (int)t;
    }
}

// Launches the three phases. block_sums must hold scan_num_blocks(n) entries (>= 1).
static inline cudaError_t exclusive_scan(const int* in, int64_t n, int* out, long long* block_sums,
                                         long long* total, cudaStream_t stream) {
    const int nb = scan_num_blocks(n) > 0 ? scan_num_blocks(n) : 1;
    scan_reduce_kernel<<<nb, SCAN_THREADS, 0, stream>>>(in, n, block_sums);
    scan_blocksums_kernel<<<1, SCAN_THREADS, 0, stream>>>(block_sums, nb, total);
    scan_downsweep_kernel<<<nb, SCAN_THREADS, 0, stream>>>(in, n, block_sums, total, out);
    return cudaGetLastError();
}

}  // namespace us3d
