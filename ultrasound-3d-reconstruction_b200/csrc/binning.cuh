// Tile binning shared by the renderers: header words of a binned workspace, and the
// per-tile ordering of bucketed instances by their 64-bit (depth key << 32 | Gaussian) key.
// Everything here has internal linkage so that each renderer's translation unit carries
// its own copy of the kernels.
#pragma once

#include "us3d_common.cuh"

namespace us3d {

constexpr int SORT_THREADS = 512;
// Tiles of up to SORT_SMEM_CAP keys are ordered in shared memory by the first sort pass
// (48 KB, four 512-thread blocks per SM); up to SORT_MID_CAP keys, when every element index of
// the call fits a 13-bit slot packing, by a pass with 64 KB (two 1024-thread blocks per SM); larger ones,
// up to SORT_BIG_CAP, by a pass with 192 KB (one block per SM); up to SORT_HUGE_CAP, when the
// bucket's keys pack into 64-bit words, by a pass with 222 KB (one block per SM); beyond that
// the network runs on global memory (one block per tile).
constexpr int SORT_SMEM_CAP = 4096;
constexpr int SORT_BIG_CAP = 16384;
constexpr int SORT_MIN_BLOCKS = 4;
// Above every real key: a key's low word is a Gaussian (or instance) index below 2^31.
constexpr unsigned long long SORT_PAD_KEY = ~0ull;

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
// index; positions >= n act as +infinity and are never touched. Used on global memory for
// buckets too large for shared memory.
static __device__ void bitonic_sort(unsigned long long* k, int* v, int n) {
    int npow = 1, lp = 0;
    while (npow < n) {
        npow <<= 1;
        ++lp;
    }
    const int half_n = npow >> 1;
    for (int ls = 1; ls <= lp; ++ls) {
        const int size = 1 << ls, lh = ls - 1, hs = size >> 1;
        for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
            const int base = (i >> lh) << ls, off = i & (hs - 1);
            const int b = base + size - 1 - off;
            if (b < n) cswap(k, v, base + off, b);
        }
        __syncthreads();
        for (int l2 = lh - 1; l2 >= 0; --l2) {
            const int h = 1 << l2;
            for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
                const int a = ((i >> l2) << (l2 + 1)) + (i & (h - 1)), b = a + h;
                if (b < n) cswap(k, v, a, b);
            }
            __syncthreads();
        }
    }
}

// ------------------------------------------------------------------------------------
// Bucket filling for renderers whose element g has the instances of a half-open rectangle
// (x0, y0, x1, y1) of a gx-wide bucket grid, enumerated row by row (nothing when x0 >= x1 or
// y0 >= y1). When the grid has at most BLOCK_BUCKETS_MAX buckets, a block first counts in
// shared memory and touches each global counter once per bucket it fills, so that a few buckets
// receiving many instances (a small image, large splats) do not serialise on same-address
// global atomics.
// ------------------------------------------------------------------------------------
constexpr int BUCKET_THREADS = 256;
constexpr int BLOCK_BUCKETS_MAX = 4096;

struct RectOf4 {
    const int4* r;
    __device__ __forceinline__ int4 operator()(int64_t g) const { return r[g]; }
};

// An inclusive 1D range (r0, r1) as the rectangle (r0, 0, r1 + 1, 1).
struct RangeOf2 {
    const int2* r;
    __device__ __forceinline__ int4 operator()(int64_t g) const {
        const int2 v = r[g];
        return make_int4(v.x, 0, v.y + 1, 1);
    }
};

static inline bool bucket_counts_in_smem(int64_t n_buckets) { return n_buckets <= BLOCK_BUCKETS_MAX; }

// Instances per bucket (count[] must be zero on entry). Dynamic shared memory: n_buckets ints
// when bucket_counts_in_smem(n_buckets), else none.
template <class Rect>
static __global__ void __launch_bounds__(BUCKET_THREADS)
rect_count_kernel(int64_t n, int gx, int n_buckets, int use_smem, Rect rect, int* __restrict__ count) {
    extern __shared__ int s_cnt[];
    if (use_smem) {
        for (int i = threadIdx.x; i < n_buckets; i += blockDim.x) s_cnt[i] = 0;
        __syncthreads();
    }
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g < n) {
        const int4 r = rect(g);
        for (int y = r.y; y < r.w; ++y)
            for (int x = r.x; x < r.z; ++x) atomicAdd(use_smem ? &s_cnt[y * gx + x] : &count[y * gx + x], 1);
    }
    if (use_smem) {
        __syncthreads();
        for (int i = threadIdx.x; i < n_buckets; i += blockDim.x)
            if (s_cnt[i] != 0) atomicAdd(&count[i], s_cnt[i]);
    }
}

// Writes element g's instances into their buckets: key (dkey[g] << 32 | g) (dkey NULL: 0),
// instance id inst_offset[g] + ordinal in enumeration order. A slot never leaves its bucket.
// Dynamic shared memory: 2 * n_buckets ints when use_smem (slots reserved once per block and
// bucket), else none.
template <class Rect>
static __global__ void __launch_bounds__(BUCKET_THREADS)
rect_scatter_kernel(int64_t n, int gx, int n_buckets, int use_smem, Rect rect, const uint32_t* __restrict__ dkey,
                    const int* __restrict__ inst_offset, const int* __restrict__ start, int* __restrict__ cursor,
                    const long long* __restrict__ header, unsigned long long* __restrict__ keys,
                    int* __restrict__ slot_inst) {
    extern __shared__ int s_buf[];
    if (header[H_FLAGS] != 0) return;
    int* s_cnt = s_buf;
    int* s_base = s_buf + n_buckets;
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int4 r = g < n ? rect(g) : make_int4(0, 0, 0, 0);
    if (use_smem) {
        for (int i = threadIdx.x; i < n_buckets; i += blockDim.x) s_cnt[i] = 0;
        __syncthreads();
        for (int y = r.y; y < r.w; ++y)
            for (int x = r.x; x < r.z; ++x) atomicAdd(&s_cnt[y * gx + x], 1);
        __syncthreads();
        for (int i = threadIdx.x; i < n_buckets; i += blockDim.x)
            if (s_cnt[i] != 0) {
                s_base[i] = atomicAdd(&cursor[i], s_cnt[i]);
                s_cnt[i] = 0;
            }
        __syncthreads();
    }
    if (r.x >= r.z || r.y >= r.w) return;
    const unsigned long long key =
        ((unsigned long long)(dkey ? dkey[g] : 0u) << 32) | (unsigned long long)(uint32_t)g;
    int inst = inst_offset[g];
    for (int y = r.y; y < r.w; ++y)
        for (int x = r.x; x < r.z; ++x) {
            const int t = y * gx + x;
            const int within = use_smem ? s_base[t] + atomicAdd(&s_cnt[t], 1) : atomicAdd(&cursor[t], 1);
            const int slot = start[t] + within;
            if (slot < start[t + 1]) {
                keys[slot] = key;
                slot_inst[slot] = inst;
            }
            ++inst;
        }
}

// Launches rect_count_kernel / rect_scatter_kernel with their shared memory.
template <class Rect>
static inline cudaError_t launch_rect_count(int64_t n, int gx, int64_t n_buckets, Rect rect, int* count,
                                            cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int sm = bucket_counts_in_smem(n_buckets) ? 1 : 0;
    rect_count_kernel<Rect><<<(unsigned)((n + BUCKET_THREADS - 1) / BUCKET_THREADS), BUCKET_THREADS,
                              sm ? (size_t)n_buckets * sizeof(int) : 0, stream>>>(n, gx, (int)n_buckets, sm, rect,
                                                                                  count);
    return cudaGetLastError();
}

template <class Rect>
static inline cudaError_t launch_rect_scatter(int64_t n, int gx, int64_t n_buckets, Rect rect, const uint32_t* dkey,
                                              const int* inst_offset, const int* start, int* cursor,
                                              const long long* header, unsigned long long* keys, int* slot_inst,
                                              cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    const int sm = bucket_counts_in_smem(n_buckets) ? 1 : 0;
    rect_scatter_kernel<Rect><<<(unsigned)((n + BUCKET_THREADS - 1) / BUCKET_THREADS), BUCKET_THREADS,
                                sm ? (size_t)n_buckets * 2 * sizeof(int) : 0, stream>>>(
        n, gx, (int)n_buckets, sm, rect, dkey, inst_offset, start, cursor, header, keys, slot_inst);
    return cudaGetLastError();
}

// Register-resident part of the shared-memory sort. A warp owns a 64-element segment; lane
// l holds its elements 2l (x0) and 2l + 1 (x1). A compare-exchange of stride h >= 2 pairs
// lane l with lane l ^ h/2 (same slot); a mirror pass over blocks of `size` pairs element
// e with e ^ (size - 1), i.e. slot 0 of lane l with slot 1 of lane l ^ (size/2 - 1).
// (Four keys per lane, 128-element segments and four fewer shared-memory passes for a 1024-key
// tile, measured slower on every renderer: bin stage 1.07 -> 1.10-1.17 ms for 16 headline
// frames, UltraGS forward 0.343 -> 0.365 ms. The compare-exchanges are the same network's.)
template <bool PAY>
struct SortEl;  // a key with (PAY) or without its int payload
template <>
struct SortEl<true> {
    unsigned long long k;
    int v;
};
template <>
struct SortEl<false> {
    unsigned long long k;
};

template <bool PAY>
static __device__ __forceinline__ SortEl<PAY> kv_shfl_xor(const SortEl<PAY>& x, int mask) {
    SortEl<PAY> y;
    y.k = __shfl_xor_sync(0xffffffffu, x.k, mask);
    if constexpr (PAY) y.v = __shfl_xor_sync(0xffffffffu, x.v, mask);
    return y;
}

// x becomes the smaller (keep_low) or the larger key of the pair; an equal key keeps x.
template <bool PAY>
static __device__ __forceinline__ void kv_keep(SortEl<PAY>& x, const SortEl<PAY>& y, bool keep_low) {
    if (keep_low ? (y.k < x.k) : (x.k < y.k)) x = y;
}

template <bool PAY>
static __device__ __forceinline__ void kv_order(SortEl<PAY>& a, SortEl<PAY>& b) {
    if (b.k < a.k) {
        const SortEl<PAY> t = a;
        a = b;
        b = t;
    }
}

template <bool PAY>
static __device__ __forceinline__ void warp_stride_pass(SortEl<PAY>& x0, SortEl<PAY>& x1, int h, int lane) {
    if (h == 1) {
        kv_order(x0, x1);
        return;
    }
    const int m = h >> 1;
    const bool low = (lane & m) == 0;
    const SortEl<PAY> y0 = kv_shfl_xor(x0, m), y1 = kv_shfl_xor(x1, m);
    kv_keep(x0, y0, low);
    kv_keep(x1, y1, low);
}

template <bool PAY>
static __device__ __forceinline__ void warp_mirror_pass(SortEl<PAY>& x0, SortEl<PAY>& x1, int size, int lane) {
    if (size == 2) {
        kv_order(x0, x1);
        return;
    }
    const int m = (size >> 1) - 1;
    const bool low = (lane & (size >> 2)) == 0;
    const SortEl<PAY> y0 = kv_shfl_xor(x1, m), y1 = kv_shfl_xor(x0, m);
    kv_keep(x0, y0, low);
    kv_keep(x1, y1, low);
}

template <bool PAY>
static __device__ __forceinline__ void seg_load(const unsigned long long* sk, const int* sv, int seg, int lane,
                                                SortEl<PAY>& x0, SortEl<PAY>& x1) {
    const ulonglong2 k = reinterpret_cast<const ulonglong2*>(sk)[seg * 32 + lane];
    x0.k = k.x;
    x1.k = k.y;
    if constexpr (PAY) {
        const int2 v = reinterpret_cast<const int2*>(sv)[seg * 32 + lane];
        x0.v = v.x;
        x1.v = v.y;
    }
}

template <bool PAY>
static __device__ __forceinline__ void seg_store(unsigned long long* sk, int* sv, int seg, int lane,
                                                 const SortEl<PAY>& x0, const SortEl<PAY>& x1) {
    reinterpret_cast<ulonglong2*>(sk)[seg * 32 + lane] = make_ulonglong2(x0.k, x1.k);
    if constexpr (PAY) reinterpret_cast<int2*>(sv)[seg * 32 + lane] = make_int2(x0.v, x1.v);
}

template <bool PAY>
static __device__ __forceinline__ void cswap_smem(unsigned long long* k, int* v, int a, int b) {
    const unsigned long long ka = k[a], kb = k[b];
    if (kb < ka) {
        k[a] = kb;
        k[b] = ka;
        if constexpr (PAY) {
            const int t = v[a];
            v[a] = v[b];
            v[b] = t;
        }
    }
}

// Ascending sort of the npow (a power of two >= 64) keys, with (PAY) or without an int payload,
// in shared memory (16-byte aligned key array, 8-byte aligned payload array), the same mirror
// network as bitonic_sort: passes that stay inside 64-element segments run in registers with
// warp shuffles, the others as shared-memory compare-exchanges between block barriers. The
// caller pads the keys past the first n with SORT_PAD_KEY and synchronises first. Every
// compare-exchange puts the smaller key at the lower index, so the padding never moves and an
// exchange whose upper index is >= n does nothing: those exchanges, and the 64-element
// segments lying wholly in the padding, are skipped.
template <bool PAY>
static __device__ void block_sort_smem(unsigned long long* sk, int* sv, int npow, int n) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int nseg = (n + 63) >> 6, half_n = npow >> 1;
    for (int s = warp; s < nseg; s += nwarp) {
        SortEl<PAY> x0, x1;
        seg_load(sk, sv, s, lane, x0, x1);
#pragma unroll
        for (int size = 2; size <= 64; size <<= 1) {
            warp_mirror_pass(x0, x1, size, lane);
#pragma unroll
            for (int h = size >> 2; h >= 1; h >>= 1) warp_stride_pass(x0, x1, h, lane);
        }
        seg_store(sk, sv, s, lane, x0, x1);
    }
    __syncthreads();
    for (int ls = 7; (1 << ls) <= npow; ++ls) {
        const int size = 1 << ls, lh = ls - 1, hs = size >> 1;
        for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
            const int base = (i >> lh) << ls, off = i & (hs - 1);
            const int b = base + size - 1 - off;
            if (b < n) cswap_smem<PAY>(sk, sv, base + off, b);
        }
        __syncthreads();
        for (int l2 = lh - 1; l2 >= 6; --l2) {
            const int h = 1 << l2;
            for (int i = threadIdx.x; i < half_n; i += blockDim.x) {
                const int a = ((i >> l2) << (l2 + 1)) + (i & (h - 1));
                if (a + h < n) cswap_smem<PAY>(sk, sv, a, a + h);
            }
            __syncthreads();
        }
        for (int s = warp; s < nseg; s += nwarp) {
            SortEl<PAY> x0, x1;
            seg_load(sk, sv, s, lane, x0, x1);
#pragma unroll
            for (int h = 32; h >= 1; h >>= 1) warp_stride_pass(x0, x1, h, lane);
            seg_store(sk, sv, s, lane, x0, x1);
        }
        __syncthreads();
    }
}

// Buckets of at most SORT_SMEM_CAP keys whose element indices (a key's low word) are below
// SORT_PACK_G can be ordered without a payload: the key (hi << 32 | g) is packed as
// (hi << 32 | g << 12 | slot), which orders like the key itself (a bucket holds an element
// once) and carries the bucket slot in its low 12 bits.
constexpr int64_t SORT_PACK_G = (1 << 20) - 1;
// Buckets of SORT_SMEM_CAP < n <= SORT_MID_CAP keys whose element indices are below
// SORT_PACK_G_MID sort the same way with a 13-bit slot field, in 64 KB (two 1024-thread blocks per SM).
constexpr int SORT_MID_CAP = 8192;
constexpr int SORT_MID_SLOT_BITS = 13;
constexpr int64_t SORT_PACK_G_MID = (1 << 19) - 1;

// The packed sort of bucket t (n keys at s0, n <= 2^slot_bits, every element index below
// 2^(32 - slot_bits)): the key (hi << 32 | g) is packed as (hi << 32 | g << slot_bits | slot),
// which orders like the key itself (a bucket holds an element once) and carries the bucket
// slot in its low slot_bits bits.
static __device__ __forceinline__ void sort_bucket_packed(unsigned long long* s_keys, int s0, int n, int slot_bits,
                                                          unsigned long long* __restrict__ keys,
                                                          const int* __restrict__ slot_inst,
                                                          int* __restrict__ sorted_gid, int* __restrict__ sorted_inst,
                                                          const uint16_t* __restrict__ slot_mask,
                                                          uint16_t* __restrict__ sorted_mask) {
    int npow = 64;
    while (npow < n) npow <<= 1;
    const unsigned long long gmask = (1ull << (32 - slot_bits)) - 1ull, smask = (1ull << slot_bits) - 1ull;
    for (int i = threadIdx.x; i < npow; i += blockDim.x) {
        const unsigned long long k = i < n ? keys[s0 + i] : 0ull;
        s_keys[i] = i < n ? ((k & 0xffffffff00000000ull) | ((k & gmask) << slot_bits) | (unsigned long long)i)
                          : SORT_PAD_KEY;
    }
    __syncthreads();
    block_sort_smem<false>(s_keys, nullptr, npow, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long k = s_keys[i];
        const int slot = (int)(k & smask);
        const uint32_t g = (uint32_t)((k >> slot_bits) & gmask);
        sorted_gid[s0 + i] = (int)g;
        sorted_inst[s0 + i] = slot_inst[s0 + slot];
        if (sorted_mask) sorted_mask[s0 + i] = slot_mask[s0 + slot];
        keys[s0 + i] = (k & 0xffffffff00000000ull) | g;
    }
}

// Orders bucket t (n keys at s0) in shared memory of capacity `cap` (a power of two >= n)
// and writes the sorted Gaussian indices, instance ids and keys; `packed`: every element index
// of the bucket is below SORT_PACK_G (then buckets of up to SORT_SMEM_CAP keys sort without a
// payload).
static __device__ __forceinline__ void sort_bucket_smem(unsigned long long* s_keys, int* s_idx, int s0, int n,
                                                        unsigned long long* __restrict__ keys,
                                                        const int* __restrict__ slot_inst,
                                                        int* __restrict__ sorted_gid, int* __restrict__ sorted_inst,
                                                        const uint16_t* __restrict__ slot_mask,
                                                        uint16_t* __restrict__ sorted_mask, bool packed) {
    if (packed && n <= SORT_SMEM_CAP) {
        sort_bucket_packed(s_keys, s0, n, 12, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
        return;
    }
    int npow = 64;
    while (npow < n) npow <<= 1;
    for (int i = threadIdx.x; i < npow; i += blockDim.x) {
        s_keys[i] = i < n ? keys[s0 + i] : SORT_PAD_KEY;
        s_idx[i] = i;
    }
    __syncthreads();
    block_sort_smem<true>(s_keys, s_idx, npow, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const unsigned long long k = s_keys[i];
        sorted_gid[s0 + i] = (int)(uint32_t)(k & 0xffffffffull);
        sorted_inst[s0 + i] = slot_inst[s0 + s_idx[i]];
        if (sorted_mask) sorted_mask[s0 + i] = slot_mask[s0 + s_idx[i]];
        keys[s0 + i] = k;
    }
}

// A bucket too large for any shared-memory pass: the network directly on global memory (the
// calling block owns the bucket), with the slot indices as payload in sorted_inst.
static __device__ void sort_bucket_global(int s0, int n, unsigned long long* __restrict__ keys,
                                          const int* __restrict__ slot_inst, int* __restrict__ sorted_gid,
                                          int* __restrict__ sorted_inst, const uint16_t* __restrict__ slot_mask,
                                          uint16_t* __restrict__ sorted_mask) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) sorted_inst[s0 + i] = i;
    __syncthreads();
    bitonic_sort(keys + s0, sorted_inst + s0, n);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int slot = sorted_inst[s0 + i];
        sorted_gid[s0 + i] = (int)(uint32_t)(keys[s0 + i] & 0xffffffffull);
        sorted_inst[s0 + i] = slot_inst[s0 + slot];
        if (sorted_mask) sorted_mask[s0 + i] = slot_mask[s0 + slot];
    }
}

// Buckets of SORT_BIG_CAP < n <= SORT_HUGE_CAP keys: when the call's element indices need
// gbits bits and every depth key of the bucket is below 2^(64 - gbits - 15), the key
// (hi << 32 | g) is packed as (hi << (gbits + 15) | g << 15 | slot) -- same order, slot in the
// low 15 bits -- and the bucket sorts in 222 KB of shared memory (the network touches only the
// first ceil(n / 64) * 64 entries); otherwise the global-memory network orders it.
constexpr int SORT_HUGE_CAP = 28416;  // 222 KB of keys + the block's static shared memory
constexpr int SORT_HUGE_SLOT_BITS = 15;
constexpr int SORT_HUGE_GRID = 148;       // one 222 KB block per SM
constexpr int SORT_HUGE_THREADS = 1024;

static __global__ void __launch_bounds__(SORT_HUGE_THREADS)
tile_sort_huge_kernel(int64_t T, const int* __restrict__ tile_start, const long long* __restrict__ header,
                      unsigned long long* __restrict__ keys, const int* __restrict__ slot_inst,
                      int* __restrict__ sorted_gid, int* __restrict__ sorted_inst,
                      const uint16_t* __restrict__ slot_mask, uint16_t* __restrict__ sorted_mask, int gbits) {
    extern __shared__ __align__(16) unsigned long long s_huge[];
    __shared__ int s_fits;
    __shared__ int s_list[SORT_HUGE_THREADS];
    __shared__ int s_n;
    if (header[H_FLAGS] != 0) return;
    const int sb = SORT_HUGE_SLOT_BITS, hi_bits = 64 - gbits - SORT_HUGE_SLOT_BITS;
    const unsigned long long gmask = (1ull << gbits) - 1ull, smask = (1ull << sb) - 1ull;
    // block b owns tiles b, b + grid, ...: its threads inspect SORT_HUGE_THREADS of them at a
    // time and the block sorts the ones in this size class, one after another
    const int64_t stride = gridDim.x;
    for (int64_t c0 = 0; c0 < T; c0 += stride * SORT_HUGE_THREADS) {
      if (threadIdx.x == 0) s_n = 0;
      __syncthreads();
      {
        const int64_t t = c0 + blockIdx.x + stride * threadIdx.x;
        if (t < T) {
            const int n = tile_start[t + 1] - tile_start[t];
            if (n > SORT_BIG_CAP && n <= SORT_HUGE_CAP) s_list[atomicAdd(&s_n, 1)] = threadIdx.x;
        }
      }
      __syncthreads();
      const int count = s_n;
      for (int kk = 0; kk < count; ++kk) {
        const int64_t t = c0 + blockIdx.x + stride * s_list[kk];
        const int s0 = tile_start[t];
        const int n = tile_start[t + 1] - s0;
        if (threadIdx.x == 0) s_fits = 1;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            if ((keys[s0 + i] >> 32) >> hi_bits) s_fits = 0;
        __syncthreads();
        if (!s_fits) {
            sort_bucket_global(s0, n, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
            __syncthreads();
            continue;
        }
        int npow = 64;
        while (npow < n) npow <<= 1;
        const int nfill = (n + 63) & ~63;
        for (int i = threadIdx.x; i < nfill; i += blockDim.x) {
            const unsigned long long k = i < n ? keys[s0 + i] : 0ull;
            s_huge[i] = i < n ? (((k >> 32) << (gbits + sb)) | ((k & gmask) << sb) | (unsigned long long)i)
                              : SORT_PAD_KEY;
        }
        __syncthreads();
        block_sort_smem<false>(s_huge, nullptr, npow, n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned long long k = s_huge[i];
            const int slot = (int)(k & smask);
            const uint32_t g = (uint32_t)((k >> sb) & gmask);
            sorted_gid[s0 + i] = (int)g;
            sorted_inst[s0 + i] = slot_inst[s0 + slot];
            if (sorted_mask) sorted_mask[s0 + i] = slot_mask[s0 + slot];
            keys[s0 + i] = ((k >> (gbits + sb)) << 32) | g;
        }
        __syncthreads();
      }
    }
}

// One block per tile: order the tile's bucket by (depth key, Gaussian index), which is the
// order the reference's stable radix sort of (tile << 32 | depth key) over instances
// enumerated Gaussian by Gaussian produces (src/mapper/wrapper_mapper.cu:134-146). Keys
// within a bucket are distinct (a Gaussian enters a tile's bucket at most once), so any
// correct sorting network gives that order. The optional 16-bit per-slot mask (slot_mask) follows
// its instance into sorted_mask.
// PACKED: every element index of the call is below SORT_PACK_G, so buckets of up to
// SORT_SMEM_CAP keys sort without a payload; the block then needs only the 32 KB key array and
// runs with 256 threads, seven blocks (tiles) per SM instead of four.
constexpr int SORT_PACKED_THREADS = 256;
constexpr int SORT_PACKED_MIN_BLOCKS = 7;

template <bool PACKED>
static __global__ void __launch_bounds__(PACKED ? SORT_PACKED_THREADS : SORT_THREADS,
                                         PACKED ? SORT_PACKED_MIN_BLOCKS : SORT_MIN_BLOCKS)
tile_sort_kernel(int64_t T, const int* __restrict__ tile_start, const long long* __restrict__ header,
                 unsigned long long* __restrict__ keys, const int* __restrict__ slot_inst,
                 int* __restrict__ sorted_gid, int* __restrict__ sorted_inst,
                 const uint16_t* __restrict__ slot_mask, uint16_t* __restrict__ sorted_mask) {
    __shared__ __align__(16) unsigned long long s_keys[SORT_SMEM_CAP];
    __shared__ __align__(16) int s_idx[PACKED ? 4 : SORT_SMEM_CAP];
    const int64_t t = blockIdx.x;
    if (t >= T || header[H_FLAGS] != 0) return;
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    if (n <= 0) return;
    if (n <= SORT_SMEM_CAP) {
        if constexpr (PACKED)
            sort_bucket_packed(s_keys, s0, n, 12, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
        else
            sort_bucket_smem(s_keys, s_idx, s0, n, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask,
                             false);
    } else if (n > SORT_HUGE_CAP) {
        sort_bucket_global(s0, n, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
    }
}

// Second pass: buckets of SORT_SMEM_CAP < n <= SORT_BIG_CAP keys with 192 KB of shared
// memory. Block b owns the tiles b, b + grid, b + 2 grid, ... (large buckets tend to be
// neighbours, so they spread over the blocks); it inspects them SORT_BIG_THREADS at a time and
// orders the large ones it finds, one after another.
constexpr int SORT_BIG_GRID = 148;      // one 192 KB block per SM
constexpr int SORT_BIG_THREADS = 1024;  // the whole SM's threads on one large bucket

// Buckets of SORT_SMEM_CAP < n <= SORT_MID_CAP keys of a call whose element indices fit the
// 13-bit-slot packing: block b orders tiles b, b + grid, ... with 64 KB of shared memory and
// 1024 threads (two blocks per SM, so that a small image's few large buckets run side by side
// with enough warps to cover the shared-memory passes: 256 tiles of ~7,400 keys sort in 140 us
// instead of 155 us with 512 threads).
constexpr int SORT_MID_GRID = 3 * 148;
constexpr int SORT_MID_THREADS = 1024;

static __global__ void __launch_bounds__(SORT_MID_THREADS)
tile_sort_mid_kernel(int64_t T, const int* __restrict__ tile_start, const long long* __restrict__ header,
                     unsigned long long* __restrict__ keys, const int* __restrict__ slot_inst,
                     int* __restrict__ sorted_gid, int* __restrict__ sorted_inst,
                     const uint16_t* __restrict__ slot_mask, uint16_t* __restrict__ sorted_mask) {
    extern __shared__ __align__(16) unsigned long long s_mid_keys[];
    __shared__ int s_list[SORT_MID_THREADS];
    __shared__ int s_n;
    if (header[H_FLAGS] != 0) return;
    // block b owns tiles b, b + grid, ...: its threads inspect SORT_MID_THREADS of them at a
    // time and the block sorts the ones in this size class, one after another
    const int64_t stride = gridDim.x;
    for (int64_t c0 = 0; c0 < T; c0 += stride * SORT_MID_THREADS) {
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        const int64_t t = c0 + blockIdx.x + stride * threadIdx.x;
        if (t < T) {
            const int n = tile_start[t + 1] - tile_start[t];
            if (n > SORT_SMEM_CAP && n <= SORT_MID_CAP) s_list[atomicAdd(&s_n, 1)] = threadIdx.x;
        }
        __syncthreads();
        const int count = s_n;
        for (int k = 0; k < count; ++k) {
            const int64_t tt = c0 + blockIdx.x + stride * s_list[k];
            const int s0 = tile_start[tt];
            sort_bucket_packed(s_mid_keys, s0, tile_start[tt + 1] - s0, SORT_MID_SLOT_BITS, keys, slot_inst,
                               sorted_gid, sorted_inst, slot_mask, sorted_mask);
            __syncthreads();
        }
    }
}

static __global__ void __launch_bounds__(SORT_BIG_THREADS)
tile_sort_big_kernel(int64_t T, const int* __restrict__ tile_start, const long long* __restrict__ header,
                     unsigned long long* __restrict__ keys, const int* __restrict__ slot_inst,
                     int* __restrict__ sorted_gid, int* __restrict__ sorted_inst,
                     const uint16_t* __restrict__ slot_mask, uint16_t* __restrict__ sorted_mask, int mid) {
    extern __shared__ __align__(16) unsigned long long s_big_keys[];
    int* s_big_idx = reinterpret_cast<int*>(s_big_keys + SORT_BIG_CAP);
    __shared__ int s_list[SORT_BIG_THREADS];
    __shared__ int s_n;
    if (header[H_FLAGS] != 0) return;
    const int64_t stride = gridDim.x;
    for (int64_t c0 = 0; c0 < T; c0 += stride * SORT_BIG_THREADS) {
        if (threadIdx.x == 0) s_n = 0;
        __syncthreads();
        const int64_t t = c0 + blockIdx.x + stride * threadIdx.x;
        if (t < T) {
            const int n = tile_start[t + 1] - tile_start[t];
            if (n > SORT_SMEM_CAP && n <= SORT_BIG_CAP && !(mid && n <= SORT_MID_CAP))
                s_list[atomicAdd(&s_n, 1)] = threadIdx.x;
        }
        __syncthreads();
        const int count = s_n;
        for (int k = 0; k < count; ++k) {
            const int64_t tt = c0 + blockIdx.x + stride * s_list[k];
            const int s0 = tile_start[tt];
            const int n = tile_start[tt + 1] - s0;
            sort_bucket_smem(s_big_keys, s_big_idx, s0, n, keys, slot_inst, sorted_gid, sorted_inst, slot_mask,
                             sorted_mask, false);
            __syncthreads();
        }
    }
}

static inline size_t tile_sort_big_smem_bytes() { return SORT_BIG_CAP * (sizeof(unsigned long long) + sizeof(int)); }
static inline size_t tile_sort_mid_smem_bytes() { return SORT_MID_CAP * sizeof(unsigned long long); }
static inline size_t tile_sort_huge_smem_bytes() { return SORT_HUGE_CAP * sizeof(unsigned long long); }
// Bits of the largest element index of a call (at least 1).
static inline int tile_sort_gbits(int64_t n_elems) {
    int b = 1;
    while (b < 31 && (int64_t(1) << b) < n_elems) ++b;
    return b;
}
static inline bool tile_sort_mid(int64_t n_elems) { return n_elems < SORT_PACK_G_MID; }

// Launches the tile sort on `stream` for keys whose low word indexes one of n_elems elements:
// the shared-memory pass over all T tiles and, for large
// buckets, the 192 KB pass. `attr_done` records per device that the second kernel's
// shared-memory limit was raised (one array per translation unit, 128 devices). slot_mask /
// sorted_mask may be NULL.
static inline cudaError_t launch_tile_sort(int64_t T, int64_t n_elems, const int* tile_start,
                                           const long long* header, unsigned long long* keys, const int* slot_inst,
                                           int* sorted_gid, int* sorted_inst, bool* attr_done, cudaStream_t stream,
                                           const uint16_t* slot_mask = nullptr,
                                           uint16_t* sorted_mask = nullptr) {
    if (T <= 0) return cudaSuccess;
    if (n_elems < SORT_PACK_G)
        tile_sort_kernel<true><<<(unsigned)T, SORT_PACKED_THREADS, 0, stream>>>(
            T, tile_start, header, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
    else
        tile_sort_kernel<false><<<(unsigned)T, SORT_THREADS, 0, stream>>>(
            T, tile_start, header, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (!(dev >= 0 && dev < 128 && attr_done[dev])) {
        e = cudaFuncSetAttribute(tile_sort_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_sort_big_smem_bytes());
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(tile_sort_mid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_sort_mid_smem_bytes());
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(tile_sort_huge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_sort_huge_smem_bytes());
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 128) attr_done[dev] = true;
    }
    const bool mid = tile_sort_mid(n_elems);
    if (mid) {
        const unsigned mgrid = (unsigned)(T < SORT_MID_GRID ? T : SORT_MID_GRID);
        tile_sort_mid_kernel<<<mgrid, SORT_MID_THREADS, tile_sort_mid_smem_bytes(), stream>>>(
            T, tile_start, header, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    const unsigned grid = (unsigned)(T < SORT_BIG_GRID ? T : SORT_BIG_GRID);
    tile_sort_big_kernel<<<grid, SORT_BIG_THREADS, tile_sort_big_smem_bytes(), stream>>>(
        T, tile_start, header, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask, mid ? 1 : 0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const unsigned hgrid = (unsigned)(T < SORT_HUGE_GRID ? T : SORT_HUGE_GRID);
    tile_sort_huge_kernel<<<hgrid, SORT_HUGE_THREADS, tile_sort_huge_smem_bytes(), stream>>>(
        T, tile_start, header, keys, slot_inst, sorted_gid, sorted_inst, slot_mask, sorted_mask,
        tile_sort_gbits(n_elems));
    return cudaGetLastError();
}

// Kernel launches launch_tile_sort makes for T > 0 tiles over n_elems elements.
static inline int tile_sort_launches(int64_t n_elems) { return 3 + (tile_sort_mid(n_elems) ? 1 : 0); }

}  // namespace us3d
