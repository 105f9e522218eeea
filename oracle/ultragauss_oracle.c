/*
 * TEST INFRASTRUCTURE ONLY — the checker for the tests and the timed CPU baseline of the
 * benchmark; nothing in the product links or calls it.
 *
 * Restatement of the reference UltraGauss algorithm (ops/ultragauss_renderer) in C, in
 * fp32 (suffix _f32) and fp64 (suffix _f64), plus the integer parts shared by both: the
 * stable LSD radix sort that stands in for cub::DeviceRadixSort::SortPairs (a stable sort
 * of 64-bit keys over bits [begin_bit, 64): equal keys keep their input order) and the
 * tile-range extraction (src/mapper/core.cu:145-164).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define UGO_TILE 16

static int ugo_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
static int ugo_thread_id(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

int ugo_num_threads(void) { return ugo_max_threads(); }
void ugo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* float -> int32 with the GPU's cvt.rzi.s32 rule: NaN -> 0, saturate at the int range. */
static int32_t ugo_to_i32_sat(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return (int32_t)-2147483647 - 1;
    return (int32_t)x;
}
/* float -> uint32 with the GPU's cvt.rzi.u32 rule: NaN and negatives -> 0, saturate high. */
static uint32_t ugo_to_u32_sat(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 4294967295.0) return 4294967295u;
    return (uint32_t)x;
}

/* Stable LSD radix sort of (key, value) pairs on key bits [begin_bit, 64), 8 bits a pass. */
void ugo_sort_pairs(int64_t n, int begin_bit, uint64_t* keys, int32_t* vals) {
    if (n <= 1) return;
    uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int32_t* v2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    uint64_t *ks = keys, *kd = k2;
    int32_t *vs = vals, *vd = v2;
    for (int shift = begin_bit; shift < 64; shift += 8) {
        const int bits = (64 - shift) < 8 ? (64 - shift) : 8;
        const uint64_t mask = (1ull << bits) - 1;
        int64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (int64_t i = 0; i < n; ++i) cnt[((ks[i] >> shift) & mask) + 1]++;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (int64_t i = 0; i < n; ++i) {
            const int64_t pos = cnt[(ks[i] >> shift) & mask]++;
            kd[pos] = ks[i];
            vd[pos] = vs[i];
        }
        uint64_t* tk = ks; ks = kd; kd = tk;
        int32_t* tv = vs; vs = vd; vd = tv;
    }
    if (ks != keys) {
        memcpy(keys, ks, sizeof(uint64_t) * (size_t)n);
        memcpy(vals, vs, sizeof(int32_t) * (size_t)n);
    }
    free(k2);
    free(v2);
}

/* Per-tile [start, end) over sorted keys; empty tiles keep -1 (src/mapper/core.cu:145-164). */
void ugo_tile_ranges(int64_t n, const uint64_t* keys, int n_tiles, int32_t* rs, int32_t* re) {
    for (int t = 0; t < n_tiles; ++t) rs[t] = re[t] = -1;
    for (int64_t i = 0; i < n; ++i) {
        const uint32_t cur = (uint32_t)(keys[i] >> 32);
        if (cur >= (uint32_t)n_tiles) continue;
        if (i == 0) rs[cur] = 0;
        else {
            const uint32_t prev = (uint32_t)(keys[i - 1] >> 32);
            if (cur != prev) {
                if (prev < (uint32_t)n_tiles) re[prev] = (int32_t)i;
                rs[cur] = (int32_t)i;
            }
        }
        if (i == n - 1) re[cur] = (int32_t)n;
    }
}

#define REAL float
#define SUFFIX _f32
#define FMAX fmaxf
#define SQRT sqrtf
#define FABS fabsf
#define FLOOR floorf
#define CEIL ceilf
#define EXP expf
#include "ultragauss_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef FMAX
#undef SQRT
#undef FABS
#undef FLOOR
#undef CEIL
#undef EXP

#define REAL double
#define SUFFIX _f64
#define FMAX fmax
#define SQRT sqrt
#define FABS fabs
#define FLOOR floor
#define CEIL ceil
#define EXP exp
#include "ultragauss_oracle_impl.h"
