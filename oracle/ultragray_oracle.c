/*
 * TEST INFRASTRUCTURE ONLY — the checker for the UltraGray tests; nothing in the product
 * links or calls it.
 *
 * Restatement of the reference UltraGray scanline renderer (ops/ultragray_renderer) in C,
 * in fp32 (suffix _f32) and fp64 (suffix _f64): ray mapper (culls, ray ranges, quantised
 * depth keys, per-ray lists ordered like the reference's stable radix sort of
 * (ray << 32 | depth) over Gaussian-major instances), forward and backward per pixel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int ugo_max_threads_ugr(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
static int ugo_thread_id_ugr(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

/* float -> int32 as the GPU's cvt.rzi.s32 (saturating, NaN -> 0). */
static int32_t ugro_i32(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return (int32_t)-2147483647 - 1;
    return (int32_t)x;
}

/* float -> uint32 as the GPU's cvt.rzi.u32 (negative and NaN -> 0, saturating). */
static uint32_t ugro_u32_sat(double x) {
    if (!(x > 0.0)) return 0u;
    if (x >= 4294967295.0) return 4294967295u;
    return (uint32_t)x;
}

#define REAL float
#define SUFFIX _f32
#define FMAX fmaxf
#define FMIN fminf
#define FABS fabsf
#define SQRT sqrtf
#define FLOOR floorf
#define CEIL ceilf
#define EXP expf
#include "ultragray_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef FMAX
#undef FMIN
#undef FABS
#undef SQRT
#undef FLOOR
#undef CEIL
#undef EXP

#define REAL double
#define SUFFIX _f64
#define FMAX fmax
#define FMIN fmin
#define FABS fabs
#define SQRT sqrt
#define FLOOR floor
#define CEIL ceil
#define EXP exp
#include "ultragray_oracle_impl.h"
