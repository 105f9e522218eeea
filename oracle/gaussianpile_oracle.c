/*
 * TEST INFRASTRUCTURE ONLY — the checker for the GaussianPile tests and part of the CPU
 * baseline; nothing in the product links or calls it. Restatement of the reference
 * GaussianPile projected-slice renderer (ops/gaussianplie_renderer) in fp32 and fp64.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* float -> int32 with the GPU's cvt.rzi.s32 rule (NaN -> 0, saturating). */
static int32_t gpo_to_i32(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return (int32_t)-2147483647 - 1;
    return (int32_t)x;
}

#define REAL float
#define SUFFIX _f32
#define GMAX fmaxf
#define GMIN fminf
#define GSQRT sqrtf
#define GABS fabsf
#define GFLOOR floorf
#define GCEIL ceilf
#define GEXP expf
#define GPOW powf
#include "gaussianpile_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef GMAX
#undef GMIN
#undef GSQRT
#undef GABS
#undef GFLOOR
#undef GCEIL
#undef GEXP
#undef GPOW

#define REAL double
#define SUFFIX _f64
#define GMAX fmax
#define GMIN fmin
#define GSQRT sqrt
#define GABS fabs
#define GFLOOR floor
#define GCEIL ceil
#define GEXP exp
#define GPOW pow
#include "gaussianpile_oracle_impl.h"
